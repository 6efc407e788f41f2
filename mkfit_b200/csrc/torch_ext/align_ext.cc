// PyTorch binding of the differentiable fit: a torch::autograd::Function
// whose forward is mkfg_align_chi2_forward (summed chi2 of the fit at
// alignment / material parameters theta) and whose backward is
// mkfg_align_chi2_backward (the hand-derived adjoint), both from the C ABI.
// Built as a Python extension module against libtorch; the kernels stay in
// libmkfit_b200.so.
//
// Streams: the kernels run on the library context's stream. Each call makes
// that stream wait for the caller's current stream, allocates its tensors
// with that stream current, and makes the caller's stream wait for it
// before returning.
#include <torch/extension.h>

#include <ATen/cuda/CUDAEvent.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>

#include "../../../include/mkfit_b200.h"

namespace {

using torch::autograd::AutogradContext;
using torch::autograd::variable_list;

void check(int rc) {
  if (rc != MKFG_OK) {
    char msg[1024];
    mkfg_last_error(msg, sizeof msg);
    TORCH_CHECK(false, "mkfit_b200 error ", rc, ": ", msg);
  }
}

// Runs fn with the context stream current, ordered after and before the
// caller's stream.
template <typename Fn>
void on_context_stream(mkfg_context* ctx, int device, Fn&& fn) {
  auto caller = c10::cuda::getCurrentCUDAStream(device);
  auto cs = c10::cuda::getStreamFromExternal(static_cast<cudaStream_t>(mkfg_context_stream(ctx)),
                                             device);
  at::cuda::CUDAEvent in_ready;
  in_ready.record(caller);
  in_ready.block(cs);
  {
    c10::cuda::CUDAStreamGuard guard(cs);
    fn();
  }
  at::cuda::CUDAEvent done;
  done.record(cs);
  done.block(caller);
}

struct Inputs {
  torch::Tensor par, err, chg, hit_pos, hit_err, layer_begin, hot;
  std::vector<int32_t> hit_layer;
  int64_t pflags;
};

mkfg_align_args make_args(const Inputs& in, const torch::Tensor& theta, const torch::Tensor& ckpt,
                          const torch::Tensor& sum) {
  const int n = static_cast<int>(in.chg.size(0));
  mkfg_align_args a{};
  a.fit.in = mkfg_tracks{in.par.data_ptr<float>(), in.err.data_ptr<float>(),
                         in.chg.data_ptr<int32_t>(), n, n};
  a.fit.out = mkfg_tracks{nullptr, nullptr, nullptr, n, n};
  a.fit.hits = mkfg_hits{in.hit_pos.data_ptr<float>(), in.hit_err.data_ptr<float>(),
                         in.layer_begin.data_ptr<int32_t>(),
                         static_cast<int32_t>(in.layer_begin.size(0) - 1),
                         static_cast<int32_t>(in.hit_pos.size(1))};
  a.fit.hot_index = in.hot.data_ptr<int32_t>();
  a.fit.hot_stride = n;
  a.fit.n_steps = static_cast<int32_t>(in.hit_layer.size());
  a.fit.hit_layer = in.hit_layer.data();
  a.fit.endcap_mask = 0;
  a.fit.pflags = static_cast<uint32_t>(in.pflags);
  a.fit.out_chi2 = nullptr;
  a.theta = theta.data_ptr<float>();
  a.checkpoint = ckpt.data_ptr<float>();
  a.chi2_sum = sum.data_ptr<double>();
  return a;
}

class AlignChi2 : public torch::autograd::Function<AlignChi2> {
 public:
  static torch::Tensor forward(AutogradContext* actx, torch::Tensor theta, int64_t handle,
                               torch::Tensor par, torch::Tensor err, torch::Tensor chg,
                               torch::Tensor hit_pos, torch::Tensor hit_err,
                               torch::Tensor layer_begin, torch::Tensor hot,
                               std::vector<int64_t> hit_layer, int64_t pflags) {
    auto* ctx = reinterpret_cast<mkfg_context*>(handle);
    TORCH_CHECK(theta.is_cuda() && par.is_cuda(), "tensors must be on the context's device");
    const int device = theta.get_device();
    Inputs in{par.contiguous(), err.contiguous(), chg.contiguous(), hit_pos.contiguous(),
              hit_err.contiguous(), layer_begin.contiguous(), hot.contiguous(), {}, pflags};
    for (auto l : hit_layer) in.hit_layer.push_back(static_cast<int32_t>(l));
    const int64_t n_steps = static_cast<int64_t>(hit_layer.size());
    TORCH_CHECK(theta.numel() == 3 * n_steps, "theta must hold 3 parameters per step");
    torch::Tensor th, ckpt, sum;
    on_context_stream(ctx, device, [&] {
      th = theta.detach().to(torch::kFloat32).contiguous();
      ckpt = torch::empty({n_steps, 27, in.chg.size(0)}, par.options().dtype(torch::kFloat32));
      sum = torch::empty({}, par.options().dtype(torch::kFloat64));
      mkfg_align_args a = make_args(in, th, ckpt, sum);
      check(mkfg_align_chi2_forward(ctx, &a));
    });
    actx->save_for_backward({th, ckpt, in.par, in.err, in.chg, in.hit_pos, in.hit_err,
                             in.layer_begin, in.hot});
    actx->saved_data["handle"] = handle;
    actx->saved_data["hit_layer"] = hit_layer;
    actx->saved_data["pflags"] = pflags;
    actx->saved_data["dtype"] = static_cast<int64_t>(theta.scalar_type());
    return sum.to(theta.scalar_type());
  }

  static variable_list backward(AutogradContext* actx, variable_list grad_outputs) {
    auto s = actx->get_saved_variables();
    auto* ctx = reinterpret_cast<mkfg_context*>(actx->saved_data["handle"].toInt());
    Inputs in{s[2], s[3], s[4], s[5], s[6], s[7], s[8], {}, actx->saved_data["pflags"].toInt()};
    for (auto l : actx->saved_data["hit_layer"].toIntVector())
      in.hit_layer.push_back(static_cast<int32_t>(l));
    const auto th = s[0], ckpt = s[1];
    const int device = th.get_device();
    torch::Tensor grad;
    on_context_stream(ctx, device, [&] {
      auto g = grad_outputs[0].to(torch::kFloat32).contiguous();
      auto sum = torch::empty({}, th.options().dtype(torch::kFloat64));
      grad = torch::empty({static_cast<int64_t>(in.hit_layer.size()), 3},
                          th.options().dtype(torch::kFloat64));
      mkfg_align_args a = make_args(in, th, ckpt, sum);
      check(mkfg_align_chi2_backward(ctx, &a, g.data_ptr<float>(), grad.data_ptr<double>()));
    });
    const auto dtype = static_cast<c10::ScalarType>(actx->saved_data["dtype"].toInt());
    variable_list out(11);
    out[0] = grad.to(dtype).reshape(th.sizes());
    return out;
  }
};

torch::Tensor align_chi2(torch::Tensor theta, int64_t handle, torch::Tensor par, torch::Tensor err,
                         torch::Tensor chg, torch::Tensor hit_pos, torch::Tensor hit_err,
                         torch::Tensor layer_begin, torch::Tensor hot,
                         std::vector<int64_t> hit_layer, int64_t pflags) {
  return AlignChi2::apply(theta, handle, par, err, chg, hit_pos, hit_err, layer_begin, hot,
                          hit_layer, pflags);
}

}  // namespace

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.doc() = "Differentiable mkfit_b200 fit (autograd Function over the C ABI)";
  m.def("align_chi2", &align_chi2,
        "Summed fit chi2 at alignment / material parameters theta [n_steps][3]; "
        "differentiable in theta.");
}
