// Kalman fit kernel: one track per thread, all layer steps in registers.
//
// Replaces the reference's MkFitter fit loop (mkFit/MkFitter.cc:286-363,
// 473-522): for each step, gather the track's hit, propagate to the hit's r
// (barrel) or z (endcap) with the configured propagation flags and apply
// the Kalman update. The track state is read once and written once; per
// step only the hit (36 B) and its index (4 B) come from HBM.
#include "internal.h"
#include "kalman.cuh"

namespace mkfg {

constexpr int kMaxFitSteps = 64;  // Config::nMaxTrkHits
constexpr int kFitBlock = 128;

struct FitKernelArgs {
  const float* in_par;
  const float* in_err;
  const int* in_chg;
  int in_stride;
  float* out_par;
  float* out_err;
  int* out_chg;
  int out_stride;
  const float* hpos;
  const float* herr;
  int hstride;
  const int* layer_begin;
  const int* hot;
  int hot_stride;
  int n;
  int n_steps;
  unsigned long long endcap_mask;
  unsigned pflags;
  Material mat;
  float* out_chi2;
  int hit_layer[kMaxFitSteps];
};

template <bool kChi2>
__global__ void __launch_bounds__(kFitBlock) fit_kernel(const FitKernelArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;

  float par[6], err[21];
#pragma unroll
  for (int e = 0; e < 6; ++e) par[e] = __ldg(a.in_par + e * a.in_stride + i);
#pragma unroll
  for (int e = 0; e < 21; ++e) err[e] = __ldg(a.in_err + e * a.in_stride + i);
  const int chg = __ldg(a.in_chg + i);

  float chi2_sum = 0.f;
  for (int s = 0; s < a.n_steps; ++s) {
    int hidx = __ldg(a.hot + s * a.hot_stride + i);
    if (hidx < 0) hidx = 0;  // reference packer's null input (hit 0)
    // An index past its layer is kept on the layer's last hit (and on hit 0
    // of the buffer when the layer is empty), so every read stays inside the
    // hit arrays; the host entry points reject such indexes before copying.
    const int lb0 = __ldg(a.layer_begin + a.hit_layer[s]);
    const int lb1 = __ldg(a.layer_begin + a.hit_layer[s] + 1);
    const int h = max(min(lb0 + hidx, lb1 - 1), 0);
    float mpos[3], merr[6];
#pragma unroll
    for (int e = 0; e < 3; ++e) mpos[e] = __ldg(a.hpos + e * a.hstride + h);
#pragma unroll
    for (int e = 0; e < 6; ++e) merr[e] = __ldg(a.herr + e * a.hstride + h);

    float ppar[6], perr[21];
    const bool endcap = (a.endcap_mask >> s) & 1ull;
    if (!endcap) {
      propagate_to_r(par, err, chg, hypot_f(mpos[0], mpos[1]), a.pflags, a.mat, false, ppar, perr);
      chi2_sum += kalman_barrel<kChi2, true>(ppar, perr, mpos, merr, par, err);
    } else {
      propagate_to_z(par, err, chg, mpos[2], a.pflags, a.mat, false, ppar, perr);
      chi2_sum += kalman_endcap<kChi2, true>(ppar, perr, mpos, merr, par, err);
    }
  }

#pragma unroll
  for (int e = 0; e < 6; ++e) a.out_par[e * a.out_stride + i] = par[e];
#pragma unroll
  for (int e = 0; e < 21; ++e) a.out_err[e * a.out_stride + i] = err[e];
  a.out_chg[i] = chg;
  if (kChi2) a.out_chi2[i] = chi2_sum;
}

namespace {

int check_fit_args(const mkfg_fit_args* a) {
  MKFG_REQUIRE(a != nullptr, "null fit args");
  MKFG_REQUIRE(a->in.n >= 0 && a->in.n <= a->in.stride, "bad input track count/stride");
  MKFG_REQUIRE(a->out.n == a->in.n && a->out.stride >= a->out.n, "bad output track count/stride");
  MKFG_REQUIRE(a->n_steps >= 0 && a->n_steps <= kMaxFitSteps, "n_steps must be in [0, %d]", kMaxFitSteps);
  MKFG_REQUIRE(a->hot_stride >= a->in.n, "hot_stride smaller than track count");
  MKFG_REQUIRE(a->hits.n_layers > 0, "no hit layers");
  MKFG_REQUIRE(a->hit_layer != nullptr || a->n_steps == 0, "null hit_layer");
  for (int s = 0; s < a->n_steps; ++s)
    MKFG_REQUIRE(a->hit_layer[s] >= 0 && a->hit_layer[s] < a->hits.n_layers,
                 "hit_layer[%d]=%d out of range", s, a->hit_layer[s]);
  return MKFG_OK;
}

}  // namespace

// Checks of a host-buffer fit call, all made before anything is copied:
// the device-pointer checks, non-null host arrays, a consistent layer
// table, and every hit index inside its layer (a negative index means the
// layer's hit 0, which must exist).
int check_fit_host_args(const mkfg_fit_args* a) {
  int rc = check_fit_args(a);
  if (rc) return rc;
  const int n = a->in.n, nl = a->hits.n_layers;
  MKFG_REQUIRE(a->hits.layer_begin != nullptr, "null layer_begin");
  MKFG_REQUIRE(a->hits.layer_begin[0] == 0, "layer_begin[0] must be 0");
  for (int l = 0; l < nl; ++l)
    MKFG_REQUIRE(a->hits.layer_begin[l + 1] >= a->hits.layer_begin[l],
                 "layer_begin decreases at layer %d", l);
  const int n_hits = a->hits.layer_begin[nl];
  MKFG_REQUIRE(n_hits <= a->hits.stride, "hit count %d exceeds hit stride %d", n_hits,
               a->hits.stride);
  if (n == 0) return MKFG_OK;
  MKFG_REQUIRE(a->in.par && a->in.err && a->in.chg && a->out.par && a->out.err && a->out.chg,
               "null host track array");
  MKFG_REQUIRE(n_hits == 0 || (a->hits.pos && a->hits.err), "null host hit array");
  MKFG_REQUIRE(a->hot_index != nullptr || a->n_steps == 0, "null hot_index");
  for (int s = 0; s < a->n_steps; ++s) {
    const int l = a->hit_layer[s];
    const int size = a->hits.layer_begin[l + 1] - a->hits.layer_begin[l];
    const int32_t* row = a->hot_index + size_t(s) * a->hot_stride;
    for (int i = 0; i < n; ++i) {
      const int h = row[i] < 0 ? 0 : row[i];
      if (h >= size)
        return set_error(MKFG_ERR_BAD_INPUT,
                         "hot_index[%d][%d] = %d outside layer %d, which holds %d hits", s, i,
                         row[i], l, size);
    }
  }
  return MKFG_OK;
}

namespace {

int launch_fit(mkfg_context* ctx, const mkfg_fit_args* a) {
  if (a->in.n == 0) return MKFG_OK;
  FitKernelArgs k;
  k.in_par = a->in.par;
  k.in_err = a->in.err;
  k.in_chg = a->in.chg;
  k.in_stride = a->in.stride;
  k.out_par = a->out.par;
  k.out_err = a->out.err;
  k.out_chg = a->out.chg;
  k.out_stride = a->out.stride;
  k.hpos = a->hits.pos;
  k.herr = a->hits.err;
  k.hstride = a->hits.stride;
  k.layer_begin = a->hits.layer_begin;
  k.hot = a->hot_index;
  k.hot_stride = a->hot_stride;
  k.n = a->in.n;
  k.n_steps = a->n_steps;
  k.endcap_mask = a->endcap_mask;
  k.pflags = a->pflags;
  k.mat = Material{ctx->d_rl, ctx->d_xi};
  k.out_chi2 = a->out_chi2;
  for (int s = 0; s < kMaxFitSteps; ++s) k.hit_layer[s] = s < a->n_steps ? a->hit_layer[s] : 0;
  const int grid = (a->in.n + kFitBlock - 1) / kFitBlock;
  if (a->out_chi2)
    fit_kernel<true><<<grid, kFitBlock, 0, ctx->stream>>>(k);
  else
    fit_kernel<false><<<grid, kFitBlock, 0, ctx->stream>>>(k);
  MKFG_CUDA_TRY(cudaGetLastError());
  return MKFG_OK;
}

}  // namespace
}  // namespace mkfg

using namespace mkfg;

extern "C" int mkfg_fit(mkfg_context* ctx, const mkfg_fit_args* args) {
  int rc = activate(ctx);
  if (rc) return rc;
  if ((rc = check_fit_args(args))) return rc;
  MKFG_REQUIRE(args->in.par && args->in.err && args->in.chg && args->out.par && args->out.err &&
                   args->out.chg && args->hits.pos && args->hits.err && args->hits.layer_begin &&
                   (args->hot_index || args->n_steps == 0),
               "null device pointer in fit args");
  return launch_fit(ctx, args);
}

namespace {

int fit_host_staged(mkfg_context* ctx, const mkfg_fit_args* args) {
  int rc;
  const int n = args->in.n;
  const int nl = args->hits.n_layers;
  const int n_hits = args->hits.layer_begin[nl];

  // Device scratch: compact strides (n for tracks, n_hits for hits).
  const size_t trk_bytes = size_t(n) * (27 * sizeof(float) + sizeof(int));
  const size_t hit_bytes = size_t(n_hits) * 9 * sizeof(float) + size_t(nl + 1) * sizeof(int) +
                           size_t(args->n_steps) * n * sizeof(int);
  if ((rc = ctx->scratch_in.ensure(trk_bytes))) return rc;
  if ((rc = ctx->scratch_out.ensure(trk_bytes + size_t(n) * sizeof(float)))) return rc;
  if ((rc = ctx->scratch_hits.ensure(hit_bytes))) return rc;
  cudaStream_t st = ctx->stream;

  float* d_in_par = ctx->scratch_in.as<float>();
  float* d_in_err = d_in_par + 6 * size_t(n);
  int* d_in_chg = reinterpret_cast<int*>(d_in_err + 21 * size_t(n));
  float* d_out_par = ctx->scratch_out.as<float>();
  float* d_out_err = d_out_par + 6 * size_t(n);
  int* d_out_chg = reinterpret_cast<int*>(d_out_err + 21 * size_t(n));
  float* d_chi2 = reinterpret_cast<float*>(d_out_chg + n);
  float* d_hpos = ctx->scratch_hits.as<float>();
  float* d_herr = d_hpos + 3 * size_t(n_hits);
  int* d_lb = reinterpret_cast<int*>(d_herr + 6 * size_t(n_hits));
  int* d_hot = d_lb + (nl + 1);

  auto h2d_rows = [&](void* dst, const void* src, int rows, size_t row_elems, size_t src_stride,
                      size_t elem) -> int {
    MKFG_CUDA_TRY(cudaMemcpy2DAsync(dst, row_elems * elem, src, src_stride * elem, row_elems * elem,
                                    rows, cudaMemcpyHostToDevice, st));
    return MKFG_OK;
  };
  if ((rc = h2d_rows(d_in_par, args->in.par, 6, n, args->in.stride, 4))) return rc;
  if ((rc = h2d_rows(d_in_err, args->in.err, 21, n, args->in.stride, 4))) return rc;
  MKFG_CUDA_TRY(cudaMemcpyAsync(d_in_chg, args->in.chg, size_t(n) * 4, cudaMemcpyHostToDevice, st));
  if (n_hits > 0) {
    if ((rc = h2d_rows(d_hpos, args->hits.pos, 3, n_hits, args->hits.stride, 4))) return rc;
    if ((rc = h2d_rows(d_herr, args->hits.err, 6, n_hits, args->hits.stride, 4))) return rc;
  }
  MKFG_CUDA_TRY(cudaMemcpyAsync(d_lb, args->hits.layer_begin, size_t(nl + 1) * 4, cudaMemcpyHostToDevice, st));
  if (args->n_steps > 0)
    if ((rc = h2d_rows(d_hot, args->hot_index, args->n_steps, n, args->hot_stride, 4))) return rc;

  mkfg_fit_args d = *args;
  d.in = mkfg_tracks{d_in_par, d_in_err, d_in_chg, n, n};
  d.out = mkfg_tracks{d_out_par, d_out_err, d_out_chg, n, n};
  d.hits = mkfg_hits{d_hpos, d_herr, d_lb, nl, n_hits > 0 ? n_hits : 1};
  d.hot_index = d_hot;
  d.hot_stride = n;
  d.out_chi2 = args->out_chi2 ? d_chi2 : nullptr;
  if ((rc = launch_fit(ctx, &d))) return rc;

  auto d2h_rows = [&](void* dst, const void* src, int rows, size_t row_elems, size_t dst_stride,
                      size_t elem) -> int {
    MKFG_CUDA_TRY(cudaMemcpy2DAsync(dst, dst_stride * elem, src, row_elems * elem, row_elems * elem,
                                    rows, cudaMemcpyDeviceToHost, st));
    return MKFG_OK;
  };
  if ((rc = d2h_rows(args->out.par, d_out_par, 6, n, args->out.stride, 4))) return rc;
  if ((rc = d2h_rows(args->out.err, d_out_err, 21, n, args->out.stride, 4))) return rc;
  MKFG_CUDA_TRY(cudaMemcpyAsync(args->out.chg, d_out_chg, size_t(n) * 4, cudaMemcpyDeviceToHost, st));
  if (args->out_chi2)
    MKFG_CUDA_TRY(cudaMemcpyAsync(args->out_chi2, d_chi2, size_t(n) * 4, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  return MKFG_OK;
}

}  // namespace

extern "C" int mkfg_fit_host(mkfg_context* ctx, const mkfg_fit_args* args) {
  int rc = activate(ctx);
  if (rc) return rc;
  if ((rc = check_fit_host_args(args))) return rc;
  if (args->in.n == 0) return MKFG_OK;
  rc = fit_host_staged(ctx, args);
  // On an error after copies were queued, let them finish before the caller
  // reuses its host buffers.
  if (rc) cudaStreamSynchronize(ctx->stream);
  return rc;
}
