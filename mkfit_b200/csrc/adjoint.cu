// Differentiable fit: summed chi2 of a barrel Kalman fit and its gradient
// with respect to per-step alignment and material parameters.
//
// Parameters per fit step s (theta[s][3]): a = hit shift along the
// transverse tangent (r-phi, cm), b = hit shift in z (cm), c = scale of the
// layer material (radiation length and xi). The loss is
//   L = sum over tracks and steps of the predicted-residual chi2
// of the fit run with those parameters (the fit of mkfg_fit: propagation to
// the shifted hit's radius with material, Kalman update).
//
// Forward kernel: one track per thread, the state in registers; the state
// entering every step is written to a checkpoint array ([n_steps][27][n],
// lane-fastest) so the backward pass never re-runs the earlier steps.
// Backward kernel: one track per thread, steps in reverse; each step
// recomputes its own forward sweep from the checkpoint and runs the
// generated reverse sweep (generated_adjoint.cuh), carrying the adjoint of
// the state to the previous step; per-step parameter adjoints are reduced
// over the block in shared memory (double) and added to the global gradient.
#include "internal.h"
#include "kalman.cuh"
#include "adjoint_step.cuh"

namespace mkfg {

constexpr int kAdjBlock = 128;
constexpr int kAdjMaxSteps = 64;

struct AdjKernelArgs {
  const float* in_par;
  const float* in_err;
  const int* in_chg;
  int in_stride;
  float* out_par;  // optional final state
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
  const float* theta;  // [n_steps][3]
  float* ckpt;         // [n_steps][27][n]
  double* chi2_sum;
  float* out_chi2;     // optional per track
  const float* grad_out;
  double* grad;        // [n_steps][3]
  adj::MatGrid mat;
  int material;
  int hit_layer[kAdjMaxSteps];
};

__device__ __forceinline__ float track_k(int chg) { return float(chg) * 100.f / (-kSol * kBfield); }

__device__ __forceinline__ void load_hit(const AdjKernelArgs& a, int s, int i, float (&m)[3],
                                         float (&me)[6]) {
  int hidx = __ldg(a.hot + s * a.hot_stride + i);
  if (hidx < 0) hidx = 0;
  const int h = __ldg(a.layer_begin + a.hit_layer[s]) + hidx;
#pragma unroll
  for (int e = 0; e < 3; ++e) m[e] = __ldg(a.hpos + e * a.hstride + h);
#pragma unroll
  for (int e = 0; e < 6; ++e) me[e] = __ldg(a.herr + e * a.hstride + h);
}

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < kAdjBlock / 32; ++i) t += red[i];
  return t;
}

template <bool kMat>
__global__ void __launch_bounds__(kAdjBlock) k_align_forward(const AdjKernelArgs a) {
  __shared__ double red[kAdjBlock / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float chi2_track = 0.f;
  if (i < a.n) {
    float par[6], err[21];
#pragma unroll
    for (int e = 0; e < 6; ++e) par[e] = __ldg(a.in_par + e * a.in_stride + i);
#pragma unroll
    for (int e = 0; e < 21; ++e) err[e] = __ldg(a.in_err + e * a.in_stride + i);
    const int chg = __ldg(a.in_chg + i);
    const float k = track_k(chg);
    for (int s = 0; s < a.n_steps; ++s) {
      float* ck = a.ckpt + (size_t)s * 27 * a.n + i;
#pragma unroll
      for (int e = 0; e < 6; ++e) ck[(size_t)e * a.n] = par[e];
#pragma unroll
      for (int e = 0; e < 21; ++e) ck[(size_t)(6 + e) * a.n] = err[e];
      float m[3], me[6];
      load_hit(a, s, i, m, me);
      const float ta = __ldg(a.theta + 3 * s), tb = __ldg(a.theta + 3 * s + 1),
                  tc = __ldg(a.theta + 3 * s + 2);
      float opar[6], oerr[21], c2;
      if (kMat)
        adj::barrel_step_fwd_mat(par, err, m, me, ta, tb, tc, k, a.mat, opar, oerr, c2);
      else
        adj::barrel_step_fwd_nomat(par, err, m, me, ta, tb, tc, k, a.mat, opar, oerr, c2);
#pragma unroll
      for (int e = 0; e < 6; ++e) par[e] = opar[e];
#pragma unroll
      for (int e = 0; e < 21; ++e) err[e] = oerr[e];
      chi2_track += c2;
    }
    if (a.out_par) {
#pragma unroll
      for (int e = 0; e < 6; ++e) a.out_par[e * a.out_stride + i] = par[e];
#pragma unroll
      for (int e = 0; e < 21; ++e) a.out_err[e * a.out_stride + i] = err[e];
      a.out_chg[i] = chg;
    }
    if (a.out_chi2) a.out_chi2[i] = chi2_track;
  }
  const double t = block_sum((double)chi2_track, red);
  if (threadIdx.x == 0) atomicAdd(a.chi2_sum, t);
}

template <bool kMat>
__global__ void __launch_bounds__(kAdjBlock) k_align_backward(const AdjKernelArgs a) {
  __shared__ double acc[kAdjMaxSteps * 3];
  for (int j = threadIdx.x; j < 3 * a.n_steps; j += blockDim.x) acc[j] = 0.0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < a.n;
  const int lane = threadIdx.x & 31;
  float par_bar[6], err_bar[21];
#pragma unroll
  for (int e = 0; e < 6; ++e) par_bar[e] = 0.f;
#pragma unroll
  for (int e = 0; e < 21; ++e) err_bar[e] = 0.f;
  const float g = *a.grad_out;
  const float k = live ? track_k(__ldg(a.in_chg + i)) : 0.f;
  for (int s = a.n_steps - 1; s >= 0; --s) {
    float ga = 0.f, gb = 0.f, gc = 0.f;
    if (live) {
      float par[6], err[21];
      const float* ck = a.ckpt + (size_t)s * 27 * a.n + i;
#pragma unroll
      for (int e = 0; e < 6; ++e) par[e] = ck[(size_t)e * a.n];
#pragma unroll
      for (int e = 0; e < 21; ++e) err[e] = ck[(size_t)(6 + e) * a.n];
      float m[3], me[6];
      load_hit(a, s, i, m, me);
      const float ta = __ldg(a.theta + 3 * s), tb = __ldg(a.theta + 3 * s + 1),
                  tc = __ldg(a.theta + 3 * s + 2);
      float pb[6], eb[21];
      if (kMat)
        adj::barrel_step_rev_mat(par, err, m, me, ta, tb, tc, k, a.mat, par_bar, err_bar, g, pb,
                                 eb, ga, gb, gc);
      else
        adj::barrel_step_rev_nomat(par, err, m, me, ta, tb, tc, k, a.mat, par_bar, err_bar, g,
                                   pb, eb, ga, gb, gc);
#pragma unroll
      for (int e = 0; e < 6; ++e) par_bar[e] = pb[e];
#pragma unroll
      for (int e = 0; e < 21; ++e) err_bar[e] = eb[e];
    }
    double da = ga, db = gb, dc = gc;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      da += __shfl_xor_sync(0xffffffffu, da, off);
      db += __shfl_xor_sync(0xffffffffu, db, off);
      dc += __shfl_xor_sync(0xffffffffu, dc, off);
    }
    if (lane == 0) {
      atomicAdd(&acc[3 * s + 0], da);
      atomicAdd(&acc[3 * s + 1], db);
      atomicAdd(&acc[3 * s + 2], dc);
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < 3 * a.n_steps; j += blockDim.x) atomicAdd(&a.grad[j], acc[j]);
}

namespace {

int fill_args(mkfg_context* ctx, const mkfg_align_args* x, AdjKernelArgs& k) {
  MKFG_REQUIRE(x != nullptr, "null align args");
  const mkfg_fit_args& f = x->fit;
  MKFG_REQUIRE(f.in.n >= 0 && f.in.n <= f.in.stride, "bad input track count/stride");
  MKFG_REQUIRE(f.in.n == 0 || (f.in.par && f.in.err && f.in.chg), "null input tracks");
  MKFG_REQUIRE(f.n_steps >= 1 && f.n_steps <= kAdjMaxSteps, "n_steps must be in [1, %d]",
               kAdjMaxSteps);
  MKFG_REQUIRE(f.endcap_mask == 0, "the differentiable fit supports barrel steps only");
  MKFG_REQUIRE((f.pflags & ~kPfMaterial) == 0,
               "the differentiable fit supports pflags 0 or material (2) only");
  MKFG_REQUIRE(f.hot_stride >= f.in.n && f.hits.n_layers > 0 && f.hit_layer != nullptr,
               "bad hit indexing");
  MKFG_REQUIRE(f.hits.pos && f.hits.err && f.hits.layer_begin && (f.hot_index || f.in.n == 0),
               "null hit pointer");
  MKFG_REQUIRE(x->theta && x->checkpoint && x->chi2_sum, "null theta / checkpoint / chi2_sum");
  MKFG_REQUIRE(!f.out.par || (f.out.err && f.out.chg && f.out.n == f.in.n &&
                              f.out.stride >= f.in.n),
               "bad output tracks");
  for (int s = 0; s < f.n_steps; ++s)
    MKFG_REQUIRE(f.hit_layer[s] >= 0 && f.hit_layer[s] < f.hits.n_layers,
                 "hit_layer[%d]=%d out of range", s, f.hit_layer[s]);
  k = AdjKernelArgs{};
  k.in_par = f.in.par;
  k.in_err = f.in.err;
  k.in_chg = f.in.chg;
  k.in_stride = f.in.stride;
  k.out_par = f.out.par;
  k.out_err = f.out.err;
  k.out_chg = f.out.chg;
  k.out_stride = f.out.stride;
  k.hpos = f.hits.pos;
  k.herr = f.hits.err;
  k.hstride = f.hits.stride;
  k.layer_begin = f.hits.layer_begin;
  k.hot = f.hot_index;
  k.hot_stride = f.hot_stride;
  k.n = f.in.n;
  k.n_steps = f.n_steps;
  k.theta = x->theta;
  k.ckpt = x->checkpoint;
  k.chi2_sum = x->chi2_sum;
  k.out_chi2 = f.out_chi2;
  k.mat = adj::MatGrid{ctx->d_rl, ctx->d_xi};
  k.material = (f.pflags & kPfMaterial) != 0;
  MKFG_REQUIRE(!k.material || ctx->d_rl, "material requested but mkfg_set_material not called");
  for (int s = 0; s < f.n_steps; ++s) k.hit_layer[s] = f.hit_layer[s];
  return MKFG_OK;
}

}  // namespace
}  // namespace mkfg

using namespace mkfg;

extern "C" int mkfg_align_chi2_forward(mkfg_context* ctx, const mkfg_align_args* args) {
  int rc = activate(ctx);
  if (rc) return rc;
  AdjKernelArgs k;
  if ((rc = fill_args(ctx, args, k))) return rc;
  MKFG_CUDA_TRY(cudaMemsetAsync(k.chi2_sum, 0, sizeof(double), ctx->stream));
  if (k.n == 0) return MKFG_OK;
  const int grid = (k.n + kAdjBlock - 1) / kAdjBlock;
  if (k.material)
    k_align_forward<true><<<grid, kAdjBlock, 0, ctx->stream>>>(k);
  else
    k_align_forward<false><<<grid, kAdjBlock, 0, ctx->stream>>>(k);
  MKFG_CUDA_TRY(cudaGetLastError());
  return MKFG_OK;
}

extern "C" int mkfg_align_chi2_backward(mkfg_context* ctx, const mkfg_align_args* args,
                                        const float* grad_out, double* grad_theta) {
  int rc = activate(ctx);
  if (rc) return rc;
  AdjKernelArgs k;
  if ((rc = fill_args(ctx, args, k))) return rc;
  MKFG_REQUIRE(grad_out && grad_theta, "null grad_out / grad_theta");
  k.grad_out = grad_out;
  k.grad = grad_theta;
  MKFG_CUDA_TRY(cudaMemsetAsync(grad_theta, 0, sizeof(double) * 3 * k.n_steps, ctx->stream));
  if (k.n == 0) return MKFG_OK;
  const int grid = (k.n + kAdjBlock - 1) / kAdjBlock;
  if (k.material)
    k_align_backward<true><<<grid, kAdjBlock, 0, ctx->stream>>>(k);
  else
    k_align_backward<false><<<grid, kAdjBlock, 0, ctx->stream>>>(k);
  MKFG_CUDA_TRY(cudaGetLastError());
  return MKFG_OK;
}
