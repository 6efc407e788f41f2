// The finding's operator table as plain calls: the three operations the
// reference selects per layer through FindingFoos (mkFit/FindingFoos.h:
// 10-38, FindingFoos.cc:7-8) -- propagation to a layer (MkBase::
// PropagateTracksToR / ToZ), propagation to the hit with the chi2
// (kalmanPropagateAndComputeChi2[Endcap]) and with the update
// (kalmanPropagateAndUpdate[Endcap], mkFit/KalmanUtilsMPlex.cc:471-544,
// 697-770) -- on caller-given states, one thread per state, with the
// device functions the fit and the finding run (kalman.cuh).
//
// Arrays are lane-fastest with an element stride (a Matriplex's NN lanes:
// element e of state i at e * stride + i), so a Matriplex's storage can be
// passed as it is. Host pointers; every call stages through the context's
// scratch and synchronizes.
#include "internal.h"
#include "kalman.cuh"

namespace mkfg {

constexpr int kOpBlock = 128;

struct OpArgs {
  int n, stride, endcap;
  unsigned pflags;
  Material mat;
  const float* par;     // [6][stride]
  const float* err;     // [21][stride]
  const int* chg;       // [stride]
  const float* target;  // [stride]: r or z to propagate to
  const float* hpos;    // [3][stride]
  const float* herr;    // [6][stride]
  float* out_par;       // [6][stride]
  float* out_err;       // [21][stride]
  int* out_chg;
  float* out_chi2;
};

__device__ __forceinline__ void op_load(const OpArgs& A, int i, float (&p)[6], float (&e)[21]) {
#pragma unroll
  for (int k = 0; k < 6; ++k) p[k] = A.par[k * A.stride + i];
#pragma unroll
  for (int k = 0; k < 21; ++k) e[k] = A.err[k * A.stride + i];
}

__device__ __forceinline__ void op_hit(const OpArgs& A, int i, float (&m)[3], float (&v)[6]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) m[k] = A.hpos[k * A.stride + i];
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = A.herr[k * A.stride + i];
}

// propagateHelixToRMPlex / propagateHelixToZMPlex to the given r / z.
__global__ void __launch_bounds__(kOpBlock) k_op_propagate(const OpArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  float p[6], e[21], op[6], oe[21];
  op_load(A, i, p, e);
  if (A.endcap)
    propagate_to_z(p, e, A.chg[i], A.target[i], A.pflags, A.mat, false, op, oe);
  else
    propagate_to_r(p, e, A.chg[i], A.target[i], A.pflags, A.mat, false, op, oe);
#pragma unroll
  for (int k = 0; k < 6; ++k) A.out_par[k * A.stride + i] = op[k];
#pragma unroll
  for (int k = 0; k < 21; ++k) A.out_err[k * A.stride + i] = oe[k];
}

// kalmanPropagateAndComputeChi2[Endcap]: propagation to the hit's radius
// (barrel) or z (endcap), then the chi2; out_par = the propagated state.
__global__ void __launch_bounds__(kOpBlock) k_op_chi2(const OpArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  float p[6], e[21], m[3], v[6], hp[6], he[21];
  op_load(A, i, p, e);
  op_hit(A, i, m, v);
  float chi2;
  if (A.endcap) {
    propagate_to_z(p, e, A.chg[i], m[2], A.pflags, A.mat, false, hp, he);
    chi2 = kalman_endcap<true, false>(hp, he, m, v, hp, he);
  } else {
    propagate_to_r(p, e, A.chg[i], hypot_f(m[0], m[1]), A.pflags, A.mat, false, hp, he);
    chi2 = kalman_barrel<true, false>(hp, he, m, v, hp, he);
  }
  A.out_chi2[i] = chi2;
#pragma unroll
  for (int k = 0; k < 6; ++k) A.out_par[k * A.stride + i] = hp[k];
}

// kalmanPropagateAndUpdate[Endcap]: propagation to the hit, the update and
// the charge flip of a negative 1/pT.
__global__ void __launch_bounds__(kOpBlock) k_op_update(const OpArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  float p[6], e[21], m[3], v[6], hp[6], he[21];
  op_load(A, i, p, e);
  op_hit(A, i, m, v);
  int chg = A.chg[i];
  if (A.endcap) {
    propagate_to_z(p, e, chg, m[2], A.pflags, A.mat, false, hp, he);
    kalman_endcap<false, true>(hp, he, m, v, p, e);
  } else {
    propagate_to_r(p, e, chg, hypot_f(m[0], m[1]), A.pflags, A.mat, false, hp, he);
    kalman_barrel<false, true>(hp, he, m, v, p, e);
  }
  if (p[3] < 0) {
    chg = -chg;
    p[3] = -p[3];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) A.out_par[k * A.stride + i] = p[k];
#pragma unroll
  for (int k = 0; k < 21; ++k) A.out_err[k * A.stride + i] = e[k];
  A.out_chg[i] = chg;
}

namespace {

enum OpKind { kOpPropagate, kOpChi2, kOpUpdate };

// Stages the arrays of one operator call, runs it and copies the results
// back.
int run_op(mkfg_context* ctx, OpKind kind, int endcap, int n, int stride, const float* par,
           const float* err, const int32_t* chg, const float* target, const float* hpos,
           const float* herr, uint32_t pflags, float* out_par, float* out_err, int32_t* out_chg,
           float* out_chi2) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(endcap == 0 || endcap == 1, "endcap must be 0 or 1");
  MKFG_REQUIRE(n >= 0 && stride >= n && stride <= (1 << 24), "n %d, stride %d", n, stride);
  MKFG_REQUIRE((pflags & ~3u) == 0, "pflags 0x%x: only bits 0 (B field) and 1 (material)", pflags);
  if (n == 0) return MKFG_OK;
  MKFG_REQUIRE(par && err && chg && out_par, "null argument");
  MKFG_REQUIRE(kind != kOpPropagate || (target && out_err), "null target / out_err");
  MKFG_REQUIRE(kind == kOpPropagate || (hpos && herr), "null hit arrays");
  MKFG_REQUIRE(kind != kOpChi2 || out_chi2, "null out_chi2");
  MKFG_REQUIRE(kind != kOpUpdate || (out_err && out_chg), "null out_err / out_chg");
  const size_t S = (size_t)stride;
  auto r = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t need = r(4 * 27 * S) + r(4 * S) * 3 + r(4 * 9 * S) + r(4 * 27 * S);
  if ((rc = ctx->scratch_misc.ensure(need))) return rc;
  char* p = ctx->scratch_misc.as<char>();
  auto take = [&](size_t bytes) {
    char* q = p;
    p += r(bytes);
    return q;
  };
  OpArgs A{};
  A.n = n;
  A.stride = stride;
  A.endcap = endcap;
  A.pflags = pflags;
  A.mat = Material{ctx->d_rl, ctx->d_xi};
  float* d_par = reinterpret_cast<float*>(take(4 * 6 * S));
  float* d_err = reinterpret_cast<float*>(take(4 * 21 * S));
  int* d_chg = reinterpret_cast<int*>(take(4 * S));
  float* d_target = reinterpret_cast<float*>(take(4 * S));
  float* d_chi2 = reinterpret_cast<float*>(take(4 * S));
  float* d_hpos = reinterpret_cast<float*>(take(4 * 3 * S));
  float* d_herr = reinterpret_cast<float*>(take(4 * 6 * S));
  float* d_opar = reinterpret_cast<float*>(take(4 * 6 * S));
  float* d_oerr = reinterpret_cast<float*>(take(4 * 21 * S));
  cudaStream_t st = ctx->stream;
  auto up = [&](void* d, const void* h, size_t bytes) {
    return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st);
  };
  MKFG_CUDA_TRY(up(d_par, par, 4 * 6 * S));
  MKFG_CUDA_TRY(up(d_err, err, 4 * 21 * S));
  MKFG_CUDA_TRY(up(d_chg, chg, 4 * S));
  if (kind == kOpPropagate) MKFG_CUDA_TRY(up(d_target, target, 4 * S));
  if (kind != kOpPropagate) {
    MKFG_CUDA_TRY(up(d_hpos, hpos, 4 * 3 * S));
    MKFG_CUDA_TRY(up(d_herr, herr, 4 * 6 * S));
  }
  A.par = d_par;
  A.err = d_err;
  A.chg = d_chg;
  A.target = d_target;
  A.hpos = d_hpos;
  A.herr = d_herr;
  A.out_par = d_opar;
  A.out_err = d_oerr;
  A.out_chg = d_chg;
  A.out_chi2 = d_chi2;
  const int grid = (n + kOpBlock - 1) / kOpBlock;
  if (kind == kOpPropagate) k_op_propagate<<<grid, kOpBlock, 0, st>>>(A);
  else if (kind == kOpChi2) k_op_chi2<<<grid, kOpBlock, 0, st>>>(A);
  else k_op_update<<<grid, kOpBlock, 0, st>>>(A);
  MKFG_CUDA_TRY(cudaGetLastError());
  // Only the states' lanes [0, n) of each element row are written back.
  auto down = [&](void* h, const void* d, int rows, size_t elem) {
    return cudaMemcpy2DAsync(h, elem * S, d, elem * S, elem * (size_t)n, rows,
                             cudaMemcpyDeviceToHost, st);
  };
  MKFG_CUDA_TRY(down(out_par, d_opar, 6, 4));
  if (kind != kOpChi2) MKFG_CUDA_TRY(down(out_err, d_oerr, 21, 4));
  if (kind == kOpChi2) MKFG_CUDA_TRY(down(out_chi2, d_chi2, 1, 4));
  if (kind == kOpUpdate) MKFG_CUDA_TRY(down(out_chg, d_chg, 1, 4));
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  return MKFG_OK;
}

}  // namespace
}  // namespace mkfg

using namespace mkfg;

extern "C" int mkfg_op_propagate(mkfg_context* ctx, int32_t endcap, int32_t n, int32_t stride,
                                 const float* par, const float* err, const int32_t* chg,
                                 const float* target, uint32_t pflags, float* out_par,
                                 float* out_err) {
  return run_op(ctx, kOpPropagate, endcap, n, stride, par, err, chg, target, nullptr, nullptr,
                pflags, out_par, out_err, nullptr, nullptr);
}

extern "C" int mkfg_op_propagate_chi2(mkfg_context* ctx, int32_t endcap, int32_t n, int32_t stride,
                                      const float* par, const float* err, const int32_t* chg,
                                      const float* hit_pos, const float* hit_err, uint32_t pflags,
                                      float* out_chi2, float* out_prop_par) {
  return run_op(ctx, kOpChi2, endcap, n, stride, par, err, chg, nullptr, hit_pos, hit_err, pflags,
                out_prop_par, nullptr, nullptr, out_chi2);
}

extern "C" int mkfg_op_propagate_update(mkfg_context* ctx, int32_t endcap, int32_t n,
                                        int32_t stride, const float* par, const float* err,
                                        const int32_t* chg, const float* hit_pos,
                                        const float* hit_err, uint32_t pflags, float* out_par,
                                        float* out_err, int32_t* out_chg) {
  return run_op(ctx, kOpUpdate, endcap, n, stride, par, err, chg, nullptr, hit_pos, hit_err,
                pflags, out_par, out_err, out_chg, nullptr);
}
