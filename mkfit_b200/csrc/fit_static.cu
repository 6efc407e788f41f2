// Host-buffer Kalman fit that allocates nothing: the inputs and outputs are
// staged through a fixed device array compiled into the library instead of
// the context's grow-only scratch (mkfg_fit_host). The fit itself is the
// device-pointer entry point mkfg_fit on pointers into that array.
//
// The array lives in this translation unit only, so with the CUDA runtime's
// lazy module loading its device memory is taken on a device the first time
// this entry point resolves its address there, not by the other entry points.
#include "internal.h"

#include <atomic>

namespace mkfg {

// 16 MiB: e.g. 16384 tracks x 10 layers (one hit per layer) with chi2 output
// need about 10.3 MiB of staging.
constexpr size_t kFitStageBytes = size_t(16) << 20;
constexpr int kFitStageMaxDevices = 64;
constexpr int kFitStageMaxSteps = 64;  // the fit's step limit

static __device__ __align__(256) unsigned char fit_stage[kFitStageBytes];

// Device address of fit_stage, resolved once per device.
static std::atomic<void*> fit_stage_addr[kFitStageMaxDevices];

static int fit_stage_address(int device, unsigned char** out) {
  MKFG_REQUIRE(device >= 0 && device < kFitStageMaxDevices, "device %d out of range", device);
  void* p = fit_stage_addr[device].load(std::memory_order_acquire);
  if (!p) {
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, fit_stage);
    if (e != cudaSuccess || !p)
      return set_error(MKFG_ERR_CUDA, "cudaGetSymbolAddress(fit_stage) failed: %s",
                       cudaGetErrorString(e));
    fit_stage_addr[device].store(p, std::memory_order_release);
  }
  *out = static_cast<unsigned char*>(p);
  return MKFG_OK;
}

static size_t stage_round(size_t bytes) { return (bytes + 255) / 256 * 256; }

}  // namespace mkfg

using namespace mkfg;

namespace {

int fit_static_staged(mkfg_context* ctx, const mkfg_fit_args* args, unsigned char* base);

}  // namespace

extern "C" int mkfg_fit_host_static(mkfg_context* ctx, const mkfg_fit_args* args) {
  int rc = activate(ctx);
  if (rc) return rc;
  // Every check, the hit indexes against their layers included, comes
  // before the first copy into the shared array.
  if ((rc = check_fit_host_args(args))) return rc;
  MKFG_REQUIRE(args->n_steps <= kFitStageMaxSteps, "n_steps must be in [0, %d]",
               kFitStageMaxSteps);
  const int n = args->in.n;
  const int nl = args->hits.n_layers;
  const int n_steps = args->n_steps;
  const int n_hits = args->hits.layer_begin[nl];
  if (n == 0) return MKFG_OK;

  // Staging layout (256-byte aligned pieces). Nothing in it has to start at
  // zero: every byte the kernel reads is copied in by this call first, and
  // the kernel writes every output element of tracks [0, n).
  const size_t nn = size_t(n), nh = size_t(n_hits);
  const size_t sz_in_par = stage_round(6 * nn * 4), sz_in_err = stage_round(21 * nn * 4);
  const size_t sz_trk_int = stage_round(nn * 4);
  const size_t sz_hpos = stage_round(3 * nh * 4), sz_herr = stage_round(6 * nh * 4);
  const size_t sz_lb = stage_round(size_t(nl + 1) * 4);
  const size_t sz_hot = stage_round(size_t(n_steps) * nn * 4);
  const size_t need = 2 * (sz_in_par + sz_in_err + sz_trk_int) + sz_trk_int + sz_hpos + sz_herr +
                      sz_lb + sz_hot;
  if (need > kFitStageBytes)
    return set_error(MKFG_ERR_BAD_INPUT,
                     "mkfg_fit_host_static: %d tracks, %d hits, %d steps need %zu bytes of "
                     "staging; the fixed device array holds %zu (use mkfg_fit_host)",
                     n, n_hits, n_steps, need, kFitStageBytes);

  unsigned char* base = nullptr;
  if ((rc = fit_stage_address(ctx->device, &base))) return rc;
  rc = fit_static_staged(ctx, args, base);
  // On an error after copies into the array were queued, let them finish:
  // the caller may start the next call as soon as this one returns.
  if (rc) cudaStreamSynchronize(ctx->stream);
  return rc;
}

namespace {

int fit_static_staged(mkfg_context* ctx, const mkfg_fit_args* args, unsigned char* base) {
  int rc;
  const int n = args->in.n;
  const int nl = args->hits.n_layers;
  const int n_steps = args->n_steps;
  const int n_hits = args->hits.layer_begin[nl];
  const size_t nn = size_t(n), nh = size_t(n_hits);
  const size_t sz_in_par = stage_round(6 * nn * 4), sz_in_err = stage_round(21 * nn * 4);
  const size_t sz_trk_int = stage_round(nn * 4);
  const size_t sz_hpos = stage_round(3 * nh * 4), sz_herr = stage_round(6 * nh * 4);
  const size_t sz_lb = stage_round(size_t(nl + 1) * 4);
  const size_t sz_hot = stage_round(size_t(n_steps) * nn * 4);
  unsigned char* p = base;
  auto take = [&p](size_t bytes) {
    unsigned char* r = p;
    p += bytes;
    return r;
  };
  float* d_in_par = reinterpret_cast<float*>(take(sz_in_par));
  float* d_in_err = reinterpret_cast<float*>(take(sz_in_err));
  int* d_in_chg = reinterpret_cast<int*>(take(sz_trk_int));
  float* d_out_par = reinterpret_cast<float*>(take(sz_in_par));
  float* d_out_err = reinterpret_cast<float*>(take(sz_in_err));
  int* d_out_chg = reinterpret_cast<int*>(take(sz_trk_int));
  float* d_chi2 = reinterpret_cast<float*>(take(sz_trk_int));
  float* d_hpos = reinterpret_cast<float*>(take(sz_hpos));
  float* d_herr = reinterpret_cast<float*>(take(sz_herr));
  int* d_lb = reinterpret_cast<int*>(take(sz_lb));
  int* d_hot = reinterpret_cast<int*>(take(sz_hot));

  cudaStream_t st = ctx->stream;
  auto h2d_rows = [&](void* dst, const void* src, int rows, size_t row_elems,
                      size_t src_stride) -> int {
    MKFG_CUDA_TRY(cudaMemcpy2DAsync(dst, row_elems * 4, src, src_stride * 4, row_elems * 4, rows,
                                    cudaMemcpyHostToDevice, st));
    return MKFG_OK;
  };
  if ((rc = h2d_rows(d_in_par, args->in.par, 6, nn, args->in.stride))) return rc;
  if ((rc = h2d_rows(d_in_err, args->in.err, 21, nn, args->in.stride))) return rc;
  MKFG_CUDA_TRY(cudaMemcpyAsync(d_in_chg, args->in.chg, nn * 4, cudaMemcpyHostToDevice, st));
  if (n_hits > 0) {
    if ((rc = h2d_rows(d_hpos, args->hits.pos, 3, nh, args->hits.stride))) return rc;
    if ((rc = h2d_rows(d_herr, args->hits.err, 6, nh, args->hits.stride))) return rc;
  }
  MKFG_CUDA_TRY(cudaMemcpyAsync(d_lb, args->hits.layer_begin, size_t(nl + 1) * 4,
                                cudaMemcpyHostToDevice, st));
  if (n_steps > 0)
    if ((rc = h2d_rows(d_hot, args->hot_index, n_steps, nn, args->hot_stride))) return rc;

  mkfg_fit_args d = *args;
  d.in = mkfg_tracks{d_in_par, d_in_err, d_in_chg, n, n};
  d.out = mkfg_tracks{d_out_par, d_out_err, d_out_chg, n, n};
  d.hits = mkfg_hits{d_hpos, d_herr, d_lb, nl, n_hits > 0 ? n_hits : 1};
  d.hot_index = d_hot;
  d.hot_stride = n;
  d.out_chi2 = args->out_chi2 ? d_chi2 : nullptr;
  if ((rc = mkfg_fit(ctx, &d))) return rc;

  auto d2h_rows = [&](void* dst, const void* src, int rows, size_t row_elems,
                      size_t dst_stride) -> int {
    MKFG_CUDA_TRY(cudaMemcpy2DAsync(dst, dst_stride * 4, src, row_elems * 4, row_elems * 4, rows,
                                    cudaMemcpyDeviceToHost, st));
    return MKFG_OK;
  };
  if ((rc = d2h_rows(args->out.par, d_out_par, 6, nn, args->out.stride))) return rc;
  if ((rc = d2h_rows(args->out.err, d_out_err, 21, nn, args->out.stride))) return rc;
  MKFG_CUDA_TRY(cudaMemcpyAsync(args->out.chg, d_out_chg, nn * 4, cudaMemcpyDeviceToHost, st));
  if (args->out_chi2)
    MKFG_CUDA_TRY(cudaMemcpyAsync(args->out_chi2, d_chi2, nn * 4, cudaMemcpyDeviceToHost, st));
  // The staging array is reused by the next call: finish before returning.
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  return MKFG_OK;
}

}  // namespace
