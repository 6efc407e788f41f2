// Context management, error reporting and the material map upload.
#include "internal.h"
#include "kalman.cuh"

#include <cstring>

namespace mkfg {

namespace {
thread_local std::string t_last_error;
}

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = buf;
  return code;
}

int activate(mkfg_context* ctx) {
  MKFG_REQUIRE(ctx != nullptr, "null context");
  MKFG_CUDA_TRY(cudaSetDevice(ctx->device));
  return MKFG_OK;
}

}  // namespace mkfg

using namespace mkfg;

extern "C" {

void mkfg_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return;
  std::strncpy(buf, t_last_error.c_str(), len - 1);
  buf[len - 1] = '\0';
}

const char* mkfg_version(void) { return "mkfit_b200 0.1 sm_100a"; }

int mkfg_context_create(int device, mkfg_context** out) {
  MKFG_REQUIRE(out != nullptr, "null output pointer");
  *out = nullptr;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0)
    return set_error(MKFG_ERR_NO_DEVICE, "no CUDA device available");
  MKFG_REQUIRE(device >= 0 && device < n_dev, "device %d out of range [0, %d)", device, n_dev);
  cudaDeviceProp prop;
  MKFG_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return set_error(MKFG_ERR_NO_DEVICE, "device %d is sm_%d%d; this build targets sm_100a",
                     device, prop.major, prop.minor);
  MKFG_CUDA_TRY(cudaSetDevice(device));
  mkfg_context* ctx = new mkfg_context;
  ctx->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
  ctx->stream = ctx->own_stream;
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_rl, sizeof(float) * kMatNZ * kMatNR);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_xi, sizeof(float) * kMatNZ * kMatNR);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_rl, 0, sizeof(float) * kMatNZ * kMatNR, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_xi, 0, sizeof(float) * kMatNZ * kMatNR, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    mkfg_context_destroy(ctx);
    return set_error(MKFG_ERR_CUDA, "context setup failed: %s", cudaGetErrorString(e));
  }
  *out = ctx;
  return MKFG_OK;
}

int mkfg_context_destroy(mkfg_context* ctx) {
  if (!ctx) return MKFG_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  finder_release(ctx);
  if (ctx->d_rl) cudaFree(ctx->d_rl);
  if (ctx->d_xi) cudaFree(ctx->d_xi);
  ctx->scratch_in.release();
  ctx->scratch_hits.release();
  ctx->scratch_out.release();
  ctx->scratch_misc.release();
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return MKFG_OK;
}

void* mkfg_context_stream(mkfg_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int mkfg_context_set_stream(mkfg_context* ctx, void* stream) {
  int rc = activate(ctx);
  if (rc) return rc;
  // Work already enqueued finishes on the stream it was enqueued on.
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return MKFG_OK;
}

int mkfg_context_synchronize(mkfg_context* ctx) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return MKFG_OK;
}

int mkfg_set_material(mkfg_context* ctx, const float* rl_grid, const float* xi_grid) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(rl_grid && xi_grid, "null material grid");
  const size_t bytes = sizeof(float) * kMatNZ * kMatNR;
  MKFG_CUDA_TRY(cudaMemcpyAsync(ctx->d_rl, rl_grid, bytes, cudaMemcpyHostToDevice, ctx->stream));
  MKFG_CUDA_TRY(cudaMemcpyAsync(ctx->d_xi, xi_grid, bytes, cudaMemcpyHostToDevice, ctx->stream));
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return MKFG_OK;
}

}  // extern "C"

//------------------------------------------------------------------------------
// FP32 CUDA-core throughput probe (roofline denominator for the kernels of
// this library, which run on the FP32 pipes, not the tensor cores).
//------------------------------------------------------------------------------
namespace mkfg {
__global__ void fma_probe_kernel(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
  float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678f) out[0] = s;  // keeps the chains live
}
}  // namespace mkfg

extern "C" int mkfg_probe_fp32_peak(mkfg_context* ctx, int iters, double* tflops) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(tflops != nullptr && iters > 0, "bad probe arguments");
  int n_sm = 0;
  MKFG_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, ctx->device));
  const int blocks = n_sm * 8, threads = 256;
  float* d_out = nullptr;
  MKFG_CUDA_TRY(cudaMalloc(&d_out, sizeof(float)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(d_out, iters / 4 + 1, 0.999999f, 1e-7f);
  cudaEventRecord(e0, ctx->stream);
  fma_probe_kernel<<<blocks, threads, 0, ctx->stream>>>(d_out, iters, 0.999999f, 1e-7f);
  cudaEventRecord(e1, ctx->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_out);
  if (e != cudaSuccess) return set_error(MKFG_ERR_CUDA, "probe failed: %s", cudaGetErrorString(e));
  const double flops = 2.0 * 8 * 16 * double(iters) * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return MKFG_OK;
}
