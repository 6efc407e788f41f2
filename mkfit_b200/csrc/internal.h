// Internal host-side helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/mkfit_b200.h"

namespace mkfg {

// Records the calling thread's last error message and returns `code`.
int set_error(int code, const char* fmt, ...);

#define MKFG_CUDA_TRY(expr)                                                        \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess)                                                         \
      return ::mkfg::set_error(MKFG_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,      \
                               cudaGetErrorString(_e), __FILE__, __LINE__);        \
  } while (0)

#define MKFG_REQUIRE(cond, ...)                                                    \
  do {                                                                             \
    if (!(cond)) return ::mkfg::set_error(MKFG_ERR_BAD_INPUT, __VA_ARGS__);       \
  } while (0)

// Grow-only device buffer owned by a context.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  int ensure(size_t need) {
    if (need <= bytes) return MKFG_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t want = need + need / 4 + 256;
    MKFG_CUDA_TRY(cudaMalloc(&ptr, want));
    bytes = want;
    return MKFG_OK;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as(size_t byte_off = 0) const {
    return reinterpret_cast<T*>(static_cast<char*>(ptr) + byte_off);
  }
};

// Grow-only pinned host buffer (staging for large host-to-device copies).
struct HostBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  int ensure(size_t need) {
    if (need <= bytes) return MKFG_OK;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t want = need + need / 4 + 256;
    MKFG_CUDA_TRY(cudaHostAlloc(&ptr, want, cudaHostAllocDefault));
    bytes = want;
    return MKFG_OK;
  }
  void release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
  }
};

}  // namespace mkfg

struct mkfg_context {
  int device = -1;
  cudaStream_t stream = nullptr;      // where the context enqueues its work
  cudaStream_t own_stream = nullptr;  // the stream the context created
  float* d_rl = nullptr;  // material grid, 300 x 120
  float* d_xi = nullptr;
  // Scratch for the host-buffer entry points.
  mkfg::DevBuf scratch_in, scratch_hits, scratch_out, scratch_misc;
  // Finding state (device geometry, event buffers) lives in find.cu.
  void* finder = nullptr;
};

namespace mkfg {
// Makes ctx->device current on the calling thread.
int activate(mkfg_context* ctx);
// Releases the finder state (find.cu).
void finder_release(mkfg_context* ctx);
// Validates a host-buffer fit call before anything is copied (fit.cu).
int check_fit_host_args(const mkfg_fit_args* a);
}  // namespace mkfg
