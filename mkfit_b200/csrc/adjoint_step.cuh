// Barrel fit step with alignment / material-scale parameters and its adjoint
// (generated_adjoint.cuh), with the elementary functions and the material
// grid lookup it calls. Host and device: float in the CUDA kernels
// (adjoint.cu), double on the host for checking the derivation.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define AD_FN __host__ __device__ __forceinline__
#else
#define AD_FN inline
#endif

namespace mkfg {
namespace adj {

AD_FN float ad_sqrt(float x) { return sqrtf(x); }
AD_FN double ad_sqrt(double x) { return sqrt(x); }
AD_FN float ad_log(float x) { return logf(x); }
AD_FN double ad_log(double x) { return log(x); }
AD_FN float ad_sin(float x) { return sinf(x); }
AD_FN double ad_sin(double x) { return sin(x); }
AD_FN float ad_cos(float x) { return cosf(x); }
AD_FN double ad_cos(double x) { return cos(x); }
AD_FN float ad_abs(float x) { return fabsf(x); }
AD_FN double ad_abs(double x) { return fabs(x); }
AD_FN float ad_max(float a, float b) { return a >= b ? a : b; }
AD_FN double ad_max(double a, double b) { return a >= b ? a : b; }

// Material grid (300 z bins x 120 r bins over 300 x 120 cm; Config.h:123-127
// of the reference), looked up at the propagated position with the
// reference's float bin arithmetic (MaterialEffects.h:8-11); nothing when
// the propagation failed or no grid is given.
struct MatGrid {
  const float* rl;
  const float* xi;
};

template <typename T>
AD_FN void mat_lookup(const MatGrid& m, T z, T r, bool fail, T& rl, T& xi) {
  rl = T(0);
  xi = T(0);
  if (fail || !m.rl) return;
  const int zb = (int)((fabsf((float)z) * 300.f) / 300.f);
  const int rb = (int)(((float)r * 120.f) / 120.f);
  if (zb >= 0 && zb < 300 && rb >= 0 && rb < 120) {
    rl = T(m.rl[zb * 120 + rb]);
    xi = T(m.xi[zb * 120 + rb]);
  }
}

}  // namespace adj
}  // namespace mkfg

#include "generated_adjoint.cuh"
