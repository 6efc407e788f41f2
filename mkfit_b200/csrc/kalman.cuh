// Device-side Kalman-filter math for one track per CUDA thread.
//
// Semantics follow the reference CPU Matriplex path (trackreco/mkFit); each
// function names the reference routine it restates. All state lives in
// registers: parameters (x, y, z, 1/pT, phi, theta) in CCS coordinates, the
// 6x6 covariance as 21 floats (packed lower triangle, same element order as
// the reference's MatriplexSym), 6x6 Jacobians as 36-float arrays whose
// known-zero entries are folded away by the generated products.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include "generated_ops.cuh"

namespace mkfg {

// Physics / math constants (Config.h:77-88, 240-245 of the reference).
constexpr float kPI = 3.14159265358979323846f;
constexpr float kTwoPI = 6.28318530717958647692f;
constexpr float kPIOver2 = kPI / 2.0f;
constexpr float kInvPI = 1.0f / kPI;
constexpr float kSol = 0.299792458f;
constexpr float kBfield = 3.8112f;
constexpr float kMagC1 = 3.8114f;
constexpr float kMagB0 = -3.94991e-06f;
constexpr float kMagB1 = 7.53701e-06f;
constexpr float kMagA = 2.43878e-11f;
constexpr int kNiter = 5;  // Config::Niter

// Material grid (Config.h:123-127): 300 z bins x 120 r bins over 300 x 120 cm.
constexpr int kMatNZ = 300;
constexpr int kMatNR = 120;
constexpr float kMatRangeZ = 300.f;
constexpr float kMatRangeR = 120.f;

// Propagation flag bits (Config.h:17-23).
constexpr unsigned kPfParamB = 0x1;
constexpr unsigned kPfMaterial = 0x2;

struct Material {
  const float* rl;  // [kMatNZ][kMatNR] radiation lengths
  const float* xi;  // [kMatNZ][kMatNR] energy-loss xi
};

__device__ __forceinline__ float sqr(float x) { return x * x; }

// Packed lower-triangle index of symmetric element (i, j).
__host__ __device__ constexpr int sidx(int i, int j) {
  return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

// Elementary functions. The reference calls the host C library's float
// functions (sinf, cosf, logf, atan2f), which are correctly rounded for
// nearly all arguments. With MKFG_LIBM_EXACT (default) the device evaluates
// them in double precision and rounds once to float, which reproduces those
// results except in rare double-rounding cases; without it the CUDA float
// versions (<= 2 ulp) are used.
#ifndef MKFG_LIBM_EXACT
#define MKFG_LIBM_EXACT 1
#endif
__device__ __forceinline__ void f_sincos(float x, float* s, float* c) {
#if MKFG_LIBM_EXACT
  double sd, cd;
  sincos((double)x, &sd, &cd);
  *s = (float)sd;
  *c = (float)cd;
#else
  sincosf(x, s, c);
#endif
}
__device__ __forceinline__ float f_sin(float x) {
#if MKFG_LIBM_EXACT
  return (float)sin((double)x);
#else
  return sinf(x);
#endif
}
__device__ __forceinline__ float f_cos(float x) {
#if MKFG_LIBM_EXACT
  return (float)cos((double)x);
#else
  return cosf(x);
#endif
}
__device__ __forceinline__ float f_log(float x) {
#if MKFG_LIBM_EXACT
  return (float)log((double)x);
#else
  return logf(x);
#endif
}
__device__ __forceinline__ float f_atan2(float y, float x) {
#if MKFG_LIBM_EXACT
  return (float)atan2((double)y, (double)x);
#else
  return atan2f(y, x);
#endif
}

// sqrt(x*x + y*y) in float, as the reference's hipo() (Matrix.h:38).
__device__ __forceinline__ float hipo(float x, float y) { return sqrtf(x * x + y * y); }

// std::hypot(float, float) as evaluated by glibc: the sum of squares is
// formed in double precision and the root is rounded once to float.
__device__ __forceinline__ float hypot_f(float x, float y) {
  const double dx = x, dy = y;
  return (float)sqrt(dx * dx + dy * dy);
}

// Magnetic field model (Config.h:434-437).
__device__ __forceinline__ float bfield_zr(float z, float r) {
  return (kMagB0 * z * z + kMagB1 * z + kMagC1) * (kMagA * r * r + 1.f);
}

// Fourth-order sin/cos polynomial of the reference (Matrix.h:48-56).
__device__ __forceinline__ void sincos4(float x, float& s, float& c) {
  const float x2 = x * x;
  c = 1.f - 0.5f * x2 + 0.04166667f * x2 * x2;
  s = x - 0.16666667f * x * x2;
}

// phi into [-pi, pi) (squashPhiMPlex, mkFit/PropagationMPlex.h:8-15).
__device__ __forceinline__ float squash_phi(float phi) {
  if (phi >= kPI) phi -= kTwoPI;
  if (phi < -kPI) phi += kTwoPI;
  return phi;
}

//------------------------------------------------------------------------------
// Helix to radius r: 5 fixed iterations with arc-length derivative tracking.
// Restates helixAtRFromIterativeCCS_impl (mkFit/PropagationMPlex.icc:5-246).
// Returns the fail flag (1 when the step would approach the apex).
//------------------------------------------------------------------------------
__device__ __forceinline__ int helix_to_r(const float (&in)[6], int chg, float r, bool param_b,
                                          float (&out)[6], float (&J)[36]) {
#pragma unroll
  for (int i = 0; i < 36; ++i) J[i] = 0.f;
  int fail = 0;

  float r0 = hipo(in[0], in[1]);
  const float bf = param_b ? bfield_zr(in[2], r0) : kBfield;
  const float k = float(chg) * 100.f / (-kSol * bf);

  const float xin = in[0], yin = in[1], ipt = in[3], phiin = in[4], theta = in[5];
  const float kinv = 1.f / k;
  const float pt = 1.f / ipt;

  float D = 0.f, cosa = 0.f, sina = 0.f, cosah = 0.f, sinah = 0.f, id = 0.f;
  float cosPorT, sinPorT;
  f_sincos(phiin, &sinPorT, &cosPorT);
  float pxin = cosPorT * pt;
  float pyin = sinPorT * pt;

  float dDdx = r0 > 0.f ? -xin / r0 : 0.f;
  float dDdy = r0 > 0.f ? -yin / r0 : 0.f;
  float dDdipt = 0.f;
  float dDdphi = 0.f;

  float ox = in[0], oy = in[1];
#pragma unroll
  for (int it = 0; it < kNiter; ++it) {
    r0 = hipo(ox, oy);
    const float oodotp = r0 * pt / (pxin * ox + pyin * oy);
    if (oodotp > 5.0f || oodotp < 0) {
      id = 0.0f;
      fail = 1;
    } else {
      id = (r - r0) * oodotp;
    }
    D += id;

    sincos4(id * ipt * kinv * 0.5f, sinah, cosah);
    cosa = 1.f - 2.f * sinah * sinah;
    sina = 2.f * sinah * cosah;

    if (it + 1 != kNiter) {
      const float x = ox, y = oy;
      const float oor0 = (r0 > 0.f && fabsf(r - r0) < 0.0001f) ? 1.f / r0 : 0.f;
      const float dadipt = id * kinv;
      const float dadx = -x * ipt * kinv * oor0;
      const float dady = -y * ipt * kinv * oor0;
      const float pxca = pxin * cosa;
      const float pxsa = pxin * sina;
      const float pyca = pyin * cosa;
      const float pysa = pyin * sina;
      float tmp = k * dadx;
      dDdx -= (x * (1.f + tmp * (pxca - pysa)) + y * tmp * (pyca + pxsa)) * oor0;
      tmp = k * dady;
      dDdy -= (x * tmp * (pxca - pysa) + y * (1.f + tmp * (pyca + pxsa))) * oor0;
      tmp = dadipt * ipt;
      dDdipt -= k * (x * (pxca * tmp - pysa * tmp - pyca - pxsa + pyin) +
                     y * (pyca * tmp + pxsa * tmp - pysa + pxca - pxin)) * pt * oor0;
      dDdphi += k * (x * (pysa - pxin + pxca) - y * (pxsa - pyin + pyca)) * oor0;
    }

    ox = ox + 2.f * k * sinah * (pxin * cosah - pyin * sinah);
    oy = oy + 2.f * k * sinah * (pyin * cosah + pxin * sinah);
    const float pxinold = pxin;
    pxin = pxin * cosa - pyin * sina;
    pyin = pyin * cosa + pxinold * sina;
  }

  const float alpha = D * ipt * kinv;
  const float dadx = dDdx * ipt * kinv;
  const float dady = dDdy * ipt * kinv;
  const float dadipt = (ipt * dDdipt + D) * kinv;
  const float dadphi = dDdphi * ipt * kinv;

  sincos4(alpha, sina, cosa);

  J[0 * 6 + 0] = 1.f + k * dadx * (cosPorT * cosa - sinPorT * sina) * pt;
  J[0 * 6 + 1] = k * dady * (cosPorT * cosa - sinPorT * sina) * pt;
  J[0 * 6 + 3] = k * (cosPorT * (ipt * dadipt * cosa - sina) + sinPorT * ((1.f - cosa) - ipt * dadipt * sina)) * pt * pt;
  J[0 * 6 + 4] = k * (cosPorT * dadphi * cosa - sinPorT * dadphi * sina - sinPorT * sina + cosPorT * cosa - cosPorT) * pt;

  J[1 * 6 + 0] = k * dadx * (sinPorT * cosa + cosPorT * sina) * pt;
  J[1 * 6 + 1] = 1.f + k * dady * (sinPorT * cosa + cosPorT * sina) * pt;
  J[1 * 6 + 3] = k * (sinPorT * (ipt * dadipt * cosa - sina) + cosPorT * (ipt * dadipt * sina - (1.f - cosa))) * pt * pt;
  J[1 * 6 + 4] = k * (sinPorT * dadphi * cosa + cosPorT * dadphi * sina + sinPorT * cosa + cosPorT * sina - sinPorT) * pt;

  float cosT, sinT;
  f_sincos(theta, &sinT, &cosT);
  const float isinT = 1.f / sinT;

  out[0] = ox;
  out[1] = oy;
  out[2] = in[2] + k * alpha * cosT * pt * isinT;
  out[3] = ipt;
  out[4] = in[4] + alpha;
  out[5] = theta;

  J[2 * 6 + 0] = k * cosT * dadx * pt * isinT;
  J[2 * 6 + 1] = k * cosT * dady * pt * isinT;
  J[2 * 6 + 2] = 1.f;
  J[2 * 6 + 3] = k * cosT * (ipt * dadipt - alpha) * pt * pt * isinT;
  J[2 * 6 + 4] = k * dadphi * cosT * pt * isinT;
  J[2 * 6 + 5] = -k * alpha * pt * isinT * isinT;

  J[3 * 6 + 3] = 1.f;

  J[4 * 6 + 0] = dadx;
  J[4 * 6 + 1] = dady;
  J[4 * 6 + 3] = dadipt;
  J[4 * 6 + 4] = 1.f + dadphi;

  J[5 * 6 + 5] = 1.f;
  return fail;
}

//------------------------------------------------------------------------------
// Helix to plane z (endcap). Restates helixAtZ (mkFit/PropagationMPlex.cc:604-712).
//------------------------------------------------------------------------------
__device__ __forceinline__ void helix_to_z(const float (&in)[6], int chg, float zout, bool param_b,
                                           float (&out)[6], float (&J)[36]) {
#pragma unroll
  for (int i = 0; i < 36; ++i) J[i] = 0.f;
  J[0 * 6 + 0] = 1.f;
  J[1 * 6 + 1] = 1.f;
  J[3 * 6 + 3] = 1.f;
  J[4 * 6 + 4] = 1.f;
  J[5 * 6 + 5] = 1.f;

  const float zin = in[2], ipt = in[3], phiin = in[4], theta = in[5];
  const float bf = param_b ? bfield_zr(zin, hipo(in[0], in[1])) : kBfield;
  const float k = float(chg) * 100.f / (-kSol * bf);
  const float kinv = 1.f / k;
  const float pt = 1.f / ipt;

  float cosP, sinP, cosT, sinT;
  f_sincos(phiin, &sinP, &cosP);
  f_sincos(theta, &sinT, &cosT);
  const float tanT = sinT / cosT;
  const float icos2T = 1.f / (cosT * cosT);
  const float pxin = cosP * pt;
  const float pyin = sinP * pt;

  const float deltaZ = zout - zin;
  const float alpha = deltaZ * tanT * ipt * kinv;

  float sinah, cosah;
  sincos4(alpha * 0.5f, sinah, cosah);
  const float cosa = 1.f - 2.f * sinah * sinah;
  const float sina = 2.f * sinah * cosah;

  out[0] = in[0] + 2.f * k * sinah * (pxin * cosah - pyin * sinah);
  out[1] = in[1] + 2.f * k * sinah * (pyin * cosah + pxin * sinah);
  out[2] = zout;
  out[3] = in[3];
  out[4] = phiin + alpha;
  out[5] = in[5];

  const float pxcaMpysa = pxin * cosa - pyin * sina;
  J[0 * 6 + 2] = -tanT * ipt * pxcaMpysa;
  J[0 * 6 + 3] = k * pt * pt * (cosP * (alpha * cosa - sina) + sinP * 2.f * sinah * (sinah - alpha * cosah));
  J[0 * 6 + 4] = -2 * k * pt * sinah * (sinP * cosah + cosP * sinah);
  J[0 * 6 + 5] = deltaZ * ipt * pxcaMpysa * icos2T;

  const float pycaPpxsa = pyin * cosa + pxin * sina;
  J[1 * 6 + 2] = -tanT * ipt * pycaPpxsa;
  J[1 * 6 + 3] = k * pt * pt * (sinP * (alpha * cosa - sina) - cosP * 2.f * sinah * (sinah - alpha * cosah));
  J[1 * 6 + 4] = 2 * k * pt * sinah * (cosP * cosah - sinP * sinah);
  J[1 * 6 + 5] = deltaZ * ipt * pycaPpxsa * icos2T;

  J[4 * 6 + 2] = -ipt * tanT * kinv;
  J[4 * 6 + 3] = tanT * deltaZ * kinv;
  J[4 * 6 + 5] = ipt * deltaZ * kinv * icos2T;
}

//------------------------------------------------------------------------------
// Multiple scattering + energy loss. Restates applyMaterialEffects
// (mkFit/PropagationMPlex.cc:716-767): updates C[3][3], C[4][4], C[5][5] of
// the (pre-similarity) covariance and 1/pT of the propagated parameters.
//------------------------------------------------------------------------------
__device__ __forceinline__ void material_effects(float radL, float xi, float prop_sign, bool is_barrel,
                                                 float (&C)[21], float (&par)[6]) {
  if (radL < 1e-13f) return;
  const float theta = par[5];
  const float pt = 1.f / par[3];
  const float p = pt / f_sin(theta);
  const float p2 = p * p;
  constexpr float mpi = 0.140f;
  constexpr float mpi2 = mpi * mpi;
  const float beta2 = p2 / (p2 + mpi2);
  const float beta = sqrtf(beta2);
  const float invCos = is_barrel ? p / pt : 1.f / fabsf(f_cos(theta));
  radL = radL * invCos;
  if (radL < 1e-13f) return;
  const float thetaMSC = 0.0136f * (1.f + 0.038f * f_log(radL)) / (beta * p);
  const float thetaMSC2 = thetaMSC * thetaMSC * radL;
  C[14] += thetaMSC2;  // (4,4)
  C[20] += thetaMSC2;  // (5,5)
  const float gamma2 = (p2 + mpi2) / mpi2;
  const float gamma = sqrtf(gamma2);
  constexpr float me = 0.0005f;
  const float wmax = 2.f * me * beta2 * gamma2 / (1.f + 2.f * gamma * me / mpi + me * me / (mpi * mpi));
  constexpr float I = (float)(16.0e-9 * 10.75);
  const float deltahalf = f_log(28.816e-9f * sqrtf(2.33f * 0.498f) / I) + f_log(beta * gamma) - 0.5f;
  const float dEdx = beta < 1.f
                         ? (2.f * (xi * invCos * (0.5f * f_log(2.f * me * beta2 * gamma2 * wmax / (I * I)) - beta2 - deltahalf) / beta2))
                         : 0.f;
  const float dP = prop_sign * dEdx / beta;
  par[3] = p / (fmaxf(p + dP, 0.001f) * pt);
  C[9] += dP * dP / (p2 * pt * pt);  // (3,3)
}

// Material grid lookup with the reference's bin arithmetic and range guard
// (MaterialEffects.h:8-11, mkFit/PropagationMPlex.cc:455-460).
__device__ __forceinline__ void material_lookup(const Material& m, float z, float r, float& rl, float& xi) {
  const int zb = (int)((fabsf(z) * kMatNZ) / kMatRangeZ);
  const int rb = (int)((r * kMatNR) / kMatRangeR);
  if (zb >= 0 && zb < kMatNZ && rb >= 0 && rb < kMatNR) {
    rl = __ldg(m.rl + zb * kMatNR + rb);
    xi = __ldg(m.xi + zb * kMatNR + rb);
  } else {
    rl = 0.f;
    xi = 0.f;
  }
}

//------------------------------------------------------------------------------
// Full propagation to radius r with material and covariance transport.
// Restates propagateHelixToRMPlex (mkFit/PropagationMPlex.cc:408-505).
// On failure the output is reset to the input (fix-up at :497-504).
//------------------------------------------------------------------------------
__device__ __forceinline__ int propagate_to_r(const float (&par)[6], const float (&err)[21], int chg,
                                              float r, unsigned pflags, const Material& mat,
                                              bool no_mat_eff, float (&opar)[6], float (&oerr)[21]) {
  float J[36];
  float p[6];
  const int fail = helix_to_r(par, chg, r, pflags & kPfParamB, p, J);
  float C[21];
#pragma unroll
  for (int i = 0; i < 21; ++i) C[i] = err[i];
  if (pflags & kPfMaterial) {
    float rl = 0.f, xi = 0.f;
    if (!(fail || no_mat_eff)) material_lookup(mat, p[2], r, rl, xi);
    const float r0 = hipo(par[0], par[1]);
    const float sign = (r > r0 ? 1.f : -1.f);
    material_effects(rl, xi, sign, true, C, p);
  }
  p[4] = squash_phi(p[4]);
  float Co[21];
  similarity_barrel(J, C, Co);
  if (fail) {
#pragma unroll
    for (int i = 0; i < 6; ++i) opar[i] = par[i];
#pragma unroll
    for (int i = 0; i < 21; ++i) oerr[i] = err[i];
  } else {
#pragma unroll
    for (int i = 0; i < 6; ++i) opar[i] = p[i];
#pragma unroll
    for (int i = 0; i < 21; ++i) oerr[i] = Co[i];
  }
  return fail;
}

// Propagation to plane z. Restates propagateHelixToZMPlex
// (mkFit/PropagationMPlex.cc:510-601); this path has no fail flag.
__device__ __forceinline__ void propagate_to_z(const float (&par)[6], const float (&err)[21], int chg,
                                               float z, unsigned pflags, const Material& mat,
                                               bool no_mat_eff, float (&opar)[6], float (&oerr)[21]) {
  float J[36];
  float p[6];
  helix_to_z(par, chg, z, pflags & kPfParamB, p, J);
  float C[21];
#pragma unroll
  for (int i = 0; i < 21; ++i) C[i] = err[i];
  if (pflags & kPfMaterial) {
    float rl = 0.f, xi = 0.f;
    if (!no_mat_eff) material_lookup(mat, z, hypot_f(p[0], p[1]), rl, xi);
    const float sign = (fabsf(z) > fabsf(par[2]) ? 1.f : -1.f);
    material_effects(rl, xi, sign, false, C, p);
  }
  p[4] = squash_phi(p[4]);
  similarity_endcap(J, C, oerr);
#pragma unroll
  for (int i = 0; i < 6; ++i) opar[i] = p[i];
}

//------------------------------------------------------------------------------
// 2x2 symmetric inverse with the determinant formed in double precision
// (CramerInverterSym<T,2,N>, Matriplex/MatriplexSym.h:422-445).
//------------------------------------------------------------------------------
__device__ __forceinline__ void invert_sym2(float& a0, float& a1, float& a2) {
  const double det = (double)a0 * a2 - (double)a1 * a1;
  const float s = (float)(1.0 / det);
  const float tmp = s * a2;
  a1 *= -s;
  a2 = s * a0;
  a0 = tmp;
}

//------------------------------------------------------------------------------
// Barrel Kalman operation: residual rotated onto the plane tangent to the
// cylinder, chi2 and/or update. Restates kalmanOperation
// (mkFit/KalmanUtilsMPlex.cc:548-681). do_update: write (opar, oerr).
//------------------------------------------------------------------------------
template <bool kChi2, bool kUpdate>
__device__ __forceinline__ float kalman_barrel(const float (&par)[6], const float (&err)[21],
                                               const float (&mpos)[3], const float (&merr)[6],
                                               float (&opar)[6], float (&oerr)[21]) {
  const float r = hypot_f(mpos[0], mpos[1]);
  const float r00 = -(mpos[1] + par[1]) / (2 * r);
  const float r01 = (mpos[0] + par[0]) / (2 * r);

  const float res0 = mpos[0] - par[0], res1 = mpos[1] - par[1], res2 = mpos[2] - par[2];
  // Covariance sum in global position coordinates (upper-left 3x3).
  const float g0 = err[0] + merr[0], g1 = err[1] + merr[1], g2 = err[2] + merr[2];
  const float g3 = err[3] + merr[3], g4 = err[4] + merr[4], g5 = err[5] + merr[5];

  // Local residual and its covariance (ProjectResErr / ProjectResErrTransp).
  const float loc0 = r00 * res0 + r01 * res1;
  const float loc1 = res2;
  const float t0 = r00 * g0 + r01 * g1;
  const float t1 = r00 * g1 + r01 * g2;
  const float t2 = r00 * g3 + r01 * g4;
  float s0 = t0 * r00 + t1 * r01;
  float s1 = g3 * r00 + g4 * r01;
  float s2 = g5;
  (void)t2;
  invert_sym2(s0, s1, s2);

  float chi2 = 0.f;
  if (kChi2) chi2 = s0 * loc0 * loc0 + s2 * loc1 * loc1 + 2 * (s1 * loc1 * loc0);

  if (kUpdate) {
    // H^T G (KalmanHTG): 3x2 live block.
    const float h00 = r00 * s0, h01 = r00 * s1;
    const float h10 = r01 * s0, h11 = r01 * s1;
    const float h20 = s1, h21 = s2;
    // Gain K = C[:, 0:3] * HTG (KalmanGain): 6x2.
    float K[12];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const float ci0 = err[sidx(i, 0)], ci1 = err[sidx(i, 1)], ci2 = err[sidx(i, 2)];
      K[2 * i + 0] = ci0 * h00 + ci1 * h10 + ci2 * h20;
      K[2 * i + 1] = ci0 * h01 + ci1 * h11 + ci2 * h21;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) opar[i] = par[i] + K[2 * i] * loc0 + K[2 * i + 1] * loc1;
    opar[4] = squash_phi(opar[4]);
    // KH (KHMult): rows (K0*r00, K0*r01, K1, 0, 0, 0).
    float KH[36];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      KH[i * 6 + 0] = K[2 * i] * r00;
      KH[i * 6 + 1] = K[2 * i] * r01;
      KH[i * 6 + 2] = K[2 * i + 1];
      KH[i * 6 + 3] = 0.f;
      KH[i * 6 + 4] = 0.f;
      KH[i * 6 + 5] = 0.f;
    }
    float KHC[21];
    khc_barrel(KH, err, KHC);
#pragma unroll
    for (int i = 0; i < 21; ++i) oerr[i] = err[i] - KHC[i];
  }
  return chi2;
}

//------------------------------------------------------------------------------
// Endcap Kalman operation: xy residual, 6x2 gain. Restates
// kalmanOperationEndcap (mkFit/KalmanUtilsMPlex.cc:774-888).
//------------------------------------------------------------------------------
template <bool kChi2, bool kUpdate>
__device__ __forceinline__ float kalman_endcap(const float (&par)[6], const float (&err)[21],
                                               const float (&mpos)[3], const float (&merr)[6],
                                               float (&opar)[6], float (&oerr)[21]) {
  const float res0 = mpos[0] - par[0], res1 = mpos[1] - par[1];
  float s0 = err[0] + merr[0], s1 = err[1] + merr[1], s2 = err[2] + merr[2];
  invert_sym2(s0, s1, s2);
  float chi2 = 0.f;
  if (kChi2) chi2 = s0 * res0 * res0 + s2 * res1 * res1 + 2 * (s1 * res1 * res0);
  if (kUpdate) {
    // K = C[:, 0:2] * S^-1 (KalmanGain62).
    float K[12];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const float ci0 = err[sidx(i, 0)], ci1 = err[sidx(i, 1)];
      K[2 * i + 0] = ci0 * s0 + ci1 * s1;
      K[2 * i + 1] = ci0 * s1 + ci1 * s2;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) opar[i] = par[i] + K[2 * i] * res0 + K[2 * i + 1] * res1;
    opar[4] = squash_phi(opar[4]);
    float KHC[21];
    khc_endcap(K, err, KHC);
#pragma unroll
    for (int i = 0; i < 21; ++i) oerr[i] = err[i] - KHC[i];
  }
  return chi2;
}

}  // namespace mkfg
