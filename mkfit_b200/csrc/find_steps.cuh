// Per-candidate and per-seed steps of one clone-engine layer iteration.
// Each function restates the cited reference routine for one candidate
// (one CUDA thread) or one seed (one warp); the plain form calls them from
// separate kernels, the batched persistent form from one kernel.
#pragma once

#include "find_dev.cuh"

namespace mkfg {

// Layer of region `reg` at layer-plan step `step` (>= 1), or -1.
__device__ __forceinline__ int plan_layer(const FindConfigDev& C, int reg, int step) {
  const int idx = C.pickup[reg] + step;
  return idx < C.plan_len[reg] ? C.plan[reg][idx] : -1;
}

__device__ __forceinline__ void load_state(const CandSoA& B, int slot, float (&par)[6],
                                           float (&err)[21]) {
#pragma unroll
  for (int e = 0; e < 6; ++e) par[e] = B.par[e * B.cap + slot];
#pragma unroll
  for (int e = 0; e < 21; ++e) err[e] = B.err[e * B.cap + slot];
}

__device__ __forceinline__ void store_state(const CandSoA& B, int slot, const float (&par)[6],
                                            const float (&err)[21]) {
#pragma unroll
  for (int e = 0; e < 6; ++e) B.par[e * B.cap + slot] = par[e];
#pragma unroll
  for (int e = 0; e < 21; ++e) B.err[e * B.cap + slot] = err[e];
}

// Appends a hit-on-track node to seed s's arena (CombCandidate::AddHit).
__device__ __forceinline__ int arena_append(const EventDev& E, int s, int index, int layer,
                                            float chi2, int prev) {
  const int pos = atomicAdd(&E.hot_size[s], 1);
  if (pos >= E.hot_cap) {
    atomicOr(E.err_flags, kErrArena);
    return prev;
  }
  const size_t k = (size_t)s * E.hot_cap + pos;
  E.node_hot[k] = hot_pack(index, layer);
  E.node_chi2[k] = chi2;
  E.node_prev[k] = prev;
  return pos;
}

__device__ __forceinline__ int node_hot_of(const EventDev& E, int s, int node) {
  return E.node_hot[(size_t)s * E.hot_cap + node];
}

// Dynamic hit-selection windows (MkFinder::getHitSelDynamicWindows,
// mkFit/MkFinder.cc:166-195).
__device__ __forceinline__ void dynamic_windows(const LayerDev& L, float invpt, float theta,
                                                float& min_dq, float& max_dq, float& min_dphi,
                                                float& max_dphi) {
  float max_invpt = invpt;
  if (invpt > 10.0) max_invpt = 10.0f;
  const float this_dq = L.c_dq_0 * max_invpt + L.c_dq_1 * theta + L.c_dq_2;
  if (L.c_dq_sf * this_dq > 0.f) {
    min_dq = L.c_dq_sf * this_dq;
    max_dq = 2.0f * min_dq;
  }
  const float this_dphi = L.c_dp_0 * max_invpt + L.c_dp_1 * theta + L.c_dp_2;
  if (L.c_dp_sf * this_dphi > min_dphi) {
    min_dphi = L.c_dp_sf * this_dphi;
    max_dphi = 2.0f * min_dphi;
  }
}

// Dynamic chi2 cut (MkFinder::getHitSelDynamicChi2Cut, :203-220).
__device__ __forceinline__ float dynamic_chi2_cut(const LayerDev& L, float chi2_min,
                                                  const float (&par)[6]) {
  const float invpt = par[3];
  const float theta = fabsf(par[5] - kPIOver2);
  float max_invpt = invpt;
  if (invpt > 10.0) max_invpt = 10.0f;
  const float this_c2 = L.c_c2_0 * max_invpt + L.c_c2_1 * theta + L.c_c2_2;
  if (L.c_c2_sf * this_c2 > chi2_min) return L.c_c2_sf * this_c2;
  return chi2_min;
}

__device__ __forceinline__ int q_bin_checked(const LayerDev& L, float q) {
  const int b = (int)((q - L.qmin) * L.fq);
  return min(max(b, 0), L.nq - 1);
}

__device__ __forceinline__ int phi_bin(float phi) {
  constexpr float fphi_fine = 1024 / kTwoPI;
  return ((int)floorf(fphi_fine * (phi + kPI))) >> 2;
}

__device__ __forceinline__ float cdist(float a) { return a > kPI ? kTwoPI - a : a; }

// SelectHitIndices for one candidate (mkFit/MkFinder.cc:227-684) including
// the sensitive-region test (TrackerInfo.h:118-138). Writes up to 16 hit
// indices (index within layer) in bin-scan order; returns XHitSize (-1 when
// outside the layer) and the WSR code.
__device__ __forceinline__ int select_hits(const EventDev& E, const LayerDev& L,
                                           const uint32_t* __restrict__ ev_bins, int hit_base,
                                           const float (&par)[6],
                                           const float (&err)[21], int* xhit, int xstride,
                                           int& wsr) {
  float min_dq = L.min_dq, max_dq = L.max_dq, min_dphi = L.min_dphi, max_dphi = L.max_dphi;
  const float invpt = par[3];
  const float theta = fabsf(par[5] - kPIOver2);
  dynamic_windows(L, invpt, theta, min_dq, max_dq, min_dphi, max_dphi);

  const float x = par[0], y = par[1];
  const float r2 = x * x + y * y;
  const float dphidx = -y / r2, dphidy = x / r2;
  const float dphi2 = dphidx * dphidx * err[0] + dphidy * dphidy * err[2] + 2 * dphidx * dphidy * err[1];
  const float phi = f_atan2(y, x);
  float dphi = fmaxf(3.f * sqrtf(fabsf(dphi2)), min_dphi);
  float q, dq;
  if (L.is_barrel) {
    const float z = par[2];
    dq = fabsf(3.f * sqrtf(err[5]));
    const float edgeCorr = fabsf(0.5f * (L.rout - L.rin) / f_tan(par[5]));
    const float d = sqrtf(dq * dq + edgeCorr * edgeCorr);
    if (z > L.zmax + d || z < L.zmin - d)
      wsr = kWsrOutside;
    else if (z < L.zmax - d && z > L.zmin + d)
      wsr = kWsrInside;
    else
      wsr = kWsrEdge;
    q = z;
  } else {
    const float r = sqrtf(r2);
    dq = 3.f * sqrtf(fabsf(x * x * err[0] + y * y * err[2] + 2 * x * y * err[1]) / r2);
    const float edgeCorr = fabsf(0.5f * (L.zmax - L.zmin) * f_tan(par[5]));
    const float d = sqrtf(dq * dq + edgeCorr * edgeCorr);
    if (r > L.rout + d || r < L.rin - d) {
      wsr = kWsrOutside;
    } else if (r < L.rout - d && r > L.rin + d) {
      wsr = kWsrInside;
      if (L.has_hole) {
        if (r < L.hole_max - d && r > L.hole_min + d)
          wsr = kWsrOutside;
        else if (r < L.hole_max + d && r > L.hole_min - d)
          wsr = kWsrEdge;
      }
    } else {
      wsr = kWsrEdge;
    }
    q = r;
  }
  if (wsr == kWsrOutside) return -1;

  dphi = fminf(fmaxf(fabsf(dphi), min_dphi), max_dphi);
  dq = fminf(fmaxf(dq, min_dq), max_dq);
  const int qb1 = q_bin_checked(L, q - dq);
  const int qb2 = q_bin_checked(L, q + dq) + 1;
  const int pb1 = phi_bin(phi - dphi);
  const int pb2 = phi_bin(phi + dphi) + 1;

  int n = 0;
  const uint32_t* bins = ev_bins + L.bin_offset;
  for (int qi = qb1; qi < qb2; ++qi) {
    for (int pi = pb1; pi < pb2; ++pi) {
      const int pb = pi & 0xff;
      const uint32_t bin = __ldg(bins + qi * 256 + pb);
      const int first = bin & 0xffff, last = bin >> 16;
      for (int hi = first; hi < last; ++hi) {
        if (n >= kMaxXHits) break;
        const int g = hit_base + hi;
        const float ddq = fabsf(q - __ldg(E.sq + g));
        const float ddphi = cdist(fabsf(phi - __ldg(E.sphi + g)));
        if (ddq >= dq) continue;
        if (ddphi >= dphi) continue;
        xhit[n * xstride] = __ldg(E.srank + g);
        ++n;
      }
    }
  }
  return n;
}

// isStripQCompatible (mkFit/MkFinder.cc:837-860).
__device__ __forceinline__ bool strip_q_compatible(bool barrel, const float (&perr)[21],
                                                   const float (&ppar)[6], const float (&mpos)[3],
                                                   const float (&merr)[6]) {
  if (barrel) {
    const float res = fabsf(mpos[2] - ppar[2]);
    const float hitHL = sqrtf(merr[5] * 3.f);
    const float qErr = sqrtf(perr[5]);
    return hitHL + fmaxf(3.f * qErr, 0.5f) > res;
  }
  const float res0 = mpos[0] - ppar[0], res1 = mpos[1] - ppar[1];
  const float hitT2 = merr[0] + merr[2];
  const float hitT2inv = 1.f / hitT2;
  const float proj0 = merr[0] * hitT2inv, proj1 = merr[1] * hitT2inv, proj2 = merr[2] * hitT2inv;
  const float qErr = sqrtf(fabsf(perr[0] * proj0 + 2.f * perr[1] * proj1 + perr[2] * proj2));
  const float resProj = sqrtf(res0 * proj0 * res0 + 2.f * res1 * proj1 * res0 + res1 * proj2 * res1);
  return sqrtf(hitT2 * 3.f) + fmaxf(3.f * qErr, 0.5f) > resProj;
}

// passStripChargePCMfromTrack (mkFit/MkFinder.cc:867-896).
__device__ __forceinline__ bool strip_charge_ok(bool barrel, unsigned pcm, const float (&ppar)[6],
                                                const float (&merr)[6]) {
  constexpr unsigned kMaxPcm = 1620 + (0xfe << 3);
  if (pcm >= kMaxPcm) return true;
  float qSF;
  if (barrel) {
    const float hitT2 = merr[0] + merr[2];
    const float hitT2inv = 1.f / hitT2;
    const float proj0 = merr[0] * hitT2inv, proj1 = merr[1] * hitT2inv, proj2 = merr[2] * hitT2inv;
    const bool detXY_OK = fabsf(proj0 * proj2 - proj1 * proj1) < 0.1f;
    const float cosP = f_cos(ppar[4]);
    const float sinP = f_sin(ppar[4]);
    const float sinT = fabsf(f_sin(ppar[5]));
    qSF = detXY_OK ? sinT * sqrtf(fabsf(1.f + cosP * cosP * proj0 + sinP * sinP * proj2 -
                                        2.f * cosP * sinP * proj1))
                   : 1.f;
  } else {
    qSF = fabsf(f_cos(ppar[5]));
  }
  const float qCorr = pcm * qSF;
  return qCorr > 1620u;
}

// HitMatchPair (mkFit/HitStructures.h:343-393).
struct HitMatchPair {
  int hit[2];
  int module[2];
  float chi2[2];
  __device__ void reset() {
    hit[0] = hit[1] = -1;
    module[0] = module[1] = -1;
    chi2[0] = chi2[1] = 1e9f;
  }
  __device__ void consider(int h, int m, float c2) {
    if (m == module[0]) {
      if (c2 < chi2[0]) { chi2[0] = c2; hit[0] = h; }
    } else if (m == module[1]) {
      if (c2 < chi2[1]) { chi2[1] = c2; hit[1] = h; }
    } else {
      if (chi2[0] > chi2[1]) {
        if (c2 < chi2[0]) { hit[0] = h; module[0] = m; chi2[0] = c2; }
      } else {
        if (c2 < chi2[1]) { hit[1] = h; module[1] = m; chi2[1] = c2; }
      }
    }
  }
  // Returns 0/1 for the chosen match, or -1.
  __device__ int find(int h, int m) const {
    (void)h;
    if (m == module[0]) return hit[1] >= 0 ? 1 : -1;
    if (m == module[1]) return hit[0] >= 0 ? 0 : -1;
    if (chi2[0] <= chi2[1]) return hit[0] >= 0 ? 0 : -1;
    return hit[1] >= 0 ? 1 : -1;
  }
};

}  // namespace mkfg
