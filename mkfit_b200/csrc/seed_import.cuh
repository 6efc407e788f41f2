// Seed import on the device: MkBuilder::import_seeds with the CMS-2017
// partition (partitionSeeds1, Geoms/CMS-2017.cc:436-549; mkFit/
// MkBuilder.cc:214-275) and the initial candidates of
// CombCandidate::ImportSeed (mkFit/HitStructures.cc:483-509), for a batch
// of events whose hits are already on the device.
//
// The same results as the host path of the upload (find_host.cc
// partition_seeds_cms2017 and the staging loop of upload_batch): every
// float operation is written out with round-to-nearest intrinsics in the
// host code's order (no contraction into FMAs), and the float library
// functions are the host-rounded versions of kalman.cuh / find_dev.cuh.
#pragma once

#include <cstdint>

#include "find_dev.cuh"
#include "find_host.h"

namespace mkfg {

constexpr int kSeedSortMax = 16384;  // seeds per event the device sort takes
constexpr int kSeedSortBlock = 1024;

// Seeds of a batch as the caller gave them, events back to back (raw
// index = first seed of the event + input index).
struct RawSeeds {
  const float* par;       // [6][S]
  const float* err;       // [21][S]
  const int* chg;
  const int* nhits;
  const int* hit_layer;   // [S][MKFG_MAX_SEED_HITS]
  const int* hit_index;   // [S][MKFG_MAX_SEED_HITS]
  const int* seed_off;    // [n_events + 1]
  int n_events;
  int n;                  // S
};

// TrackBase kinematics and the helix steps partitionSeeds1 uses
// (Track.h:105-130, Track.cc:53-100), as find_host.cc SeedTrack.
struct DevSeedTrack {
  float x, y, z, ipt;
  int chg;
  float pt, px, py, pz;
  __device__ DevSeedTrack(float x_, float y_, float z_, float ipt_, float phi, float theta, int c)
      : x(x_), y(y_), z(z_), ipt(ipt_), chg(c) {
    pt = fabsf(__fdiv_rn(1.f, ipt));
    px = __fmul_rn(pt, f_cos(phi));
    py = __fmul_rn(pt, f_sin(phi));
    pz = __fdiv_rn(pt, f_tan(theta));
  }
  __device__ float max_reach_radius() const {
    const float k = __fdiv_rn(chg < 0 ? 100.0f : -100.0f, __fmul_rn(0.299792458f, 3.8112f));
    const float abs_ooc_half = fabsf(__fmul_rn(k, pt));
    const float xc = __fsub_rn(x, __fmul_rn(k, py));
    const float yc = __fadd_rn(y, __fmul_rn(k, px));
    return __fadd_rn(hypot_f(xc, yc), abs_ooc_half);
  }
  __device__ float z_at_r(float R) const {
    float xc = x, yc = y, pxc = px, pyc = py;
    const float kinv = __fmul_rn(__fmul_rn(chg < 0 ? 0.01f : -0.01f, 0.299792458f), 3.8112f);
    const float k = __fdiv_rn(1.0f, kinv);
    const float c = __fmul_rn(__fmul_rn(0.5f, kinv), ipt);
    const float ooc = __fdiv_rn(1.0f, c);
    const float lambda = __fmul_rn(pz, ipt);
    float D = 0;
    for (int i = 0; i < 5; ++i) {
      const float r0 = hypot_f(xc, yc);
      const float td = __fmul_rn(__fsub_rn(R, r0), c);
      const float id = __fmul_rn(__fmul_rn(ooc, td),
                                 __fadd_rn(1.0f, __fmul_rn(__fmul_rn(0.16666666f, td), td)));
      D = __fadd_rn(D, id);
      const float arg = __fmul_rn(__fmul_rn(id, ipt), kinv);
      const float cosa = f_cos(arg);
      const float sina = f_sin(arg);
      const float omc = __fsub_rn(1.0f, cosa);
      xc = __fadd_rn(xc, __fmul_rn(k, __fsub_rn(__fmul_rn(pxc, sina), __fmul_rn(pyc, omc))));
      yc = __fadd_rn(yc, __fmul_rn(k, __fadd_rn(__fmul_rn(pyc, sina), __fmul_rn(pxc, omc))));
      const float pxo = pxc;
      pxc = __fsub_rn(__fmul_rn(pxc, cosa), __fmul_rn(pyc, sina));
      pyc = __fadd_rn(__fmul_rn(pyc, cosa), __fmul_rn(pxo, sina));
    }
    return __fadd_rn(z, __fmul_rn(lambda, D));
  }
};

// Region of one seed (partitionSeeds1's decision tree, with the tests of
// each pair short-circuited as on the host).
__device__ __forceinline__ int seed_region(const DevSeedTrack& S, const RegionCuts& r) {
  const float maxR = S.max_reach_radius();
  auto barrel_pos = [&](float rin, float zmax) { return maxR > rin && S.z_at_r(rin) < zmax; };
  auto barrel_neg = [&](float rin, float zmin) { return maxR > rin && S.z_at_r(rin) > zmin; };
  auto endcap_pos = [&](float rout, float rin, float zmin) {
    return maxR > rout ? S.z_at_r(rout) > zmin : (maxR > rin && S.z_at_r(maxR) > zmin);
  };
  auto endcap_neg = [&](float rout, float rin, float zmax) {
    return maxR > rout ? S.z_at_r(rout) < zmax : (maxR > rin && S.z_at_r(maxR) < zmax);
  };
  if (S.pz > 0) {
    if (!(barrel_pos(r.tib1_rin, r.tib1_zmax) || barrel_pos(r.tob1_rin, r.tob1_zmax))) return 4;
    const bool in_endcap = endcap_pos(r.tidp_rout, r.tidp_rin, r.tidp1_zmin) ||
                           endcap_pos(r.tecp_rout, r.tecp_rin, r.tecp1_zmin);
    return in_endcap ? 3 : 2;
  }
  if (!(barrel_neg(r.tib1_rin, r.tib1_zmin) || barrel_neg(r.tob1_rin, r.tob1_zmin))) return 0;
  const bool in_endcap = endcap_neg(r.tidn_rout, r.tidn_rin, r.tidn1_zmax) ||
                         endcap_neg(r.tecn_rout, r.tecn_rin, r.tecn1_zmax);
  return in_endcap ? 1 : 2;
}

// Kernel 1: region and sort key of every seed (raw order): key = 7 (region
// - 2) + eta of the seed's last hit (Hit::eta).
__global__ void k_seed_keys(const RawSeeds R, const EventDev E, const RegionCuts cuts,
                            int* __restrict__ region, float* __restrict__ key,
                            int* __restrict__ seed_event) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R.n) return;
  int e_lo = 0, e_hi = R.n_events - 1;  // the event with seed_off[e] <= i < seed_off[e + 1]
  while (e_lo < e_hi) {
    const int mid = (e_lo + e_hi + 1) >> 1;
    if (R.seed_off[mid] <= i) e_lo = mid;
    else e_hi = mid - 1;
  }
  const int e = e_lo;
  seed_event[i] = e;
  const DevSeedTrack S(R.par[i], R.par[R.n + i], R.par[2 * R.n + i], R.par[3 * R.n + i],
                       R.par[4 * R.n + i], R.par[5 * R.n + i], R.chg[i]);
  const int last = R.nhits[i] - 1;
  const int hl = R.hit_layer[i * MKFG_MAX_SEED_HITS + last];
  const int hi = R.hit_index[i * MKFG_MAX_SEED_HITS + last];
  const int h = E.layer_begin[e * E.lb_stride + hl] + hi;
  const float hx = E.hpos[h], hy = E.hpos[E.hstride + h], hz = E.hpos[2 * E.hstride + h];
  const float theta = f_atan2(__fsqrt_rn(__fadd_rn(__fmul_rn(hx, hx), __fmul_rn(hy, hy))), hz);
  const float eta = __fmul_rn(-1.0f, f_log(f_tan(__fdiv_rn(theta, 2.0f))));
  const int reg = seed_region(S, cuts);
  region[i] = reg;
  key[i] = __fadd_rn(__fmul_rn(7.0f, (float)(reg - 2)), eta);
}

// Order-preserving integer image of a float key (-0 taken as +0; NaN
// above every number).
__device__ __forceinline__ uint32_t float_order_bits(float v) {
  v = __fadd_rn(v, 0.f);
  if (v != v) return 0xffffffffu;
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Kernel 2: per event (one block), the seeds sorted by key with ties in
// input order (std::stable_sort in import_seeds): a bitonic sort of
// (key, input index) pairs in shared memory. order[first + k] = raw index
// of the event's k-th seed.
__global__ void __launch_bounds__(kSeedSortBlock) k_seed_sort(const RawSeeds R,
                                                             const float* __restrict__ key,
                                                             int* __restrict__ order) {
  extern __shared__ unsigned long long s_pair[];
  const int e = blockIdx.x;
  const int first = R.seed_off[e], n = R.seed_off[e + 1] - first;
  if (n <= 0) return;
  int np = 1;
  while (np < n) np <<= 1;
  for (int t = threadIdx.x; t < np; t += blockDim.x)
    s_pair[t] = t < n ? ((unsigned long long)float_order_bits(key[first + t]) << 32) | (uint32_t)t
                      : ~0ull;
  __syncthreads();
  for (int k = 2; k <= np; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < np; t += blockDim.x) {
        const int u = t ^ j;
        if (u > t) {
          const unsigned long long a = s_pair[t], b = s_pair[u];
          const bool up = (t & k) == 0;
          if ((a > b) == up) {
            s_pair[t] = b;
            s_pair[u] = a;
          }
        }
      }
      __syncthreads();
    }
  for (int t = threadIdx.x; t < n; t += blockDim.x)
    order[first + t] = first + (int)(uint32_t)(s_pair[t] & 0xffffffffull);
}

// Kernel 3: the initial candidate of every seed in sorted order (the
// staging loop of the host path): state, hit counters from the seed's
// hits, the seed's hit-on-track nodes, getScoreCand, and
// MkBuilder::seed_post_cleaning's drop of a seed with a negative
// diagonal or a non-finite covariance element (nfound = -1).
__global__ void k_seed_import(const RawSeeds R, const int* __restrict__ order,
                              const int* __restrict__ region, const int* __restrict__ raw_event,
                              EventDev E, int* __restrict__ seed_hot) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= R.n) return;
  const int i = order[s];
  const CandSoA& B = E.init;
  E.seed_label[s] = i;
  E.seed_event[s] = raw_event[i];
  E.region[s] = region[i];
  const int nhs = R.nhits[i];
  E.pickup_layer[s] = R.hit_layer[i * MKFG_MAX_SEED_HITS + nhs - 1];
  float par3 = 0.f;
  for (int c = 0; c < 6; ++c) {
    const float v = R.par[c * R.n + i];
    B.par[c * B.cap + s] = v;
    if (c == 3) par3 = v;
  }
  bool silly = false;
  for (int a = 0, c = 0; a < 6; ++a)
    for (int b = 0; b <= a; ++b, ++c) {
      const float v = R.err[c * R.n + i];
      B.err[c * B.cap + s] = v;
      if ((a == b && v < 0.f) || !isfinite(v)) silly = true;
    }
  B.chg[s] = R.chg[i];
  int nf = 0, nm = 0, nin = 0, ntl = 0;
  for (int h = 0; h < MKFG_MAX_SEED_HITS; ++h) {
    if (h >= nhs) {
      seed_hot[MKFG_MAX_SEED_HITS * s + h] = 0;
      continue;
    }
    const int hi = R.hit_index[i * MKFG_MAX_SEED_HITS + h], hl = R.hit_layer[i * MKFG_MAX_SEED_HITS + h];
    seed_hot[MKFG_MAX_SEED_HITS * s + h] = (hi & 0xffffff) | (hl << 24);
    if (hi >= 0 || hi == -9) {
      ++nf;
      nin += ntl;
      ntl = 0;
    } else {
      ++nm;
      if (hi == -1) ++ntl;
    }
  }
  E.init_hot[s] = nhs;
  B.last[s] = nhs - 1;
  if (silly) nf = -1;
  B.nfound[s] = nf;
  B.nmiss[s] = nm;
  B.ninside[s] = nin;
  B.ntail[s] = ntl;
  B.chi2[s] = 0.f;
  B.nover[s] = 0;
  // getScoreCand(cand) with default arguments (mkFit/HitStructures.h:519-531).
  const float pt = fabsf(__fdiv_rn(1.f, par3));
  float bonus = __fadd_rn(__fmul_rn(0.2f, (float)nf), 4.0f), penalty = 8.0f;
  if (pt < 0.9f) {
    penalty = __fmul_rn(penalty, 1.5f);
    bonus = fminf(bonus, 8.0f);
  }
  float t = __fadd_rn(__fmul_rn(bonus, (float)nf), 0.0f);
  t = __fsub_rn(t, __fmul_rn(penalty, (float)nin));
  B.score[s] = __fsub_rn(__fsub_rn(t, 0.0f), 0.0f);
}

}  // namespace mkfg
