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
// the sensitive-region test (TrackerInfo.h:118-138). `bins` is the layer's
// (q bin, phi bin) table of the candidate's event. Writes up to 16 hit
// indices (index within layer) in bin-scan order; returns XHitSize (-1 when
// outside the layer) and the WSR code. kGenericBins: `bins` may point to
// shared memory (a staged copy of the table), so it is read with generic
// loads rather than through the read-only data path.
template <bool kGenericBins = false>
__device__ __forceinline__ int select_hits(const EventDev& E, const LayerDev& L,
                                           const uint32_t* __restrict__ bins, int hit_base,
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

  // Bins in scan order (q row, then phi bin mod 256), read eight at a time
  // so the loads of a row are in flight together.
  constexpr int kBinChunk = 8;
  int n = 0;
  for (int qi = qb1; qi < qb2; ++qi) {
    const uint32_t* row = bins + qi * 256;
    for (int p0 = pb1; p0 < pb2; p0 += kBinChunk) {
      uint32_t bv[kBinChunk];
#pragma unroll
      for (int k = 0; k < kBinChunk; ++k)
        bv[k] = p0 + k < pb2 ? (kGenericBins ? row[(p0 + k) & 0xff] : __ldg(row + ((p0 + k) & 0xff)))
                             : 0u;
#pragma unroll
      for (int k = 0; k < kBinChunk; ++k) {
        const int first = bv[k] & 0xffff, last = bv[k] >> 16;
        for (int hi = first; hi < last; ++hi) {
          if (n >= kMaxXHits) break;
          const float4 hs = __ldg(reinterpret_cast<const float4*>(E.sorted_hits + hit_base + hi));
          const float ddq = fabsf(q - hs.x);
          const float ddphi = cdist(fabsf(phi - hs.y));
          if (ddq >= dq) continue;
          if (ddphi >= dphi) continue;
          xhit[n * xstride] = __float_as_int(hs.z);
          ++n;
        }
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

namespace mkfg {

//------------------------------------------------------------------------------
// Shared step implementations (plain kernels and the fused persistent kernel)
//------------------------------------------------------------------------------

struct NewCand {
  int parent;    // candidate slot (0..7) the new candidate copies
  int hit;       // added hit index (or hole code)
  float chi2hit;
  int ov;        // overlap: match index 0/1 in the parent's pair, or -1
  float score;
  int is_extra;  // 1: held-back copy (extra), 2: extra with a stop (-2) node
};

// Every value is loaded before the first store: the compiler cannot tell
// the two buffers apart, and interleaved loads and stores would wait for
// one another (37 memory round trips instead of one).
__device__ __forceinline__ void copy_slot(const CandSoA& from, int fs, const CandSoA& to, int ts) {
  float par[6], err[21];
#pragma unroll
  for (int e = 0; e < 6; ++e) par[e] = from.par[e * from.cap + fs];
#pragma unroll
  for (int e = 0; e < 21; ++e) err[e] = from.err[e * from.cap + fs];
  const int chg = from.chg[fs], last = from.last[fs], nfound = from.nfound[fs];
  const int nmiss = from.nmiss[fs], nover = from.nover[fs], ninside = from.ninside[fs];
  const int ntail = from.ntail[fs];
  const float chi2 = from.chi2[fs], score = from.score[fs];
#pragma unroll
  for (int e = 0; e < 6; ++e) to.par[e * to.cap + ts] = par[e];
#pragma unroll
  for (int e = 0; e < 21; ++e) to.err[e * to.cap + ts] = err[e];
  to.chg[ts] = chg;
  to.chi2[ts] = chi2;
  to.score[ts] = score;
  to.last[ts] = last;
  to.nfound[ts] = nfound;
  to.nmiss[ts] = nmiss;
  to.nover[ts] = nover;
  to.ninside[ts] = ninside;
  to.ntail[ts] = ntail;
}

// TrackCand::addHitIdx counters (mkFit/HitStructures.h:714-735).
__device__ __forceinline__ void add_hit_counts(int hit, float chi2, int& nfound, int& nmiss,
                                               int& ninside, int& ntail, float& tchi2) {
  if (hit >= 0 || hit == -9) {
    ++nfound;
    tchi2 += chi2;
    ninside += ntail;
    ntail = 0;
  } else {
    ++nmiss;
    if (hit == -1) ++ntail;
  }
}

// Seed state at the start of layer-plan step `step`: a dormant seed starts
// finding at the step after its pickup layer (find_tracks_unroll_candidates,
// mkFit/MkBuilder.cc:1503-1566).
__device__ __forceinline__ int wake_seed(const FindConfigDev& C, int reg, int layer, int step,
                                         int state, int pickup_layer) {
  if (layer >= 0 && state == kDormant && pickup_layer == C.plan[reg][C.pickup[reg] + step - 1])
    return kFinding;
  return state;
}

// Output of the candidate preparation of one layer step.
struct PrepOut {
  bool active = false;  // candidate takes part in this layer
  int xs = 0;           // XHitSize
  int wsr = kWsrOutside;
  int extra = 0;        // held back: 1 plain copy, 2 copy with a stop node
  int extra_last = -1;  // arena node of the stop node (extra == 2)
  bool hole = false;    // a hole record was produced
  int hole_hit = 0;
  float hole_score = 0.f;
  float ppar[6];
  float perr[21];
};

// Unroll + looper stop (mkFit/MkBuilder.cc:1503-1566) for a candidate of a
// seed already in Finding state: a candidate whose last node is a stop (-2)
// is inactive; a low-pT looper outside r = 25 cm turning back gets a stop
// node and is inactive. Returns whether the candidate is active.
__device__ __forceinline__ bool cand_is_active(const EventDev& E, const CandSoA& B, int s, int slot,
                                               int layer, bool looper_stop) {
  // Parameters first: their loads overlap the stop-node lookup.
  const float x = B.par[0 * B.cap + slot], y = B.par[1 * B.cap + slot];
  const float ipt = B.par[3 * B.cap + slot], phi = B.par[4 * B.cap + slot];
  const int last = B.last[slot];
  if (hot_index(node_hot_of(E, s, last)) == -2) return false;
  const float pt = fabsf(1.f / ipt);
  if (looper_stop && pt < 1.2f) {  // IT_FwdSearch only
    const float dphi = fabsf(f_atan2(y, x) - phi);
    if (x * x + y * y > 625.f && dphi > 1.371f && dphi < 4.512f) {
      B.last[slot] = arena_append(E, s, -2, layer, 0.f, last);
      B.nmiss[slot] += 1;
      return false;
    }
  }
  return true;
}

// cand_is_active, loading the state of an active candidate.
__device__ __forceinline__ bool activate_cand(const EventDev& E, const CandSoA& B, int s, int slot,
                                              int layer, bool looper_stop, float (&par)[6],
                                              float (&err)[21], int& chg) {
  if (!cand_is_active(E, B, s, slot, layer, looper_stop)) return false;
  load_state(B, slot, par, err);
  chg = B.chg[slot];
  return true;
}

// Propagation to the layer, SelectHitIndices, missed-layer handling
// (mkFit/MkBuilder.cc:1568-1637) and the hole record (MkFinder.cc:1245-1283)
// for an active candidate. xhit receives up to 16 indices with stride xstride.
template <bool kGenericBins = false>
__device__ __forceinline__ void select_cand(const EventDev& E, const FindConfigDev& C,
                                            const LayerDev& L, const uint32_t* layer_bins,
                                            int hit_base, int reg, int layer, int s,
                                            const CandSoA& B, int slot, const float (&ppar)[6],
                                            const float (&perr)[21], int* xhit, int xstride,
                                            PrepOut& o);

template <bool kGenericBins = false>
__device__ __forceinline__ void prep_cand(const EventDev& E, const FindConfigDev& C,
                                          const LayerDev& L, const uint32_t* layer_bins,
                                          int hit_base, int reg, int layer, int s, const CandSoA& B,
                                          int slot, const float (&par)[6], const float (&err)[21],
                                          int chg, int* xhit, int xstride, PrepOut& o) {
  if (L.is_barrel)
    propagate_to_r(par, err, chg, L.propagate_to, C.inter_pflags, C.mat, false, o.ppar, o.perr);
  else
    propagate_to_z(par, err, chg, L.propagate_to, C.inter_pflags, C.mat, false, o.ppar, o.perr);
  select_cand<kGenericBins>(E, C, L, layer_bins, hit_base, reg, layer, s, B, slot, o.ppar, o.perr,
                            xhit, xstride, o);
}

// The part of prep_cand after the propagation: SelectHitIndices on the
// propagated state, missed-layer handling and the hole record.
template <bool kGenericBins>
__device__ __forceinline__ void select_cand(const EventDev& E, const FindConfigDev& C,
                                            const LayerDev& L, const uint32_t* layer_bins,
                                            int hit_base, int reg, int layer, int s,
                                            const CandSoA& B, int slot, const float (&ppar)[6],
                                            const float (&perr)[21], int* xhit, int xstride,
                                            PrepOut& o) {
  o.active = true;
  o.xs = select_hits<kGenericBins>(E, L, layer_bins, hit_base, ppar, perr, xhit, xstride, o.wsr);
  const float cand_r = hypot_f(ppar[0], ppar[1]);
  if (L.is_barrel && cand_r < L.rin) {
    o.xs = 0;
    o.wsr = kWsrOutside;
    o.extra = (reg == 2) ? 2 : 1;
    if (o.extra == 2) o.extra_last = arena_append(E, s, -2, layer, 0.f, B.last[slot]);
  } else if (o.wsr == kWsrOutside) {
    o.extra = 1;
  }
  if (o.xs < 0) o.xs = 0;
  if (o.wsr != kWsrOutside) {
    const int nin = B.ninside[slot], ntl = B.ntail[slot];
    int fake = ((nin + ntl) < C.max_holes && ntl < C.max_consec_holes) ? -1 : -2;
    if (o.wsr == kWsrEdge) fake = -3;
    const int ntail_rec = fake == -1 ? ntl + 1 : ntl;
    const float pt = fabsf(1.0f / ppar[3]);
    o.hole = true;
    o.hole_hit = fake;
    o.hole_score = score_struct(B.nfound[slot], ntail_rec, B.nover[slot], nin, B.chi2[slot], pt);
  }
}

// The chi2 and the cuts of one (candidate, hit) evaluation
// (MkFinder::FindCandidatesCloneEngine, mkFit/MkFinder.cc:1142-1193, with
// kalmanPropagateAndComputeChi2[Endcap]): dynamic chi2 cut, strip
// compatibility and strip charge. The pixel same-layer check is the
// caller's. Returns whether the hit passes; fills chi2 and module.
__device__ __forceinline__ bool pair_accept(const EventDev& E, const FindConfigDev& C,
                                            const LayerDev& L, int g, const float (&ppar)[6],
                                            const float (&perr)[21], int chg, float& chi2_out,
                                            int& module_out) {
  float mpos[3], merr[6];
  load_hit(E, g, mpos, merr);
  const uint32_t info = __ldg(E.hinfo + g);
  float hpar[6], herr_[21];
  float chi2;
  if (L.is_barrel) {
    propagate_to_r(ppar, perr, chg, hypot_f(mpos[0], mpos[1]), C.intra_pflags, C.mat, false, hpar,
                   herr_);
    chi2 = kalman_barrel<true, false>(hpar, herr_, mpos, merr, hpar, herr_);
  } else {
    propagate_to_z(ppar, perr, chg, mpos[2], C.intra_pflags, C.mat, false, hpar, herr_);
    chi2 = kalman_endcap<true, false>(hpar, herr_, mpos, merr, hpar, herr_);
  }
  chi2 = fabsf(chi2);
  bool ok = chi2 < dynamic_chi2_cut(L, C.chi2_cut_min, ppar);
  if (ok && !L.is_pix) {
    ok = strip_q_compatible(L.is_barrel, perr, hpar, mpos, merr);
    ok &= strip_charge_ok(L.is_barrel, info >> 12, hpar, merr);
  }
  chi2_out = chi2;
  module_out = info & 0xfff;
  return ok;
}

// Score of an accepted hit record (IdxChi2List with nhits + 1, no tail
// holes, MkFinder.cc:1222-1233).
__device__ __forceinline__ float hit_record_score(const float (&ppar)[6], int nfound, int nover,
                                                  int nholes, float cand_chi2, float chi2) {
  const float pt = fabsf(1.0f / ppar[3]);
  return score_struct(nfound + 1, 0, nover, nholes, cand_chi2 + chi2, pt);
}

// One (candidate, hit) evaluation (MkFinder::FindCandidatesCloneEngine,
// mkFit/MkFinder.cc:1142-1240). Returns whether the hit is accepted; fills
// chi2, score, module.
__device__ __forceinline__ bool eval_pair(const EventDev& E, const FindConfigDev& C,
                                          const LayerDev& L, int layer, int s, int g,
                                          const float (&ppar)[6], const float (&perr)[21], int chg,
                                          int nfound, int nover, int nholes, float cand_chi2,
                                          float& chi2_out, float& score_out, int& module_out) {
  float chi2;
  bool ok = pair_accept(E, C, L, g, ppar, perr, chg, chi2, module_out);
  if (ok && L.is_pix) {
    // No second hit on a pixel layer of the first three hit-on-track nodes
    // (MkFinder.cc:1195-1210: ccand.m_hots[0 .. min(nFound, 2)]). Those are
    // the seed's own nodes, the first ones of its arena; for a seed with
    // fewer than three hits the reference reads past the nodes it holds, so
    // only the seed's nodes are checked here.
    const int n_seed = E.init_hot[s];
    for (int i = 0; i <= nfound && i <= 2 && i < n_seed; ++i)
      if (hot_layer(node_hot_of(E, s, i)) == layer) ok = false;
  }
  if (!ok) return false;
  chi2_out = chi2;
  score_out = hit_record_score(ppar, nfound, nover, nholes, cand_chi2, chi2);
  return true;
}

// UpdateWithLastHit on a state in registers (mkFit/MkFinder.cc:1291-1308;
// kalmanPropagateAndUpdate[Endcap], KalmanUtilsMPlex.cc:471-505, 697-731):
// propagation to the hit with the inter-layer flags, the update, and the
// charge flip of a negative 1/pT; g is the hit's global index.
__device__ __forceinline__ void update_state(const EventDev& E, const FindConfigDev& C,
                                             const LayerDev& L, int g, float (&par)[6],
                                             float (&err)[21], int& chg) {
  float mpos[3], merr[6];
  load_hit(E, g, mpos, merr);
  float ppar[6], perr[21];
  if (L.is_barrel) {
    propagate_to_r(par, err, chg, hypot_f(mpos[0], mpos[1]), C.inter_pflags, C.mat, false, ppar, perr);
    kalman_barrel<false, true>(ppar, perr, mpos, merr, par, err);
  } else {
    propagate_to_z(par, err, chg, mpos[2], C.inter_pflags, C.mat, false, ppar, perr);
    kalman_endcap<false, true>(ppar, perr, mpos, merr, par, err);
  }
  if (par[3] < 0) {
    chg = -chg;
    par[3] = -par[3];
  }
}

// UpdateWithLastHit + CopyOutParErr for one candidate slot of buffer B
// (MkFinder.cc:1291-1335), given the hit's global index g and its layer.
__device__ __forceinline__ void update_cand_at(const EventDev& E, const FindConfigDev& C,
                                               const LayerDev& L, int g, const CandSoA& B,
                                               int slot) {
  float par[6], err[21];
  load_state(B, slot, par, err);
  int chg = B.chg[slot];
  update_state(E, C, L, g, par, err, chg);
  store_state(B, slot, par, err);
  B.chg[slot] = chg;
}

// UpdateWithLastHit with the hit found from the candidate's last node.
// Returns false if the last node is not a hit.
__device__ __forceinline__ bool update_cand(const EventDev& E, const FindConfigDev& C, int s,
                                            const int* lb, const CandSoA& B, int slot) {
  const int hv = node_hot_of(E, s, B.last[slot]);
  const int hl = hot_layer(hv);
  // After an arena overflow (reported through err_flags) the last node may
  // not be a hit: skip rather than read outside the hit arrays.
  if (hot_index(hv) < 0 || hl < 0 || hl >= C.n_layers) return false;
  update_cand_at(E, C, C.layer[hl], lb[hl] + hot_index(hv), B, slot);
  return true;
}

// Records and per-candidate step results of one seed, wherever they live
// (global memory in the plain form, shared memory in the fused form).
struct SeedRecords {
  const Record* rec_;      // kRecPerSeed records
  const uint32_t* mask_;   // per candidate: bit h set = record h present
  const int* wsr_;         // WSR code | extra kind << 8, per candidate
  const int* extra_last_;  // stop node of a kind-2 extra, per candidate
  int* upd_;               // per new candidate: 1 + index in its layer of the hit
                           // to update with (the last one added), 0 = none;
                           // null: returned only
  __device__ Record rec(int idx) const { return rec_[idx]; }
  __device__ uint32_t mask(int c) const { return mask_[c]; }
  __device__ int extra_kind(int c) const { return wsr_[c] >> 8; }
  __device__ int extra_last(int c) const { return extra_last_[c]; }
  __device__ void set_upd(int i, int v) const {
    if (upd_) upd_[i] = v;
  }
};

// Total order of record scores as integers: the float order, with -0 taken
// as +0 and NaN below every number (NaN records go last, in record order).
__device__ __forceinline__ int score_key(float score) {
  const float z = __fadd_rn(score, 0.f);
  const int k = __float_as_int(z);
  return z != z ? INT_MIN : (k >= 0 ? k : k ^ 0x7fffffff);
}

// Copy of the parameters and covariance of new candidates i < n (parent
// slot parent_i, lane i of `parent`) from buffer B to buffer N, in two
// halves so a caller can issue the loads early: load_par_err into seven
// registers per lane, store_par_err from them. Lane t moves element
// t / 8 + 4 k of candidate t % 8: each access of the warp covers four whole
// 32-byte sectors (a seed's 8 slots are contiguous).
__device__ __forceinline__ void load_par_err(const CandSoA& B, int s, int n, int parent, int lane,
                                             float (&v)[7]) {
  const int c = lane & 7;
  const int pc = __shfl_sync(0xffffffffu, parent, c);
  const int src = s * kSlots + pc;
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    const int e = (lane >> 3) + 4 * k;
    v[k] = 0.f;
    if (c < n && e < 27) v[k] = (e < 6 ? B.par + e * B.cap : B.err + (e - 6) * B.cap)[src];
  }
}
__device__ __forceinline__ void store_par_err(const CandSoA& N, int s, int n, int lane,
                                              const float (&v)[7]) {
  const int c = lane & 7;
  if (c >= n) return;
  const int dst = s * kSlots + c;
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    const int e = (lane >> 3) + 4 * k;
    float* to = e < 6 ? N.par + e * N.cap : N.err + (e - 6) * N.cap;
    if (e < 27) to[dst] = v[k];
  }
}
// Both halves at once (all loads before the first store).
__device__ __forceinline__ void copy_par_err(const CandSoA& B, const CandSoA& N, int s, int n,
                                             int parent, int lane) {
  float v[7];
  load_par_err(B, s, n, parent, lane, v);
  store_par_err(N, s, n, lane, v);
}

// Writes a hit-on-track node at arena position pos of seed s (allocated by
// the caller); returns pos, or prev after an overflow (flagged).
__device__ __forceinline__ int arena_put(const EventDev& E, int s, int pos, int index, int layer,
                                         float chi2, int prev) {
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

// Shared-memory scratch of one warp's clone step: the ranked records with
// their fields, and the counters of the seed's candidates.
struct CloneScratch {
  int rec[32];
  int hit[32];
  float score[32];
  float chi2[32];
  int module[32];
  // Per candidate: chg, chi2 bits, last, nfound, nmiss, nover, ninside,
  // ntail, score bits, 1/pT bits, extra kind.
  int cand[11][kSlots];
};

// CandCloner::ProcessSeedRange for one seed (mkFit/CandCloner.cc:36-189),
// executed by one warp. Returns the new candidate count, or -1 when the
// seed's candidates are unchanged; upd_out: lane i's new candidate's
// update code (SeedRecords::upd_); n_records_out (optional): the records
// present; parent_out (optional, kSlots entries): each new candidate's
// parent slot. The warp owns the seed's arena counter.
__device__ __forceinline__ int clone_seed(const EventDev& E, const FindConfigDev& C, int s,
                                          int layer, int state, int ncand, int cur,
                                          const SeedRecords& R, HitMatchPair* hm,
                                          CloneScratch& X, int& upd_out, int lane,
                                          int* n_records_out = nullptr,
                                          int* parent_out = nullptr) {
  constexpr unsigned kFull = 0xffffffffu;
  const CandSoA& B = E.cand[cur];
  const CandSoA& N = E.cand[cur ^ 1];
  const int M = C.max_cands;
  upd_out = 0;
  const int hot0 = E.hot_size[s];
  // The best short candidate's flag and score, loaded with the seed's
  // other data rather than one after the other where they are used.
  const int bs_valid = E.bshort_valid[s];
  const float bs_score_in = E.bshort.score[s];

  // Per-candidate values, staged by lane c for candidate c.
  const int cslot = s * kSlots + (lane < kSlots ? lane : 0);
  const bool is_cand = lane < ncand;
  const int c_kind = (is_cand && state == kFinding) ? R.extra_kind(lane) : 0;
  if (is_cand) {
    X.cand[8][lane] = __float_as_int(B.score[cslot]);
    X.cand[9][lane] = __float_as_int(B.par[3 * B.cap + cslot]);
    X.cand[10][lane] = c_kind;
    X.cand[0][lane] = B.chg[cslot];
    X.cand[1][lane] = __float_as_int(B.chi2[cslot]);
    X.cand[2][lane] = B.last[cslot];
    X.cand[3][lane] = B.nfound[cslot];
    X.cand[4][lane] = B.nmiss[cslot];
    X.cand[5][lane] = B.nover[cslot];
    X.cand[6][lane] = B.ninside[cslot];
    X.cand[7][lane] = B.ntail[cslot];
  }

  constexpr int kPer = (kRecPerSeed + 31) / 32;  // present records per lane, at most
  // Records present: the mask bits of candidates [0, ncand) (lane c holds
  // candidate c's mask). In record order they get compacted indices
  // p = 0 .. n_valid - 1; cincl is the inclusive count up to candidate c.
  const uint32_t cm = is_cand ? R.mask(lane) : 0u;
  const int ccount = __popc(cm);
  int cincl = ccount;
#pragma unroll
  for (int off = 1; off < kSlots; off <<= 1) {
    const int v = __shfl_up_sync(kFull, cincl, off);
    if (lane >= off) cincl += v;
  }
  const int n_valid = __shfl_sync(kFull, cincl, kSlots - 1);
  if (n_records_out) *n_records_out = n_valid;
  // Record index of present record p < n_valid (warp-collective).
  auto locate = [&](int p) {
    int c = 0;
#pragma unroll
    for (int j = 0; j < kSlots - 1; ++j) c += p >= __shfl_sync(kFull, cincl, j) ? 1 : 0;
    const uint32_t m = __shfl_sync(kFull, cm, c);
    const int first = __shfl_sync(kFull, cincl - ccount, c);
    return c * kRecPerCand + (int)(__fns(m, 0, p - first + 1) & 31u);
  };
  const bool mine = lane < n_valid;
  const int my_idx = locate(lane);
  Record my_r{0, 0, 0.f, 0.f};
  if (mine) my_r = R.rec(my_idx);

  // Overlap candidates per parent (consulted at CandCloner.cc:120-124),
  // filled in hit order as MkFinder does (:1212-1216): lane c considers
  // candidate c's hit records under the overlap chi2 cut.
  if (lane < kSlots) {
    HitMatchPair p;
    p.reset();
    uint32_t m = cm & ((1u << kMaxXHits) - 1u);
    while (m) {
      const int h = __ffs(m) - 1;
      m &= m - 1;
      const Record q = R.rec(lane * kRecPerCand + h);
      if (q.chi2 < C.chi2_cut_overlap) p.consider(q.hit, q.module, q.chi2);
    }
    hm[lane] = p;
  }

  // Extras (held-back candidates) in candidate order (MkBuilder.cc:1600-1626).
  const unsigned extra_mask = __ballot_sync(kFull, c_kind != 0);
  const int n_extras = __popc(extra_mask);
  __syncwarp();

  if (n_valid == 0) {
    // hitsForSeed empty (CandCloner.cc:163-172): the extras survive.
    if (state != kFinding) return -1;

    // Lane i: the i-th extra.
    int c = 0;
    if (lane < n_extras) {
      unsigned mm = extra_mask;
      for (int k = 0; k < lane; ++k) mm &= mm - 1;
      c = __ffs(mm) - 1;
    }
    copy_par_err(B, N, s, n_extras, c, lane);
    if (lane < n_extras) {
      if (parent_out) parent_out[lane] = c;
      const int src = s * kSlots + c, dst = s * kSlots + lane;
      // Loads first (see copy_slot).
      const int chg = B.chg[src], nfound = B.nfound[src], nover = B.nover[src];
      const int ninside = B.ninside[src], ntail = B.ntail[src], nmiss = B.nmiss[src];
      const float chi2 = B.chi2[src], score = B.score[src];
      const bool stop = R.extra_kind(c) == 2;
      const int last = stop ? R.extra_last(c) : B.last[src];
      N.chg[dst] = chg;
      N.chi2[dst] = chi2;
      N.score[dst] = score;
      N.nfound[dst] = nfound;
      N.nover[dst] = nover;
      N.ninside[dst] = ninside;
      N.ntail[dst] = ntail;
      N.last[dst] = last;
      N.nmiss[dst] = nmiss + (stop ? 1 : 0);
      R.set_upd(lane, 0);
    }
    return n_extras;
  }

  // Top-num_hits records in (score desc, record index asc) order: the
  // reference's std::sort by score; on exact score ties this order is the
  // stable one. Lane i receives the i-th record and its fields.
  const int num_hits = min(n_valid, M);
  const bool has_rec = lane < num_hits;
  int my_rec = 0, r_hit = 0, r_module = 0;
  float r_score = 0.f, r_chi2 = 0.f;
  if (n_valid <= 32) {
    // Lane p holds present record p: rank each against all others, place
    // the first num_hits by rank.
    const int key = mine ? score_key(my_r.score) : INT_MIN;
    int rank = 0;
    for (int j = 0; j < n_valid; ++j) {
      const int kj = __shfl_sync(kFull, key, j);
      rank += (kj > key) || (kj == key && j < lane);
    }
    if (mine && rank < num_hits) {
      X.rec[rank] = my_idx;
      X.hit[rank] = my_r.hit;
      X.score[rank] = my_r.score;
      X.chi2[rank] = my_r.chi2;
      X.module[rank] = my_r.module;
    }
    __syncwarp();
    if (has_rec) {
      my_rec = X.rec[lane];
      r_hit = X.hit[lane];
      r_score = X.score[lane];
      r_chi2 = X.chi2[lane];
      r_module = X.module[lane];
    }
  } else {
    // More records than lanes: num_hits rounds of a warp arg-max over the
    // compacted indices (their order is the record order).
    int key[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int p = lane + 32 * k;
      const int idx = locate(p);
      key[k] = p < n_valid ? score_key(R.rec(idx).score) : INT_MIN;
    }
    bool left[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) left[k] = lane + 32 * k < n_valid;
    int my_p = 0;
    for (int i = 0; i < num_hits; ++i) {
      int best = INT_MIN, bidx = INT_MAX;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        const int p = lane + 32 * k;
        if (left[k] && (key[k] > best || (key[k] == best && p < bidx))) {
          best = key[k];
          bidx = p;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const int ob = __shfl_xor_sync(kFull, best, off);
        const int oi = __shfl_xor_sync(kFull, bidx, off);
        if (ob > best || (ob == best && oi < bidx)) {
          best = ob;
          bidx = oi;
        }
      }
      if (lane == i) my_p = bidx;
#pragma unroll
      for (int k = 0; k < kPer; ++k)
        if (lane + 32 * k == bidx) left[k] = false;
    }
    my_rec = locate(my_p);
    if (has_rec) {
      const Record q = R.rec(my_rec);
      r_hit = q.hit;
      r_score = q.score;
      r_chi2 = q.chi2;
      r_module = q.module;
    }
  }

  // Build the new candidate list (logic of ProcessSeedRange); lane i keeps
  // new candidate i.
  NewCand nc{0, 0, 0.f, -1, 0.f, 0};
  int n_pushed = 0;
  float bs_score = bs_valid ? bs_score_in : -1e16f;  // getScoreWorstPossible
  int bs_from = -1;
  if (extra_mask == 0) {
    // No extras: the new candidates are the records in order, less the
    // stop (-2) records, of which the first (best) may replace the best
    // short candidate. All lanes at once.
    const bool is_stop = has_rec && r_hit == -2;
    const unsigned stop_mask = __ballot_sync(kFull, is_stop);
    const unsigned push_mask = __ballot_sync(kFull, has_rec && !is_stop);
    n_pushed = __popc(push_mask);
    if (stop_mask) {
      const int f = __ffs(stop_mask) - 1;
      const float sc = __shfl_sync(kFull, r_score, f);
      const int rec = __shfl_sync(kFull, my_rec, f);
      if (sc > bs_score) {
        bs_score = sc;
        bs_from = rec;
      }
    }
    const int src = stop_mask ? (int)__fns(push_mask, 0, lane + 1) & 31 : lane;
    const int idx = __shfl_sync(kFull, my_rec, src);
    const int hit = __shfl_sync(kFull, r_hit, src);
    const float score = __shfl_sync(kFull, r_score, src);
    const float chi2hit = __shfl_sync(kFull, r_chi2, src);
    const int module = __shfl_sync(kFull, r_module, src);
    const int parent = idx / kRecPerCand;
    if (lane < n_pushed) {
      const float ppt = fabsf(1.f / __int_as_float(X.cand[9][parent]));
      int ov = -1;
      if (ppt > C.pt_cut_overlap && hit >= 0) ov = hm[parent].find(hit, module);
      nc = NewCand{parent, hit, chi2hit, ov, score, 0};
    }
  }
  auto push = [&](const NewCand& v) {
    if (lane == n_pushed) nc = v;
    ++n_pushed;
  };
  unsigned em = extra_mask;  // extras not yet taken, in candidate order
  // With extras: sequentially, identically in every lane from the
  // broadcast values.
  for (int ih = 0; ih < (extra_mask ? num_hits : 0); ++ih) {
    const int idx = __shfl_sync(kFull, my_rec, ih);
    const int hit = __shfl_sync(kFull, r_hit, ih);
    const float score = __shfl_sync(kFull, r_score, ih);
    const float chi2hit = __shfl_sync(kFull, r_chi2, ih);
    const int module = __shfl_sync(kFull, r_module, ih);
    const int parent = idx / kRecPerCand;
    if (hit == -2) {
      if (score > bs_score) {
        bs_score = score;
        bs_from = idx;
      }
      continue;
    }
    while (em && n_pushed < M) {
      const int c = __ffs(em) - 1;
      if (!(__int_as_float(X.cand[8][c]) > score)) break;
      push(NewCand{c, 0, 0.f, -1, 0.f, X.cand[10][c]});
      em &= em - 1;
    }
    if (n_pushed >= M) break;
    int ov = -1;
    const float ppt = fabsf(1.f / __int_as_float(X.cand[9][parent]));
    if (ppt > C.pt_cut_overlap && hit >= 0) ov = hm[parent].find(hit, module);
    push(NewCand{parent, hit, chi2hit, ov, score, 0});
  }
  while (em && n_pushed < M) {
    const int c = __ffs(em) - 1;
    push(NewCand{c, 0, 0.f, -1, 0.f, X.cand[10][c]});
    em &= em - 1;
  }

  // The parents' parameters and covariances are loaded now, so the loads
  // overlap the node and best-short bookkeeping (stored at the end).
  float pe[7];
  load_par_err(B, s, n_pushed, nc.parent, lane, pe);
  // Arena nodes of this step, one allocation for the seed: the best short
  // candidate's hole node first, then one or two nodes per new candidate
  // with a hit, in candidate order.
  const bool own = lane < n_pushed && !nc.is_extra;
  const int n_nodes = own ? 1 + (nc.ov >= 0) : 0;
  int node_off = n_nodes;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int v = __shfl_up_sync(kFull, node_off, off);
    if (lane >= off) node_off += v;
  }
  const int nodes_total = __shfl_sync(kFull, node_off, 31) + (bs_from >= 0);
  node_off -= n_nodes;
  if (lane == 0 && nodes_total) E.hot_size[s] = hot0 + nodes_total;
  const int node_base = hot0 + (bs_from >= 0);

  // Best short candidate (a -2 record scoring above the current best).
  if (bs_from >= 0) {
    const int parent = bs_from / kRecPerCand;
    const int src = s * kSlots + parent;
    if (lane < 27) {
      if (lane < 6) E.bshort.par[lane * E.bshort.cap + s] = B.par[lane * B.cap + src];
      else E.bshort.err[(lane - 6) * E.bshort.cap + s] = B.err[(lane - 6) * B.cap + src];
    }
    if (lane == 0) {
      int nfound = B.nfound[src], nmiss = B.nmiss[src], nin = B.ninside[src], ntl = B.ntail[src];
      float chi2 = B.chi2[src];
      const int chg = B.chg[src], nover = B.nover[src], last = B.last[src];
      add_hit_counts(-2, 0.f, nfound, nmiss, nin, ntl, chi2);
      E.bshort.last[s] = arena_put(E, s, node_base - 1, -2, layer, 0.f, last);
      E.bshort.chg[s] = chg;
      E.bshort.chi2[s] = chi2;
      E.bshort.score[s] = bs_score;
      E.bshort.nfound[s] = nfound;
      E.bshort.nmiss[s] = nmiss;
      E.bshort.nover[s] = nover;
      E.bshort.ninside[s] = nin;
      E.bshort.ntail[s] = ntl;
      E.bshort_valid[s] = 1;
    }
  }

  // Materialize the new candidates into the other buffer: parameters and
  // covariance by all lanes, counters and hit-on-track nodes of new
  // candidate i by lane i.
  store_par_err(N, s, n_pushed, lane, pe);
  if (lane < n_pushed) {
    if (parent_out) parent_out[lane] = nc.parent;
    const int pc = nc.parent, dst = s * kSlots + lane;
    int nfound = X.cand[3][pc], nmiss = X.cand[4][pc], nin = X.cand[6][pc], ntl = X.cand[7][pc];
    int nover = X.cand[5][pc];
    float chi2 = __int_as_float(X.cand[1][pc]);
    int last = X.cand[2][pc];
    float score = __int_as_float(X.cand[8][pc]);
    int upd = 0;
    if (nc.is_extra) {
      if (nc.is_extra == 2) {
        last = R.extra_last(nc.parent);
        ++nmiss;
      }
    } else {
      const int pos = node_base + node_off;
      add_hit_counts(nc.hit, nc.chi2hit, nfound, nmiss, nin, ntl, chi2);
      last = arena_put(E, s, pos, nc.hit, layer, nc.chi2hit, last);
      score = nc.score;
      if (nc.ov >= 0) {
        const HitMatchPair& p = hm[nc.parent];
        add_hit_counts(p.hit[nc.ov], p.chi2[nc.ov], nfound, nmiss, nin, ntl, chi2);
        last = arena_put(E, s, pos + 1, p.hit[nc.ov], layer, p.chi2[nc.ov], last);
        ++nover;
      }
      // UpdateWithLastHit uses the last hit added: the overlap hit if any.
      if (nc.hit >= 0) upd = 1 + (nc.ov >= 0 ? hm[nc.parent].hit[nc.ov] : nc.hit);
    }
    N.chg[dst] = X.cand[0][pc];
    N.chi2[dst] = chi2;
    N.score[dst] = score;
    N.last[dst] = last;
    N.nfound[dst] = nfound;
    N.nmiss[dst] = nmiss;
    N.nover[dst] = nover;
    N.ninside[dst] = nin;
    N.ntail[dst] = ntl;
    R.set_upd(lane, upd);
    upd_out = upd;
  }
  return n_pushed;
}

// Candidate score for the final merge: getScoreCand with default arguments
// (mkFit/HitStructures.h:519-531).
__device__ __forceinline__ float cand_score(const CandSoA& B, int slot) {
  const float pt = fabsf(1.f / B.par[3 * B.cap + slot]);
  float chi2 = B.chi2[slot];
  if (chi2 < 0) chi2 = 0.f;
  return score_calc(B.nfound[slot], 0, B.nover[slot], B.ninside[slot], chi2, pt, false);
}

// CombCandidate::MergeCandsAndBestShortOne(update_score, sort_cands)
// (mkFit/HitStructures.cc:511-552) for one seed; writes the final list into
// buffer cur ^ 1 and returns the final candidate count. When the list
// stays as it is (already in score order, no best short candidate to
// insert) only the scores are written, in place, and `moved` is false.
__device__ __forceinline__ int merge_seed(const EventDev& E, const FindConfigDev& C, int s,
                                          int n, int cur, bool& moved) {
  const CandSoA& B = E.cand[cur];
  const CandSoA& N = E.cand[cur ^ 1];
  float score[kSlots + 1];
  int order[kSlots + 1];
  for (int c = 0; c < n; ++c) {
    score[c] = cand_score(B, s * kSlots + c);
    order[c] = c;
  }
  // Insertion sort by score, descending (std::sort on <= 16 elements).
  for (int i = 1; i < n; ++i) {
    const int o = order[i];
    const float v = score[o];
    int j = i;
    while (j > 0 && score[order[j - 1]] < v) {
      order[j] = order[j - 1];
      --j;
    }
    order[j] = o;
  }
  const bool has_bs = E.bshort_valid[s];
  // With candidates left the best short candidate's score is recomputed
  // with theirs; with none it is appended as it is, keeping the score of
  // the record that made it (getScoreStruct, in-finding weights, tail holes
  // counted) -- HitStructures.cc:515-548.
  const float bs = has_bs ? (n > 0 ? cand_score(E.bshort, s) : E.bshort.score[s]) : 0.f;
  int ins = -1;
  if (n > 0) {
    if (has_bs && bs > score[order[n - 1]]) {
      int ci = 0;
      while (score[order[ci]] > bs) ++ci;
      if (n >= C.max_cands) --n;
      ins = ci;
    }
  } else if (has_bs) {
    ins = 0;
  }
  bool identity = ins < 0;
  for (int i = 0; i < n && identity; ++i) identity = order[i] == i;
  moved = !identity;
  if (identity) {
    for (int c = 0; c < n; ++c) B.score[s * kSlots + c] = score[c];
    E.bshort_valid[s] = 0;
    return n;
  }
  int w = 0;
  for (int i = 0; i <= n; ++i) {
    if (i == ins) {
      const int dst = s * kSlots + w;
      copy_slot(E.bshort, s, N, dst);
      N.score[dst] = bs;
      ++w;
    }
    if (i == n) break;
    const int src = s * kSlots + order[i];
    const int dst = s * kSlots + w;
    copy_slot(B, src, N, dst);
    N.score[dst] = score[order[i]];
    ++w;
  }
  E.bshort_valid[s] = 0;
  return w;
}

}  // namespace mkfg
