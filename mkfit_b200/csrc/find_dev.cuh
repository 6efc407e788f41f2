// Device data structures and per-candidate building blocks of the
// clone-engine combinatorial finder. Used by the plain (one launch per layer
// step) and the batched persistent forms.
#pragma once

#include <cstdint>

#include "kalman.cuh"

namespace mkfg {

constexpr int kSlots = 8;               // candidate slots per seed (maxCandsPerSeed <= 8)
constexpr int kMaxXHits = 16;           // MkFinder::MPlexHitIdxMax
constexpr int kRecPerCand = kMaxXHits + 1;
constexpr int kRecPerSeed = kSlots * kRecPerCand;
// Work counters per layer-plan step (EventDev::work): active candidates,
// Kalman updates, (candidate, hit) pairs, seeds cloned, records present at
// the clone step, new candidates written by it.
constexpr int kWorkN = 6;
constexpr int kMaxLayers = 128;
// find_list entry info: current buffer (bit 0), candidate count (bits
// 1-4), layer (bits 5-12).
__host__ __device__ constexpr int find_info_pack(int cur, int ncand, int layer) {
  return cur | (ncand << 1) | (layer << 5);
}
static_assert(kSlots <= 15 && kMaxLayers <= 256, "find_info_pack field widths");

constexpr int kMaxPlan = 64;
constexpr int kMaxRegions = 8;
constexpr int kExportHits = 64;         // Config::nMaxTrkHits
constexpr int kRecInvalid = -1000000;

// A hit of the layer index in sorted order, in one 16-byte word so the
// hit selection reads the window test's inputs and the hit's index in the
// layer's input order together: q (z in the barrel, r in the endcaps; +inf
// for a hit masked by an earlier iteration), phi, and that index.
struct __align__(16) SortedHit {
  float q, phi;
  int rank, unused;
};

// One IdxChi2List entry of a candidate: a hit (index within the layer) or
// a hole code (-1, -2, -3), with its module, chi2 and candidate score.
struct __align__(16) Record {
  int hit;
  int module;
  float chi2;
  float score;
};

enum SeedState { kDormant = 0, kFinding = 1, kFinished = 2 };
enum WsrCode { kWsrInside = 0, kWsrEdge = 1, kWsrOutside = 2 };
enum ErrBits { kErrArena = 1, kErrLayerSize = 2, kErrStage = 4 };
enum StepCount {
  kCntActBarrel = 0, kCntActEndcap, kCntPairBarrel, kCntPairEndcap, kCntUpdBarrel, kCntUpdEndcap,
  kCntFind, kCntN = 8
};

struct LayerDev {
  float rin, rout, zmin, zmax, propagate_to;
  float hole_min, hole_max;
  float min_dphi, max_dphi, min_dq, max_dq;
  float c_dp_sf, c_dp_0, c_dp_1, c_dp_2;
  float c_dq_sf, c_dq_0, c_dq_1, c_dq_2;
  float c_c2_sf, c_c2_0, c_c2_1, c_c2_2;
  float qmin, fq;
  int nq, bin_offset;
  int is_barrel, has_hole, is_pix, is_stereo;
};

struct FindConfigDev {
  LayerDev layer[kMaxLayers];
  int plan[kMaxRegions][kMaxPlan];
  int plan_len[kMaxRegions];
  int pickup[kMaxRegions];
  int n_layers, n_regions, max_steps;
  int max_cands, max_holes, max_consec_holes;
  float chi2_cut_min, chi2_cut_overlap, pt_cut_overlap;
  unsigned inter_pflags, intra_pflags;
  Material mat;
  int looper_stop;  // forward search: stop low-pT loopers turning back
};

// Candidate state, structure of arrays over slots (seed * kSlots + c).
struct CandSoA {
  float* par;  // [6][cap]
  float* err;  // [21][cap]
  int* chg;
  float* chi2;
  float* score;
  int* last;   // arena index of the last hit-on-track node
  int* nfound;
  int* nmiss;
  int* nover;
  int* ninside;  // TrackCand::nInsideMinusOneHits_
  int* ntail;    // TrackCand::nTailMinusOneHits_
  int cap;
};

// One event (or a batch of events laid out back to back) on the device.
struct EventDev {
  // Hits (original order within each layer; global index = layer_begin + i).
  const float* hpos;
  const float* herr;
  int hstride;
  // The same positions and errors packed per hit for the gathers of the
  // (candidate, hit) steps: x y z e0 | e1 e2 e3 e4 | e5 - - -.
  const float4* hit4;
  const uint32_t* hinfo;  // detid (12 bit) | charge per cm << 12
  const int* layer_begin; // [n_events][lb_stride]: global index of each layer's first hit
  int lb_stride;          // n_layers + 1
  int n_bins;             // bins per event
  // Per-layer bins: (first | last << 16) over nq x 256 bins; sorted hits.
  const uint32_t* bins;
  const SortedHit* sorted_hits;
  // Seeds in sorted order (index = seed slot s).
  int n_seeds;
  int* seed_label;   // input index
  int* seed_event;   // event of the seed (batched form)
  int* region;
  int* pickup_layer;
  int* state;
  int* n_cands;
  int* cur;          // which candidate buffer holds the seed's current candidates
  int* hot_size;
  // Candidates: two buffers, kSlots per seed; best short candidate per seed.
  CandSoA cand[2];
  CandSoA bshort;
  int* bshort_valid;
  int* removed;    // the seed's comb candidate was dropped by a quality filter
  // Hit-on-track arena, hot_cap nodes per seed.
  int* node_hot;   // index (24 bit, signed) | layer << 24 (HitOnTrack layout)
  float* node_chi2;
  int* node_prev;
  int hot_cap;
  // Step scratch per candidate slot.
  float* ppar;     // [6][S*kSlots] state propagated to the layer
  float* perr;     // [21][S*kSlots]
  int* xhit;       // [kMaxXHits][S*kSlots] hit index within layer
  int* wsr;        // WSR code | extra kind << 8
  int* extra_last; // arena node of the held-back copy (kind 2)
  int* upd;        // needs UpdateWithLastHit (per slot of the new buffer)
  // Records (IdxChi2List) per seed: kRecPerSeed slots, kRecPerCand per
  // candidate (its hits in bin-scan order, then the hole record); a slot
  // holds a record when its bit of the candidate's mask is set.
  Record* rec;
  uint32_t* rmask;  // per candidate slot
  // (cand slot, hit) pairs for the chi2 pass; in the plain form barrel
  // pairs fill the array from the front and endcap pairs from the back.
  int* pairs;
  int* pair_count; // [max_steps + 2] pairs per step
  int pair_cap;
  // Plain form, per step: compact lists of the active candidate slots and
  // of the slots that take a Kalman update (barrel from the front, endcap
  // from the back); counts in step_count[step][kCnt*].
  int* act_list;
  int* upd_list;
  int* upd_hit;    // global index of the hit each listed update uses
  int list_cap;
  // Plain form, per step: seeds finding at the step (for the clone kernel),
  // and per entry the seed's buffer, candidate count and layer at the step
  // (find_info_pack), so the clone kernel starts its loads from one read.
  int* find_list;
  int* find_info;
  // Beside the update list: the candidate's buffer and layer
  // (find_info_pack without the count), so the update starts its loads
  // from its list entry.
  int* upd_info;
  int* step_count; // [max_steps + 2][kCntN]
  int* err_flags;
  // Pristine initial state (restored by the reset kernel before every run).
  CandSoA init;
  int* init_hot;   // number of seed nodes per seed
  // Work counters per step: [step][0] active candidates, [1] updates.
  int* work;
};

// Position and error of hit g (global index) from the packed copy: three
// 16-byte loads instead of nine 4-byte ones from separate rows.
__device__ __forceinline__ void load_hit(const EventDev& E, int g, float (&m)[3], float (&v)[6]) {
  const float4* h = E.hit4 + 3 * (size_t)g;
  const float4 a = __ldg(h), b = __ldg(h + 1), c = __ldg(h + 2);
  m[0] = a.x;
  m[1] = a.y;
  m[2] = a.z;
  v[0] = a.w;
  v[1] = b.x;
  v[2] = b.y;
  v[3] = b.z;
  v[4] = b.w;
  v[5] = c.x;
}

__device__ __forceinline__ int hot_pack(int index, int layer) {
  return (index & 0xffffff) | (layer << 24);
}
__device__ __forceinline__ int hot_index(int v) { return (v << 8) >> 8; }  // sign-extend 24 bit
__device__ __forceinline__ int hot_layer(int v) { return v >> 24; }

// getScoreCalc (Track.h:648-670).
__device__ __forceinline__ float score_calc(int nfound, int ntail, int nover, int nmiss, float chi2,
                                            float pt, bool in_find) {
  const float maxBonus = 8.0f;
  float bonus = 0.2f * nfound + 4.0f;
  float penalty = 8.0f;
  const float tailPenalty = 3.0f;
  const float overlapBonus = 0.0f;
  if (pt < 0.9f) {
    penalty *= in_find ? 1.7f : 1.5f;
    bonus = fminf(bonus * (in_find ? 0.9f : 1.0f), maxBonus);
  }
  return __fsub_rn(__fsub_rn(__fsub_rn(__fadd_rn(__fmul_rn(bonus, (float)nfound),
                                                 __fmul_rn(overlapBonus, (float)nover)),
                                        __fmul_rn(penalty, (float)nmiss)),
                             __fmul_rn(tailPenalty, (float)ntail)),
                   chi2);
}

// getScoreStruct (Track.h:685-697): inFindCandidates = true.
__device__ __forceinline__ float score_struct(int nhits, int ntail, int nover, int nholes,
                                              float chi2, float pt) {
  if (chi2 < 0) chi2 = 0.f;
  return score_calc(nhits, ntail, nover, nholes, chi2, pt, true);
}

// std::tan(float) as the host C library rounds it.
__device__ __forceinline__ float f_tan(float x) {
#if MKFG_LIBM_EXACT
  return (float)tan((double)x);
#else
  return tanf(x);
#endif
}

// Track::momEta / getEta(theta) (Hit.h:77-79) with the float libm calls.
__device__ __forceinline__ float eta_of_theta(float theta) {
  return -1.0f * f_log(f_tan(theta / 2.0f));
}

// Helix radius per GeV of pT in cm, signed as TrackBase::d0BeamSpot takes
// it: ((charge < 0) ? 100 : -100) / (Config::sol * Config::Bfield), in
// float as the reference's constants.
constexpr float kSolBfield = 0.299792458f * 3.8112f;
constexpr float kD0KNeg = 100.0f / kSolBfield;
constexpr float kD0KPos = -100.0f / kSolBfield;

// TrackBase::d0BeamSpot, not linearised (Track.cc:195-210): the distance of
// the helix centre from the beam spot less the helix radius. The reference
// build contracts x - k*py and y + k*px into FMAs; d0 is a difference of two
// numbers near the helix radius, so the rounding decides near-ties.
__device__ __forceinline__ float d0_beam_spot(float x, float y, float ipt, float phi, int q, float bx,
                                              float by) {
  const float k = q < 0 ? kD0KNeg : kD0KPos;
  const float pt = fabsf(1.f / ipt);
  const float abs_ooc_half = fabsf(__fmul_rn(k, pt));
  float sp, cp;
  f_sincos(phi, &sp, &cp);
  const float px = __fmul_rn(pt, cp), py = __fmul_rn(pt, sp);
  const float xc = fmaf(-k, py, x);
  const float yc = fmaf(k, px, y);
  return __fsub_rn(hypot_f(__fsub_rn(xc, bx), __fsub_rn(yc, by)), abs_ooc_half);
}

}  // namespace mkfg
