// Fused clone-engine finding: one thread block carries a chunk of W
// consecutive seeds through every layer-plan step and the final merge in a
// single launch. Per step the block runs the same four phases as the plain
// form's four kernels (prep, chi2, clone, update), separated by block
// barriers, but the step scratch -- states propagated to the layer, selected
// hit lists, the (candidate, hit) pair list, the IdxChi2List records, the
// overlap pairs and the update flags -- lives in shared memory and never
// goes to DRAM. Candidate buffers, seed scalars and the hit-on-track arena
// stay in global memory (each seed's data is touched by one block only, so
// they stay in L1/L2 between phases).
//
// The per-candidate and per-seed work is the code the plain kernels call
// (find_steps.cuh), so results are the plain form's; a chunk stops stepping
// once none of its seeds can change any more.
#pragma once

#include "find_steps.cuh"

namespace mkfg {

template <int W>
struct FusedShared {
  static constexpr int T = W * kSlots;  // threads: one per candidate slot
  float ppar[6 * T];
  float perr[21 * T];
  int xhit[kMaxXHits * T];
  int wsr[T];
  int extra_last[T];
  int upd[T];
  Record rec[W * kRecPerSeed];
  uint32_t rmask[T];
  unsigned short pairs[T * kMaxXHits];
  HitMatchPair hm[T / 32][kSlots];
  CloneScratch scratch[T / 32];
  int n_pairs;
};

template <int W>
__global__ void __launch_bounds__(W * kSlots) k_find_fused(EventDev E,
                                                           const FindConfigDev* __restrict__ Cp) {
  constexpr int T = W * kSlots;
  static_assert(T % 32 == 0, "chunk must fill whole warps");
  extern __shared__ __align__(16) unsigned char fused_smem[];
  FusedShared<W>& S = *reinterpret_cast<FusedShared<W>*>(fused_smem);
  const FindConfigDev& C = *Cp;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int s0 = blockIdx.x * W;
  const int ls = tid / kSlots, c = tid % kSlots;  // local seed, candidate slot
  const int s = s0 + ls;
  const bool in_range = s < E.n_seeds;
  const int slot = s * kSlots + c;
  const unsigned grp = 0xffu << (lane & ~7);
  const int reg = in_range ? E.region[s] : 0;
  const int ev = in_range ? E.seed_event[s] : 0;
  const int pickup_layer = in_range ? E.pickup_layer[s] : -1;
  const int* lb = E.layer_begin + ev * E.lb_stride;
  const int n_local = min(W, E.n_seeds - s0);

  S.upd[tid] = 0;
  if (tid == 0) S.n_pairs = 0;
  __syncthreads();

  for (int step = 1; step <= C.max_steps; ++step) {
    //-------------------------------------------------------------- prep
    int layer = -1, state = kFinished, ncand = 0, buf = 0;
    if (in_range) {
      layer = plan_layer(C, reg, step);
      state = wake_seed(C, reg, layer, step, E.state[s], pickup_layer);
      ncand = E.n_cands[s];
      buf = E.cur[s];
    }
    const CandSoA& B = E.cand[buf];
    float par[6], err[21];
    int chg = 0;
    const bool active = in_range && layer >= 0 && state == kFinding && c < ncand &&
                        activate_cand(E, B, s, slot, layer, C.looper_stop != 0, par, err, chg);
    const unsigned act = __ballot_sync(0xffffffffu, active) & grp;
    {
      const unsigned all = __ballot_sync(0xffffffffu, active);
      if (lane == 0 && all) atomicAdd(&E.work[step * kWorkN + 0], __popc(all));
    }
    if (in_range && c == 0) {
      if (layer >= 0 && state == kFinding && act == 0) state = kFinished;
      E.state[s] = state;
    }
    const int rbase = ls * kRecPerSeed + c * kRecPerCand;
    PrepOut o;
    if (active) {
      const LayerDev& L = C.layer[layer];
      prep_cand(E, C, L, E.bins + (size_t)ev * E.n_bins + L.bin_offset, lb[layer], reg, layer, s,
                B, slot, par, err, chg, S.xhit + tid, T, o);
      if (o.extra == 2) S.extra_last[tid] = o.extra_last;
#pragma unroll
      for (int e = 0; e < 6; ++e) S.ppar[e * T + tid] = o.ppar[e];
#pragma unroll
      for (int e = 0; e < 21; ++e) S.perr[e * T + tid] = o.perr[e];
      if (o.xs > 0) {
        const int base = atomicAdd(&S.n_pairs, o.xs);
        for (int h = 0; h < o.xs; ++h) S.pairs[base + h] = (unsigned short)(tid * kMaxXHits + h);
      }
    }
    if (o.hole) S.rec[rbase + kMaxXHits] = Record{o.hole_hit, -1, 0.f, o.hole_score};
    S.rmask[tid] = o.hole ? 1u << kMaxXHits : 0u;
    S.wsr[tid] = o.wsr | (o.extra << 8);
    __syncthreads();

    //-------------------------------------------------------------- chi2
    const int np = S.n_pairs;
    if (tid == 0 && np) {
      atomicAdd(&E.pair_count[step], np);
      atomicAdd(&E.work[step * kWorkN + 2], np);
    }
    for (int p = tid; p < np; p += T) {
      const int code = S.pairs[p];
      const int lt = code / kMaxXHits, h = code % kMaxXHits;
      const int pls = lt / kSlots, pc = lt % kSlots;
      const int ps = s0 + pls, pslot = ps * kSlots + pc;
      const int player = plan_layer(C, E.region[ps], step);
      const LayerDev& L = C.layer[player];
      float ppar[6], perr[21];
#pragma unroll
      for (int e = 0; e < 6; ++e) ppar[e] = S.ppar[e * T + lt];
#pragma unroll
      for (int e = 0; e < 21; ++e) perr[e] = S.perr[e * T + lt];
      const CandSoA& PB = E.cand[E.cur[ps]];
      const int hidx = S.xhit[h * T + lt];
      const int g = E.layer_begin[E.seed_event[ps] * E.lb_stride + player] + hidx;
      float chi2, score;
      int module;
      const int r = pls * kRecPerSeed + pc * kRecPerCand + h;
      if (eval_pair(E, C, L, player, ps, g, ppar, perr, PB.chg[pslot], PB.nfound[pslot],
                    PB.nover[pslot], PB.ninside[pslot] + PB.ntail[pslot], PB.chi2[pslot], chi2,
                    score, module)) {
        S.rec[r] = Record{hidx, module, chi2, score};
        atomicOr(S.rmask + lt, 1u << h);
      }
    }
    __syncthreads();

    //-------------------------------------------------------------- clone
    if (tid == 0) S.n_pairs = 0;
    for (int wl = warp; wl < n_local; wl += T / 32) {
      const int ws = s0 + wl;
      const int wlayer = plan_layer(C, E.region[ws], step);
      if (wlayer < 0) continue;
      const int wstate = E.state[ws];
      if (wstate != kFinding) continue;
      const int cur = E.cur[ws];
      if (lane == 0) atomicAdd(&E.work[step * kWorkN + 3], 1);
      const int rb = wl * kRecPerSeed;
      const SeedRecords R{S.rec + rb, S.rmask + wl * kSlots, S.wsr + wl * kSlots,
                          S.extra_last + wl * kSlots, S.upd + wl * kSlots};
      int upd = 0;
      const int n = clone_seed(E, C, ws, wlayer, wstate, E.n_cands[ws], cur, R, S.hm[warp],
                               S.scratch[warp], upd, lane);
      if (n >= 0 && lane == 0) {
        E.n_cands[ws] = n;
        E.cur[ws] = cur ^ 1;
      }
      __syncwarp();
    }
    __syncthreads();

    //-------------------------------------------------------------- update
    if (in_range && layer >= 0 && c < E.n_cands[s] && S.upd[tid]) {
      S.upd[tid] = 0;
      atomicAdd(&E.work[step * kWorkN + 1], 1);
      update_cand(E, C, s, lb, E.cand[E.cur[s]], slot);
    }
    // A seed can still change if it is dormant (it may wake up) or finding
    // with layers left in its plan.
    bool live = false;
    if (in_range && c == 0)
      live = state == kDormant || (state == kFinding && plan_layer(C, reg, step + 1) >= 0);
    if (!__syncthreads_or(live)) break;
  }

  //---------------------------------------------------------------- merge
  if (tid < n_local) {
    const int ms = s0 + tid;
    const int cur = E.cur[ms];
    bool moved = true;
    E.n_cands[ms] = merge_seed(E, C, ms, E.n_cands[ms], cur, moved);
    if (moved) E.cur[ms] = cur ^ 1;
  }
}

}  // namespace mkfg
