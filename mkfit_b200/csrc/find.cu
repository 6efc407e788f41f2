// Clone-engine combinatorial track finding: device kernels and C ABI.
//
// Plain form (the drop-in for MkBuilder::FindTracksCloneEngine,
// mkFit/MkBuilder.cc:1847-2058): for every layer-plan step, five launches
//   1. activate : seed activation, candidate unroll + low-pT looper stop,
//                 compact list of the active candidates (one thread per
//                 candidate slot; barrel and endcap candidates listed apart)
//   2. propagate: propagation to the layer, SelectHitIndices, missed-layer
//                 handling, hole records (one thread per active candidate)
//   3. chi2     : propagate to each selected hit, chi2, strip checks,
//                 hit records (one thread per (cand, hit) pair)
//   4. clone    : per-seed ranking of the records (warp top-M selection),
//                 overlap hits, extras, best short candidate, new
//                 candidates (one warp per seed) -- CandCloner::ProcessSeedRange
//   5. update   : UpdateWithLastHit for the listed candidates that took a hit
//                 (barrel and endcap candidates listed apart)
// then one merge launch (MergeCandsAndBestShortOne) and one export launch.
#include "internal.h"
#include "find_host.h"
#include "find_fused.cuh"
#include "layer_hits.cuh"
#include "find_steps.cuh"
#include "seed_import.cuh"
#include "quality.cuh"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <thread>
#include <vector>

namespace mkfg {

constexpr int kBlock = 256;
// Minimum resident blocks per SM requested for the heavy per-candidate
// kernels (propagate, chi2, update): trades registers for occupancy.
#ifndef MKFG_HEAVY_MIN_BLOCKS
#define MKFG_HEAVY_MIN_BLOCKS 2
#endif
// The propagation kernel gains from 4 (64 registers, a few spilled to L1;
// measured on the 64-event batch: 18.98 vs 20.06 ms per step; 3 and 5 give
// 5.74 and 5.55 ms against 5.25 ms for the kernel). The chi2 kernel gains
// from 3 (2.45 vs 2.71 ms per step); update stays at 2.
#ifndef MKFG_PROP_MIN_BLOCKS
#define MKFG_PROP_MIN_BLOCKS 4
#endif
#ifndef MKFG_CHI2_MIN_BLOCKS
#define MKFG_CHI2_MIN_BLOCKS 3
#endif
#ifndef MKFG_UPD_MIN_BLOCKS
#define MKFG_UPD_MIN_BLOCKS MKFG_HEAVY_MIN_BLOCKS
#endif
// The activation kernel at full occupancy (32 registers): 18.90 vs 19.07 ms.
#ifndef MKFG_ACT_MIN_BLOCKS
#define MKFG_ACT_MIN_BLOCKS 8
#endif
// The same for the clone kernel (one warp per seed, latency bound: the
// full 64 warps per SM pay for the few registers spilled to L1).
#ifndef MKFG_CLONE_MIN_BLOCKS
#define MKFG_CLONE_MIN_BLOCKS 8
#endif


// Appends `value` for the lanes where `want` holds to a two-ended list:
// barrel entries from the front (counter cnt[0]), endcap entries from the
// back (counter cnt[1]). One atomic per warp and end; all lanes call it.
__device__ __forceinline__ void append_two_ended(bool want, bool barrel, int value, int* list,
                                                 int cap, int* cnt, int lane, int value2 = 0,
                                                 int* list2 = nullptr) {
  const unsigned mb = __ballot_sync(0xffffffffu, want && barrel);
  const unsigned me = __ballot_sync(0xffffffffu, want && !barrel);
  int bb = 0, be = 0;
  if (lane == 0) {
    if (mb) bb = atomicAdd(cnt + 0, __popc(mb));
    if (me) be = atomicAdd(cnt + 1, __popc(me));
  }
  bb = __shfl_sync(0xffffffffu, bb, 0);
  be = __shfl_sync(0xffffffffu, be, 0);
  const unsigned below = (1u << lane) - 1u;
  const int at = !want ? -1 : barrel ? bb + __popc(mb & below) : cap - 1 - (be + __popc(me & below));
  if (want) {
    list[at] = value;
    if (list2) list2[at] = value2;
  }
}

// Block-aggregated forms of the appends: one atomic per block (and end)
// instead of one per warp, for lists every warp of a busy grid appends to
// (same-address atomics serialise in L2). Every thread of the block calls
// them, the same number of times: they synchronise the block.
struct BlockAppend {
  int n[kBlock / 32][2];
  int base[kBlock / 32][2];
};

__device__ __forceinline__ void append_two_ended_block(bool want, bool barrel, int value, int* list,
                                                       int cap, int* cnt, BlockAppend& sh,
                                                       int value2 = 0, int* list2 = nullptr,
                                                       int value3 = 0, int* list3 = nullptr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned mb = __ballot_sync(0xffffffffu, want && barrel);
  const unsigned me = __ballot_sync(0xffffffffu, want && !barrel);
  if (lane == 0) {
    sh.n[warp][0] = __popc(mb);
    sh.n[warp][1] = __popc(me);
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    const int end = threadIdx.x;
    int tot = 0;
    for (int w = 0; w < kBlock / 32; ++w) {
      sh.base[w][end] = tot;
      tot += sh.n[w][end];
    }
    const int b = tot ? atomicAdd(cnt + end, tot) : 0;
    for (int w = 0; w < kBlock / 32; ++w) sh.base[w][end] += b;
  }
  __syncthreads();
  const unsigned below = (1u << lane) - 1u;
  if (want) {
    const int at = barrel ? sh.base[warp][0] + __popc(mb & below)
                          : cap - 1 - (sh.base[warp][1] + __popc(me & below));
    list[at] = value;
    if (list2) list2[at] = value2;
    if (list3) list3[at] = value3;
  }
}

// Block-aggregated reservation of `count` consecutive entries of a
// two-ended list per thread: returns the thread's first position counted
// from its end (barrel: list[pos + i], endcap: list[cap - 1 - (pos + i)]).
__device__ __forceinline__ int reserve_two_ended_block(int count, bool barrel, int* cnt,
                                                       BlockAppend& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cb = barrel ? count : 0, ce = barrel ? 0 : count;
  int ib = cb, ie = ce;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int vb = __shfl_up_sync(0xffffffffu, ib, off);
    const int ve = __shfl_up_sync(0xffffffffu, ie, off);
    if (lane >= off) {
      ib += vb;
      ie += ve;
    }
  }
  if (lane == 31) {
    sh.n[warp][0] = ib;
    sh.n[warp][1] = ie;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    const int end = threadIdx.x;
    int tot = 0;
    for (int w = 0; w < kBlock / 32; ++w) {
      sh.base[w][end] = tot;
      tot += sh.n[w][end];
    }
    const int b = tot ? atomicAdd(cnt + end, tot) : 0;
    for (int w = 0; w < kBlock / 32; ++w) sh.base[w][end] += b;
  }
  __syncthreads();
  return barrel ? sh.base[warp][0] + ib - cb : sh.base[warp][1] + ie - ce;
}

// One-ended block-aggregated append (counter cnt[0]); uses sh.n[.][0] and
// sh.base[.][0] only after the block synchronises, like the two-ended form.
__device__ __forceinline__ void append_list_block(bool want, int value, int* list, int* cnt,
                                                  BlockAppend& sh) {
  append_two_ended_block(want, true, value, list, 0, cnt, sh);
}

// Warp-aggregated append of `value` for the lanes where `want` holds.
__device__ __forceinline__ void append_list(bool want, int value, int* list, int* cnt, int lane) {
  const unsigned m = __ballot_sync(0xffffffffu, want);
  if (!m) return;
  int base = 0;
  if (lane == 0) base = atomicAdd(cnt, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (want) list[base + __popc(m & ((1u << lane) - 1u))] = value;
}

//------------------------------------------------------------------------------
// Kernel 1a: activation (one thread per candidate slot, light): seed wake-up,
// unroll + looper stop, seed state, compact list of the active candidates.
//------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock, MKFG_ACT_MIN_BLOCKS) k_activate(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                     int step) {
  const FindConfigDev& C = *Cp;
  const int lane = threadIdx.x & 31;
  const unsigned grp = 0xffu << (lane & ~7);
  int* cnt = E.step_count + step * kCntN;
  // One thread per candidate slot, seeds in order (coalesced seed data).
  {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in_range = t < E.n_seeds * kSlots;
    const int s = in_range ? t / kSlots : 0, c = t % kSlots;
    int reg = 0, layer = -1, state = kFinished, ncand = 0, buf = 0;
    if (in_range) {
      reg = E.region[s];
      layer = plan_layer(C, reg, step);
      state = wake_seed(C, reg, layer, step, E.state[s], E.pickup_layer[s]);
      ncand = E.n_cands[s];
      buf = E.cur[s];
    }
    const int slot = s * kSlots + c;
    const bool active = in_range && layer >= 0 && state == kFinding && c < ncand &&
                        cand_is_active(E, E.cand[buf], s, slot, layer, C.looper_stop != 0);
    const unsigned act = __ballot_sync(0xffffffffu, active) & grp;
    const bool seed_finding = layer >= 0 && state == kFinding && act != 0;
    if (in_range && c == 0) {
      if (layer >= 0 && state == kFinding && act == 0) state = kFinished;
      E.state[s] = state;
    }
    const bool barrel = active && C.layer[layer].is_barrel;
    __shared__ BlockAppend sh;
    append_two_ended_block(active, barrel, slot, E.act_list, E.list_cap, cnt + kCntActBarrel, sh);
    // Seeds finding at this step go to the clone step.
    append_two_ended_block(in_range && c == 0 && seed_finding, true, s, E.find_list, 0,
                           cnt + kCntFind, sh, find_info_pack(buf, ncand, layer), E.find_info);
    // The clone step reads the records and extra flags of candidates
    // [0, ncand) of seeds still finding: an inactive one among them has
    // neither.
    if (seed_finding && !active && c < ncand) {
      E.rmask[slot] = 0u;
      E.wsr[slot] = kWsrOutside;
    }
  }
}

//------------------------------------------------------------------------------
// Kernel 1b: propagation to the layer, hit selection, missed-layer handling
// and hole record for the active candidates (compact list; barrel and
// endcap candidates in separate runs of the list).
//------------------------------------------------------------------------------
// Bulk copy global -> shared memory completing on an mbarrier (TMA,
// cp.async.bulk; no cluster multicast).
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bulk_to_shared(void* dst, const void* src, unsigned bytes,
                                               uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Waits for the barrier's phase `parity` to complete, at most kMaxPolls
// polls; false when it did not.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  constexpr int kMaxPolls = 1 << 22;
  for (int i = 0; i < kMaxPolls; ++i) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// kStageBins: each chunk of the active list first copies the bin table of
// its first candidate's (event, layer) into shared memory (one bulk copy
// of nq x 256 words, at most `stage_words`); the chunk's candidates on
// that (event, layer) scan the copy, the others the global table. The
// active list holds a seed's candidates together and the seeds of an
// event and region consecutively, so a chunk seldom spans two tables.
template <bool kStageBins>
__global__ void __launch_bounds__(kBlock, MKFG_PROP_MIN_BLOCKS) k_propagate(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                      int step, int stage_words) {
  const FindConfigDev& C = *Cp;
  int* cnt = E.step_count + step * kCntN;
  const int nb = cnt[kCntActBarrel], ne = cnt[kCntActEndcap];
  const int stride = E.cand[0].cap;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&E.work[step * kWorkN + 0], nb + ne);
  __shared__ BlockAppend sh;
  extern __shared__ __align__(128) uint32_t s_bins[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ int s_key;       // (event, layer) staged for this chunk, -1 none
  __shared__ int s_pending;   // a copy may still be in flight (a wait gave up)
  unsigned parity = 0;
  if (kStageBins) {
    if (threadIdx.x == 0) {
      mbar_init(&s_bar);
      s_pending = 0;
    }
    __syncthreads();
  }
  // Block-uniform loop: the pair-list reservation synchronises the block.
  for (int j0 = blockIdx.x * kBlock; j0 < nb + ne; j0 += gridDim.x * kBlock) {
    const int j = j0 + threadIdx.x;
    if (kStageBins) {
      __syncthreads();  // the previous chunk's scans are done with the copy
      if (threadIdx.x == 0) {
        int key = -1;
        if (!s_pending) {
          const int sl = j0 < nb ? E.act_list[j0] : E.act_list[E.list_cap - 1 - (j0 - nb)];
          const int ss = sl / kSlots;
          const int lay = plan_layer(C, E.region[ss], step);
          const LayerDev& SL = C.layer[lay];
          const int ev0 = E.seed_event[ss];
          if (SL.nq * 256 <= stage_words) {
            key = ev0 * kMaxLayers + lay;
            bulk_to_shared(s_bins, E.bins + (size_t)ev0 * E.n_bins + SL.bin_offset,
                           (unsigned)(SL.nq * 256 * 4), &s_bar);
          }
        }
        s_key = key;
      }
      __syncthreads();
      if (s_key >= 0) {
        const bool ok = mbar_wait(&s_bar, parity);
        parity ^= 1u;
        if (!__syncthreads_and(ok)) {
          // The copy did not complete in time: no more staging in this
          // block, the chunk reads the global table.
          if (threadIdx.x == 0) {
            atomicOr(E.err_flags, kErrStage);
            s_pending = 1;
            s_key = -1;
          }
          __syncthreads();
        }
      }
    }
    int xs = 0, slot = 0;
    bool barrel = true;
    if (j < nb + ne) {
      slot = j < nb ? E.act_list[j] : E.act_list[E.list_cap - 1 - (j - nb)];
      const int s = slot / kSlots, c = slot % kSlots;
      const int reg = E.region[s];
      const int layer = plan_layer(C, reg, step);
      const CandSoA& B = E.cand[E.cur[s]];
      float par[6], err[21];
      load_state(B, slot, par, err);
      const int chg = B.chg[slot];
      const LayerDev& L = C.layer[layer];
      const int ev = E.seed_event[s];
      const int hit0 = E.layer_begin[ev * E.lb_stride + layer];
      PrepOut o;
      const uint32_t* gbins = E.bins + (size_t)ev * E.n_bins + L.bin_offset;
      if (kStageBins)
        prep_cand<true>(E, C, L, s_key == ev * kMaxLayers + layer ? s_bins : gbins,
                        hit0, reg, layer, s, B, slot, par, err, chg, E.xhit + slot, stride, o);
      else
        prep_cand(E, C, L, gbins, hit0, reg, layer, s, B, slot, par, err, chg, E.xhit + slot,
                  stride, o);
      if (o.extra == 2) E.extra_last[slot] = o.extra_last;
#pragma unroll
      for (int e = 0; e < 6; ++e) E.ppar[e * stride + slot] = o.ppar[e];
#pragma unroll
      for (int e = 0; e < 21; ++e) E.perr[e * stride + slot] = o.perr[e];
      // The chi2 pass adds the bits of the accepted hits.
      if (o.hole)
        E.rec[(size_t)s * kRecPerSeed + c * kRecPerCand + kMaxXHits] =
            Record{o.hole_hit, -1, 0.f, o.hole_score};
      E.rmask[slot] = o.hole ? 1u << kMaxXHits : 0u;
      E.wsr[slot] = o.wsr | (o.extra << 8);
      xs = max(o.xs, 0);
      barrel = L.is_barrel;
    }
    const int base = reserve_two_ended_block(xs, barrel, cnt + kCntPairBarrel, sh);
    for (int h = 0; h < xs; ++h)
      E.pairs[barrel ? base + h : E.pair_cap - 1 - (base + h)] = slot * kMaxXHits + h;
  }
  // A copy whose wait gave up may still be writing shared memory: wait for
  // it once more (bounded) before the block exits.
  if (kStageBins && s_pending && threadIdx.x == 0) mbar_wait(&s_bar, parity ^ 1u);
}

//------------------------------------------------------------------------------
// Kernel 2: chi2 of every (candidate, selected hit) pair
// (MkFinder::FindCandidatesCloneEngine, mkFit/MkFinder.cc:1116-1240).
//------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock, MKFG_CHI2_MIN_BLOCKS) k_chi2(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                 int step) {
  const FindConfigDev& C = *Cp;
  const int* cnt = E.step_count + step * kCntN;
  const int nb = cnt[kCntPairBarrel], ne = cnt[kCntPairEndcap];
  const int n_pairs = nb + ne;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    atomicAdd(&E.work[step * kWorkN + 2], n_pairs);
    E.pair_count[step] = n_pairs;
  }
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_pairs; p += gridDim.x * blockDim.x) {
    const int code = p < nb ? E.pairs[p] : E.pairs[E.pair_cap - 1 - (p - nb)];
    const int slot = code / kMaxXHits, h = code % kMaxXHits;
    const int s = slot / kSlots, c = slot % kSlots;
    const int layer = plan_layer(C, E.region[s], step);
    const LayerDev& L = C.layer[layer];
    const int stride = E.cand[0].cap;
    float ppar[6], perr[21];
#pragma unroll
    for (int e = 0; e < 6; ++e) ppar[e] = E.ppar[e * stride + slot];
#pragma unroll
    for (int e = 0; e < 21; ++e) perr[e] = E.perr[e * stride + slot];
    const CandSoA& B = E.cand[E.cur[s]];
    const int hidx = E.xhit[h * stride + slot];
    const int g = E.layer_begin[E.seed_event[s] * E.lb_stride + layer] + hidx;
    float chi2, score;
    int module;
    const size_t r = (size_t)s * kRecPerSeed + c * kRecPerCand + h;
    if (eval_pair(E, C, L, layer, s, g, ppar, perr, B.chg[slot], B.nfound[slot], B.nover[slot],
                  B.ninside[slot] + B.ntail[slot], B.chi2[slot], chi2, score, module)) {
      E.rec[r] = Record{hidx, module, chi2, score};
      atomicOr(E.rmask + slot, 1u << h);
    }
  }
}

//------------------------------------------------------------------------------
// Kernel 3: per-seed candidate cloning (CandCloner::ProcessSeedRange,
// mkFit/CandCloner.cc:36-189). One warp per seed.
//------------------------------------------------------------------------------
// kCount: also count the records present and the new candidates (work
// counters 4 and 5). The eager launch sequence counts; the graph form, whose
// kernel sits at its register cap, does not.
template <bool kCount>
__global__ void __launch_bounds__(kBlock, MKFG_CLONE_MIN_BLOCKS) k_clone(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                  int step) {
  const FindConfigDev& C = *Cp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ HitMatchPair s_hm[kBlock / 32][kSlots];
  __shared__ CloneScratch s_scratch[kBlock / 32];
  __shared__ BlockAppend sh;
  __shared__ int s_work[2];  // records present, new candidates (this block)
  HitMatchPair* hm = s_hm[warp];
  int* cnt = E.step_count + step * kCntN;
  const int n_find = cnt[kCntFind];
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&E.work[step * kWorkN + 3], n_find);
  if (kCount) {
    if (threadIdx.x < 2) s_work[threadIdx.x] = 0;
    __syncthreads();
  }
  // Block-uniform loop (the update-list append synchronises the block):
  // warp `warp` of the block takes seed base + warp of each round.
  for (int base = blockIdx.x * (kBlock / 32); base < n_find; base += gridDim.x * (kBlock / 32)) {
    const int w = base + warp;
    int u = 0, g = 0, slot = 0, upd_info = 0;
    bool barrel = true;
    if (w < n_find) {
      // A seed finding at this step (listed by the activation kernel).
      const int s = E.find_list[w];
      const int info = E.find_info[w];
      const int cur = info & 1, ncand = (info >> 1) & 15, layer = info >> 5;
      const size_t rb = (size_t)s * kRecPerSeed;
      const int hit0 = E.layer_begin[E.seed_event[s] * E.lb_stride + layer];
      const SeedRecords R{E.rec + rb, E.rmask + s * kSlots, E.wsr + s * kSlots,
                          E.extra_last + s * kSlots, nullptr};
      int upd = 0, n_rec = 0;
      const int n = clone_seed(E, C, s, layer, kFinding, ncand, cur, R, hm, s_scratch[warp], upd,
                               lane, kCount ? &n_rec : nullptr);
      if (n >= 0 && lane == 0) {
        E.n_cands[s] = n;
        E.cur[s] = cur ^ 1;
      }
      if (kCount && lane == 0) {
        atomicAdd(s_work, n_rec);
        atomicAdd(s_work + 1, max(n, 0));
      }
      // The new candidates that take a Kalman update, with the global index
      // of the hit to update with (on this step's layer).
      slot = s * kSlots + lane;
      u = lane < n ? upd : 0;
      g = u ? hit0 + (u - 1) : 0;
      barrel = C.layer[layer].is_barrel;
      // The new candidates sit in the other buffer.
      upd_info = find_info_pack(cur ^ 1, 0, layer);
    }
    append_two_ended_block(u != 0, barrel, slot, E.upd_list, E.list_cap, cnt + kCntUpdBarrel, sh, g,
                           E.upd_hit, upd_info, E.upd_info);
    __syncwarp();  // hm and scratch are reused by the next seed of this warp
  }
  if (kCount) {
    __syncthreads();
    if (threadIdx.x < 2 && s_work[threadIdx.x])
      atomicAdd(&E.work[step * kWorkN + 4 + threadIdx.x], s_work[threadIdx.x]);
  }
}

//------------------------------------------------------------------------------
// Kernel 4: UpdateWithLastHit + CopyOutParErr for the listed candidates.
//------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock, MKFG_UPD_MIN_BLOCKS) k_update(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                   int step) {
  const FindConfigDev& C = *Cp;
  const int* cnt = E.step_count + step * kCntN;
  const int nb = cnt[kCntUpdBarrel], ne = cnt[kCntUpdEndcap];
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&E.work[step * kWorkN + 1], nb + ne);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nb + ne; j += gridDim.x * blockDim.x) {
    const int at = j < nb ? j : E.list_cap - 1 - (j - nb);
    const int slot = E.upd_list[at];
    const int info = E.upd_info[at];
    const LayerDev& L = C.layer[info >> 5];
    update_cand_at(E, C, L, E.upd_hit[at], E.cand[info & 1], slot);
  }
}

//------------------------------------------------------------------------------
// Reset: restore the imported seeds as the only candidates (the state after
// MkBuilder::find_tracks_load_seeds), so every run starts from the upload.
//------------------------------------------------------------------------------
__global__ void k_reset(EventDev E, int n_work) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n_work) E.work[t] = 0;
  if (t == 0) E.err_flags[0] = 0;
  const int s = t / kSlots, c = t % kSlots;
  if (s >= E.n_seeds) return;
  E.upd[t] = 0;
  if (c == 0) {
    copy_slot(E.init, s, E.cand[0], t);
    // A seed the upload's post-cleaning dropped (nfound < 0) has no
    // candidate and takes no part in the run.
    const bool dropped = E.init.nfound[s] < 0;
    E.n_cands[s] = dropped ? 0 : 1;
    E.state[s] = dropped ? kFinished : kDormant;
    E.cur[s] = 0;
    E.hot_size[s] = E.init_hot[s];
    E.bshort_valid[s] = 0;
    E.removed[s] = dropped ? 1 : 0;
  }
}

// Writes every seed's own hits as the first nodes of its hit-on-track
// arena (CombCandidate::ImportSeed); appends during a run start after them.
// The packed copy of the hits (EventDev::hit4), one thread per hit.
__global__ void k_pack_hits(const float* __restrict__ pos, const float* __restrict__ err,
                            int stride, int n, float4* __restrict__ out) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= n) return;
  float v[9];
#pragma unroll
  for (int k = 0; k < 3; ++k) v[k] = pos[(size_t)k * stride + h];
#pragma unroll
  for (int k = 0; k < 6; ++k) v[3 + k] = err[(size_t)k * stride + h];
  out[3 * (size_t)h] = make_float4(v[0], v[1], v[2], v[3]);
  out[3 * (size_t)h + 1] = make_float4(v[4], v[5], v[6], v[7]);
  out[3 * (size_t)h + 2] = make_float4(v[8], 0.f, 0.f, 0.f);
}

__global__ void k_seed_nodes(EventDev E, const int* __restrict__ seed_hot) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E.n_seeds) return;
  const int nhs = E.init_hot[s];
  for (int h = 0; h < nhs; ++h) {
    const size_t k = (size_t)s * E.hot_cap + h;
    E.node_hot[k] = seed_hot[MKFG_MAX_SEED_HITS * s + h];
    E.node_chi2[k] = 0.f;
    E.node_prev[k] = h - 1;
  }
}

//------------------------------------------------------------------------------
// Kernel 5: CombCandidate::MergeCandsAndBestShortOne (one thread per seed).
//------------------------------------------------------------------------------
__global__ void k_merge(EventDev E, const FindConfigDev* __restrict__ Cp) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E.n_seeds) return;
  // A region without a plan (backward search) leaves its seeds as they are.
  if (Cp->plan_len[E.region[s]] == 0) return;
  const int cur = E.cur[s];
  bool moved = true;
  E.n_cands[s] = merge_seed(E, *Cp, s, E.n_cands[s], cur, moved);
  if (moved) E.cur[s] = cur ^ 1;
}

//------------------------------------------------------------------------------
// Backward search (run_OneIteration with m_backward_search,
// mkFit/buildtestMPlex.cc:700-714): after the backward fit, every seed's best
// candidate is searched again through the plan's first layers in reverse.
// Begin: CombCandidate::CompactifyHitStorageForBestCand (without dropping
// seed hits) + BeginBkwSearch (mkFit/HitStructures.cc:554-674): one
// candidate per seed, whose "last" hit-on-track node becomes the first one
// (the seed's innermost hit, arena node 0), with its inside/tail hole counts
// saved and reset; the seed turns dormant with that node's layer as pickup.
// End: EndBkwSearch (:676-702) for the merged best candidate: the nodes added
// by the search are re-linked to follow the first node, and the forward
// chain's end and hole counts come back.
//------------------------------------------------------------------------------
struct BkSearchSave {
  int* last;
  int* ninside;
  int* ntail;
};

__global__ void k_bks_begin(EventDev E, const FindConfigDev* __restrict__ Cp, BkSearchSave V) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E.n_seeds) return;
  if (Cp->plan_len[E.region[s]] == 0 || E.n_cands[s] == 0) {
    E.state[s] = kFinished;
    V.last[s] = -1;
    return;
  }
  const CandSoA& B = E.cand[E.cur[s]];
  const int slot = s * kSlots;
  E.n_cands[s] = 1;
  V.last[s] = B.last[slot];
  V.ninside[s] = B.ninside[slot];
  V.ntail[s] = B.ntail[slot];
  B.last[slot] = 0;
  B.ninside[slot] = 0;
  B.ntail[slot] = 0;
  E.state[s] = kDormant;
  E.pickup_layer[s] = hot_layer(node_hot_of(E, s, 0));
  E.bshort_valid[s] = 0;
}

__global__ void k_bks_end(EventDev E, BkSearchSave V) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E.n_seeds || V.last[s] < 0) return;
  const CandSoA& B = E.cand[E.cur[s]];
  const int slot = s * kSlots;
  int* prev = E.node_prev + (size_t)s * E.hot_cap;
  int curr = B.last[slot];
  if (curr != 0) {
    int last = -1, p;
    // Bounded by the arena size (the chain visits each node once).
    for (int guard = 0; guard < E.hot_cap; ++guard) {
      p = prev[curr];
      prev[curr] = last;
      last = curr;
      curr = p;
      if (p == -1) break;
    }
  }
  B.last[slot] = V.last[s];
  B.ninside[slot] += V.ninside[s];
  B.ntail[slot] += V.ntail[s];
}

//------------------------------------------------------------------------------
// Backward fit of every seed's best candidate (MkBuilder::BackwardFit +
// fit_cands, mkFit/MkBuilder.cc:2153-2253; MkFinder::BkFitInputTracks /
// BkFitFitTracks / BkFitOutputTracks, mkFit/MkFinder.cc:1368-1452,
// 1573-1742). The reference fits seeds in groups of NN consecutive seeds
// (its Matriplex width) and the group's members interact: a layer where no
// member has a hit is skipped by all of them, and on a layer where some
// member has one the others are updated with a stand-in measurement at
// their own position (variance 666, no material). Here each group runs on
// `nn` lanes of a warp, which make those decisions with group ballots.
//------------------------------------------------------------------------------
struct BkFitArgs {
  const int2* groups;  // (first position, count) in the seed order below
  const int* members;  // sorted seeds left by the quality filters; NULL: all
  int n_groups;
  int nn;              // lanes per group (8 or 16)
  unsigned pflags;
  int bkfit_last[kMaxRegions];
};

__global__ void __launch_bounds__(kBlock) k_bkfit(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                  const BkFitArgs A) {
  const FindConfigDev& C = *Cp;
  const int lane = threadIdx.x & 31;
  const int per_warp = 32 / A.nn;
  const int g = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * per_warp + lane / A.nn;
  if (g >= A.n_groups) return;  // whole groups leave together
  const int k = lane % A.nn;
  const int base = lane - k;
  const unsigned gmask = (A.nn == 32 ? 0xffffffffu : ((1u << A.nn) - 1u)) << base;
  const int2 grp = A.groups[g];
  const unsigned tracks = (grp.y >= 32 ? 0xffffffffu : ((1u << grp.y) - 1u)) << base;
  const int pos = grp.x + (k < grp.y ? k : 0);
  const int s = A.members ? A.members[pos] : pos;
  const int first = A.members ? A.members[grp.x] : grp.x;
  const bool member = k < grp.y;
  const CandSoA& B = E.cand[E.cur[s]];
  const int slot = s * kSlots;
  const bool present = member && E.n_cands[s] > 0;
  float par[6], err[21];
  int chg = 1, node = -1;
  if (present) {
    load_state(B, slot, par, err);
#pragma unroll
    for (int e = 0; e < 21; ++e) err[e] *= 100.f;  // Err[iC].Scale(100)
    chg = B.chg[slot];
    node = B.last[slot];
  } else {
#pragma unroll
    for (int e = 0; e < 6; ++e) par[e] = 1.f;
#pragma unroll
    for (int e = 0; e < 21; ++e) err[e] = 1.f;
  }
  float chi2 = 0.f;
  const int reg = E.region[first];
  const int* lb = E.layer_begin + E.seed_event[first] * E.lb_stride;
  for (int li = C.plan_len[reg] - 1; li >= A.bkfit_last[reg]; --li) {
    const int layer = C.plan[reg][li];
    while (node >= 0 && hot_index(node_hot_of(E, s, node)) < 0)
      node = E.node_prev[(size_t)s * E.hot_cap + node];
    const bool done = node < 0;
    const bool here = !done && hot_layer(node_hot_of(E, s, node)) == layer;
    float mpos[3], merr[6];
    if (here) {
      // The first of the candidate's consecutive nodes on this layer (an
      // overlap hit follows the hit it pairs with).
      int prev = E.node_prev[(size_t)s * E.hot_cap + node];
      while (prev >= 0 && hot_layer(node_hot_of(E, s, prev)) == layer) {
        node = prev;
        prev = E.node_prev[(size_t)s * E.hot_cap + node];
      }
      const int gi = lb[layer] + hot_index(node_hot_of(E, s, node));
      load_hit(E, gi, mpos, merr);
      node = prev;
    } else {
      mpos[0] = par[0];
      mpos[1] = par[1];
      mpos[2] = par[2];
      merr[0] = 666.f; merr[1] = 0.f; merr[2] = 666.f;
      merr[3] = 0.f; merr[4] = 0.f; merr[5] = 666.f;
    }
    const unsigned done_m = __ballot_sync(gmask, member && done) & tracks;
    const unsigned here_m = __ballot_sync(gmask, member && here) & tracks;
    if (done_m == tracks) break;
    if (here_m == 0) continue;
    if (member) {
      const LayerDev& L = C.layer[layer];
      float ppar[6], perr[21];
      float c2;
      if (L.is_barrel) {
        propagate_to_r(par, err, chg, hypot_f(mpos[0], mpos[1]), A.pflags, C.mat, !here, ppar, perr);
        c2 = kalman_barrel<true, true>(ppar, perr, mpos, merr, par, err);
      } else {
        propagate_to_z(par, err, chg, mpos[2], A.pflags, C.mat, !here, ppar, perr);
        c2 = kalman_endcap<true, true>(ppar, perr, mpos, merr, par, err);
      }
      if (par[3] < 0) {
        chg = -chg;
        par[3] = -par[3];
      }
      chi2 += c2;
    }
  }
  if (!present) return;
  // Parameters, errors, chi2 and score go back to the candidate; the charge
  // stays as found (BkFitOutputTracks copies no charge).
  store_state(B, slot, par, err);
  B.chi2[slot] = chi2;
  if (!isnan(chi2)) B.score[slot] = cand_score(B, slot);
}

//------------------------------------------------------------------------------
// Output selection of run_OneIteration (mkFit/buildtestMPlex.cc:721-731):
// qfilter_nan_n_silly on every seed's best candidate, export of the best
// candidates without their missing hits, then duplicate removal
// (find_duplicates_sharedhits_pixelseed, mkFit/MkStdSeqs.cc:510-603: the
// variant of the iterations with m_requires_dupclean_tight). A pair's
// verdict depends only on the pair, so every pair is tested at once; of a
// duplicate pair the lower score loses (the earlier track on a tie).
//------------------------------------------------------------------------------
// Duplicate removal modes (MKFG_DUP_*): the branches of
// find_and_remove_duplicates (mkFit/MkStdSeqs.cc:605-630) and none.
enum DupMode { kDupPixelSeed = 0, kDupSharedHits = 1, kDupEtaPhi = 2, kDupNone = 3 };

struct SelectArgs {
  int* hot;       // [S][kExportHits] hits of the exported best candidate
  int* nhit;      // [S]
  float* phi;
  float* cth;     // 1 / tan(theta)
  float* ipt;
  float* eta;     // Track::momEta
  float* pt;      // Track::pT
  float* score;
  int* nfound;
  int* keep;      // [S] 1: exported and not (yet) a duplicate
  int mode;
  int algorithm;
  float frac, drth_central, drth_obarrel, drth_forward;
  float maxd1pt, maxdphi, maxdcth, maxcth_ob, maxcth_fw;
  // find_duplicates (Config::maxdPt, maxdPhi, maxdEta, maxdR,
  // minFracHitsShared, useHitsForDuplicates).
  float ep_max_dpt, ep_max_dphi, ep_max_deta, ep_max_dr, ep_min_frac;
  int ep_use_hits;
};

__global__ void k_select_prep(EventDev E, const SelectArgs A) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E.n_seeds) return;
  A.keep[s] = 0;
  A.nhit[s] = 0;
  if (E.n_cands[s] == 0) return;  // empty comb candidate: nothing exported
  const CandSoA& B = E.cand[E.cur[s]];
  const int slot = s * kSlots;
  if (silly_errors(B, slot)) return;
  // exportTrack(true): the found hits in order (TrackCand, HitStructures.cc:448-478).
  const int nfound = B.nfound[slot];
  int node = B.last[slot];
  int pos = min(nfound, kExportHits);
  for (int k = B.nfound[slot] + B.nmiss[slot] - 1; k >= 0 && node >= 0; --k) {
    const int hv = node_hot_of(E, s, node);
    if (hot_index(hv) >= 0 && pos > 0) A.hot[(size_t)s * kExportHits + (--pos)] = hv;
    node = E.node_prev[(size_t)s * E.hot_cap + node];
  }
  A.nhit[s] = min(nfound, kExportHits);
  A.phi[s] = B.par[4 * B.cap + slot];
  A.cth[s] = 1.f / f_tan(B.par[5 * B.cap + slot]);
  A.ipt[s] = B.par[3 * B.cap + slot];
  if (A.mode == kDupEtaPhi) {
    A.eta[s] = eta_of_theta(B.par[5 * B.cap + slot]);
    A.pt[s] = fabsf(1.f / B.par[3 * B.cap + slot]);
  }
  A.score[s] = B.score[slot];
  A.nfound[s] = nfound;
  A.keep[s] = 1;
}

__device__ __forceinline__ float squash_phi_minimal(float phi) {
  return phi >= kPI ? phi - kTwoPI : (phi < -kPI ? phi + kTwoPI : phi);
}

// find_duplicates (mkFit/MkStdSeqs.cc:334-423) for track i: pairs close in
// (dphi, deta), or close in 1/pT and sharing most hits, lose their
// lower-score member. Tracks of the pixelLess and tobTec algorithms (9, 10)
// mark nothing; all tracks here share one algorithm.
__device__ void select_dups_eta_phi(const EventDev& E, const SelectArgs& A, int i, int* __restrict__ dup) {
  if (A.algorithm == 9 || A.algorithm == 10) return;
  const int ev = E.seed_event[i];
  const float eta1 = A.eta[i], phi1 = A.phi[i], pt1 = A.pt[i], sc1 = A.score[i];
  const int label1 = E.seed_label[i];
  float max_dr2 = __fmul_rn(A.ep_max_dr, A.ep_max_dr);
  if (fabsf(eta1) > 2.5f) max_dr2 = __fmul_rn(max_dr2, 16.0f);
  else if (fabsf(eta1) > 1.44f) max_dr2 = __fmul_rn(max_dr2, 9.0f);
  const int* h1 = A.hot + (size_t)i * kExportHits;
  const int n1 = A.nhit[i];
  for (int j = i + 1; j < E.n_seeds && E.seed_event[j] == ev; ++j) {
    if (!A.keep[j] || E.seed_label[j] == label1) continue;
    const float deta = fabsf(__fsub_rn(A.eta[j], eta1));
    if (deta > A.ep_max_deta) continue;
    const float dphi = fabsf(squash_phi_minimal(__fsub_rn(phi1, A.phi[j])));
    if (dphi > A.ep_max_dphi) continue;
    // dphi * dphi + deta * deta, the first product fused as the reference
    // build contracts it.
    if (fmaf(dphi, dphi, __fmul_rn(deta, deta)) < max_dr2) {
      dup[sc1 > A.score[j] ? j : i] = 1;
      continue;
    }
    const float pt2 = A.pt[j];
    if (pt1 == 0.f || pt2 == 0.f) continue;
    if (!(fabsf(__fsub_rn(__fdiv_rn(1.f, pt2), __fdiv_rn(1.f, pt1))) < A.ep_max_dpt)) continue;
    if (A.ep_use_hits) {
      // Hits of track j also on track i (each of j's hits counted once).
      const int* h2 = A.hot + (size_t)j * kExportHits;
      const int n2 = A.nhit[j];
      int shared = 0;
      for (int b = 0; b < n2; ++b) {
        bool on = false;
        for (int a = 0; a < n1 && !on; ++a) on = h1[a] == h2[b];
        shared += on;
      }
      const float frac = __fdiv_rn((float)shared, (float)min(A.nfound[i], A.nfound[j]));
      if (frac < A.ep_min_frac) continue;
    }
    dup[sc1 > A.score[j] ? j : i] = 1;
  }
}

__global__ void k_select_dups(EventDev E, const SelectArgs A, int* __restrict__ dup) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= E.n_seeds || !A.keep[i] || A.mode == kDupNone) return;
  if (A.mode == kDupEtaPhi) {
    select_dups_eta_phi(E, A, i, dup);
    return;
  }
  const bool pixelseed = A.mode == kDupPixelSeed;
  const int ev = E.seed_event[i];
  const float phi1 = A.phi[i], cth1 = A.cth[i], ipt1 = A.ipt[i], sc1 = A.score[i];
  const int label1 = E.seed_label[i];
  float max_dr2 = __fmul_rn(A.drth_central, A.drth_central);
  if (fabsf(cth1) > A.maxcth_fw) max_dr2 = __fmul_rn(A.drth_forward, A.drth_forward);
  else if (fabsf(cth1) > A.maxcth_ob) max_dr2 = __fmul_rn(A.drth_obarrel, A.drth_obarrel);
  const int* h1 = A.hot + (size_t)i * kExportHits;
  const int n1 = A.nhit[i];
  for (int j = i + 1; j < E.n_seeds && E.seed_event[j] == ev; ++j) {
    if (!A.keep[j] || (pixelseed && E.seed_label[j] == label1)) continue;
    const float dcth = fabsf(__fsub_rn(A.cth[j], cth1));
    if (dcth > (pixelseed ? A.maxdcth : 1.f)) continue;
    const float dphi = fabsf(squash_phi_minimal(__fsub_rn(phi1, A.phi[j])));
    if (dphi > (pixelseed ? A.maxdphi : 1.f)) continue;
    // dphi * dphi + dcth * dcth, the first product fused as the reference
    // build contracts it.
    bool is_dup = pixelseed && fmaf(dphi, dphi, __fmul_rn(dcth, dcth)) < max_dr2;
    if (!is_dup) {
      if (pixelseed && fabsf(__fsub_rn(A.ipt[j], ipt1)) > A.maxd1pt) continue;
      const int* h2 = A.hot + (size_t)j * kExportHits;
      const int n2 = A.nhit[j];
      int shared = 0, shared_first = 0;
      for (int a = 0; a < n1; ++a)
        for (int b = 0; b < n2; ++b)
          if (h1[a] == h2[b]) {
            ++shared;
            if (a == 0 && b == 0) ++shared_first;
          }
      const int min_found = min(A.nfound[i], A.nfound[j]);
      is_dup = (float)(shared - shared_first) >= (float)(min_found - shared_first) * A.frac;
    }
    if (is_dup) dup[sc1 > A.score[j] ? j : i] = 1;
  }
}

//------------------------------------------------------------------------------
// Quality filter of every seed's best candidate (MkBuilder::filter_comb_cands,
// mkFit/MkBuilder.cc:279-318, with one of the StdSeq filters): the verdict
// by input seed (1 pass, 0 fail, -1 no candidate) and, with `remove`, the
// failing seeds lose their comb candidate.
//------------------------------------------------------------------------------
__global__ void k_qfilter(EventDev E, const FindConfigDev* __restrict__ Cp, const QFilterParams P,
                          int remove, int* __restrict__ pass_by_label) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E.n_seeds) return;
  int res = -1;
  if (E.n_cands[s] > 0) {
    const bool pass = qfilter_pass(E, *Cp, E.cand[E.cur[s]], s, s * kSlots, P);
    res = pass ? 1 : 0;
    if (!pass && remove) {
      E.n_cands[s] = 0;
      E.removed[s] = 1;
    }
  }
  pass_by_label[E.seed_label[s]] = res;
}

//------------------------------------------------------------------------------
// MkFinder::SelectHitIndices as a plain worker call (mkFit/MkFinder.cc:
// 227-684): for caller-given states on layer `layer` of uploaded event
// `event`, the hit window, the sensitive-region test and the first
// kMaxXHits hits of the bin scan (indices within the layer; size -1 when
// the state is outside the layer).
//------------------------------------------------------------------------------
__global__ void k_select_hit_indices(EventDev E, const FindConfigDev* __restrict__ Cp, int event,
                                     int layer, int n, const float* __restrict__ par,
                                     const float* __restrict__ err, int* __restrict__ xsize,
                                     int* __restrict__ xhits, int* __restrict__ wsr_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float p[6], e[21];
#pragma unroll
  for (int k = 0; k < 6; ++k) p[k] = par[(size_t)k * n + i];
#pragma unroll
  for (int k = 0; k < 21; ++k) e[k] = err[(size_t)k * n + i];
  const LayerDev& L = Cp->layer[layer];
  const uint32_t* bins = E.bins + (size_t)event * E.n_bins + L.bin_offset;
  const int hit_base = E.layer_begin[event * E.lb_stride + layer];
  int wsr = kWsrInside;
  const int x = select_hits(E, L, bins, hit_base, p, e, xhits + (size_t)i * kMaxXHits, 1, wsr);
  xsize[i] = x;
  if (wsr_out) wsr_out[i] = wsr;
}

//------------------------------------------------------------------------------
// MkFinder::FindCandidatesCloneEngine as a plain worker call (mkFit/
// MkFinder.cc:1116-1284): for caller-given states on layer `layer` with the
// hit lists of SelectHitIndices, the records (IdxChi2List) each candidate
// hands to the cloner, in the order it hands them: the accepted hits in
// XHitArr order, then the hole record. One thread per candidate.
//------------------------------------------------------------------------------
struct CeArgs {
  int event, layer, n;
  const float* par;      // [6][n]
  const float* err;      // [21][n]
  const int* chg;
  const int* nfound;
  const int* nover;
  const int* ninside;
  const int* ntail;
  const float* chi2;
  const int* hot_layers; // [n][3] or null
  const int* xsize;
  const int* xidx;       // [n][kMaxXHits]
  const int* wsr;
  int* n_rec;
  Record* rec;           // [n][kRecPerCand]
};

__global__ void k_ce_records(EventDev E, const FindConfigDev* __restrict__ Cp, const CeArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const FindConfigDev& C = *Cp;
  const LayerDev& L = C.layer[A.layer];
  float p[6], e[21];
#pragma unroll
  for (int k = 0; k < 6; ++k) p[k] = A.par[(size_t)k * A.n + i];
#pragma unroll
  for (int k = 0; k < 21; ++k) e[k] = A.err[(size_t)k * A.n + i];
  const int chg = A.chg[i], nf = A.nfound[i], nov = A.nover[i], nin = A.ninside[i],
            ntl = A.ntail[i];
  const float c2 = A.chi2[i];
  const int hit_base = E.layer_begin[A.event * E.lb_stride + A.layer];
  Record* out = A.rec + (size_t)i * kRecPerCand;
  int k = 0;
  const int xs = min(A.xsize[i], kMaxXHits);
  for (int h = 0; h < xs; ++h) {
    const int hidx = A.xidx[(size_t)i * kMaxXHits + h];
    float chi2;
    int module;
    bool ok = pair_accept(E, C, L, hit_base + hidx, p, e, chg, chi2, module);
    // Pixel same-layer check on the comb candidate's first three nodes
    // (MkFinder.cc:1195-1210), from the layers the caller gives.
    if (ok && L.is_pix && A.hot_layers)
      for (int j = 0; j <= nf && j <= 2; ++j)
        if (A.hot_layers[(size_t)i * 3 + j] == A.layer) ok = false;
    if (!ok) continue;
    out[k++] = Record{hidx, module, chi2, hit_record_score(p, nf, nov, nin + ntl, c2, chi2)};
  }
  // The hole record (MkFinder.cc:1245-1283) unless the state is outside the
  // layer; -7 (inactive module) is not produced: no module is inactive.
  const int w = A.wsr[i];
  if (w != kWsrOutside) {
    int fake = ((nin + ntl) < C.max_holes && ntl < C.max_consec_holes) ? -1 : -2;
    if (w == kWsrEdge) fake = -3;
    const int ntail_rec = fake == -1 ? ntl + 1 : ntl;
    out[k++] = Record{fake, -1, 0.f, score_struct(nf, ntail_rec, nov, nin, c2, fabsf(1.0f / p[3]))};
  }
  A.n_rec[i] = k;
}

//------------------------------------------------------------------------------
// MkFinder::UpdateWithLastHit + CopyOutParErr as a plain worker call
// (mkFit/MkFinder.cc:1291-1335): caller-given states updated with one hit
// each of layer `layer` (index within the layer). One thread per state.
//------------------------------------------------------------------------------
__global__ void k_update_last_hit(EventDev E, const FindConfigDev* __restrict__ Cp, int event,
                                  int layer, int n, const int* __restrict__ hit,
                                  float* __restrict__ par, float* __restrict__ err,
                                  int* __restrict__ chg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const FindConfigDev& C = *Cp;
  float p[6], e[21];
#pragma unroll
  for (int k = 0; k < 6; ++k) p[k] = par[(size_t)k * n + i];
#pragma unroll
  for (int k = 0; k < 21; ++k) e[k] = err[(size_t)k * n + i];
  int q = chg[i];
  update_state(E, C, C.layer[layer], E.layer_begin[event * E.lb_stride + layer] + hit[i], p, e, q);
#pragma unroll
  for (int k = 0; k < 6; ++k) par[(size_t)k * n + i] = p[k];
#pragma unroll
  for (int k = 0; k < 21; ++k) err[(size_t)k * n + i] = e[k];
  chg[i] = q;
}

//------------------------------------------------------------------------------
// CandCloner::ProcessSeedRange as a plain worker call (mkFit/CandCloner.cc:
// 36-189): the clone step of the graph form (clone_seed) run on
// caller-given candidates and records held in a private EventDev. One warp
// per seed.
//------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_clone_worker(EventDev W, const FindConfigDev* __restrict__ Cp,
                                                         int layer, int* __restrict__ n_new,
                                                         int* __restrict__ parent) {
  const FindConfigDev& C = *Cp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __shared__ HitMatchPair s_hm[kBlock / 32][kSlots];
  __shared__ CloneScratch s_scratch[kBlock / 32];
  const int s = blockIdx.x * (kBlock / 32) + warp;
  if (s >= W.n_seeds) return;
  const SeedRecords R{W.rec + (size_t)s * kRecPerSeed, W.rmask + s * kSlots, W.wsr + s * kSlots,
                      W.extra_last + s * kSlots, W.upd + s * kSlots};
  int upd = 0;
  const int n = clone_seed(W, C, s, layer, kFinding, W.n_cands[s], 0, R, s_hm[warp], s_scratch[warp],
                           upd, lane, nullptr, parent + s * kSlots);
  if (lane == 0) n_new[s] = n;
}

__global__ void k_select_out(EventDev E, const SelectArgs A, const int* __restrict__ dup,
                             int* __restrict__ keep_by_label) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E.n_seeds) return;
  keep_by_label[E.seed_label[s]] = A.keep[s] && !dup[s];
}

//------------------------------------------------------------------------------
// Kernel 6: export (TrackCand::exportTrack, mkFit/HitStructures.cc:448-478).
//------------------------------------------------------------------------------
struct FindOutDev {
  int* n_cands;
  int* region;
  float* par;
  float* err;
  int* chg;
  float* chi2;
  float* score;
  int* nfound;
  int* ntot;
  int* noverlap;
  int* ninside;
  int* ntail;
  int* hit_idx;
  int* hit_lyr;
  int m;  // output slots per seed
};

__global__ void k_export(EventDev E, FindOutDev O) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = t / kSlots, c = t % kSlots;
  if (s >= E.n_seeds || c >= O.m) return;
  const int label = E.seed_label[s];
  const int n = E.n_cands[s];
  if (c == 0) {
    O.n_cands[label] = min(n, O.m);
    O.region[label] = E.region[s];
  }
  const int o = label * O.m + c;
  if (c >= n) {
    // Unused slot: defined contents (zeros, empty hit list).
    for (int e = 0; e < 6; ++e) O.par[o * 6 + e] = 0.f;
    for (int e = 0; e < 21; ++e) O.err[o * 21 + e] = 0.f;
    O.chg[o] = 0;
    O.chi2[o] = 0.f;
    O.score[o] = 0.f;
    O.nfound[o] = O.ntot[o] = O.noverlap[o] = O.ninside[o] = O.ntail[o] = 0;
    for (int k = 0; k < kExportHits; ++k) {
      O.hit_idx[o * kExportHits + k] = -100;
      O.hit_lyr[o * kExportHits + k] = -100;
    }
    return;
  }
  const CandSoA& B = E.cand[E.cur[s]];
  const int slot = s * kSlots + c;
  // Every value is loaded before the first store, so the loads are in
  // flight together (the output arrays may alias them as far as the
  // compiler knows).
  float par[6], err[21];
  load_state(B, slot, par, err);
  const int chg = B.chg[slot], nfound = B.nfound[slot], nmiss = B.nmiss[slot];
  const int nover = B.nover[slot], ninside = B.ninside[slot], ntail = B.ntail[slot];
  const float chi2 = B.chi2[slot], score = B.score[slot];
  int node = B.last[slot];
#pragma unroll
  for (int e = 0; e < 6; ++e) O.par[o * 6 + e] = par[e];
#pragma unroll
  for (int e = 0; e < 21; ++e) O.err[o * 21 + e] = err[e];
  O.chg[o] = chg;
  O.chi2[o] = chi2;
  O.score[o] = score;
  O.nfound[o] = nfound;
  const int ntot = nfound + nmiss;
  O.ntot[o] = ntot;
  O.noverlap[o] = nover;
  O.ninside[o] = ninside;
  O.ntail[o] = ntail;
  for (int k = kExportHits - 1; k >= 0; --k) {
    O.hit_idx[o * kExportHits + k] = -100;
    O.hit_lyr[o * kExportHits + k] = -100;
  }
  for (int k = ntot - 1; k >= 0; --k) {
    const int hv = node_hot_of(E, s, node);
    if (k < kExportHits) {
      O.hit_idx[o * kExportHits + k] = hot_index(hv);
      O.hit_lyr[o * kExportHits + k] = hot_layer(hv);
    }
    node = E.node_prev[(size_t)s * E.hot_cap + node];
    if (node < 0) break;
  }
}

//------------------------------------------------------------------------------
// Host side
//------------------------------------------------------------------------------
struct Finder {
  bool configured = false;
  FindConfigDev host_cfg;
  FindConfigDev* d_cfg = nullptr;
  std::vector<LayerBinning> binning;
  std::vector<float> layer_desc;  // n_layers x LC_COUNT
  int n_bins = 0;
  // Event device memory (grow-only arenas).
  DevBuf hits, seeds, cands, scratch, recs, arena, outb;
  EventDev ev{};
  int n_seeds = 0;
  int n_events = 0;
  int events_loaded = 0;
  cudaGraphExec_t graph = nullptr;  // captured run sequence
  // The device view the graph was captured with: an upload that leaves it
  // unchanged (same seed count, same buffers) replays the same graph.
  EventDev graph_ev{};
  int fused_w = 16;                 // seeds per block of the fused form
  int max_nq = 1;                   // largest number of q bins of a layer
  // Layer steps a backward search can take (the longest plan less its
  // first entry); per-step buffers and the hit-on-track arena hold a
  // forward run plus a backward search of that length.
  int bks_steps = 0;
  bool sort_seed_hits = false;  // IterationConfig::m_requires_seed_hit_sorting
  int arena_cap = 0;            // hit-on-track nodes per seed; 0 = sized for the plans
  int64_t last_chi2_evals = 0, last_seeds_cloned = 0, last_records = 0, last_new_cands = 0;
  // Per-launch device times of the last timed run: [max_steps][5] for the
  // layer-step kernels (activate, propagate, chi2, clone, update).
  std::vector<float> last_step_ms;
  // Resident blocks (all SMs) of propagate, chi2, clone, update; 0 = not
  // yet queried.
  int resident[4] = {0, 0, 0, 0};
  // Host copies for the backward fit's seed groups: region of every sorted
  // seed and the first sorted seed of every event.
  std::vector<int> h_region;
  std::vector<int> h_seed_off;
  std::vector<int> h_hit_off;
  DevBuf bk;  // backward-fit seed groups
  DevBuf bks;  // backward-search saved counts
  FindConfigDev* d_cfg_bks = nullptr;  // backward-search plans
  float* d_mat = nullptr;  // material map (radiation lengths, then xi) taken at setup
  DevBuf sel;  // output selection scratch
  DevBuf wrk;  // staging of the per-layer worker calls
  DevBuf seed_raw;  // the batch's seeds as given, for the device seed import
  // Seed import on the host (partition, sort and initial candidates by the
  // upload's worker threads) instead of on the device.
  bool seed_import_host = false;
  // Bin tables staged in shared memory by the propagation kernel.
  bool stage_bins = false;
  // Grids of the list-driven kernels (propagate, chi2, clone, update) as
  // multiples of their resident blocks on the device; tuned by
  // mkfg_find_autotune_graph.
  int grid_mult[4] = {4, 1, 2, 4};
  // Global index of every uploaded event's layer starts ([n_events][L + 1]),
  // for checking the hit indices the worker calls are given.
  std::vector<int> h_lb;
  // Hits of layer `layer` of uploaded event `event`.
  int layer_size(int event, int layer) const {
    const size_t o = (size_t)event * (host_cfg.n_layers + 1) + layer;
    return h_lb[o + 1] - h_lb[o];
  }
  // A quality filter removed comb candidates since the upload (the device
  // flags in ev.removed, cleared by every run, say which).
  bool filter_removed = false;
  HostBuf hits_h;  // pinned mirror of the hits buffer for the upload
  HostBuf seeds_h; // pinned staging of the initial candidates for the upload
  HostBuf outb_h;  // pinned mirror of the export buffer for the download
  void drop_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
};

namespace {

Finder* finder_of(mkfg_context* ctx) {
  if (!ctx->finder) ctx->finder = new Finder;
  return static_cast<Finder*>(ctx->finder);
}

template <typename T>
T* carve(char*& p, size_t n) {
  T* r = reinterpret_cast<T*>(p);
  p += ((n * sizeof(T) + 255) / 256) * 256;
  return r;
}
size_t rounded(size_t bytes) { return ((bytes + 255) / 256) * 256; }

}  // namespace

void finder_release(mkfg_context* ctx) {
  if (!ctx || !ctx->finder) return;
  Finder* f = static_cast<Finder*>(ctx->finder);
  if (f->d_cfg) cudaFree(f->d_cfg);
  if (f->d_cfg_bks) cudaFree(f->d_cfg_bks);
  if (f->d_mat) cudaFree(f->d_mat);
  f->bks.release();
  f->drop_graph();
  f->bk.release();
  f->sel.release();
  f->wrk.release();
  f->seed_raw.release();
  f->hits_h.release();
  f->outb_h.release();
  f->seeds_h.release();
  f->hits.release();
  f->seeds.release();
  f->cands.release();
  f->scratch.release();
  f->recs.release();
  f->arena.release();
  f->outb.release();
  delete f;
  ctx->finder = nullptr;
}

}  // namespace mkfg

using namespace mkfg;

extern "C" int mkfg_finder_setup(mkfg_context* ctx, const mkfg_find_config* cfg) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(cfg && cfg->layer_desc && cfg->plans && cfg->plan_len && cfg->pickup,
               "null finder configuration");
  MKFG_REQUIRE(cfg->n_layers > 0 && cfg->n_layers <= kMaxLayers, "n_layers out of range");
  MKFG_REQUIRE(cfg->n_regions > 0 && cfg->n_regions <= kMaxRegions, "n_regions out of range");
  MKFG_REQUIRE(cfg->max_plan > 0 && cfg->max_plan <= kMaxPlan, "max_plan out of range");
  MKFG_REQUIRE(cfg->max_cands_per_seed >= 1 && cfg->max_cands_per_seed <= kSlots,
               "max_cands_per_seed must be in [1, %d]", kSlots);
  MKFG_REQUIRE(cfg->sort_seed_hits == 0 || cfg->sort_seed_hits == 1, "sort_seed_hits must be 0 or 1");
  MKFG_REQUIRE(cfg->requires_prop_to_hit == 1,
               "only the propagate-to-hit finding mode (CMS geometries) is implemented");
  Finder* f = finder_of(ctx);
  FindConfigDev& H = f->host_cfg;
  std::memset(&H, 0, sizeof(H));
  f->layer_desc.assign(cfg->layer_desc, cfg->layer_desc + (size_t)cfg->n_layers * LC_COUNT);
  f->binning.resize(cfg->n_layers);
  int off = 0;
  for (int l = 0; l < cfg->n_layers; ++l) {
    const float* d = cfg->layer_desc + (size_t)l * LC_COUNT;
    LayerBinning b = setup_layer_binning(d);
    b.bin_offset = off;
    off += b.nq * kPhiBins;
    f->binning[l] = b;
    LayerDev& L = H.layer[l];
    L.rin = d[LC_RIN];
    L.rout = d[LC_ROUT];
    L.zmin = d[LC_ZMIN];
    L.zmax = d[LC_ZMAX];
    L.propagate_to = d[LC_PROPAGATE_TO];
    L.hole_min = d[LC_HOLE_MIN];
    L.hole_max = d[LC_HOLE_MAX];
    L.min_dphi = d[LC_MIN_DPHI];
    L.max_dphi = d[LC_MAX_DPHI];
    L.min_dq = d[LC_MIN_DQ];
    L.max_dq = d[LC_MAX_DQ];
    L.c_dp_sf = d[LC_C_DP_SF]; L.c_dp_0 = d[LC_C_DP_0]; L.c_dp_1 = d[LC_C_DP_1]; L.c_dp_2 = d[LC_C_DP_2];
    L.c_dq_sf = d[LC_C_DQ_SF]; L.c_dq_0 = d[LC_C_DQ_0]; L.c_dq_1 = d[LC_C_DQ_1]; L.c_dq_2 = d[LC_C_DQ_2];
    L.c_c2_sf = d[LC_C_C2_SF]; L.c_c2_0 = d[LC_C_C2_0]; L.c_c2_1 = d[LC_C_C2_1]; L.c_c2_2 = d[LC_C_C2_2];
    L.qmin = b.qmin;
    L.fq = b.fq;
    L.nq = b.nq;
    L.bin_offset = b.bin_offset;
    L.is_barrel = b.barrel;
    L.has_hole = d[LC_HAS_HOLE] > 0.5f;
    L.is_pix = d[LC_IS_PIX] > 0.5f;
    L.is_stereo = d[LC_IS_STEREO] > 0.5f;
  }
  f->n_bins = off;
  f->max_nq = 1;
  for (const auto& b : f->binning) f->max_nq = std::max(f->max_nq, b.nq);
  MKFG_REQUIRE(hits_smem_bytes(f->max_nq) <= 200 * 1024,
               "a layer has %d q bins; the device hit-index build supports up to %d",
               f->max_nq, 200 * 1024 / (2 * kFineStride));
  H.n_layers = cfg->n_layers;
  H.n_regions = cfg->n_regions;
  int max_steps = 0;
  f->bks_steps = 0;
  f->sort_seed_hits = cfg->sort_seed_hits != 0;
  for (int r = 0; r < cfg->n_regions; ++r) {
    H.plan_len[r] = cfg->plan_len[r];
    H.pickup[r] = cfg->pickup[r];
    MKFG_REQUIRE(cfg->plan_len[r] <= kMaxPlan && cfg->pickup[r] >= 0 &&
                     cfg->pickup[r] < std::max(1, cfg->plan_len[r]),
                 "bad plan for region %d", r);
    for (int i = 0; i < cfg->plan_len[r]; ++i) {
      const int l = cfg->plans[r * cfg->max_plan + i];
      MKFG_REQUIRE(l >= 0 && l < cfg->n_layers, "plan layer out of range");
      H.plan[r][i] = l;
    }
    max_steps = std::max(max_steps, cfg->plan_len[r] - cfg->pickup[r] - 1);
    f->bks_steps = std::max(f->bks_steps, cfg->plan_len[r] - 1);
  }
  H.max_steps = max_steps;
  H.max_cands = cfg->max_cands_per_seed;
  H.max_holes = cfg->max_holes_per_cand;
  H.max_consec_holes = cfg->max_consec_holes;
  H.chi2_cut_min = cfg->chi2_cut_min;
  H.chi2_cut_overlap = cfg->chi2_cut_overlap;
  H.pt_cut_overlap = cfg->pt_cut_overlap;
  H.inter_pflags = cfg->inter_layer_pflags;
  H.intra_pflags = cfg->intra_layer_pflags;
  // The finder keeps its own copy of the context's material map: a later
  // mkfg_set_material (a fit on another detector through the same context)
  // does not change what the finding propagates through.
  const size_t mat_n = (size_t)kMatNZ * kMatNR;
  if (!f->d_mat) MKFG_CUDA_TRY(cudaMalloc(&f->d_mat, 2 * mat_n * sizeof(float)));
  MKFG_CUDA_TRY(cudaMemcpyAsync(f->d_mat, ctx->d_rl, mat_n * sizeof(float), cudaMemcpyDeviceToDevice,
                                ctx->stream));
  MKFG_CUDA_TRY(cudaMemcpyAsync(f->d_mat + mat_n, ctx->d_xi, mat_n * sizeof(float),
                                cudaMemcpyDeviceToDevice, ctx->stream));
  H.mat = Material{f->d_mat, f->d_mat + mat_n};
  H.looper_stop = 1;
  if (!f->d_cfg) MKFG_CUDA_TRY(cudaMalloc(&f->d_cfg, sizeof(FindConfigDev)));
  MKFG_CUDA_TRY(cudaMemcpyAsync(f->d_cfg, &H, sizeof(H), cudaMemcpyHostToDevice, ctx->stream));
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  f->configured = true;
  // Buffers, launch sequence and graph follow the configuration: the next
  // run needs a new upload.
  f->drop_graph();
  f->events_loaded = 0;
  return MKFG_OK;
}

namespace mkfg {

// Host preparation + upload of a batch of events (one event for the plain
// drop-in form) into the finder's device buffers. Hits and seeds of all
// events are laid out back to back; every seed knows its event.
// Row width of an event's seed-hit arrays (0 means 4).
static int seed_hit_stride(const mkfg_event* ev) { return ev->seed_hit_stride ? ev->seed_hit_stride : 4; }


// Track::sortHitsByLayer (Track.cc:241-245: a stable sort by layer) of every
// seed of `ev` into hl / hi ([n_seeds][sw], like the event's own rows).
static void sort_seed_hits_by_layer(const mkfg_event* ev, int sw, std::vector<int32_t>& hl,
                                    std::vector<int32_t>& hi) {
  hl.assign(ev->seed_hit_layer, ev->seed_hit_layer + (size_t)ev->n_seeds * sw);
  hi.assign(ev->seed_hit_index, ev->seed_hit_index + (size_t)ev->n_seeds * sw);
  std::vector<std::pair<int32_t, int32_t>> hs;
  for (int i = 0; i < ev->n_seeds; ++i) {
    const int nhs = ev->seed_nhits[i];
    hs.clear();
    for (int h = 0; h < nhs; ++h) hs.emplace_back(hl[(size_t)i * sw + h], hi[(size_t)i * sw + h]);
    std::stable_sort(hs.begin(), hs.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (int h = 0; h < nhs; ++h) {
      hl[(size_t)i * sw + h] = hs[h].first;
      hi[(size_t)i * sw + h] = hs[h].second;
    }
  }
}

static int upload_batch(mkfg_context* ctx, Finder* f, const mkfg_event* evs, int n_ev) {
  const int L = f->host_cfg.n_layers;
  MKFG_REQUIRE(n_ev >= 1, "empty batch");
  std::vector<int> hit_off(n_ev + 1, 0), seed_off(n_ev + 1, 0);
  for (int e = 0; e < n_ev; ++e) {
    const mkfg_event* ev = evs + e;
    MKFG_REQUIRE(ev->n_layers == L, "event %d has %d layers, configuration %d", e, ev->n_layers, L);
    for (int l = 0; l < L; ++l)
      MKFG_REQUIRE(ev->layer_begin[l + 1] - ev->layer_begin[l] <= 65535,
                   "event %d layer %d holds more than 65535 hits", e, l);
    const int sw = seed_hit_stride(ev);
    MKFG_REQUIRE(sw >= 1 && sw <= MKFG_MAX_SEED_HITS, "event %d: seed_hit_stride %d", e, sw);
    for (int s = 0; s < ev->n_seeds; ++s) {
      MKFG_REQUIRE(ev->seed_nhits[s] >= 1 && ev->seed_nhits[s] <= sw, "seed %d hit count", s);
      // A seed's hits become hit-on-track nodes that the backward fit
      // reads: a hit index (>= 0) must name a hit of its layer.
      for (int h = 0; h < ev->seed_nhits[s]; ++h) {
        const int hl = ev->seed_hit_layer[(size_t)s * sw + h], hi = ev->seed_hit_index[(size_t)s * sw + h];
        if (hi < 0) continue;
        MKFG_REQUIRE(hl >= 0 && hl < L && hi < ev->layer_begin[hl + 1] - ev->layer_begin[hl],
                     "event %d seed %d hit %d: index %d on layer %d is not a hit of the layer", e, s,
                     h, hi, hl);
      }
    }
    hit_off[e + 1] = hit_off[e] + ev->layer_begin[L];
    seed_off[e + 1] = seed_off[e] + ev->n_seeds;
  }
  const int NH = hit_off[n_ev], S = seed_off[n_ev];
  // Work-list entries pack (candidate slot, hit) into 32-bit integers:
  // seed count * 8 slots * 16 hits must stay below 2^31.
  MKFG_REQUIRE(S <= (1 << 24), "%d seeds in the batch; at most %d", S, 1 << 24);
  const int nb = f->n_bins;

  // Hits go to the device in one copy from a pinned host mirror: positions,
  // errors, module ids, charges and layer offsets, which every event's
  // worker writes; the hit index (module info, bin table, sorted (q, phi)
  // and ranks) is then built on the device (layer_hits.cuh).
  const int NHs = std::max(NH, 1);
  const size_t n_lb = (size_t)(L + 1) * n_ev, n_bins_all = (size_t)nb * n_ev;
  bool any_mask = false;
  for (int e = 0; e < n_ev; ++e) any_mask |= evs[e].hit_mask != nullptr;
  const size_t up_bytes = rounded(12 * (size_t)NHs) + rounded(24 * (size_t)NHs) +
                          2 * rounded(4 * (size_t)NHs) + rounded(4 * n_lb) + rounded((size_t)NHs);
  const size_t hit_bytes = up_bytes + rounded(4 * (size_t)NHs) + rounded(4 * n_bins_all) +
                           rounded(16 * (size_t)NHs) + rounded(48 * (size_t)NHs);
  int rc;
  if ((rc = f->hits.ensure(hit_bytes))) return rc;
  if ((rc = f->hits_h.ensure(up_bytes))) return rc;
  struct HitsLayout {
    float* pos;
    float* err;
    int* detid;
    int* cpcm;
    int* lb;
    uint8_t* mask;  // hits masked by earlier iterations (1 = skip)
    uint32_t* info;
    uint32_t* bins;
    SortedHit* sorted;
    float4* hit4;
  };
  auto layout = [&](char* p, bool device) {
    HitsLayout h{};
    h.pos = carve<float>(p, 3 * (size_t)NHs);
    h.err = carve<float>(p, 6 * (size_t)NHs);
    h.detid = carve<int>(p, NHs);
    h.cpcm = carve<int>(p, NHs);
    h.lb = carve<int>(p, n_lb);
    h.mask = carve<uint8_t>(p, NHs);
    if (device) {
      h.info = carve<uint32_t>(p, NHs);
      h.bins = carve<uint32_t>(p, n_bins_all);
      h.sorted = carve<SortedHit>(p, NHs);
      h.hit4 = carve<float4>(p, 3 * (size_t)NHs);
    }
    return h;
  };
  const HitsLayout hh = layout(static_cast<char*>(f->hits_h.ptr), false);
  const HitsLayout dh = layout(f->hits.as<char>(), true);

  // Initial candidates (CombCandidate::ImportSeed, mkFit/HitStructures.cc:
  // 483-509), staged in pinned memory by the per-event workers: each
  // event's seeds in sorted order, one initial candidate per seed, and the
  // seed's hits as its first hit-on-track nodes (at most MKFG_MAX_SEED_HITS).
  const int SS = std::max(S, 1);
  struct SeedStage {
    float* par;    // [6][SS]
    float* err;    // [21][SS]
    float* score;
    int* chg;
    int* last;
    int* nfound;
    int* nmiss;
    int* ninside;
    int* ntail;
    int* label;
    int* sev;
    int* region;
    int* pickup;
    int* hot_size;
    int* seed_hot;  // [SS][MKFG_MAX_SEED_HITS]
  };
  // The device imports the seeds (seed_import.cuh) unless the iteration
  // sorts seed hits on the host first, an event holds more seeds than the
  // device sort takes, or the host path was asked for.
  // The device reads each seed's last hit (its eta sets the order): a seed
  // whose last hit is not one of the event's hits keeps the upload on the
  // host path, which handles it as before.
  bool dev_import = !f->seed_import_host && !f->sort_seed_hits && S > 0;
  for (int e = 0; e < n_ev && dev_import; ++e) {
    const mkfg_event* ev = evs + e;
    dev_import &= ev->n_seeds <= kSeedSortMax;
    const int sw = seed_hit_stride(ev);
    for (int k = 0; k < ev->n_seeds && dev_import; ++k) {
      const int last = ev->seed_nhits[k] - 1;
      const int hl = ev->seed_hit_layer[(size_t)k * sw + last], hi = ev->seed_hit_index[(size_t)k * sw + last];
      dev_import &= hl >= 0 && hl < L && hi >= 0 && hi < ev->layer_begin[hl + 1] - ev->layer_begin[hl];
    }
  }
  if ((rc = f->seeds_h.ensure(rounded(4 * (size_t)SS) * (27 + 14 + 2 * MKFG_MAX_SEED_HITS) +
                              rounded(4 * (size_t)(n_ev + 1)) + 4096)))
    return rc;
  // Raw seeds for the device import, in the same pinned buffer.
  struct RawStage {
    float* par;   // [6][SS]
    float* err;   // [21][SS]
    int* chg;
    int* nhits;
    int* hl;      // [SS][MKFG_MAX_SEED_HITS]
    int* hi;
    int* seed_off;
  } rs{};
  size_t raw_bytes = 0;
  if (dev_import) {
    char* p = static_cast<char*>(f->seeds_h.ptr);
    rs.par = carve<float>(p, 6 * (size_t)SS);
    rs.err = carve<float>(p, 21 * (size_t)SS);
    rs.chg = carve<int>(p, SS);
    rs.nhits = carve<int>(p, SS);
    rs.hl = carve<int>(p, MKFG_MAX_SEED_HITS * (size_t)SS);
    rs.hi = carve<int>(p, MKFG_MAX_SEED_HITS * (size_t)SS);
    rs.seed_off = carve<int>(p, n_ev + 1);
    raw_bytes = (size_t)(p - static_cast<char*>(f->seeds_h.ptr));
    for (int e = 0; e <= n_ev; ++e) rs.seed_off[e] = seed_off[e];
  }
  SeedStage ss;
  if (!dev_import) {
    char* p = static_cast<char*>(f->seeds_h.ptr);
    ss.par = carve<float>(p, 6 * (size_t)SS);
    ss.err = carve<float>(p, 21 * (size_t)SS);
    ss.score = carve<float>(p, SS);
    ss.chg = carve<int>(p, SS);
    ss.last = carve<int>(p, SS);
    ss.nfound = carve<int>(p, SS);
    ss.nmiss = carve<int>(p, SS);
    ss.ninside = carve<int>(p, SS);
    ss.ntail = carve<int>(p, SS);
    ss.label = carve<int>(p, SS);
    ss.sev = carve<int>(p, SS);
    ss.region = carve<int>(p, SS);
    ss.pickup = carve<int>(p, SS);
    ss.hot_size = carve<int>(p, SS);
    ss.seed_hot = carve<int>(p, MKFG_MAX_SEED_HITS * (size_t)SS);
  }

  // Per-event host work (seed order and initial candidates; hit copies into
  // the pinned mirror), in parallel.
  std::vector<SeedOrder> orders(n_ev);
  std::vector<int> n_silly(n_ev, 0);
  {
    auto work = [&](int e) {
      const mkfg_event* ev = evs + e;
      const int nh = ev->layer_begin[L], o = hit_off[e];
      const int sw = seed_hit_stride(ev);
      const int32_t* seed_hl = ev->seed_hit_layer;
      const int32_t* seed_hi = ev->seed_hit_index;
      std::vector<int32_t> sorted_hl, sorted_hi;
      if (f->sort_seed_hits) {
        sort_seed_hits_by_layer(ev, sw, sorted_hl, sorted_hi);
        seed_hl = sorted_hl.data();
        seed_hi = sorted_hi.data();
      }
      if (!dev_import) {
        SeedInput si{ev->n_seeds, ev->seed_par, ev->seed_chg, ev->seed_nhits, seed_hl, seed_hi, sw};
        partition_seeds_cms2017(f->layer_desc.data(), L, si, ev->layer_begin, ev->pos, nh,
                                orders[e]);
      }
      for (int r = 0; r < 3; ++r)
        std::memcpy(hh.pos + (size_t)r * NHs + o, ev->pos + (size_t)r * nh, 4 * (size_t)nh);
      for (int r = 0; r < 6; ++r)
        std::memcpy(hh.err + (size_t)r * NHs + o, ev->err + (size_t)r * nh, 4 * (size_t)nh);
      std::memcpy(hh.detid + o, ev->detid, 4 * (size_t)nh);
      std::memcpy(hh.cpcm + o, ev->cpcm, 4 * (size_t)nh);
      if (any_mask) {
        if (ev->hit_mask)
          std::memcpy(hh.mask + o, ev->hit_mask, (size_t)nh);
        else
          std::memset(hh.mask + o, 0, (size_t)nh);
      }
      for (int l = 0; l <= L; ++l) hh.lb[(size_t)e * (L + 1) + l] = o + ev->layer_begin[l];
      const int n = ev->n_seeds;
      if (dev_import) {
        // The seeds as given; partition, order and initial candidates are
        // made on the device.
        const size_t so = seed_off[e];
        for (int c = 0; c < 6; ++c)
          std::memcpy(rs.par + c * (size_t)SS + so, ev->seed_par + (size_t)c * n, 4 * (size_t)n);
        for (int c = 0; c < 21; ++c)
          std::memcpy(rs.err + c * (size_t)SS + so, ev->seed_err + (size_t)c * n, 4 * (size_t)n);
        std::memcpy(rs.chg + so, ev->seed_chg, 4 * (size_t)n);
        std::memcpy(rs.nhits + so, ev->seed_nhits, 4 * (size_t)n);
        for (int k = 0; k < n; ++k)
          for (int h = 0; h < MKFG_MAX_SEED_HITS; ++h) {
            const bool in = h < sw;
            rs.hl[(so + k) * MKFG_MAX_SEED_HITS + h] = in ? seed_hl[(size_t)k * sw + h] : 0;
            rs.hi[(so + k) * MKFG_MAX_SEED_HITS + h] = in ? seed_hi[(size_t)k * sw + h] : 0;
          }
        return;
      }
      for (int k = 0; k < n; ++k) {
        const int s = seed_off[e] + k;
        const int i = orders[e].order[k];
        ss.label[s] = seed_off[e] + i;
        ss.sev[s] = e;
        ss.region[s] = orders[e].region[i];
        const int nhs = ev->seed_nhits[i];
        ss.pickup[s] = seed_hl[i * sw + nhs - 1];
        for (int c = 0; c < 6; ++c) ss.par[c * (size_t)SS + s] = ev->seed_par[c * n + i];
        for (int c = 0; c < 21; ++c) ss.err[c * (size_t)SS + s] = ev->seed_err[c * n + i];
        ss.chg[s] = ev->seed_chg[i];
        int nf = 0, nm = 0, nin = 0, ntl = 0;
        for (int h = 0; h < MKFG_MAX_SEED_HITS; ++h) {
          if (h >= nhs) {
            ss.seed_hot[MKFG_MAX_SEED_HITS * (size_t)s + h] = 0;
            continue;
          }
          const int hi = seed_hi[i * sw + h], hl = seed_hl[i * sw + h];
          ss.seed_hot[MKFG_MAX_SEED_HITS * (size_t)s + h] = (hi & 0xffffff) | (hl << 24);
          if (hi >= 0 || hi == -9) {
            ++nf;
            nin += ntl;
            ntl = 0;
          } else {
            ++nm;
            if (hi == -1) ++ntl;
          }
        }
        ss.hot_size[s] = nhs;
        ss.last[s] = nhs - 1;
        // MkBuilder::seed_post_cleaning (mkFit/MkBuilder.cc:1151-1198, run
        // by run_OneIteration before the seeds are loaded): a seed whose
        // covariance has a negative diagonal or a non-finite element is
        // dropped. nfound = -1 marks it; the per-run reset leaves it without
        // a candidate.
        bool silly = false;
        for (int a = 0, c = 0; a < 6; ++a)
          for (int b = 0; b <= a; ++b, ++c) {
            const float v = ev->seed_err[c * n + i];
            if ((a == b && v < 0.f) || !std::isfinite(v)) silly = true;
          }
        if (silly) {
          nf = -1;
          n_silly[e] += 1;
        }
        ss.nfound[s] = nf;
        ss.nmiss[s] = nm;
        ss.ninside[s] = nin;
        ss.ntail[s] = ntl;
        // getScoreCand(cand) with default arguments (mkFit/HitStructures.h:519-531).
        const float pt = std::abs(1.f / ss.par[3 * (size_t)SS + s]);
        float bonus = 0.2f * nf + 4.0f, penalty = 8.0f;
        if (pt < 0.9f) {
          penalty *= 1.5f;
          bonus = std::min(bonus * 1.0f, 8.0f);
        }
        ss.score[s] = bonus * nf + 0.0f * 0 - penalty * nin - 3.0f * 0 - 0.0f;
      }
    };
    // The calling thread issues the hit copies as the events' workers
    // finish, so the transfers overlap the host copies.
    cudaStream_t st = ctx->stream;
    std::vector<std::atomic<int>> ready(n_ev);
    for (auto& r : ready) r.store(0);
    const int nthr = std::max(1, std::min(n_ev, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    std::atomic<int> next(0);
    for (int t = 0; t < nthr; ++t)
      pool.emplace_back([&] {
        for (int e = next++; e < n_ev; e = next++) {
          work(e);
          ready[e].store(1, std::memory_order_release);
        }
      });
    char* hbase = static_cast<char*>(f->hits_h.ptr);
    char* dbase = f->hits.as<char>();
    cudaError_t ce = cudaSuccess;
    auto copy_rows = [&](const void* h0, size_t row_stride, int rows, size_t off, size_t bytes) {
      for (int r = 0; r < rows && ce == cudaSuccess && bytes; ++r) {
        const char* h = static_cast<const char*>(h0) + r * row_stride + off;
        ce = cudaMemcpyAsync(dbase + (h - hbase), h, bytes, cudaMemcpyHostToDevice, st);
      }
    };
    // Events' hits are consecutive in every row of the mirror: each run of
    // events that became ready goes in one copy per row (at least
    // kCopyEvents events a time but the last), so few large transfers
    // follow the workers.
    constexpr int kCopyEvents = 8;
    for (int e0 = 0; e0 < n_ev;) {
      int e1 = e0;
      while (e1 < n_ev && (e1 - e0 < kCopyEvents || ready[e1].load(std::memory_order_acquire))) {
        while (!ready[e1].load(std::memory_order_acquire)) std::this_thread::yield();
        ++e1;
      }
      const size_t o = 4 * (size_t)hit_off[e0], nb = 4 * (size_t)(hit_off[e1] - hit_off[e0]);
      copy_rows(hh.pos, 4 * (size_t)NHs, 3, o, nb);
      copy_rows(hh.err, 4 * (size_t)NHs, 6, o, nb);
      copy_rows(hh.detid, 0, 1, o, nb);
      copy_rows(hh.cpcm, 0, 1, o, nb);
      if (any_mask) copy_rows(hh.mask, 0, 1, o / 4, nb / 4);
      e0 = e1;
    }
    for (auto& th : pool) th.join();
    copy_rows(hh.lb, 0, 1, 0, 4 * n_lb);
    if (ce != cudaSuccess) return set_error(MKFG_ERR_CUDA, "hit upload: %s", cudaGetErrorString(ce));
  }

  cudaStream_t st = ctx->stream;
  auto up = [&](void* d, const void* h, size_t bytes) -> int {
    if (bytes == 0) return MKFG_OK;
    MKFG_CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
    return MKFG_OK;
  };
  {
    LayerHitsArgs A;
    A.pos = dh.pos;
    A.hstride = NHs;
    A.detid = dh.detid;
    A.cpcm = dh.cpcm;
    A.layer_begin = dh.lb;
    A.lb_stride = L + 1;
    A.n_layers = L;
    A.hinfo = dh.info;
    A.bins = dh.bins;
    A.n_bins = nb;
    A.sorted = dh.sorted;
    A.mask = any_mask ? dh.mask : nullptr;
    const int smem = hits_smem_bytes(f->max_nq);
    MKFG_CUDA_TRY(cudaFuncSetAttribute(k_layer_hits, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_layer_hits<<<n_ev * L, kHitsBlock, smem, st>>>(A, f->d_cfg);
    MKFG_CUDA_TRY(cudaGetLastError());
  }
  if (NH > 0) k_pack_hits<<<(NH + 255) / 256, 256, 0, st>>>(dh.pos, dh.err, NHs, NH, dh.hit4);
  MKFG_CUDA_TRY(cudaGetLastError());
  f->ev.hpos = dh.pos;
  f->ev.herr = dh.err;
  f->ev.hit4 = dh.hit4;
  f->ev.hstride = NHs;
  f->ev.hinfo = dh.info;
  f->ev.layer_begin = dh.lb;
  f->ev.lb_stride = L + 1;
  f->ev.n_bins = nb;
  f->ev.bins = dh.bins;
  f->ev.sorted_hits = dh.sorted;
  // ---- seeds, candidates, scratch, records, arena
  const int SC = SS * kSlots;
  // Per-step buffers cover the forward run or a backward search, whichever
  // is longer; the arena holds both (the search appends to the run's nodes).
  const int max_steps = std::max(f->host_cfg.max_steps, f->bks_steps);
  const int M = f->host_cfg.max_cands;
  const int hot_cap_auto =
      ((MKFG_MAX_SEED_HITS + 4 + (f->host_cfg.max_steps + f->bks_steps) * (2 * M + 3)) + 31) / 32 * 32;
  const int hot_cap = f->arena_cap > 0 ? std::min(f->arena_cap, hot_cap_auto) : hot_cap_auto;
  {
    const size_t need = 3 * rounded(4 * (size_t)SC) * 37 + rounded(4 * (size_t)SS) * 47 + 4096;
    if ((rc = f->cands.ensure(need))) return rc;
    char* p = f->cands.as<char>();
    auto mk = [&](int cap) {
      CandSoA b;
      b.cap = cap;
      b.par = carve<float>(p, 6 * (size_t)cap);
      b.err = carve<float>(p, 21 * (size_t)cap);
      b.chg = carve<int>(p, cap);
      b.chi2 = carve<float>(p, cap);
      b.score = carve<float>(p, cap);
      b.last = carve<int>(p, cap);
      b.nfound = carve<int>(p, cap);
      b.nmiss = carve<int>(p, cap);
      b.nover = carve<int>(p, cap);
      b.ninside = carve<int>(p, cap);
      b.ntail = carve<int>(p, cap);
      return b;
    };
    f->ev.cand[0] = mk(SC);
    f->ev.cand[1] = mk(SC);
    f->ev.init = mk(SS);
    f->ev.bshort = mk(SS);
    f->ev.init_hot = carve<int>(p, SS);
    f->ev.seed_label = carve<int>(p, SS);
    f->ev.seed_event = carve<int>(p, SS);
    f->ev.region = carve<int>(p, SS);
    f->ev.pickup_layer = carve<int>(p, SS);
    f->ev.state = carve<int>(p, SS);
    f->ev.n_cands = carve<int>(p, SS);
    f->ev.cur = carve<int>(p, SS);
    f->ev.hot_size = carve<int>(p, SS);
    f->ev.bshort_valid = carve<int>(p, SS);
    f->ev.removed = carve<int>(p, SS);
  }
  {
    const size_t need = rounded(4 * (size_t)SC) * (27 + 10) + 2 * rounded(4 * (size_t)SC * kMaxXHits) +
                        rounded(4 * (size_t)(max_steps + 2)) * (1 + kWorkN + kCntN) + rounded(64) + 8192;
    if ((rc = f->scratch.ensure(need))) return rc;
    char* p = f->scratch.as<char>();
    f->ev.ppar = carve<float>(p, 6 * (size_t)SC);
    f->ev.perr = carve<float>(p, 21 * (size_t)SC);
    f->ev.xhit = carve<int>(p, (size_t)kMaxXHits * SC);
    f->ev.wsr = carve<int>(p, SC);
    f->ev.extra_last = carve<int>(p, SC);
    f->ev.upd = carve<int>(p, SC);
    f->ev.pairs = carve<int>(p, (size_t)SC * kMaxXHits);
    f->ev.pair_cap = SC * kMaxXHits;
    f->ev.pair_count = carve<int>(p, max_steps + 2);
    f->ev.act_list = carve<int>(p, SC);
    f->ev.upd_list = carve<int>(p, SC);
    f->ev.upd_hit = carve<int>(p, SC);
    f->ev.upd_info = carve<int>(p, SC);
    f->ev.find_list = carve<int>(p, SS);
    f->ev.find_info = carve<int>(p, SS);
    f->ev.list_cap = SC;
    f->ev.step_count = carve<int>(p, (size_t)kCntN * (max_steps + 2));
    f->ev.err_flags = carve<int>(p, 16);
    f->ev.work = carve<int>(p, kWorkN * (size_t)(max_steps + 2));
  }
  {
    const size_t nrec = (size_t)SS * kRecPerSeed;
    if ((rc = f->recs.ensure(rounded(sizeof(Record) * nrec) + rounded(4 * (size_t)SC) + 4096)))
      return rc;
    char* p = f->recs.as<char>();
    f->ev.rec = carve<Record>(p, nrec);
    f->ev.rmask = carve<uint32_t>(p, SC);
  }
  {
    const size_t nn = (size_t)SS * hot_cap;
    if ((rc = f->arena.ensure(rounded(4 * nn) * 3 + 4096))) return rc;
    char* p = f->arena.as<char>();
    f->ev.node_hot = carve<int>(p, nn);
    f->ev.node_chi2 = carve<float>(p, nn);
    f->ev.node_prev = carve<int>(p, nn);
    f->ev.hot_cap = hot_cap;
  }
  f->ev.n_seeds = S;

  // The initial candidates from the pinned staging (the per-run reset sets
  // the candidate counts, seed states and buffers from them).
  CandSoA& B0 = f->ev.init;
  std::vector<int> h_nfound;
  if ((rc = f->seeds.ensure(rounded(4 * MKFG_MAX_SEED_HITS * (size_t)SS)))) return rc;
  if (dev_import) {
    if ((rc = f->seed_raw.ensure(raw_bytes + 4 * rounded(4 * (size_t)SS) + 4096))) return rc;
    char* draw = f->seed_raw.as<char>();
    MKFG_CUDA_TRY(cudaMemcpyAsync(draw, f->seeds_h.ptr, raw_bytes, cudaMemcpyHostToDevice, st));
    auto dev = [&](const void* h) {
      return draw + (static_cast<const char*>(h) - static_cast<const char*>(f->seeds_h.ptr));
    };
    RawSeeds R;
    R.par = reinterpret_cast<const float*>(dev(rs.par));
    R.err = reinterpret_cast<const float*>(dev(rs.err));
    R.chg = reinterpret_cast<const int*>(dev(rs.chg));
    R.nhits = reinterpret_cast<const int*>(dev(rs.nhits));
    R.hit_layer = reinterpret_cast<const int*>(dev(rs.hl));
    R.hit_index = reinterpret_cast<const int*>(dev(rs.hi));
    R.seed_off = reinterpret_cast<const int*>(dev(rs.seed_off));
    R.n_events = n_ev;
    R.n = S;
    char* q = draw + raw_bytes;
    int* d_region = carve<int>(q, SS);
    float* d_key = carve<float>(q, SS);
    int* d_event = carve<int>(q, SS);
    int* d_order = carve<int>(q, SS);
    const RegionCuts cuts = region_cuts_cms2017(f->layer_desc.data());
    k_seed_keys<<<(S + 127) / 128, 128, 0, st>>>(R, f->ev, cuts, d_region, d_key, d_event);
    MKFG_CUDA_TRY(cudaGetLastError());
    const int smem = 8 * kSeedSortMax;
    MKFG_CUDA_TRY(cudaFuncSetAttribute(k_seed_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_seed_sort<<<n_ev, kSeedSortBlock, smem, st>>>(R, d_key, d_order);
    MKFG_CUDA_TRY(cudaGetLastError());
    k_seed_import<<<(S + 127) / 128, 128, 0, st>>>(R, d_order, d_region, d_event, f->ev,
                                                   f->seeds.as<int>());
    MKFG_CUDA_TRY(cudaGetLastError());
    // The host keeps the regions (backward-fit seed groups) and the seeds
    // the post-cleaning dropped.
    f->h_region.resize(S);
    h_nfound.resize(S);
    MKFG_CUDA_TRY(cudaMemcpyAsync(f->h_region.data(), f->ev.region, 4 * (size_t)S,
                                  cudaMemcpyDeviceToHost, st));
    MKFG_CUDA_TRY(cudaMemcpyAsync(h_nfound.data(), B0.nfound, 4 * (size_t)S, cudaMemcpyDeviceToHost,
                                  st));
  } else {
  if ((rc = up(B0.par, ss.par, 4 * 6 * (size_t)SS))) return rc;
  if ((rc = up(B0.err, ss.err, 4 * 21 * (size_t)SS))) return rc;
  if ((rc = up(B0.chg, ss.chg, 4 * (size_t)SS))) return rc;
  MKFG_CUDA_TRY(cudaMemsetAsync(B0.chi2, 0, 4 * (size_t)SS, st));
  if ((rc = up(B0.score, ss.score, 4 * (size_t)SS))) return rc;
  if ((rc = up(B0.last, ss.last, 4 * (size_t)SS))) return rc;
  if ((rc = up(B0.nfound, ss.nfound, 4 * (size_t)SS))) return rc;
  if ((rc = up(B0.nmiss, ss.nmiss, 4 * (size_t)SS))) return rc;
  MKFG_CUDA_TRY(cudaMemsetAsync(B0.nover, 0, 4 * (size_t)SS, st));
  if ((rc = up(B0.ninside, ss.ninside, 4 * (size_t)SS))) return rc;
  if ((rc = up(B0.ntail, ss.ntail, 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.seed_label, ss.label, 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.seed_event, ss.sev, 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.region, ss.region, 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.pickup_layer, ss.pickup, 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.init_hot, ss.hot_size, 4 * (size_t)SS))) return rc;
  if ((rc = up(f->seeds.ptr, ss.seed_hot, 4 * MKFG_MAX_SEED_HITS * (size_t)SS))) return rc;
  }
  if (S > 0) k_seed_nodes<<<(S + 127) / 128, 128, 0, st>>>(f->ev, f->seeds.as<int>());
  MKFG_CUDA_TRY(cudaGetLastError());
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.upd, 0, 4 * (size_t)SC, st));
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.err_flags, 0, 64, st));
  // The pinned staging is reused by the next upload: wait for the copies.
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  f->n_seeds = S;
  f->n_events = n_ev;
  if (dev_import) {
    for (int e = 0; e < n_ev; ++e)
      for (int k = seed_off[e]; k < seed_off[e + 1]; ++k) n_silly[e] += h_nfound[k] < 0;
  } else {
    f->h_region.assign(ss.region, ss.region + S);
  }
  f->h_seed_off = seed_off;
  f->h_hit_off = hit_off;
  f->h_lb.assign(hh.lb, hh.lb + n_lb);
  f->events_loaded = 1;
  // Seeds dropped by the post-cleaning are absent from the backward fit's
  // seed groups, as filtered ones are.
  f->filter_removed = false;
  for (int e = 0; e < n_ev; ++e) f->filter_removed |= n_silly[e] > 0;
  return MKFG_OK;
}

// Launch grids of the plain sequence. The list-driven kernels loop over
// their lists, so their grids stop at a few waves of resident blocks:
// one for chi2 (uniform work per pair), more where the work per list entry
// varies and later waves balance the load.
struct StepGrids {
  int activate, propagate, chi2, clone, update;
};

// The propagation launch of one layer step, with the bin tables staged in
// shared memory when the finder asks for it (mkfg_find_set_bin_staging).
static cudaError_t launch_propagate(const Finder* f, int grid, cudaStream_t st,
                                    const FindConfigDev* cfg, int step) {
  if (!f->stage_bins) {
    k_propagate<false><<<grid, kBlock, 0, st>>>(f->ev, cfg, step, 0);
    return cudaGetLastError();
  }
  const int words = f->max_nq * 256;
  const size_t smem = 4 * (size_t)words;
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_propagate<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_propagate<true><<<grid, kBlock, smem, st>>>(f->ev, cfg, step, words);
  return cudaGetLastError();
}

static StepGrids step_grids(Finder* f) {
  if (!f->resident[0]) {
    int dev = 0, n_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const void* fn[4] = {(const void*)k_propagate<false>, (const void*)k_chi2, (const void*)k_clone<false>,
                         (const void*)k_update};
    for (int k = 0; k < 4; ++k) {
      int per_sm = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn[k], kBlock, 0);
      f->resident[k] = std::max(1, n_sm * std::max(per_sm, 1));
    }
  }
  const int S = f->n_seeds;
  const int grid_c = (S * kSlots + kBlock - 1) / kBlock;
  StepGrids g;
  g.activate = grid_c;
  g.propagate = std::min(grid_c, f->grid_mult[0] * f->resident[0]);
  g.chi2 = std::min((S * kSlots * 4 + kBlock - 1) / kBlock, f->grid_mult[1] * f->resident[1]);
  g.clone = std::min((S * 32 + kBlock - 1) / kBlock, f->grid_mult[2] * f->resident[2]);
  g.update = std::min(grid_c, f->grid_mult[3] * f->resident[3]);
  return g;
}

// Enqueues the whole finding sequence of the uploaded batch on `st`:
// reset, then for every layer-plan step prep -> chi2 -> clone -> update,
// then the final merge.
static int enqueue_run(Finder* f, cudaStream_t st, bool count_clone = false) {
  const int S = f->n_seeds;
  const int n_work = kWorkN * (f->host_cfg.max_steps + 2);
  const int grid_c = (S * kSlots + kBlock - 1) / kBlock;
  const StepGrids g = step_grids(f);
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.pair_count, 0, 4 * (size_t)(f->host_cfg.max_steps + 2), st));
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.step_count, 0,
                                4 * (size_t)kCntN * (f->host_cfg.max_steps + 2), st));
  k_reset<<<std::max(grid_c, (n_work + kBlock - 1) / kBlock), kBlock, 0, st>>>(f->ev, n_work);
  for (int step = 1; step <= f->host_cfg.max_steps; ++step) {
    k_activate<<<g.activate, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
    MKFG_CUDA_TRY(launch_propagate(f, g.propagate, st, f->d_cfg, step));
    k_chi2<<<g.chi2, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
    if (count_clone)
      k_clone<true><<<g.clone, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
    else
      k_clone<false><<<g.clone, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
    k_update<<<g.update, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
  }
  k_merge<<<(S + 127) / 128, 128, 0, st>>>(f->ev, f->d_cfg);
  MKFG_CUDA_TRY(cudaGetLastError());
  return MKFG_OK;
}

template <int W>
static int launch_fused(Finder* f, cudaStream_t st) {
  const int smem = (int)sizeof(FusedShared<W>);
  MKFG_CUDA_TRY(cudaFuncSetAttribute(k_find_fused<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int grid = (f->n_seeds + W - 1) / W;
  k_find_fused<W><<<grid, W * kSlots, smem, st>>>(f->ev, f->d_cfg);
  MKFG_CUDA_TRY(cudaGetLastError());
  return MKFG_OK;
}

// Reset + one fused launch (all layer steps and the merge).
static int enqueue_fused(Finder* f, cudaStream_t st, int w) {
  const int S = f->n_seeds;
  const int n_work = kWorkN * (f->host_cfg.max_steps + 2);
  const int grid_c = (S * kSlots + kBlock - 1) / kBlock;
  k_reset<<<std::max(grid_c, (n_work + kBlock - 1) / kBlock), kBlock, 0, st>>>(f->ev, n_work);
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.pair_count, 0, 4 * (size_t)(f->host_cfg.max_steps + 2), st));
  switch (w) {
    case 4: return launch_fused<4>(f, st);
    case 8: return launch_fused<8>(f, st);
    case 16: return launch_fused<16>(f, st);
    default: return set_error(MKFG_ERR_BAD_INPUT, "seeds_per_block must be 4, 8 or 16 (got %d)", w);
  }
}

// The plain sequence with an event after every launch: device time per
// kernel class (0 reset, 1 activate, 2 propagate, 3 chi2, 4 clone,
// 5 update, 6 merge), summed over the layer steps.
static int run_timed(mkfg_context* ctx, Finder* f, float* ms) {
  for (int k = 0; k < 7; ++k) ms[k] = 0.f;
  if (f->n_seeds == 0) return MKFG_OK;
  cudaStream_t st = ctx->stream;
  const int S = f->n_seeds;
  const int n_work = kWorkN * (f->host_cfg.max_steps + 2);
  const int grid_c = (S * kSlots + kBlock - 1) / kBlock;
  const StepGrids g = step_grids(f);
  const int n_ev = 2 + 5 * f->host_cfg.max_steps + 1;
  std::vector<cudaEvent_t> ev(n_ev);
  std::vector<int> cls(n_ev, -1);
  for (auto& e : ev) MKFG_CUDA_TRY(cudaEventCreate(&e));
  int i = 0;
  auto mark = [&](int c) { cls[i] = c; return cudaEventRecord(ev[i++], st); };
  int rc = MKFG_OK;
  do {
    if (mark(-1) != cudaSuccess) { rc = set_error(MKFG_ERR_CUDA, "event record"); break; }
    cudaMemsetAsync(f->ev.pair_count, 0, 4 * (size_t)(f->host_cfg.max_steps + 2), st);
    cudaMemsetAsync(f->ev.step_count, 0, 4 * (size_t)kCntN * (f->host_cfg.max_steps + 2), st);
    k_reset<<<std::max(grid_c, (n_work + kBlock - 1) / kBlock), kBlock, 0, st>>>(f->ev, n_work);
    mark(0);
    for (int step = 1; step <= f->host_cfg.max_steps; ++step) {
      k_activate<<<g.activate, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
      mark(1);
      MKFG_CUDA_TRY(launch_propagate(f, g.propagate, st, f->d_cfg, step));
      mark(2);
      k_chi2<<<g.chi2, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
      mark(3);
      k_clone<false><<<g.clone, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
      mark(4);
      k_update<<<g.update, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
      mark(5);
    }
    k_merge<<<(S + 127) / 128, 128, 0, st>>>(f->ev, f->d_cfg);
    mark(6);
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(ev[i - 1]) != cudaSuccess) {
      rc = set_error(MKFG_ERR_CUDA, "timed run failed");
      break;
    }
    f->last_step_ms.assign(5 * (size_t)f->host_cfg.max_steps, 0.f);
    for (int k = 1; k < i; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[k - 1], ev[k]);
      if (cls[k] >= 0) ms[cls[k]] += t;
      // Events 2 .. 1 + 5 max_steps close the layer-step launches.
      if (cls[k] >= 1 && cls[k] <= 5) f->last_step_ms[k - 2] = t;
    }
  } while (false);
  for (auto& e : ev) cudaEventDestroy(e);
  return rc;
}

// The eager launch sequence also fills the clone-step counters
// (mkfg_find_work_clone).
static int run_plain(mkfg_context* ctx, Finder* f) {
  if (f->n_seeds == 0) return MKFG_OK;
  return enqueue_run(f, ctx->stream, true);
}

// Same sequence captured once into a CUDA graph and replayed: one launch
// for the whole batch of events and all layer steps.
static int run_graph(mkfg_context* ctx, Finder* f) {
  if (f->n_seeds == 0) return MKFG_OK;
  cudaStream_t st = ctx->stream;
  // The launches take the device view by value: a graph captured with
  // another one is stale.
  if (f->graph && std::memcmp(&f->graph_ev, &f->ev, sizeof(EventDev)) != 0) f->drop_graph();
  if (!f->graph) {
    f->graph_ev = f->ev;
    cudaGraph_t g = nullptr;
    step_grids(f);  // occupancy queries before the capture
    MKFG_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_run(f, st);
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return set_error(MKFG_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&f->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      f->graph = nullptr;
      return set_error(MKFG_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ei));
    }
  }
  MKFG_CUDA_TRY(cudaGraphLaunch(f->graph, st));
  return MKFG_OK;
}

// Exports m_out candidate slots per seed (max_cands: all; 1: the best).
static int download(mkfg_context* ctx, Finder* f, mkfg_find_out* out, int n_seeds_in, int m_out) {
  const int S = f->n_seeds;
  const int m = m_out;
  const size_t no = (size_t)std::max(n_seeds_in, 1) * m;
  const size_t need = rounded(4 * (size_t)std::max(n_seeds_in, 1)) * 2 +
                      rounded(4 * no) * (6 + 21 + 9) + rounded(4 * no * kExportHits) * 2;
  int rc;
  if ((rc = f->outb.ensure(need))) return rc;
  char* p = f->outb.as<char>();
  FindOutDev O;
  O.m = m;
  O.n_cands = carve<int>(p, std::max(n_seeds_in, 1));
  O.region = carve<int>(p, std::max(n_seeds_in, 1));
  O.par = carve<float>(p, 6 * no);
  O.err = carve<float>(p, 21 * no);
  O.chg = carve<int>(p, no);
  O.chi2 = carve<float>(p, no);
  O.score = carve<float>(p, no);
  O.nfound = carve<int>(p, no);
  O.ntot = carve<int>(p, no);
  O.noverlap = carve<int>(p, no);
  O.ninside = carve<int>(p, no);
  O.ntail = carve<int>(p, no);
  O.hit_idx = carve<int>(p, no * kExportHits);
  O.hit_lyr = carve<int>(p, no * kExportHits);
  cudaStream_t st = ctx->stream;
  MKFG_CUDA_TRY(cudaMemsetAsync(O.n_cands, 0, 4 * (size_t)n_seeds_in, st));
  if (S > 0) k_export<<<(S * kSlots + 127) / 128, 128, 0, st>>>(f->ev, O);
  MKFG_CUDA_TRY(cudaGetLastError());
  // One device-to-host copy of the whole export into a pinned mirror, then
  // the fields the caller asked for are copied out in parallel.
  const size_t used = (size_t)(p - f->outb.as<char>());
  if ((rc = f->outb_h.ensure(used + 64))) return rc;
  char* hbase = static_cast<char*>(f->outb_h.ptr);
  MKFG_CUDA_TRY(cudaMemcpyAsync(hbase, f->outb.ptr, used, cudaMemcpyDeviceToHost, st));
  int* flags = reinterpret_cast<int*>(hbase + used);
  MKFG_CUDA_TRY(cudaMemcpyAsync(flags, f->ev.err_flags, 4, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  const size_t ns = n_seeds_in;
  struct Field {
    void* dst;
    const void* dev;
    size_t bytes;
  };
  const Field fields[] = {
      {out->n_cands, O.n_cands, 4 * ns},         {out->region, O.region, 4 * ns},
      {out->par, O.par, 4 * 6 * ns * m},         {out->err, O.err, 4 * 21 * ns * m},
      {out->chg, O.chg, 4 * ns * m},             {out->chi2, O.chi2, 4 * ns * m},
      {out->score, O.score, 4 * ns * m},         {out->nfound, O.nfound, 4 * ns * m},
      {out->ntot, O.ntot, 4 * ns * m},           {out->noverlap, O.noverlap, 4 * ns * m},
      {out->ninside, O.ninside, 4 * ns * m},     {out->ntail, O.ntail, 4 * ns * m},
      {out->hit_idx, O.hit_idx, 4 * ns * m * kExportHits},
      {out->hit_lyr, O.hit_lyr, 4 * ns * m * kExportHits}};
  // The fields in chunks of at most 4 MB, spread over the host threads.
  struct Chunk {
    char* dst;
    const char* src;
    size_t bytes;
  };
  std::vector<Chunk> chunks;
  constexpr size_t kChunk = size_t(4) << 20;
  for (const Field& fd : fields) {
    if (!fd.dst || !fd.bytes) continue;
    const char* src = hbase + (static_cast<const char*>(fd.dev) - f->outb.as<char>());
    for (size_t o = 0; o < fd.bytes; o += kChunk)
      chunks.push_back({static_cast<char*>(fd.dst) + o, src + o, std::min(kChunk, fd.bytes - o)});
  }
  const int nthr = std::max(1, std::min((int)chunks.size(), (int)std::thread::hardware_concurrency()));
  if (used > (size_t(8) << 20) && nthr > 1) {
    std::atomic<int> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nthr; ++t)
      pool.emplace_back([&] {
        for (int i = next++; i < (int)chunks.size(); i = next++)
          std::memcpy(chunks[i].dst, chunks[i].src, chunks[i].bytes);
      });
    for (auto& th : pool) th.join();
  } else {
    for (const Chunk& c : chunks) std::memcpy(c.dst, c.src, c.bytes);
  }
  const int flag_bits = *flags;
  if (flag_bits & kErrArena)
    return set_error(MKFG_ERR_OVERFLOW, "hit-on-track arena overflow (capacity %d per seed)",
                     f->ev.hot_cap);
  return MKFG_OK;
}

}  // namespace mkfg

extern "C" int mkfg_find_upload(mkfg_context* ctx, const mkfg_event* ev) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(ev != nullptr, "null event");
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured, "mkfg_finder_setup was not called");
  return upload_batch(ctx, f, ev, 1);
}

extern "C" int mkfg_find_upload_batch(mkfg_context* ctx, const mkfg_event* evs, int32_t n_events) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(evs != nullptr && n_events >= 1, "empty batch");
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured, "mkfg_finder_setup was not called");
  return upload_batch(ctx, f, evs, n_events);
}

extern "C" int mkfg_find_run(mkfg_context* ctx) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  return run_plain(ctx, f);
}

extern "C" int mkfg_find_run_graph(mkfg_context* ctx) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  return run_graph(ctx, f);
}

extern "C" int mkfg_find_run_timed(mkfg_context* ctx, float* kernel_ms) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  MKFG_REQUIRE(kernel_ms != nullptr, "null kernel_ms");
  return run_timed(ctx, f, kernel_ms);
}

extern "C" int mkfg_find_step_profile(mkfg_context* ctx, float* launch_ms, int32_t* counts) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  const int ns = f->host_cfg.max_steps;
  if (launch_ms) {
    MKFG_REQUIRE(f->last_step_ms.size() == 5 * (size_t)ns, "no timed run");
    std::memcpy(launch_ms, f->last_step_ms.data(), sizeof(float) * 5 * ns);
  }
  if (counts) {
    std::vector<int> all((size_t)kCntN * (ns + 2));
    MKFG_CUDA_TRY(cudaMemcpyAsync(all.data(), f->ev.step_count, 4 * all.size(),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int st = 1; st <= ns; ++st)
      for (int k = 0; k < 7; ++k) counts[(st - 1) * 7 + k] = all[(size_t)st * kCntN + k];
  }
  return MKFG_OK;
}

extern "C" int mkfg_find_run_fused(mkfg_context* ctx, int32_t seeds_per_block) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  if (f->n_seeds == 0) return MKFG_OK;
  return enqueue_fused(f, ctx->stream, seeds_per_block ? seeds_per_block : f->fused_w);
}

extern "C" int mkfg_find_autotune(mkfg_context* ctx, int32_t* seeds_per_block, float* ms_per_run) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  float best_ms = 0.f;
  int best_w = f->fused_w;
  if (f->n_seeds > 0) {
    cudaStream_t st = ctx->stream;
    cudaEvent_t e0, e1;
    MKFG_CUDA_TRY(cudaEventCreate(&e0));
    MKFG_CUDA_TRY(cudaEventCreate(&e1));
    best_ms = -1.f;
    for (int w : {4, 8, 16}) {
      if ((rc = enqueue_fused(f, st, w))) break;  // warm-up
      if (cudaEventRecord(e0, st) != cudaSuccess) { rc = set_error(MKFG_ERR_CUDA, "event record"); break; }
      for (int i = 0; i < 2 && !rc; ++i) rc = enqueue_fused(f, st, w);
      if (rc) break;
      if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
        rc = set_error(MKFG_ERR_CUDA, "event timing failed");
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms *= 0.5f;
      if (best_ms < 0.f || ms < best_ms) {
        best_ms = ms;
        best_w = w;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    f->fused_w = best_w;
    // Leave the outputs of a completed run of the chosen configuration.
    if ((rc = enqueue_fused(f, st, best_w))) return rc;
    MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  }
  if (seeds_per_block) *seeds_per_block = best_w;
  if (ms_per_run) *ms_per_run = best_ms;
  return MKFG_OK;
}

extern "C" int mkfg_find_set_graph_tuning(mkfg_context* ctx, const mkfg_graph_tuning* t) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(t != nullptr, "null tuning");
  for (int k = 0; k < 4; ++k)
    MKFG_REQUIRE(t->grid_mult[k] >= 1 && t->grid_mult[k] <= 64, "grid_mult[%d] = %d outside [1, 64]",
                 k, t->grid_mult[k]);
  MKFG_REQUIRE(t->stage_bins == 0 || t->stage_bins == 1, "stage_bins must be 0 or 1");
  Finder* f = finder_of(ctx);
  for (int k = 0; k < 4; ++k) f->grid_mult[k] = t->grid_mult[k];
  f->stage_bins = t->stage_bins != 0;
  f->drop_graph();
  return MKFG_OK;
}

extern "C" int mkfg_find_get_graph_tuning(mkfg_context* ctx, mkfg_graph_tuning* t) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(t != nullptr, "null tuning");
  const Finder* f = finder_of(ctx);
  for (int k = 0; k < 4; ++k) t->grid_mult[k] = f->grid_mult[k];
  t->stage_bins = f->stage_bins;
  t->ms_before = t->ms_after = 0.f;
  return MKFG_OK;
}

extern "C" int mkfg_find_autotune_graph(mkfg_context* ctx, int32_t reps, mkfg_graph_tuning* out) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  MKFG_REQUIRE(reps >= 1 && reps <= 16, "reps %d outside [1, 16]", reps);
  float ms[7];
  // Kernel times of a run (min over reps per kernel, their sum the step).
  auto measure = [&](float* best) -> int {
    for (int k = 0; k < 7; ++k) best[k] = 1e30f;
    for (int r = 0; r < reps; ++r) {
      const int e = run_timed(ctx, f, ms);
      if (e) return e;
      for (int k = 0; k < 7; ++k) best[k] = std::min(best[k], ms[k]);
    }
    return MKFG_OK;
  };
  auto total = [](const float* t) {
    float x = 0.f;
    for (int k = 0; k < 7; ++k) x += t[k];
    return x;
  };
  float cur[7];
  if ((rc = measure(cur))) return rc;  // also the warm-up
  if ((rc = measure(cur))) return rc;
  const float before = total(cur);
  // One kernel at a time: its grid multiple (its own time decides), then
  // the bin staging (the propagation kernel's time decides). Kernel
  // times index: 2 propagate, 3 chi2, 4 clone, 5 update.
  static const int kMults[] = {1, 2, 3, 4, 6, 8, 12, 16};
  for (int k = 0; k < 4; ++k) {
    const int keep = f->grid_mult[k];
    int best_m = keep;
    float best_t = cur[2 + k];
    for (int m : kMults) {
      if (m == keep) continue;
      f->grid_mult[k] = m;
      float t[7];
      if ((rc = measure(t))) return rc;
      if (t[2 + k] < best_t) {
        best_t = t[2 + k];
        best_m = m;
      }
    }
    f->grid_mult[k] = best_m;
    if ((rc = measure(cur))) return rc;
  }
  {
    const bool keep = f->stage_bins;
    f->stage_bins = !keep;
    float t[7];
    if ((rc = measure(t))) return rc;
    if (!(t[2] < cur[2])) f->stage_bins = keep;
  }
  f->drop_graph();
  if ((rc = measure(cur))) return rc;
  if (out) {
    for (int k = 0; k < 4; ++k) out->grid_mult[k] = f->grid_mult[k];
    out->stage_bins = f->stage_bins;
    out->ms_before = before;
    out->ms_after = total(cur);
  }
  return MKFG_OK;
}

extern "C" int mkfg_find_backward_search(mkfg_context* ctx, const int32_t* bksearch_pickup) {
  return mkfg_find_backward_search_with(ctx, bksearch_pickup, nullptr);
}

extern "C" int mkfg_find_backward_search_with(mkfg_context* ctx, const int32_t* bksearch_pickup,
                                              const mkfg_search_params* params) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  MKFG_REQUIRE(bksearch_pickup != nullptr, "null bksearch_pickup");
  MKFG_REQUIRE(params == nullptr ||
                   (params->max_cands_per_seed >= 1 && params->max_cands_per_seed <= kSlots),
               "max_cands_per_seed must be in [1, %d]", kSlots);
  // The backward plans: for a region with a pickup index p, the forward
  // plan's entries p, p-1, ..., 0 (SteeringParams::make_iterator with
  // IT_BkwSearch, mkFit/SteeringParams.h:140-144), entry 0 being the pickup;
  // p = -1 means no backward plan (the region's seeds are left alone).
  FindConfigDev H = f->host_cfg;
  int max_steps = 0;
  for (int r = 0; r < H.n_regions; ++r) {
    const int p = bksearch_pickup[r];
    MKFG_REQUIRE(p >= -1 && p < f->host_cfg.plan_len[r], "bksearch_pickup[%d] = %d out of range", r, p);
    H.pickup[r] = 0;
    H.plan_len[r] = p + 1;
    for (int i = 0; i <= p; ++i) H.plan[r][i] = f->host_cfg.plan[r][p - i];
    max_steps = std::max(max_steps, p);
  }
  H.max_steps = max_steps;
  H.looper_stop = 0;
  if (params) {
    // IterationConfig::m_backward_params (find_tracks_in_layers takes them
    // for IT_BkwSearch, mkFit/MkBuilder.cc:1924-1926).
    H.max_cands = params->max_cands_per_seed;
    H.max_holes = params->max_holes_per_cand;
    H.max_consec_holes = params->max_consec_holes;
    H.chi2_cut_min = params->chi2_cut_min;
    H.chi2_cut_overlap = params->chi2_cut_overlap;
    H.pt_cut_overlap = params->pt_cut_overlap;
  }
  if (!f->d_cfg_bks) MKFG_CUDA_TRY(cudaMalloc(&f->d_cfg_bks, sizeof(FindConfigDev)));
  cudaStream_t st = ctx->stream;
  MKFG_CUDA_TRY(cudaMemcpyAsync(f->d_cfg_bks, &H, sizeof(FindConfigDev), cudaMemcpyHostToDevice, st));
  const int S = f->n_seeds;
  if (S == 0) {
    MKFG_CUDA_TRY(cudaStreamSynchronize(st));
    return MKFG_OK;
  }
  if ((rc = f->bks.ensure(3 * rounded(4 * (size_t)S) + 1024))) return rc;
  BkSearchSave V;
  {
    char* p = f->bks.as<char>();
    V.last = carve<int>(p, S);
    V.ninside = carve<int>(p, S);
    V.ntail = carve<int>(p, S);
  }
  // Per-step buffers were sized for the longest plan at upload.
  MKFG_REQUIRE(max_steps <= std::max(f->host_cfg.max_steps, f->bks_steps),
               "backward plan longer than the configured plans");
  const int n_work = kWorkN * (max_steps + 2);
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.pair_count, 0, 4 * (size_t)(max_steps + 2), st));
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.step_count, 0, 4 * (size_t)kCntN * (max_steps + 2), st));
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.work, 0, 4 * (size_t)n_work, st));
  const StepGrids g = step_grids(f);
  k_bks_begin<<<(S + 127) / 128, 128, 0, st>>>(f->ev, f->d_cfg_bks, V);
  for (int step = 1; step <= max_steps; ++step) {
    k_activate<<<g.activate, kBlock, 0, st>>>(f->ev, f->d_cfg_bks, step);
    MKFG_CUDA_TRY(launch_propagate(f, g.propagate, st, f->d_cfg_bks, step));
    k_chi2<<<g.chi2, kBlock, 0, st>>>(f->ev, f->d_cfg_bks, step);
    k_clone<false><<<g.clone, kBlock, 0, st>>>(f->ev, f->d_cfg_bks, step);
    k_update<<<g.update, kBlock, 0, st>>>(f->ev, f->d_cfg_bks, step);
  }
  k_merge<<<(S + 127) / 128, 128, 0, st>>>(f->ev, f->d_cfg_bks);
  k_bks_end<<<(S + 127) / 128, 128, 0, st>>>(f->ev, V);
  MKFG_CUDA_TRY(cudaGetLastError());
  int flag_bits = 0;
  MKFG_CUDA_TRY(cudaMemcpyAsync(&flag_bits, f->ev.err_flags, 4, cudaMemcpyDeviceToHost, st));
  // H is a host stack object read by the configuration copy.
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  if (flag_bits & kErrArena)
    return set_error(MKFG_ERR_OVERFLOW, "hit-on-track arena overflow (capacity %d per seed)",
                     f->ev.hot_cap);
  return MKFG_OK;
}

extern "C" int mkfg_find_backward_fit(mkfg_context* ctx, const int32_t* bkfit_last,
                                      uint32_t pflags, int32_t group_width) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured && f->events_loaded, "no event uploaded");
  const int nn = group_width ? group_width : 8;
  MKFG_REQUIRE(nn == 8 || nn == 16, "group_width must be 8 or 16 (got %d)", group_width);
  MKFG_REQUIRE((pflags & ~3u) == 0, "unknown propagation flags 0x%x", pflags);
  BkFitArgs A{};
  A.nn = nn;
  A.pflags = pflags;
  for (int r = 0; r < f->host_cfg.n_regions; ++r) {
    A.bkfit_last[r] = bkfit_last ? bkfit_last[r] : 0;
    MKFG_REQUIRE(A.bkfit_last[r] >= 0 && A.bkfit_last[r] <= f->host_cfg.plan_len[r],
                 "bkfit_last[%d] out of range", r);
  }
  if (f->n_seeds == 0) return MKFG_OK;
  // Seed groups as MkBuilder::BackwardFit forms them: per event and eta
  // region, the region's seed range is cut into tasks with grain
  // clamp(n_seeds + 1, 4, 32) (numThreadsEvents = numThreadsFinder = 1,
  // numSeedsPerTask = 32: the reference defaults), and fit_cands fits each
  // task in groups of NN from its start. The task cut is the one of the
  // task pool the reference is built with here: ceil(n / grain) pieces of
  // near-equal size, the first n % pieces one seed longer.
  // Seeds whose comb candidate a quality filter removed are gone from the
  // reference's candidate vector (MkBuilder::filter_comb_cands keeps the
  // others in order): the groups are formed over the survivors.
  std::vector<int> members;
  bool filtered = false;
  if (f->filter_removed) {
    std::vector<int> removed(f->n_seeds);
    MKFG_CUDA_TRY(cudaMemcpyAsync(removed.data(), f->ev.removed, 4 * (size_t)f->n_seeds,
                                  cudaMemcpyDeviceToHost, ctx->stream));
    MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < f->n_seeds; ++i)
      if (!removed[i]) members.push_back(i);
    filtered = (int)members.size() != f->n_seeds;
  }
  // Position p of the seed order: members[p] when seeds were removed.
  std::vector<int> ev_off(f->h_seed_off);
  if (filtered)
    for (size_t e = 0; e < ev_off.size(); ++e)
      ev_off[e] = (int)(std::lower_bound(members.begin(), members.end(), f->h_seed_off[e]) - members.begin());
  auto seed_at = [&](int p) { return filtered ? members[p] : p; };
  std::vector<int2> groups;
  for (int e = 0; e + 1 < (int)ev_off.size(); ++e) {
    const int b = ev_off[e], end = ev_off[e + 1];
    const int grain = std::min(std::max(end - b + 1, 4), 32);
    for (int r0 = b; r0 < end;) {
      int r1 = r0;
      while (r1 < end && f->h_region[seed_at(r1)] == f->h_region[seed_at(r0)]) ++r1;
      const int n = r1 - r0;
      const int pieces = (n + grain - 1) / grain;
      const int base = n / pieces, extra = n % pieces;
      int t0 = r0;
      for (int i = 0; i < pieces; ++i) {
        const int t1 = t0 + base + (i < extra ? 1 : 0);
        for (int g0 = t0; g0 < t1; g0 += nn) groups.push_back(make_int2(g0, std::min(nn, t1 - g0)));
        t0 = t1;
      }
      r0 = r1;
    }
  }
  if (groups.empty()) return MKFG_OK;
  const size_t gbytes = rounded(groups.size() * sizeof(int2));
  if ((rc = f->bk.ensure(gbytes + 4 * members.size()))) return rc;
  MKFG_CUDA_TRY(cudaMemcpyAsync(f->bk.ptr, groups.data(), groups.size() * sizeof(int2),
                                cudaMemcpyHostToDevice, ctx->stream));
  A.groups = f->bk.as<int2>();
  A.members = nullptr;
  if (filtered) {
    int* dm = reinterpret_cast<int*>(f->bk.as<char>() + gbytes);
    MKFG_CUDA_TRY(cudaMemcpyAsync(dm, members.data(), 4 * members.size(), cudaMemcpyHostToDevice,
                                  ctx->stream));
    A.members = dm;
  }
  A.n_groups = (int)groups.size();
  const int per_block = (kBlock / 32) * (32 / nn);
  k_bkfit<<<(A.n_groups + per_block - 1) / per_block, kBlock, 0, ctx->stream>>>(f->ev, f->d_cfg, A);
  MKFG_CUDA_TRY(cudaGetLastError());
  // The group list is host memory: finish the copy before it goes away.
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return MKFG_OK;
}

extern "C" int mkfg_find_hit_index(mkfg_context* ctx, int32_t event, uint32_t* bins,
                                   int32_t* srank) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->events_loaded, "no event uploaded");
  MKFG_REQUIRE(event >= 0 && event < f->n_events, "event %d out of range", event);
  const int nh = f->h_hit_off[event + 1] - f->h_hit_off[event];
  if (bins)
    MKFG_CUDA_TRY(cudaMemcpyAsync(bins, f->ev.bins + (size_t)event * f->ev.n_bins,
                                  4 * (size_t)f->ev.n_bins, cudaMemcpyDeviceToHost, ctx->stream));
  if (srank && nh > 0)  // the rank column of the sorted hits
    MKFG_CUDA_TRY(cudaMemcpy2DAsync(srank, 4, &f->ev.sorted_hits[f->h_hit_off[event]].rank,
                                    sizeof(SortedHit), 4, nh, cudaMemcpyDeviceToHost,
                                    ctx->stream));
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return MKFG_OK;
}

extern "C" int mkfg_find_select(mkfg_context* ctx, const mkfg_select_config* cfg, int32_t n_seeds,
                                int32_t* keep) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(cfg != nullptr && keep != nullptr, "null argument");
  MKFG_REQUIRE(f->events_loaded && n_seeds == f->n_seeds, "seed count mismatch");
  const int S = f->n_seeds;
  if (S == 0) return MKFG_OK;
  MKFG_REQUIRE(cfg->mode >= 0 && cfg->mode <= MKFG_DUP_NONE, "unknown duplicate mode %d", cfg->mode);
  const size_t need = rounded(4 * (size_t)S * kExportHits) + 11 * rounded(4 * (size_t)S) + 4096;
  if ((rc = f->sel.ensure(need))) return rc;
  char* p = f->sel.as<char>();
  SelectArgs A;
  A.hot = carve<int>(p, (size_t)S * kExportHits);
  A.nhit = carve<int>(p, S);
  A.phi = carve<float>(p, S);
  A.cth = carve<float>(p, S);
  A.ipt = carve<float>(p, S);
  A.eta = carve<float>(p, S);
  A.pt = carve<float>(p, S);
  A.score = carve<float>(p, S);
  A.nfound = carve<int>(p, S);
  A.keep = carve<int>(p, S);
  int* dup = carve<int>(p, S);
  int* d_keep = carve<int>(p, S);
  A.frac = cfg->frac_shared_hits;
  A.drth_central = cfg->drth_central;
  A.drth_obarrel = cfg->drth_obarrel;
  A.drth_forward = cfg->drth_forward;
  A.maxd1pt = cfg->max_d_invpt;
  A.maxdphi = cfg->max_d_phi;
  A.maxdcth = cfg->max_d_cottheta;
  A.maxcth_ob = cfg->max_cottheta_obarrel;
  A.maxcth_fw = cfg->max_cottheta_forward;
  A.mode = cfg->mode;
  A.algorithm = cfg->algorithm;
  A.ep_max_dpt = cfg->ep_max_d_pt;
  A.ep_max_dphi = cfg->ep_max_d_phi;
  A.ep_max_deta = cfg->ep_max_d_eta;
  A.ep_max_dr = cfg->ep_max_dr;
  A.ep_min_frac = cfg->ep_min_frac_hits_shared;
  A.ep_use_hits = cfg->ep_use_hits;
  cudaStream_t st = ctx->stream;
  MKFG_CUDA_TRY(cudaMemsetAsync(dup, 0, 4 * (size_t)S, st));
  const int grid = (S + 127) / 128;
  k_select_prep<<<grid, 128, 0, st>>>(f->ev, A);
  k_select_dups<<<grid, 128, 0, st>>>(f->ev, A, dup);
  k_select_out<<<grid, 128, 0, st>>>(f->ev, A, dup, d_keep);
  MKFG_CUDA_TRY(cudaGetLastError());
  MKFG_CUDA_TRY(cudaMemcpyAsync(keep, d_keep, 4 * (size_t)S, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  return MKFG_OK;
}

extern "C" int mkfg_find_select_hit_indices(mkfg_context* ctx, int32_t event, int32_t layer, int32_t n,
                                            const float* par, const float* err, int32_t* xhit_size,
                                            int32_t* xhit_idx, int32_t* wsr) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->events_loaded, "no event uploaded");
  MKFG_REQUIRE(event >= 0 && event < f->n_events, "event %d out of range", event);
  MKFG_REQUIRE(layer >= 0 && layer < f->host_cfg.n_layers, "layer %d out of range", layer);
  MKFG_REQUIRE(n >= 0 && (n == 0 || (par && err && xhit_size && xhit_idx)), "null argument");
  if (n == 0) return MKFG_OK;
  const size_t in_bytes = rounded(4 * 27 * (size_t)n), out_bytes = rounded(4 * (size_t)n) * 2 +
                                                                  rounded(4 * (size_t)n * kMaxXHits);
  if ((rc = f->sel.ensure(in_bytes + out_bytes))) return rc;
  char* p = f->sel.as<char>();
  float* d_par = carve<float>(p, 6 * (size_t)n);
  float* d_err = carve<float>(p, 21 * (size_t)n);
  int* d_size = carve<int>(p, n);
  int* d_wsr = carve<int>(p, n);
  int* d_idx = carve<int>(p, (size_t)n * kMaxXHits);
  cudaStream_t st = ctx->stream;
  MKFG_CUDA_TRY(cudaMemcpyAsync(d_par, par, 4 * 6 * (size_t)n, cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(d_err, err, 4 * 21 * (size_t)n, cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemsetAsync(d_idx, 0xff, 4 * (size_t)n * kMaxXHits, st));
  k_select_hit_indices<<<(n + 127) / 128, 128, 0, st>>>(f->ev, f->d_cfg, event, layer, n, d_par, d_err,
                                                        d_size, d_idx, d_wsr);
  MKFG_CUDA_TRY(cudaGetLastError());
  MKFG_CUDA_TRY(cudaMemcpyAsync(xhit_size, d_size, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(xhit_idx, d_idx, 4 * (size_t)n * kMaxXHits, cudaMemcpyDeviceToHost, st));
  if (wsr) MKFG_CUDA_TRY(cudaMemcpyAsync(wsr, d_wsr, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  return MKFG_OK;
}

namespace {

// Host -> device staging of a worker call's arrays in the finder's worker
// buffer: reserve() every array first (sizes only), then ensure() once and
// put() / get() them in the same order.
struct Staging {
  Finder* f;
  cudaStream_t st;
  size_t need = 0;
  char* at = nullptr;
  int rc = MKFG_OK;
  void reserve(size_t bytes) { need += rounded(bytes); }
  char* end = nullptr;
  int ensure() {
    const size_t bytes = need + 64 * 256;  // slack for the per-array rounding
    if ((rc = f->wrk.ensure(bytes))) return rc;
    at = f->wrk.as<char>();
    end = at + bytes;
    return MKFG_OK;
  }
  template <typename T>
  T* take(size_t n) {
    const size_t bytes = rounded(n * sizeof(T));
    if (at + bytes > end) {
      if (rc == MKFG_OK) rc = set_error(MKFG_ERR_CUDA, "worker staging sized short by %zu bytes",
                                        (size_t)(at + bytes - end));
      return reinterpret_cast<T*>(f->wrk.ptr);
    }
    T* d = reinterpret_cast<T*>(at);
    at += bytes;
    return d;
  }
  template <typename T>
  T* put(const T* h, size_t n) {
    T* d = take<T>(n);
    if (rc == MKFG_OK && n) {
      const cudaError_t ce = cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, st);
      if (ce != cudaSuccess) rc = set_error(MKFG_ERR_CUDA, "worker staging: %s", cudaGetErrorString(ce));
    }
    return d;
  }
  template <typename T>
  void get(T* h, const T* d, size_t n) {
    if (rc == MKFG_OK && n) {
      const cudaError_t ce = cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, st);
      if (ce != cudaSuccess) rc = set_error(MKFG_ERR_CUDA, "worker readback: %s", cudaGetErrorString(ce));
    }
  }
};

// Common checks of the event / layer worker calls.
int check_worker(Finder* f, int event, int layer) {
  MKFG_REQUIRE(f->configured, "mkfg_finder_setup was not called");
  MKFG_REQUIRE(f->events_loaded, "no event uploaded");
  MKFG_REQUIRE(event >= 0 && event < f->n_events, "event %d out of range", event);
  MKFG_REQUIRE(layer >= 0 && layer < f->host_cfg.n_layers, "layer %d out of range", layer);
  return MKFG_OK;
}

constexpr int kWorkerHotCap = 40;  // 16 setup nodes + a best short node + 2 per new candidate

}  // namespace

extern "C" int mkfg_find_candidates_clone_engine(mkfg_context* ctx, int32_t event, int32_t layer,
                                                 int32_t n, const float* par, const float* err,
                                                 const int32_t* chg, const mkfg_cand_counts* counts,
                                                 const int32_t* seed_hot_layers,
                                                 const int32_t* xhit_size, const int32_t* xhit_idx,
                                                 const int32_t* wsr, mkfg_ce_records* out) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  if ((rc = check_worker(f, event, layer))) return rc;
  MKFG_REQUIRE(n >= 0, "negative candidate count");
  if (n == 0) return MKFG_OK;
  MKFG_REQUIRE(par && err && chg && counts && xhit_size && xhit_idx && wsr && out, "null argument");
  MKFG_REQUIRE(counts->nfound && counts->nover && counts->ninside && counts->ntail && counts->chi2,
               "null candidate counter array");
  MKFG_REQUIRE(out->n && out->hit && out->module && out->chi2 && out->score, "null record array");
  const int lsize = f->layer_size(event, layer);
  for (int i = 0; i < n; ++i) {
    MKFG_REQUIRE(xhit_size[i] <= kMaxXHits, "xhit_size[%d] = %d above %d", i, xhit_size[i], kMaxXHits);
    MKFG_REQUIRE(wsr[i] >= kWsrInside && wsr[i] <= kWsrOutside, "wsr[%d] = %d", i, wsr[i]);
    for (int h = 0; h < xhit_size[i]; ++h) {
      const int x = xhit_idx[(size_t)i * kMaxXHits + h];
      MKFG_REQUIRE(x >= 0 && x < lsize, "xhit_idx[%d][%d] = %d outside layer %d, which holds %d hits",
                   i, h, x, layer, lsize);
    }
  }
  cudaStream_t st = ctx->stream;
  Staging S{f, st};
  const size_t N = (size_t)n;
  S.reserve(4 * 27 * N);
  S.reserve(4 * 6 * N);
  if (seed_hot_layers) S.reserve(4 * 3 * N);
  S.reserve(4 * (2 + kMaxXHits) * N);
  S.reserve(4 * N + sizeof(Record) * kRecPerCand * N);
  if ((rc = S.ensure())) return rc;
  CeArgs A{};
  A.event = event;
  A.layer = layer;
  A.n = n;
  A.par = S.put(par, 6 * N);
  A.err = S.put(err, 21 * N);
  A.chg = S.put(chg, N);
  A.nfound = S.put(counts->nfound, N);
  A.nover = S.put(counts->nover, N);
  A.ninside = S.put(counts->ninside, N);
  A.ntail = S.put(counts->ntail, N);
  A.chi2 = S.put(counts->chi2, N);
  A.hot_layers = seed_hot_layers ? S.put(seed_hot_layers, 3 * N) : nullptr;
  A.xsize = S.put(xhit_size, N);
  A.xidx = S.put(xhit_idx, kMaxXHits * N);
  A.wsr = S.put(wsr, N);
  A.n_rec = S.take<int>(N);
  A.rec = S.take<Record>(kRecPerCand * N);
  if (S.rc) return S.rc;
  k_ce_records<<<(n + 127) / 128, 128, 0, st>>>(f->ev, f->d_cfg, A);
  MKFG_CUDA_TRY(cudaGetLastError());
  std::vector<Record> rec(kRecPerCand * N);
  S.get(out->n, A.n_rec, N);
  S.get(rec.data(), A.rec, rec.size());
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  if (S.rc) return S.rc;
  for (size_t i = 0; i < N; ++i)
    for (int k = 0; k < kRecPerCand; ++k) {
      const size_t j = i * kRecPerCand + k;
      const bool live = k < out->n[i];
      out->hit[j] = live ? rec[j].hit : 0;
      out->module[j] = live ? rec[j].module : 0;
      out->chi2[j] = live ? rec[j].chi2 : 0.f;
      out->score[j] = live ? rec[j].score : 0.f;
    }
  return MKFG_OK;
}

extern "C" int mkfg_find_update_with_last_hit(mkfg_context* ctx, int32_t event, int32_t layer,
                                              int32_t n, const float* par, const float* err,
                                              const int32_t* chg, const int32_t* hit_idx,
                                              float* out_par, float* out_err, int32_t* out_chg) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  if ((rc = check_worker(f, event, layer))) return rc;
  MKFG_REQUIRE(n >= 0, "negative candidate count");
  if (n == 0) return MKFG_OK;
  MKFG_REQUIRE(par && err && chg && hit_idx && out_par && out_err && out_chg, "null argument");
  const int lsize = f->layer_size(event, layer);
  for (int i = 0; i < n; ++i)
    MKFG_REQUIRE(hit_idx[i] >= 0 && hit_idx[i] < lsize,
                 "hit_idx[%d] = %d outside layer %d, which holds %d hits", i, hit_idx[i], layer, lsize);
  cudaStream_t st = ctx->stream;
  Staging S{f, st};
  const size_t N = (size_t)n;
  S.reserve(4 * 27 * N);
  S.reserve(4 * 2 * N);
  if ((rc = S.ensure())) return rc;
  float* d_par = S.put(par, 6 * N);
  float* d_err = S.put(err, 21 * N);
  int* d_chg = S.put(chg, N);
  const int* d_hit = S.put(hit_idx, N);
  if (S.rc) return S.rc;
  k_update_last_hit<<<(n + 127) / 128, 128, 0, st>>>(f->ev, f->d_cfg, event, layer, n, d_hit, d_par,
                                                     d_err, d_chg);
  MKFG_CUDA_TRY(cudaGetLastError());
  S.get(out_par, d_par, 6 * N);
  S.get(out_err, d_err, 21 * N);
  S.get(out_chg, d_chg, N);
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  return S.rc;
}

extern "C" int mkfg_find_clone_seeds(mkfg_context* ctx, int32_t layer, const mkfg_clone_in* in,
                                     mkfg_clone_out* out) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->configured, "mkfg_finder_setup was not called");
  MKFG_REQUIRE(in && out, "null argument");
  MKFG_REQUIRE(layer >= 0 && layer < f->host_cfg.n_layers, "layer %d out of range", layer);
  const int S = in->n_seeds;
  MKFG_REQUIRE(S >= 0 && S <= (1 << 24), "seed count %d out of range", S);
  if (S == 0) return MKFG_OK;
  MKFG_REQUIRE(in->n_cands && in->par && in->err && in->chg && in->chi2 && in->score && in->nfound &&
                   in->nmiss && in->nover && in->ninside && in->ntail && in->held_back && in->n_rec &&
                   in->rec_hit && in->rec_module && in->rec_chi2 && in->rec_score &&
                   in->bshort_valid && in->bshort_score,
               "null input array");
  MKFG_REQUIRE(out->n_cands && out->par && out->err && out->chg && out->chi2 && out->score &&
                   out->nfound && out->nmiss && out->nover && out->ninside && out->ntail &&
                   out->parent && out->hit && out->overlap_hit && out->update_hit &&
                   out->bshort_valid && out->bshort_score && out->bshort_nfound && out->bshort_chi2,
               "null output array");
  const int M = f->host_cfg.max_cands;
  const size_t SC = (size_t)S * kSlots;
  // Records into the graph form's layout: a candidate's hit records at
  // positions 0.. in the given order, its hole record at kMaxXHits.
  std::vector<Record> rec((size_t)S * kRecPerSeed, Record{0, 0, 0.f, 0.f});
  std::vector<uint32_t> rmask(SC, 0u);
  std::vector<int> wsr(SC, 0), extra_last(SC, -1), last(SC, 0);
  std::vector<int> node_hot((size_t)S * kWorkerHotCap, 0), node_prev((size_t)S * kWorkerHotCap, -1);
  std::vector<int> hot_size(S, 2 * kSlots);
  for (int s = 0; s < S; ++s) {
    const int nc = in->n_cands[s];
    MKFG_REQUIRE(nc >= 1 && nc <= M, "n_cands[%d] = %d outside [1, %d]", s, nc, M);
    for (int c = 0; c < kSlots; ++c) {
      const size_t k = (size_t)s * kSlots + c;
      // Setup nodes: node c ends candidate c's list; node kSlots + c is the
      // stop node of a candidate held back with one.
      last[k] = c;
      if (c >= nc) continue;
      const int hb = in->held_back[k];
      MKFG_REQUIRE(hb >= 0 && hb <= 2, "held_back[%d][%d] = %d", s, c, hb);
      wsr[k] = hb << 8;
      if (hb == 2) {
        const size_t node = (size_t)s * kWorkerHotCap + kSlots + c;
        node_hot[node] = (-2 & 0xffffff) | (layer << 24);
        node_prev[node] = c;
        extra_last[k] = kSlots + c;
      }
      const int nr = in->n_rec[k];
      MKFG_REQUIRE(nr >= 0 && nr <= kRecPerCand, "n_rec[%d][%d] = %d", s, c, nr);
      int nh = 0, nholes = 0;
      for (int j = 0; j < nr; ++j) {
        const size_t src = k * kRecPerCand + j;
        const int hit = in->rec_hit[src];
        int pos;
        if (hit >= 0) {
          MKFG_REQUIRE(nh < kMaxXHits, "seed %d candidate %d: more than %d hit records", s, c, kMaxXHits);
          pos = nh++;
        } else {
          MKFG_REQUIRE(hit == -1 || hit == -2 || hit == -3,
                       "seed %d candidate %d: record hit %d is neither a hit nor a hole code", s, c, hit);
          MKFG_REQUIRE(nholes == 0, "seed %d candidate %d: more than one hole record", s, c);
          ++nholes;
          pos = kMaxXHits;
        }
        rec[(size_t)s * kRecPerSeed + c * kRecPerCand + pos] =
            Record{hit, in->rec_module[src], in->rec_chi2[src], in->rec_score[src]};
        rmask[k] |= 1u << pos;
      }
    }
  }
  cudaStream_t st = ctx->stream;
  Staging St{f, st};
  St.reserve(4 * 27 * SC * 2);           // par / err, both buffers
  St.reserve(4 * 11 * SC);               // counters and scores, input buffer
  St.reserve(4 * 11 * SC);               // output buffer
  St.reserve(4 * 27 * (size_t)S + 4 * 12 * (size_t)S);  // best short candidate
  St.reserve(4 * 3 * (size_t)S * kWorkerHotCap + 4 * (size_t)S * 4);
  St.reserve(sizeof(Record) * rec.size() + 4 * 6 * SC + 64);
  if ((rc = St.ensure())) return rc;
  auto cand_view = [&](size_t cap) {
    CandSoA c{};
    c.par = St.take<float>(6 * cap);
    c.err = St.take<float>(21 * cap);
    c.chg = St.take<int>(cap);
    c.chi2 = St.take<float>(cap);
    c.score = St.take<float>(cap);
    c.last = St.take<int>(cap);
    c.nfound = St.take<int>(cap);
    c.nmiss = St.take<int>(cap);
    c.nover = St.take<int>(cap);
    c.ninside = St.take<int>(cap);
    c.ntail = St.take<int>(cap);
    c.cap = (int)cap;
    return c;
  };
  EventDev W{};
  W.n_seeds = S;
  W.cand[0] = cand_view(SC);
  W.cand[1] = cand_view(SC);
  W.bshort = cand_view((size_t)S);
  auto up = [&](void* d, const void* h, size_t bytes) {
    if (St.rc == MKFG_OK && bytes) {
      const cudaError_t ce = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st);
      if (ce != cudaSuccess) St.rc = set_error(MKFG_ERR_CUDA, "worker staging: %s", cudaGetErrorString(ce));
    }
  };
  const CandSoA& B = W.cand[0];
  up(B.par, in->par, 4 * 6 * SC);
  up(B.err, in->err, 4 * 21 * SC);
  up(B.chg, in->chg, 4 * SC);
  up(B.chi2, in->chi2, 4 * SC);
  up(B.score, in->score, 4 * SC);
  up(B.last, last.data(), 4 * SC);
  up(B.nfound, in->nfound, 4 * SC);
  up(B.nmiss, in->nmiss, 4 * SC);
  up(B.nover, in->nover, 4 * SC);
  up(B.ninside, in->ninside, 4 * SC);
  up(B.ntail, in->ntail, 4 * SC);
  up(W.bshort.score, in->bshort_score, 4 * (size_t)S);
  W.bshort_valid = St.put(in->bshort_valid, (size_t)S);
  W.n_cands = St.put(in->n_cands, (size_t)S);
  W.hot_size = St.put(hot_size.data(), (size_t)S);
  W.node_hot = St.put(node_hot.data(), node_hot.size());
  W.node_prev = St.put(node_prev.data(), node_prev.size());
  W.node_chi2 = St.take<float>((size_t)S * kWorkerHotCap);
  W.hot_cap = kWorkerHotCap;
  W.rec = St.put(rec.data(), rec.size());
  W.rmask = St.put(rmask.data(), SC);
  W.wsr = St.put(wsr.data(), SC);
  W.extra_last = St.put(extra_last.data(), SC);
  W.upd = St.take<int>(SC);
  int* d_new = St.take<int>((size_t)S);
  int* d_parent = St.take<int>(SC);
  W.err_flags = St.take<int>(16);
  if (St.rc) return St.rc;
  MKFG_CUDA_TRY(cudaMemsetAsync(W.err_flags, 0, 4, st));
  MKFG_CUDA_TRY(cudaMemsetAsync(W.upd, 0, 4 * SC, st));
  MKFG_CUDA_TRY(cudaMemsetAsync(d_parent, 0xff, 4 * SC, st));
  const int blocks = (S + kBlock / 32 - 1) / (kBlock / 32);
  k_clone_worker<<<blocks, kBlock, 0, st>>>(W, f->d_cfg, layer, d_new, d_parent);
  MKFG_CUDA_TRY(cudaGetLastError());
  // Read back.
  const CandSoA& N = W.cand[1];
  std::vector<int> nnew(S), parent(SC), upd(SC), nlast(SC), flags(1);
  std::vector<int> bvalid(S), bnfound(S);
  std::vector<float> bscore(S), bchi2(S);
  St.get(nnew.data(), d_new, (size_t)S);
  St.get(parent.data(), d_parent, SC);
  St.get(upd.data(), W.upd, SC);
  St.get(out->par, N.par, 6 * SC);
  St.get(out->err, N.err, 21 * SC);
  St.get(out->chg, N.chg, SC);
  St.get(out->chi2, N.chi2, SC);
  St.get(out->score, N.score, SC);
  St.get(nlast.data(), N.last, SC);
  St.get(out->nfound, N.nfound, SC);
  St.get(out->nmiss, N.nmiss, SC);
  St.get(out->nover, N.nover, SC);
  St.get(out->ninside, N.ninside, SC);
  St.get(out->ntail, N.ntail, SC);
  St.get(bvalid.data(), W.bshort_valid, (size_t)S);
  St.get(bscore.data(), W.bshort.score, (size_t)S);
  St.get(bchi2.data(), W.bshort.chi2, (size_t)S);
  St.get(bnfound.data(), W.bshort.nfound, (size_t)S);
  St.get(node_hot.data(), W.node_hot, node_hot.size());
  St.get(node_prev.data(), W.node_prev, node_prev.size());
  St.get(flags.data(), W.err_flags, 1);
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  if (St.rc) return St.rc;
  if (flags[0] & kErrArena) return set_error(MKFG_ERR_OVERFLOW, "clone worker arena overflow");
  auto hot_idx = [&](int s, int node) { return (node_hot[(size_t)s * kWorkerHotCap + node] << 8) >> 8; };
  for (int s = 0; s < S; ++s) {
    out->n_cands[s] = nnew[s];
    out->bshort_valid[s] = bvalid[s];
    out->bshort_score[s] = bvalid[s] ? bscore[s] : -1e16f;  // getScoreWorstPossible
    out->bshort_nfound[s] = bvalid[s] ? bnfound[s] : 0;
    out->bshort_chi2[s] = bvalid[s] ? bchi2[s] : 0.f;
    for (int c = 0; c < kSlots; ++c) {
      const size_t k = (size_t)s * kSlots + c;
      out->parent[k] = -1;
      out->hit[k] = MKFG_NO_HIT;
      out->overlap_hit[k] = -1;
      out->update_hit[k] = -1;
      if (c >= nnew[s]) continue;
      out->parent[k] = parent[k];
      out->update_hit[k] = upd[k] - 1;
      // The nodes this step added (above the setup nodes): the hit or hole,
      // then the overlap hit, if any.
      const int l1 = nlast[k];
      if (l1 < 2 * kSlots) continue;  // held back: no node of its own
      const int l0 = node_prev[(size_t)s * kWorkerHotCap + l1];
      if (l0 >= 2 * kSlots) {
        out->hit[k] = hot_idx(s, l0);
        out->overlap_hit[k] = hot_idx(s, l1);
      } else {
        out->hit[k] = hot_idx(s, l1);
      }
    }
  }
  return MKFG_OK;
}

extern "C" int mkfg_find_filter(mkfg_context* ctx, const mkfg_qfilter_config* cfg, int32_t n_seeds,
                                int32_t remove, int32_t* pass) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(cfg != nullptr, "null config");
  MKFG_REQUIRE(f->events_loaded && n_seeds == f->n_seeds, "seed count mismatch");
  MKFG_REQUIRE(cfg->kind >= 0 && cfg->kind < kQfCount, "unknown quality filter %d", cfg->kind);
  const int S = f->n_seeds;
  if (S == 0) return MKFG_OK;
  if ((rc = f->sel.ensure(rounded(4 * (size_t)S)))) return rc;
  int* d_pass = f->sel.as<int>();
  QFilterParams P;
  P.kind = cfg->kind;
  P.min_hits = cfg->min_hits;
  P.beam_x = cfg->beam_spot_x;
  P.beam_y = cfg->beam_spot_y;
  cudaStream_t st = ctx->stream;
  k_qfilter<<<(S + 127) / 128, 128, 0, st>>>(f->ev, f->d_cfg, P, remove ? 1 : 0, d_pass);
  MKFG_CUDA_TRY(cudaGetLastError());
  if (pass) MKFG_CUDA_TRY(cudaMemcpyAsync(pass, d_pass, 4 * (size_t)S, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  if (remove) f->filter_removed = true;
  return MKFG_OK;
}

extern "C" int mkfg_find_work(mkfg_context* ctx, int64_t* active_cands, int64_t* hit_pairs,
                              int64_t* updates, int32_t* steps) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->events_loaded, "no event uploaded");
  const int ns = f->host_cfg.max_steps + 2;
  std::vector<int> work(kWorkN * (size_t)ns), pairs(ns);
  MKFG_CUDA_TRY(cudaMemcpyAsync(work.data(), f->ev.work, 4 * work.size(), cudaMemcpyDeviceToHost, ctx->stream));
  MKFG_CUDA_TRY(cudaMemcpyAsync(pairs.data(), f->ev.pair_count, 4 * pairs.size(), cudaMemcpyDeviceToHost, ctx->stream));
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  int64_t a = 0, p = 0, u = 0, p2 = 0, cs = 0, rec = 0, nc = 0;
  for (int i = 0; i < ns; ++i) {
    a += work[kWorkN * i];
    u += work[kWorkN * i + 1];
    p2 += work[kWorkN * i + 2];
    cs += work[kWorkN * i + 3];
    rec += work[kWorkN * i + 4];
    nc += work[kWorkN * i + 5];
    p += pairs[i];
  }
  f->last_chi2_evals = p2;
  f->last_seeds_cloned = cs;
  f->last_records = rec;
  f->last_new_cands = nc;
  if (active_cands) *active_cands = a;
  if (hit_pairs) *hit_pairs = p;
  if (updates) *updates = u;
  if (steps) *steps = f->host_cfg.max_steps;
  return MKFG_OK;
}

extern "C" int mkfg_find_download(mkfg_context* ctx, int n_seeds, mkfg_find_out* out) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(out != nullptr, "null output");
  MKFG_REQUIRE(f->events_loaded && n_seeds == f->n_seeds, "seed count mismatch");
  return download(ctx, f, out, n_seeds, f->host_cfg.max_cands);
}

extern "C" int mkfg_find_download_best(mkfg_context* ctx, int n_seeds, mkfg_find_out* out) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(out != nullptr, "null output");
  MKFG_REQUIRE(f->events_loaded && n_seeds == f->n_seeds, "seed count mismatch");
  return download(ctx, f, out, n_seeds, 1);
}

extern "C" int mkfg_find_event(mkfg_context* ctx, const mkfg_event* ev, mkfg_find_out* out) {
  int rc;
  if ((rc = mkfg_find_upload(ctx, ev))) return rc;
  if ((rc = mkfg_find_run(ctx))) return rc;
  return mkfg_find_download(ctx, ev->n_seeds, out);
}

extern "C" int mkfg_prepare_event_host(const mkfg_find_config* cfg, const mkfg_event* ev,
                                       uint32_t* bins, int32_t* n_bins, int32_t* srank,
                                       int32_t* seed_order, int32_t* seed_region) {
  MKFG_REQUIRE(cfg && ev && n_bins, "null argument");
  MKFG_REQUIRE(cfg->n_layers > 0 && cfg->n_layers <= kMaxLayers && ev->n_layers == cfg->n_layers,
               "layer count mismatch");
  std::vector<LayerBinning> lb(cfg->n_layers);
  int off = 0;
  for (int l = 0; l < cfg->n_layers; ++l) {
    lb[l] = setup_layer_binning(cfg->layer_desc + (size_t)l * LC_COUNT);
    lb[l].bin_offset = off;
    off += lb[l].nq * kPhiBins;
  }
  *n_bins = off;
  if (!bins) return MKFG_OK;
  const int nh = ev->layer_begin[cfg->n_layers];
  EventHitsPrep prep;
  prepare_event_hits(lb, ev->layer_begin, cfg->n_layers, ev->pos, nh, ev->detid, ev->cpcm, prep);
  std::copy(prep.bins.begin(), prep.bins.end(), bins);
  if (srank) std::copy(prep.srank.begin(), prep.srank.end(), srank);
  if (seed_order || seed_region) {
    const int sw = seed_hit_stride(ev);
    std::vector<int32_t> hl, hi;
    if (cfg->sort_seed_hits) sort_seed_hits_by_layer(ev, sw, hl, hi);
    SeedInput si{ev->n_seeds, ev->seed_par, ev->seed_chg, ev->seed_nhits,
                 cfg->sort_seed_hits ? hl.data() : ev->seed_hit_layer,
                 cfg->sort_seed_hits ? hi.data() : ev->seed_hit_index, sw};
    SeedOrder so;
    partition_seeds_cms2017(cfg->layer_desc, cfg->n_layers, si, ev->layer_begin, ev->pos, nh, so);
    if (seed_order) std::copy(so.order.begin(), so.order.end(), seed_order);
    if (seed_region) std::copy(so.region.begin(), so.region.end(), seed_region);
  }
  return MKFG_OK;
}

// Diagnostic counters of the last mkfg_find_work call: chi2 evaluations seen
// by the chi2 kernel and seed-steps handled by the clone kernel.
extern "C" int mkfg_find_work_detail(mkfg_context* ctx, int64_t* chi2_evals, int64_t* seeds_cloned) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  if (chi2_evals) *chi2_evals = f->last_chi2_evals;
  if (seeds_cloned) *seeds_cloned = f->last_seeds_cloned;
  return MKFG_OK;
}

// Clone-step counters of the last mkfg_find_work call: records (IdxChi2List
// entries) present when the seeds were ranked, and new candidates written.
extern "C" int mkfg_find_set_arena_capacity(mkfg_context* ctx, int32_t nodes_per_seed) {
  int rc = activate(ctx);
  if (rc) return rc;
  // Seed nodes are written unconditionally at upload: the arena must hold
  // them and at least one node found by the search.
  MKFG_REQUIRE(nodes_per_seed == 0 || nodes_per_seed >= MKFG_MAX_SEED_HITS + 2,
               "arena capacity %d: 0 (automatic) or at least %d nodes per seed", nodes_per_seed,
               MKFG_MAX_SEED_HITS + 2);
  finder_of(ctx)->arena_cap = nodes_per_seed;
  return MKFG_OK;
}

extern "C" int mkfg_find_set_bin_staging(mkfg_context* ctx, int32_t on) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(on == 0 || on == 1, "on must be 0 or 1, got %d", on);
  Finder* f = finder_of(ctx);
  if (f->stage_bins != (on != 0)) f->drop_graph();
  f->stage_bins = on != 0;
  return MKFG_OK;
}

extern "C" int mkfg_find_set_seed_import(mkfg_context* ctx, int32_t on_host) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(on_host == 0 || on_host == 1, "on_host must be 0 or 1, got %d", on_host);
  finder_of(ctx)->seed_import_host = on_host != 0;
  return MKFG_OK;
}

extern "C" int mkfg_find_work_clone(mkfg_context* ctx, int64_t* records, int64_t* new_cands) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  if (records) *records = f->last_records;
  if (new_cands) *new_cands = f->last_new_cands;
  return MKFG_OK;
}
