// Device build of the per-layer hit index (LayerOfHits::SuckInHits +
// EndRegistrationOfHits, mkFit/HitStructures.cc:77-338): for every hit of a
// layer its q bin and fine phi bin, a stable sort of the hits by the key
// (q bin, fine phi bin), the (q bin, phi bin) table of sorted-position
// ranges, the sorted (q, phi) and the original index of every sorted hit.
//
// One thread block per (event, layer). The sort is a counting sort over the
// layer's nq x 1025 fine keys in shared memory: a histogram, an exclusive
// scan (which also gives the bin table), then a scatter in hit order in
// which equal keys take consecutive positions in order of their hit index
// -- the stable order of the reference's sort, whatever the warp schedule.
// The counters are 16 bits, two to a 32-bit word (a layer holds at most
// 65535 hits, which the upload checks, so no count, start or end of a key
// reaches the upper half): 55 KB for the 27 q bins of the largest layer,
// four blocks of 512 threads per SM.
#pragma once

#include "find_dev.cuh"

namespace mkfg {

constexpr int kHitsBlock = 512;
constexpr int kPhiFine = 1024;  // fine phi bins (4 per phi bin)
// Fine keys per q bin: phi = +pi (or a value rounding to it) gives fine
// bin 1024, which the reference keeps as a key of its own, sorted after
// 1023 (its bin-table entry then replaces the one of phi bin 0).
constexpr int kFineStride = kPhiFine + 1;
constexpr int kLayerPhiBins = 256;

// Hit::setupAsStrip / setupAsPixel charge code, decoded back to charge per
// cm (Hit.h:285-300): what the strip charge cut compares.
__device__ __forceinline__ uint32_t decoded_charge_pcm_dev(int cpcm) {
  unsigned code;
  if (cpcm < 0)
    code = 0xff;
  else if (cpcm < 1620)
    code = 0;
  else
    code = min(0xff, ((cpcm - 1620) >> 3) + 1);
  return code == 0 ? 0u : ((code - 1) << 3) + 1620;
}

struct LayerHitsArgs {
  const float* pos;      // [3][hstride]
  int hstride;
  const int* detid;      // [NH]
  const int* cpcm;       // [NH]
  const int* layer_begin;  // [n_events][lb_stride], global indices
  int lb_stride;
  int n_layers;
  uint32_t* hinfo;       // [NH] out, original order
  uint32_t* bins;        // [n_events][n_bins] out
  int n_bins;
  SortedHit* sorted;     // [NH] out, sorted order
  const uint8_t* mask;   // [NH] hits masked by earlier iterations, or NULL
};

// Dynamic shared memory: nq_max * kFineStride 16-bit counters, rounded up
// to whole words (hits_smem_bytes).
__host__ __device__ constexpr int hits_smem_words(int nq) { return (nq * kFineStride + 1) / 2; }
__host__ __device__ constexpr int hits_smem_bytes(int nq) { return 4 * hits_smem_words(nq); }

// 16-bit counter k of the packed table.
__device__ __forceinline__ uint32_t cnt16_get(const uint32_t* w, int k) {
  return (w[k >> 1] >> ((k & 1) * 16)) & 0xffffu;
}
// Four blocks per SM (32 registers, a few spilled): the build is latency
// bound (its scatter steps the block's warps in turn), and the 64-event
// batch's 4608 blocks take 326 us against 496 us at two blocks per SM (62
// registers) and 379 us at three.
#ifndef MKFG_HITS_MIN_BLOCKS
#define MKFG_HITS_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(kHitsBlock, MKFG_HITS_MIN_BLOCKS) k_layer_hits(const LayerHitsArgs A,
                                                           const FindConfigDev* __restrict__ Cp) {
  extern __shared__ uint32_t cntw[];
  __shared__ uint32_t warp_tot[kHitsBlock / 32];
  __shared__ uint32_t warp_base[kHitsBlock / 32];
  const FindConfigDev& C = *Cp;
  const int layer = blockIdx.x % A.n_layers, ev = blockIdx.x / A.n_layers;
  const LayerDev& L = C.layer[layer];
  const int h0 = A.layer_begin[ev * A.lb_stride + layer];
  const int n = A.layer_begin[ev * A.lb_stride + layer + 1] - h0;
  const int nkeys = L.nq * kFineStride;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float* X = A.pos;
  const float* Y = A.pos + A.hstride;
  const float* Z = A.pos + 2 * (size_t)A.hstride;
  constexpr float fphi_fine = kPhiFine / kTwoPI;

  auto hit_key = [&](int h, float& q, float& phi) {
    const float x = X[h], y = Y[h];
    phi = f_atan2(y, x);                                                  // Hit::phi()
    q = L.is_barrel ? Z[h] : __fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)));  // z / r
    // In [0, 1024] for any finite position; the clamp only keeps invalid
    // (NaN) input inside the table.
    const int fine = min(max((int)floorf(__fmul_rn(fphi_fine, __fadd_rn(phi, kPI))), 0), kPhiFine);
    const int qb = min(max((int)__fmul_rn(__fsub_rn(q, L.qmin), L.fq), 0), L.nq - 1);
    return qb * kFineStride + fine;
  };

  const int nwords = (nkeys + 1) / 2;
  for (int k = tid; k < nwords; k += kHitsBlock) cntw[k] = 0;
  __syncthreads();
  for (int i = tid; i < n; i += kHitsBlock) {
    float q, phi;
    const int key = hit_key(h0 + i, q, phi);
    atomicAdd(&cntw[key >> 1], 1u << ((key & 1) * 16));
    A.hinfo[h0 + i] = (uint32_t(A.detid[h0 + i]) & 0xfffu) |
                      (decoded_charge_pcm_dev(A.cpcm[h0 + i]) << 12);
  }
  __syncthreads();

  // Exclusive scan of the counters: thread t owns a contiguous segment of
  // whole words (both halves of a word are its own).
  const int seg = 2 * ((nwords + kHitsBlock - 1) / kHitsBlock);
  const int k0 = min(tid * seg, nkeys), k1 = min(k0 + seg, nkeys);
  uint32_t local = 0;
  for (int k = k0; k < k1; k += 2) {
    const uint32_t v = cntw[k >> 1];
    local += (v & 0xffffu) + (v >> 16);
  }
  uint32_t incl = local;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += v;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < kHitsBlock / 32 ? warp_tot[lane] : 0u;
    uint32_t ti = t;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, ti, off);
      if (lane >= off) ti += v;
    }
    if (lane < kHitsBlock / 32) warp_base[lane] = ti - t;
  }
  __syncthreads();
  uint32_t run = warp_base[warp] + incl - local;
  for (int k = k0; k < k1; k += 2) {
    // A key past the end (odd nkeys) shares the last word and counts 0.
    const uint32_t v = cntw[k >> 1];
    const uint32_t lo = run, hi = run + (v & 0xffffu);
    cntw[k >> 1] = lo | (hi << 16);
    run = hi + (v >> 16);
  }
  __syncthreads();

  // Bin table: (q bin, phi bin) covers fine keys q * kFineStride + 4 * phi
  // bin + 0..3; fine key 1024, when present, takes over phi bin 0.
  uint32_t* bins = A.bins + (size_t)ev * A.n_bins + L.bin_offset;
  auto key_end = [&](int k) { return k < nkeys ? cnt16_get(cntw, k) : (uint32_t)n; };
  for (int b = tid; b < L.nq * kLayerPhiBins; b += kHitsBlock) {
    const int qb = b / kLayerPhiBins, pb = b % kLayerPhiBins;
    int k = qb * kFineStride + 4 * pb;
    uint32_t first = cnt16_get(cntw, k), last = key_end(k + 4);
    if (pb == 0) {
      const int k1024 = qb * kFineStride + kPhiFine;
      if (key_end(k1024 + 1) != cnt16_get(cntw, k1024)) {
        first = cnt16_get(cntw, k1024);
        last = key_end(k1024 + 1);
      }
    }
    bins[b] = first == last ? 0u : (first | (last << 16));
  }
  __syncthreads();

  // Scatter in hit order: chunks of the block, warps of a chunk in turn.
  for (int c0 = 0; c0 < n; c0 += kHitsBlock) {
    const int i = c0 + tid;
    const bool valid = i < n;
    float q = 0.f, phi = 0.f;
    const int key = valid ? hit_key(h0 + i, q, phi) : -1;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    for (int w = 0; w < kHitsBlock / 32; ++w) {
      if (warp == w && valid) {
        const unsigned peers = __match_any_sync(vmask, key);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (lane == leader) {
          // Leaders of the two keys of a word may meet here: add, not store.
          const int sh = (key & 1) * 16;
          base = (atomicAdd(&cntw[key >> 1], (uint32_t)__popc(peers) << sh) >> sh) & 0xffffu;
        }
        base = __shfl_sync(peers, base, leader);
        const uint32_t at = base + __popc(peers & ((1u << lane) - 1u));
        // A masked hit (IterationMaskIfc, skipped by
        // MkFinder::SelectHitIndices, mkFit/MkFinder.cc:476-482) keeps its
        // bin but gets q = +inf, which no search window holds.
        const bool masked = A.mask != nullptr && A.mask[h0 + i] != 0;
        A.sorted[h0 + at] = SortedHit{masked ? __int_as_float(0x7f800000) : q, phi, i, 0};
      }
      __syncthreads();
    }
  }
}

}  // namespace mkfg
