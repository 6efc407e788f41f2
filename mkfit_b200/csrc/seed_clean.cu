// Seed cleaning on the device: StdSeq::clean_cms_seedtracks_iter
// (mkFit/MkStdSeqs.cc:115-311) for a batch of events.
//
// The reference compares every ordered pair (ts < tss) of an event's seeds
// with an elliptical (dz, dR) window and, for each overlapping pair it
// examines, drops the seed with the larger transverse impact parameter and
// merges the dropped seed's hits into the kept one. Which pairs it examines
// depends on the order: the outer loop skips a seed that an earlier seed
// already dropped. Here:
//   1. k_clean_features (thread per seed): the per-seed quantities the
//      window uses, the seed's eta bin and the per-event eta histogram;
//   2. k_clean_bins (block per event): bin starts and seeds sorted by bin;
//   3. k_clean_pairs (thread per seed): the seed's window test against every
//      later seed (by index) of its event in the eta bins within reach (an
//      overlap needs |d eta| < drmax), appending overlapping pairs;
//   4. k_clean_resolve (block per event): the event's pairs sorted by
//      (ts, tss) in shared memory, then one thread replays the reference's
//      loop over them in that order (skip, drop, hit merge, layer sort).
// Overlapping pairs are rare, so step 4 is short; the O(n^2) scan of the
// reference becomes a scan over eta neighbours.
#include "internal.h"
#include "find_dev.cuh"

#include <algorithm>
#include <climits>
#include <vector>

namespace mkfg {
namespace {

constexpr int kCleanBlock = 256;
constexpr int kEtaBins = 1024;
constexpr float kEtaLo = -4.f, kEtaHi = 4.f;
constexpr int kResolveBlock = 512;
constexpr int kMaxEventPairs = 4096;  // overlapping pairs per event resolved in shared memory

struct CleanParams {
  float ptthr;
  float dz2inv_bh, dr2inv_bh, dz2inv_bl, dr2inv_bl;
  float dz2inv_eh, dr2inv_eh, dz2inv_el, dr2inv_el;
  float beam_x, beam_y;
  int reach;           // eta bins scanned on each side
};

struct CleanDev {
  int n_events;
  const int* ev_begin;  // [n_events + 1]
  const int* ev_of;     // [n] event of each seed
  int n;
  const float* par;     // [6][n]
  const int* chg;
  float* pt;
  float* eta;
  float* phi;
  float* pos2;
  float* ctheta;
  float* invptq;
  float* d0;
  int* ebin;            // [n]
  int* bin_count;       // [n_events][kEtaBins + 1]
  int* order;           // [n] seeds of each event by eta bin
  int2* pairs;          // overlapping (ts, tss), global seed indices
  int* pair_ev;         // event of each pair
  int* n_pairs;
  int pair_cap;
  int max_hits;
  int* nh;              // [n]
  int* hl;              // [n][max_hits] hit layer
  int* hi;              // [n][max_hits] hit index
  int* keep;            // [n]
  int* err;             // bit 0: pair pool overflow, bit 1: per-event pair overflow
};

__global__ void k_clean_features(CleanDev D, CleanParams P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D.n) return;
  const float x = D.par[0 * D.n + i], y = D.par[1 * D.n + i], z = D.par[2 * D.n + i];
  const float ipt = D.par[3 * D.n + i], phi = D.par[4 * D.n + i], theta = D.par[5 * D.n + i];
  const int q = D.chg[i];
  (void)z;
  const float pt = fabsf(1.f / ipt);
  D.pt[i] = pt;
  const float eta = eta_of_theta(theta);
  D.eta[i] = eta;
  D.phi[i] = phi;
  // std::pow(float, 2) is evaluated in double; the sum is stored as float.
  D.pos2[i] = (float)((double)x * (double)x + (double)y * (double)y);
  D.ctheta[i] = 1.f / f_tan(theta);
  D.invptq[i] = __fmul_rn((float)q, ipt);
  D.d0[i] = d0_beam_spot(x, y, ipt, phi, q, P.beam_x, P.beam_y);
  // Eta bin (NaN and out-of-range values go to the edge bins: only the
  // window test decides, the bins only bound the scan).
  const float f = (eta - kEtaLo) * (kEtaBins / (kEtaHi - kEtaLo));
  const int b = f >= 0.f ? min((int)f, kEtaBins - 1) : 0;
  D.ebin[i] = b;
  atomicAdd(&D.bin_count[D.ev_of[i] * (kEtaBins + 1) + b], 1);
  D.keep[i] = 1;
}

// Exclusive scan of an event's histogram into bin starts, then the seeds
// scattered by bin (order within a bin does not matter: pairs are sorted
// before they are resolved).
__global__ void __launch_bounds__(kCleanBlock) k_clean_bins(CleanDev D) {
  __shared__ int s_cnt[kEtaBins + 1];
  __shared__ int s_warp[kCleanBlock / 32];
  const int e = blockIdx.x;
  int* cnt = D.bin_count + e * (kEtaBins + 1);
  constexpr int kPer = kEtaBins / kCleanBlock;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int v[kPer], local = 0;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    v[k] = cnt[tid * kPer + k];
    local += v[k];
  }
  int incl = local;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += t;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  int base = 0;
  for (int w = 0; w < warp; ++w) base += s_warp[w];
  int run = base + incl - local;
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    s_cnt[tid * kPer + k] = run;
    run += v[k];
  }
  if (tid == kCleanBlock - 1) s_cnt[kEtaBins] = run;
  __syncthreads();
  // Bin starts (relative to the event) stay in the histogram array.
  for (int b = tid; b <= kEtaBins; b += kCleanBlock) cnt[b] = s_cnt[b];
  __syncthreads();
  const int s0 = D.ev_begin[e], s1 = D.ev_begin[e + 1];
  for (int i = s0 + tid; i < s1; i += kCleanBlock) {
    const int at = atomicAdd(&s_cnt[D.ebin[i]], 1);
    D.order[s0 + at] = i;
  }
}

// The window test of one (ts, tss) pair, ts < tss (MkStdSeqs.cc:196-265).
__device__ __forceinline__ bool seeds_overlap(const CleanDev& D, const CleanParams& P, int ts,
                                              int tss) {
  constexpr float kDptCommon = 0.25f;    // Config::c_dpt_common
  constexpr float kEtaMaxBrl = 0.9f;     // Config::c_etamax_brl
  constexpr float kInvR1GeV = 1.f / 87.6f;  // 1 / Config::track1GeVradius
  if (D.chg[tss] != D.chg[ts]) return false;
  const float Pt1 = D.pt[ts], Pt2 = D.pt[tss];
  if (fabsf(__fsub_rn(Pt2, Pt1)) > __fmul_rn(kDptCommon, Pt1)) return false;
  const float Eta1 = D.eta[ts];
  const float de = __fsub_rn(Eta1, D.eta[tss]);
  const float deta2 = __fmul_rn(de, de);
  const float sign05 = D.pos2[tss] > D.pos2[ts] ? -0.5f : 0.5f;
  const float dx = __fsub_rn(D.par[0 * D.n + ts], D.par[0 * D.n + tss]);
  const float dy = __fsub_rn(D.par[1 * D.n + ts], D.par[1 * D.n + tss]);
  const float dxy = (float)((double)sign05 * sqrt((double)dx * (double)dx + (double)dy * (double)dy));
  // Rounded as the reference build evaluates it: the products that feed a
  // single add or subtract are contracted into FMAs.
  const float t = __fmul_rn(dxy, kInvR1GeV);
  const float newPhi1 = fmaf(-t, D.invptq[ts], D.phi[ts]);
  const float newPhi2 = fmaf(t, D.invptq[tss], D.phi[tss]);
  float dphi = fabsf(__fsub_rn(newPhi1, newPhi2));
  if (dphi > kPI) dphi = __fsub_rn(kTwoPI, dphi);  // cdist
  const float dr2 = fmaf(dphi, dphi, deta2);
  const float dz = fmaf(-dxy, __fadd_rn(D.ctheta[ts], D.ctheta[tss]),
                        __fsub_rn(D.par[2 * D.n + ts], D.par[2 * D.n + tss]));
  const float dz2 = __fmul_rn(dz, dz);
  float dzi, dri;
  if (fabsf(Eta1) < kEtaMaxBrl) {
    dzi = Pt1 > P.ptthr ? P.dz2inv_bh : P.dz2inv_bl;
    dri = Pt1 > P.ptthr ? P.dr2inv_bh : P.dr2inv_bl;
  } else {
    dzi = Pt1 > P.ptthr ? P.dz2inv_eh : P.dz2inv_el;
    dri = Pt1 > P.ptthr ? P.dr2inv_eh : P.dr2inv_el;
  }
  return fmaf(dz2, dzi, __fmul_rn(dr2, dri)) < 1.0f;
}

__global__ void __launch_bounds__(kCleanBlock) k_clean_pairs(CleanDev D, CleanParams P) {
  const int ts = blockIdx.x * blockDim.x + threadIdx.x;
  if (ts >= D.n) return;
  const int e = D.ev_of[ts];
  const int s0 = D.ev_begin[e];
  const int* start = D.bin_count + e * (kEtaBins + 1);
  const int b = D.ebin[ts];
  const int b0 = max(b - P.reach, 0), b1 = min(b + P.reach, kEtaBins - 1);
  for (int k = start[b0]; k < start[b1 + 1]; ++k) {
    const int tss = D.order[s0 + k];
    if (tss <= ts || !seeds_overlap(D, P, ts, tss)) continue;
    const int at = atomicAdd(D.n_pairs, 1);
    if (at >= D.pair_cap) {
      atomicOr(D.err, 1);
      continue;
    }
    D.pairs[at] = make_int2(ts, tss);
    D.pair_ev[at] = e;
  }
}

// Appends the hits of seed `from` that `to` does not hold yet (same index
// and layer), while `to` has fewer than 15; returns how many were added
// (MkStdSeqs.cc:276-301).
__device__ int merge_seed_hits(const CleanDev& D, int to, int from) {
  int added = 0;
  int nt = D.nh[to];
  if (nt >= 15) return 0;
  const int nf = D.nh[from];
  const int* fl = D.hl + (size_t)from * D.max_hits;
  const int* fi = D.hi + (size_t)from * D.max_hits;
  int* tl = D.hl + (size_t)to * D.max_hits;
  int* ti = D.hi + (size_t)to * D.max_hits;
  for (int j = 0; j < nf; ++j) {
    const int idx = fi[j], lyr = fl[j];
    if (idx < 0) continue;
    bool unique = true;
    for (int i = 0; i < nt; ++i)
      if (idx == ti[i] && lyr == tl[i]) {
        unique = false;
        break;
      }
    if (!unique) continue;
    if (nt < D.max_hits) {
      ti[nt] = idx;
      tl[nt] = lyr;
    }
    ++nt;
    ++added;
    if (nt >= 15) break;
  }
  D.nh[to] = min(nt, D.max_hits);
  return added;
}

// Track::sortHitsByLayer: stable sort of the hit list by layer.
__device__ void sort_seed_hits(const CleanDev& D, int s) {
  int* l = D.hl + (size_t)s * D.max_hits;
  int* x = D.hi + (size_t)s * D.max_hits;
  const int n = D.nh[s];
  for (int i = 1; i < n; ++i) {
    const int kl = l[i], kx = x[i];
    int j = i;
    while (j > 0 && l[j - 1] > kl) {
      l[j] = l[j - 1];
      x[j] = x[j - 1];
      --j;
    }
    l[j] = kl;
    x[j] = kx;
  }
}

__global__ void __launch_bounds__(kResolveBlock) k_clean_resolve(CleanDev D) {
  __shared__ long long s_key[kMaxEventPairs];
  __shared__ int s_n;
  const int e = blockIdx.x, tid = threadIdx.x;
  if (tid == 0) s_n = 0;
  __syncthreads();
  const int np = min(*D.n_pairs, D.pair_cap);
  for (int p = tid; p < np; p += kResolveBlock) {
    if (D.pair_ev[p] != e) continue;
    const int at = atomicAdd(&s_n, 1);
    if (at < kMaxEventPairs)
      s_key[at] = ((long long)D.pairs[p].x << 32) | (unsigned)D.pairs[p].y;
    else
      atomicOr(D.err, 2);
  }
  __syncthreads();
  const int n = min(s_n, kMaxEventPairs);
  int m = 1;
  while (m < n) m <<= 1;
  for (int i = n + tid; i < m; i += kResolveBlock) s_key[i] = LLONG_MAX;
  __syncthreads();
  // Bitonic sort of the event's pairs by (ts, tss).
  for (int k = 2; k <= m; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < m; i += kResolveBlock) {
        const int l = i ^ j;
        if (l > i) {
          const long long a = s_key[i], b = s_key[l];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            s_key[i] = b;
            s_key[l] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  if (tid != 0) return;
  // The reference's loops over the overlapping pairs, in its order.
  int cur = -1, added = 0;
  bool skip = false;
  for (int p = 0; p < n; ++p) {
    const int ts = (int)(s_key[p] >> 32), tss = (int)(s_key[p] & 0xffffffffLL);
    if (ts != cur) {
      cur = ts;
      skip = !D.keep[ts];  // dropped by an earlier seed: the outer loop skips it
      added = 0;
    }
    if (skip) continue;
    int i1 = ts, i2 = tss;
    if (D.d0[tss] > D.d0[ts]) {
      D.keep[tss] = 0;
    } else {
      D.keep[ts] = 0;
      i1 = tss;
      i2 = ts;
    }
    added += merge_seed_hits(D, i1, i2);
    if (added > 0) sort_seed_hits(D, i1);
  }
}

}  // namespace
}  // namespace mkfg

using namespace mkfg;

extern "C" int mkfg_clean_seeds(mkfg_context* ctx, const mkfg_seed_clean_params* p, int32_t n_events,
                                const int32_t* event_seed_begin, const float* seed_par,
                                const int32_t* seed_chg, const int32_t* seed_nhits,
                                const int32_t* seed_hit_layer, const int32_t* seed_hit_index,
                                int32_t in_hits, int32_t max_hits, int32_t* keep,
                                int32_t* out_nhits, int32_t* out_hit_layer,
                                int32_t* out_hit_index) {
  int rc = activate(ctx);
  if (rc) return rc;
  MKFG_REQUIRE(p && event_seed_begin && n_events >= 0, "bad arguments");
  MKFG_REQUIRE(in_hits >= 1 && max_hits >= 15 && max_hits >= in_hits && max_hits <= 64,
               "bad hit-row widths (max_hits must hold the 15 hits a merge can reach)");
  const int n = n_events ? event_seed_begin[n_events] : 0;
  MKFG_REQUIRE(event_seed_begin[0] == 0 || n_events == 0, "event_seed_begin[0] must be 0");
  for (int e = 0; e < n_events; ++e)
    MKFG_REQUIRE(event_seed_begin[e + 1] >= event_seed_begin[e], "event_seed_begin not sorted");
  if (n == 0) return MKFG_OK;
  MKFG_REQUIRE(seed_par && seed_chg && seed_nhits && seed_hit_layer && seed_hit_index && keep &&
                   out_nhits && out_hit_layer && out_hit_index,
               "null array");
  for (int i = 0; i < n; ++i)
    MKFG_REQUIRE(seed_nhits[i] >= 0 && seed_nhits[i] <= in_hits, "seed %d: bad hit count", i);

  CleanParams P;
  auto inv2 = [](float v) { return 1.f / (v * v); };
  P.ptthr = p->pt_thr;
  P.dz2inv_bh = inv2(p->dzmax_bh);
  P.dr2inv_bh = inv2(p->drmax_bh);
  P.dz2inv_bl = inv2(p->dzmax_bl);
  P.dr2inv_bl = inv2(p->drmax_bl);
  P.dz2inv_eh = inv2(p->dzmax_eh);
  P.dr2inv_eh = inv2(p->drmax_eh);
  P.dz2inv_el = inv2(p->dzmax_el);
  P.dr2inv_el = inv2(p->drmax_el);
  P.beam_x = p->beam_x;
  P.beam_y = p->beam_y;
  const float drmax = std::max(std::max(p->drmax_bh, p->drmax_bl), std::max(p->drmax_eh, p->drmax_el));
  MKFG_REQUIRE(drmax > 0.f && drmax < 1.f, "drmax out of range");
  P.reach = (int)std::ceil(drmax * (kEtaBins / (kEtaHi - kEtaLo))) + 1;

  std::vector<int> ev_of(n);
  for (int e = 0; e < n_events; ++e)
    for (int i = event_seed_begin[e]; i < event_seed_begin[e + 1]; ++i) ev_of[i] = e;
  std::vector<int> hl((size_t)n * max_hits, 0), hi((size_t)n * max_hits, 0);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < seed_nhits[i]; ++k) {
      hl[(size_t)i * max_hits + k] = seed_hit_layer[(size_t)i * in_hits + k];
      hi[(size_t)i * max_hits + k] = seed_hit_index[(size_t)i * in_hits + k];
    }

  const int pair_cap = 8 * n + 1024;
  const size_t f_bytes = 4 * (size_t)n;
  const size_t need = 6 * f_bytes * 4 + 4 * (size_t)n_events * (kEtaBins + 1) + 4 * (size_t)(n_events + 1) +
                      12 * (size_t)pair_cap + 8 * (size_t)n * max_hits + 64 + 64 * 256;
  if ((rc = ctx->scratch_misc.ensure(need))) return rc;
  char* base = ctx->scratch_misc.as<char>();
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* r = base + off;
    off += (bytes + 255) / 256 * 256;
    return r;
  };
  CleanDev D;
  D.n_events = n_events;
  D.n = n;
  D.max_hits = max_hits;
  D.pair_cap = pair_cap;
  float* par = (float*)take(6 * f_bytes);
  int* chg = (int*)take(f_bytes);
  D.par = par;
  D.chg = chg;
  int* evb = (int*)take(4 * (size_t)(n_events + 1));
  int* evo = (int*)take(f_bytes);
  D.ev_begin = evb;
  D.ev_of = evo;
  D.pt = (float*)take(f_bytes);
  D.eta = (float*)take(f_bytes);
  D.phi = (float*)take(f_bytes);
  D.pos2 = (float*)take(f_bytes);
  D.ctheta = (float*)take(f_bytes);
  D.invptq = (float*)take(f_bytes);
  D.d0 = (float*)take(f_bytes);
  D.ebin = (int*)take(f_bytes);
  D.bin_count = (int*)take(4 * (size_t)n_events * (kEtaBins + 1));
  D.order = (int*)take(f_bytes);
  D.pairs = (int2*)take(8 * (size_t)pair_cap);
  D.pair_ev = (int*)take(4 * (size_t)pair_cap);
  D.nh = (int*)take(f_bytes);
  D.hl = (int*)take(4 * (size_t)n * max_hits);
  D.hi = (int*)take(4 * (size_t)n * max_hits);
  D.keep = (int*)take(f_bytes);
  int* flags = (int*)take(64);
  D.n_pairs = flags;
  D.err = flags + 1;
  MKFG_REQUIRE(off <= ctx->scratch_misc.bytes, "scratch sizing");

  cudaStream_t st = ctx->stream;
  MKFG_CUDA_TRY(cudaMemcpyAsync(par, seed_par, 6 * f_bytes, cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(chg, seed_chg, f_bytes, cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(evb, event_seed_begin, 4 * (size_t)(n_events + 1), cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(evo, ev_of.data(), f_bytes, cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(D.nh, seed_nhits, f_bytes, cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(D.hl, hl.data(), 4 * hl.size(), cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(D.hi, hi.data(), 4 * hi.size(), cudaMemcpyHostToDevice, st));
  MKFG_CUDA_TRY(cudaMemsetAsync(D.bin_count, 0, 4 * (size_t)n_events * (kEtaBins + 1), st));
  MKFG_CUDA_TRY(cudaMemsetAsync(flags, 0, 64, st));
  const int grid = (n + kCleanBlock - 1) / kCleanBlock;
  k_clean_features<<<grid, kCleanBlock, 0, st>>>(D, P);
  k_clean_bins<<<n_events, kCleanBlock, 0, st>>>(D);
  k_clean_pairs<<<grid, kCleanBlock, 0, st>>>(D, P);
  k_clean_resolve<<<n_events, kResolveBlock, 0, st>>>(D);
  MKFG_CUDA_TRY(cudaGetLastError());
  int h_flags[2] = {0, 0};
  MKFG_CUDA_TRY(cudaMemcpyAsync(keep, D.keep, f_bytes, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(out_nhits, D.nh, f_bytes, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(out_hit_layer, D.hl, 4 * hl.size(), cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(out_hit_index, D.hi, 4 * hi.size(), cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaMemcpyAsync(h_flags, flags, 8, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_flags[1] & 1) return set_error(MKFG_ERR_OVERFLOW, "seed cleaning: more than %d overlapping pairs", pair_cap);
  if (h_flags[1] & 2)
    return set_error(MKFG_ERR_OVERFLOW, "seed cleaning: more than %d overlapping pairs in one event", kMaxEventPairs);
  return MKFG_OK;
}
