// Clone-engine combinatorial track finding: device kernels and C ABI.
//
// Plain form (the drop-in for MkBuilder::FindTracksCloneEngine,
// mkFit/MkBuilder.cc:1847-2058): for every layer-plan step, four launches
//   1. prep   : seed activation, candidate unroll + low-pT looper stop,
//               propagation to the layer, SelectHitIndices, missed-layer
//               handling, hole records        (one thread per candidate)
//   2. chi2   : propagate to each selected hit, chi2, strip checks,
//               hit records                   (one thread per (cand, hit))
//   3. clone  : per-seed ranking of the records (warp top-M selection),
//               overlap hits, extras, best short candidate, new candidates
//               (one warp per seed) -- CandCloner::ProcessSeedRange
//   4. update : UpdateWithLastHit for candidates that took a hit
// then one merge launch (MergeCandsAndBestShortOne) and one export launch.
#include "internal.h"
#include "find_host.h"
#include "find_fused.cuh"
#include "find_steps.cuh"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstring>
#include <thread>
#include <vector>

namespace mkfg {

constexpr int kBlock = 256;

//------------------------------------------------------------------------------
// Kernel 1: prep
//------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_prep(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                 int step) {
  const FindConfigDev& C = *Cp;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = t / kSlots, c = t % kSlots;
  const bool in_range = s < E.n_seeds;
  const int lane = threadIdx.x & 31;
  const unsigned grp = 0xffu << (lane & ~7);

  int reg = 0, layer = -1, state = kFinished, ncand = 0, buf = 0;
  if (in_range) {
    reg = E.region[s];
    layer = plan_layer(C, reg, step);
    state = wake_seed(C, reg, layer, step, E.state[s], E.pickup_layer[s]);
    ncand = E.n_cands[s];
    buf = E.cur[s];
  }
  const int slot = s * kSlots + c;
  const CandSoA& B = E.cand[buf];
  float par[6], err[21];
  int chg = 0;
  const bool active = in_range && layer >= 0 && state == kFinding && c < ncand &&
                      activate_cand(E, B, s, slot, layer, par, err, chg);
  const unsigned act = __ballot_sync(0xffffffffu, active) & grp;
  {
    const unsigned all = __ballot_sync(0xffffffffu, active);
    if (lane == 0 && all) atomicAdd(&E.work[step * 4 + 0], __popc(all));
  }
  if (in_range && c == 0) {
    if (layer >= 0 && state == kFinding && act == 0) state = kFinished;
    E.state[s] = state;
  }
  if (!in_range) return;

  const size_t rbase = (size_t)s * kRecPerSeed + c * kRecPerCand;
  PrepOut o;
  if (active) {
    const LayerDev& L = C.layer[layer];
    const int ev = E.seed_event[s];
    const int stride = E.cand[0].cap;
    prep_cand(E, C, L, E.bins + (size_t)ev * E.n_bins + L.bin_offset,
              E.layer_begin[ev * E.lb_stride + layer], reg, layer, s, B, slot, par, err, chg,
              E.xhit + slot, stride, o);
    if (o.extra == 2) E.extra_last[slot] = o.extra_last;
#pragma unroll
    for (int e = 0; e < 6; ++e) E.ppar[e * stride + slot] = o.ppar[e];
#pragma unroll
    for (int e = 0; e < 21; ++e) E.perr[e * stride + slot] = o.perr[e];
    if (o.xs > 0) {
      const int base = atomicAdd(&E.pair_count[step], o.xs);
      for (int h = 0; h < o.xs; ++h) E.pairs[base + h] = slot * kMaxXHits + h;
    }
  }
  const size_t r = rbase + kMaxXHits;
  if (o.hole) {
    E.rhit[r] = o.hole_hit;
    E.rmodule[r] = -1;
    E.rchi2hit[r] = 0.f;
    E.rscore[r] = o.hole_score;
  } else {
    E.rhit[r] = kRecInvalid;
  }
  for (int h = o.xs; h < kMaxXHits; ++h) E.rhit[rbase + h] = kRecInvalid;
  E.wsr[slot] = o.wsr | (o.extra << 8);
}

//------------------------------------------------------------------------------
// Kernel 2: chi2 of every (candidate, selected hit) pair
// (MkFinder::FindCandidatesCloneEngine, mkFit/MkFinder.cc:1116-1240).
//------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_chi2(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                 int step) {
  const FindConfigDev& C = *Cp;
  const int n_pairs = E.pair_count[step];
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&E.work[step * 4 + 2], n_pairs);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n_pairs; p += gridDim.x * blockDim.x) {
    const int code = E.pairs[p];
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
      E.rhit[r] = hidx;
      E.rmodule[r] = module;
      E.rchi2hit[r] = chi2;
      E.rscore[r] = score;
    } else {
      E.rhit[r] = kRecInvalid;
    }
  }
}

//------------------------------------------------------------------------------
// Kernel 3: per-seed candidate cloning (CandCloner::ProcessSeedRange,
// mkFit/CandCloner.cc:36-189). One warp per seed.
//------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_clone(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                  int step) {
  const FindConfigDev& C = *Cp;
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  __shared__ HitMatchPair s_hm[kBlock / 32][kSlots];
  if (s >= E.n_seeds) return;
  const int layer = plan_layer(C, E.region[s], step);
  if (layer < 0) return;
  const int state = E.state[s];
  if (state == kDormant) return;
  const int cur = E.cur[s];
  if (lane == 0) atomicAdd(&E.work[step * 4 + 3], 1);
  const size_t rb = (size_t)s * kRecPerSeed;
  const SeedRecords R{E.rhit + rb,          E.rscore + rb,           E.rchi2hit + rb,
                        E.rmodule + rb,       E.wsr + s * kSlots,      E.extra_last + s * kSlots,
                        E.upd + s * kSlots};
  const int n = clone_seed(E, C, s, layer, state, E.n_cands[s], cur, R, s_hm[threadIdx.x >> 5], lane);
  if (n >= 0 && lane == 0) {
    E.n_cands[s] = n;
    E.cur[s] = cur ^ 1;
  }
}

//------------------------------------------------------------------------------
// Kernel 4: UpdateWithLastHit + CopyOutParErr for candidates that took a hit.
//------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_update(EventDev E, const FindConfigDev* __restrict__ Cp,
                                                   int step) {
  const FindConfigDev& C = *Cp;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = t / kSlots, c = t % kSlots;
  if (s >= E.n_seeds) return;
  if (plan_layer(C, E.region[s], step) < 0) return;
  if (c >= E.n_cands[s]) return;
  const int slot = s * kSlots + c;
  if (!E.upd[slot]) return;
  E.upd[slot] = 0;
  atomicAdd(&E.work[step * 4 + 1], 1);
  update_cand(E, C, s, E.layer_begin + E.seed_event[s] * E.lb_stride, E.cand[E.cur[s]], slot);
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
  copy_slot(E.init, t, E.cand[0], t);
  E.upd[t] = 0;
  if (c == 0) {
    E.n_cands[s] = 1;
    E.state[s] = kDormant;
    E.cur[s] = 0;
    E.hot_size[s] = E.init_hot[s];
    E.bshort_valid[s] = 0;
  }
}

//------------------------------------------------------------------------------
// Kernel 5: CombCandidate::MergeCandsAndBestShortOne (one thread per seed).
//------------------------------------------------------------------------------
__global__ void k_merge(EventDev E, const FindConfigDev* __restrict__ Cp) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= E.n_seeds) return;
  const int cur = E.cur[s];
  E.n_cands[s] = merge_seed(E, *Cp, s, E.n_cands[s], cur);
  E.cur[s] = cur ^ 1;
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
  for (int e = 0; e < 6; ++e) O.par[o * 6 + e] = B.par[e * B.cap + slot];
  for (int e = 0; e < 21; ++e) O.err[o * 21 + e] = B.err[e * B.cap + slot];
  O.chg[o] = B.chg[slot];
  O.chi2[o] = B.chi2[slot];
  O.score[o] = B.score[slot];
  O.nfound[o] = B.nfound[slot];
  const int ntot = B.nfound[slot] + B.nmiss[slot];
  O.ntot[o] = ntot;
  O.noverlap[o] = B.nover[slot];
  O.ninside[o] = B.ninside[slot];
  O.ntail[o] = B.ntail[slot];
  int node = B.last[slot];
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
  cudaGraphExec_t graph = nullptr;  // captured run sequence of the current upload
  int fused_w = 16;                 // seeds per block of the fused form
  int64_t last_chi2_evals = 0, last_seeds_cloned = 0;
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
  f->drop_graph();
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
  }
  f->n_bins = off;
  H.n_layers = cfg->n_layers;
  H.n_regions = cfg->n_regions;
  int max_steps = 0;
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
  H.mat = Material{ctx->d_rl, ctx->d_xi};
  if (!f->d_cfg) MKFG_CUDA_TRY(cudaMalloc(&f->d_cfg, sizeof(FindConfigDev)));
  MKFG_CUDA_TRY(cudaMemcpyAsync(f->d_cfg, &H, sizeof(H), cudaMemcpyHostToDevice, ctx->stream));
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  f->configured = true;
  return MKFG_OK;
}

namespace mkfg {

// Host preparation + upload of a batch of events (one event for the plain
// drop-in form) into the finder's device buffers. Hits and seeds of all
// events are laid out back to back; every seed knows its event.
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
    for (int s = 0; s < ev->n_seeds; ++s)
      MKFG_REQUIRE(ev->seed_nhits[s] >= 1 && ev->seed_nhits[s] <= 4, "seed %d hit count", s);
    hit_off[e + 1] = hit_off[e] + ev->layer_begin[L];
    seed_off[e + 1] = seed_off[e] + ev->n_seeds;
  }
  const int NH = hit_off[n_ev], S = seed_off[n_ev];
  const int nb = f->n_bins;

  // Per-event host preparation (hit index, seed order), in parallel.
  std::vector<EventHitsPrep> preps(n_ev);
  std::vector<SeedOrder> orders(n_ev);
  {
    auto work = [&](int e) {
      const mkfg_event* ev = evs + e;
      const int nh = ev->layer_begin[L];
      prepare_event_hits(f->binning, ev->layer_begin, L, ev->pos, nh, ev->detid, ev->cpcm, preps[e]);
      SeedInput si{ev->n_seeds, ev->seed_par, ev->seed_chg, ev->seed_nhits, ev->seed_hit_layer,
                   ev->seed_hit_index};
      partition_seeds_cms2017(f->layer_desc.data(), L, si, ev->layer_begin, ev->pos, nh, orders[e]);
    };
    const int nthr = std::max(1, std::min(n_ev, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    std::atomic<int> next(0);
    for (int t = 0; t < nthr; ++t)
      pool.emplace_back([&] {
        for (int e = next++; e < n_ev; e = next++) work(e);
      });
    for (auto& th : pool) th.join();
  }

  // Host staging of the concatenated arrays.
  const int NHs = std::max(NH, 1);
  std::vector<float> h_pos(3 * (size_t)NHs), h_err(6 * (size_t)NHs), h_sphi(NHs), h_sq(NHs);
  std::vector<uint32_t> h_info(NHs), h_bins((size_t)nb * n_ev);
  std::vector<int> h_srank(NHs), h_lb((size_t)(L + 1) * n_ev);
  for (int e = 0; e < n_ev; ++e) {
    const mkfg_event* ev = evs + e;
    const int nh = ev->layer_begin[L], o = hit_off[e];
    for (int r = 0; r < 3; ++r)
      std::memcpy(&h_pos[(size_t)r * NHs + o], ev->pos + (size_t)r * nh, 4 * (size_t)nh);
    for (int r = 0; r < 6; ++r)
      std::memcpy(&h_err[(size_t)r * NHs + o], ev->err + (size_t)r * nh, 4 * (size_t)nh);
    std::copy(preps[e].sphi.begin(), preps[e].sphi.end(), h_sphi.begin() + o);
    std::copy(preps[e].sq.begin(), preps[e].sq.end(), h_sq.begin() + o);
    std::copy(preps[e].srank.begin(), preps[e].srank.end(), h_srank.begin() + o);
    std::copy(preps[e].hinfo.begin(), preps[e].hinfo.end(), h_info.begin() + o);
    std::copy(preps[e].bins.begin(), preps[e].bins.end(), h_bins.begin() + (size_t)e * nb);
    for (int l = 0; l <= L; ++l) h_lb[(size_t)e * (L + 1) + l] = o + ev->layer_begin[l];
  }

  cudaStream_t st = ctx->stream;
  int rc;
  auto up = [&](void* d, const void* h, size_t bytes) -> int {
    if (bytes == 0) return MKFG_OK;
    MKFG_CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
    return MKFG_OK;
  };
  // ---- hits
  {
    const size_t need = rounded(12 * (size_t)NHs) + rounded(24 * (size_t)NHs) + 4 * rounded(4 * (size_t)NHs) +
                        rounded(4 * h_lb.size()) + rounded(4 * h_bins.size()) + 4096;
    if ((rc = f->hits.ensure(need))) return rc;
    char* p = f->hits.as<char>();
    float* d_pos = carve<float>(p, 3 * (size_t)NHs);
    float* d_err = carve<float>(p, 6 * (size_t)NHs);
    uint32_t* d_info = carve<uint32_t>(p, NHs);
    int* d_lb = carve<int>(p, h_lb.size());
    uint32_t* d_bins = carve<uint32_t>(p, h_bins.size());
    float* d_sphi = carve<float>(p, NHs);
    float* d_sq = carve<float>(p, NHs);
    int* d_srank = carve<int>(p, NHs);
    if ((rc = up(d_pos, h_pos.data(), 4 * h_pos.size()))) return rc;
    if ((rc = up(d_err, h_err.data(), 4 * h_err.size()))) return rc;
    if ((rc = up(d_info, h_info.data(), 4 * h_info.size()))) return rc;
    if ((rc = up(d_lb, h_lb.data(), 4 * h_lb.size()))) return rc;
    if ((rc = up(d_bins, h_bins.data(), 4 * h_bins.size()))) return rc;
    if ((rc = up(d_sphi, h_sphi.data(), 4 * h_sphi.size()))) return rc;
    if ((rc = up(d_sq, h_sq.data(), 4 * h_sq.size()))) return rc;
    if ((rc = up(d_srank, h_srank.data(), 4 * h_srank.size()))) return rc;
    f->ev.hpos = d_pos;
    f->ev.herr = d_err;
    f->ev.hstride = NHs;
    f->ev.hinfo = d_info;
    f->ev.layer_begin = d_lb;
    f->ev.lb_stride = L + 1;
    f->ev.n_bins = nb;
    f->ev.bins = d_bins;
    f->ev.sphi = d_sphi;
    f->ev.sq = d_sq;
    f->ev.srank = d_srank;
  }
  // ---- seeds, candidates, scratch, records, arena
  const int SS = std::max(S, 1);
  const int SC = SS * kSlots;
  const int max_steps = f->host_cfg.max_steps;
  const int M = f->host_cfg.max_cands;
  const int hot_cap = ((8 + max_steps * (2 * M + 3)) + 31) / 32 * 32;
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
    f->ev.init = mk(SC);
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
  }
  {
    const size_t need = rounded(4 * (size_t)SC) * (27 + 5) + 2 * rounded(4 * (size_t)SC * kMaxXHits) +
                        rounded(4 * (size_t)(max_steps + 2)) * 5 + rounded(64) + 4096;
    if ((rc = f->scratch.ensure(need))) return rc;
    char* p = f->scratch.as<char>();
    f->ev.ppar = carve<float>(p, 6 * (size_t)SC);
    f->ev.perr = carve<float>(p, 21 * (size_t)SC);
    f->ev.xhit = carve<int>(p, (size_t)kMaxXHits * SC);
    f->ev.wsr = carve<int>(p, SC);
    f->ev.extra_last = carve<int>(p, SC);
    f->ev.upd = carve<int>(p, SC);
    f->ev.pairs = carve<int>(p, (size_t)SC * kMaxXHits);
    f->ev.pair_count = carve<int>(p, max_steps + 2);
    f->ev.err_flags = carve<int>(p, 16);
    f->ev.work = carve<int>(p, 4 * (size_t)(max_steps + 2));
  }
  {
    const size_t nrec = (size_t)SS * kRecPerSeed;
    if ((rc = f->recs.ensure(rounded(4 * nrec) * 4 + 4096))) return rc;
    char* p = f->recs.as<char>();
    f->ev.rscore = carve<float>(p, nrec);
    f->ev.rchi2hit = carve<float>(p, nrec);
    f->ev.rhit = carve<int>(p, nrec);
    f->ev.rmodule = carve<int>(p, nrec);
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

  // Initial candidates: each event's seeds in sorted order
  // (CombCandidate::ImportSeed, mkFit/HitStructures.cc:483-509).
  std::vector<float> par(6 * (size_t)SC, 0.f), err(21 * (size_t)SC, 0.f), score(SC, 0.f);
  std::vector<int> chg(SC, 0), last(SC, 0), nfound(SC, 0), nmiss(SC, 0), ninside(SC, 0), ntail(SC, 0);
  std::vector<int> label(SS, 0), sev(SS, 0), region(SS, 0), pickup(SS, 0), state(SS, kDormant),
      ncand(SS, 1), cur(SS, 0), hot_size(SS, 0);
  std::vector<int> node_hot((size_t)SS * hot_cap, 0), node_prev((size_t)SS * hot_cap, -1);
  for (int e = 0; e < n_ev; ++e) {
    const mkfg_event* ev = evs + e;
    const int n = ev->n_seeds;
    for (int k = 0; k < n; ++k) {
      const int s = seed_off[e] + k;
      const int i = orders[e].order[k];
      label[s] = seed_off[e] + i;
      sev[s] = e;
      region[s] = orders[e].region[i];
      const int nhs = ev->seed_nhits[i];
      pickup[s] = ev->seed_hit_layer[i * 4 + nhs - 1];
      const int slot = s * kSlots;
      for (int c = 0; c < 6; ++c) par[c * (size_t)SC + slot] = ev->seed_par[c * n + i];
      for (int c = 0; c < 21; ++c) err[c * (size_t)SC + slot] = ev->seed_err[c * n + i];
      chg[slot] = ev->seed_chg[i];
      int nf = 0, nm = 0, nin = 0, ntl = 0, prev = -1;
      for (int h = 0; h < nhs; ++h) {
        const int hi = ev->seed_hit_index[i * 4 + h], hl = ev->seed_hit_layer[i * 4 + h];
        node_hot[(size_t)s * hot_cap + h] = (hi & 0xffffff) | (hl << 24);
        node_prev[(size_t)s * hot_cap + h] = prev;
        prev = h;
        if (hi >= 0 || hi == -9) {
          ++nf;
          nin += ntl;
          ntl = 0;
        } else {
          ++nm;
          if (hi == -1) ++ntl;
        }
      }
      hot_size[s] = nhs;
      last[slot] = nhs - 1;
      nfound[slot] = nf;
      nmiss[slot] = nm;
      ninside[slot] = nin;
      ntail[slot] = ntl;
      // getScoreCand(cand) with default arguments (mkFit/HitStructures.h:519-531).
      const float pt = std::abs(1.f / par[3 * (size_t)SC + slot]);
      float bonus = 0.2f * nf + 4.0f, penalty = 8.0f;
      if (pt < 0.9f) {
        penalty *= 1.5f;
        bonus = std::min(bonus * 1.0f, 8.0f);
      }
      score[slot] = bonus * nf + 0.0f * 0 - penalty * nin - 3.0f * 0 - 0.0f;
    }
  }
  f->drop_graph();
  CandSoA& B0 = f->ev.init;
  if ((rc = up(B0.par, par.data(), 4 * par.size()))) return rc;
  if ((rc = up(B0.err, err.data(), 4 * err.size()))) return rc;
  if ((rc = up(B0.chg, chg.data(), 4 * (size_t)SC))) return rc;
  MKFG_CUDA_TRY(cudaMemsetAsync(B0.chi2, 0, 4 * (size_t)SC, st));
  if ((rc = up(B0.score, score.data(), 4 * (size_t)SC))) return rc;
  if ((rc = up(B0.last, last.data(), 4 * (size_t)SC))) return rc;
  if ((rc = up(B0.nfound, nfound.data(), 4 * (size_t)SC))) return rc;
  if ((rc = up(B0.nmiss, nmiss.data(), 4 * (size_t)SC))) return rc;
  MKFG_CUDA_TRY(cudaMemsetAsync(B0.nover, 0, 4 * (size_t)SC, st));
  if ((rc = up(B0.ninside, ninside.data(), 4 * (size_t)SC))) return rc;
  if ((rc = up(B0.ntail, ntail.data(), 4 * (size_t)SC))) return rc;
  if ((rc = up(f->ev.seed_label, label.data(), 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.seed_event, sev.data(), 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.region, region.data(), 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.pickup_layer, pickup.data(), 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.state, state.data(), 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.n_cands, ncand.data(), 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.cur, cur.data(), 4 * (size_t)SS))) return rc;
  if ((rc = up(f->ev.init_hot, hot_size.data(), 4 * (size_t)SS))) return rc;
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.bshort_valid, 0, 4 * (size_t)SS, st));
  if ((rc = up(f->ev.node_hot, node_hot.data(), 4 * node_hot.size()))) return rc;
  if ((rc = up(f->ev.node_prev, node_prev.data(), 4 * node_prev.size()))) return rc;
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.node_chi2, 0, 4 * node_hot.size(), st));
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.upd, 0, 4 * (size_t)SC, st));
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.err_flags, 0, 64, st));
  // The staging vectors die at return: wait for the copies.
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  f->n_seeds = S;
  f->n_events = n_ev;
  f->events_loaded = 1;
  return MKFG_OK;
}

// Enqueues the whole finding sequence of the uploaded batch on `st`:
// reset, then for every layer-plan step prep -> chi2 -> clone -> update,
// then the final merge.
static int enqueue_run(Finder* f, cudaStream_t st) {
  const int S = f->n_seeds;
  const int n_work = 4 * (f->host_cfg.max_steps + 2);
  const int threads_c = S * kSlots;
  const int grid_c = (threads_c + kBlock - 1) / kBlock;
  const int grid_w = (S * 32 + kBlock - 1) / kBlock;
  const int grid_p = std::min((S * kSlots * 4 + kBlock - 1) / kBlock, 148 * 16);
  k_reset<<<std::max(grid_c, (n_work + kBlock - 1) / kBlock), kBlock, 0, st>>>(f->ev, n_work);
  MKFG_CUDA_TRY(cudaMemsetAsync(f->ev.pair_count, 0, 4 * (size_t)(f->host_cfg.max_steps + 2), st));
  for (int step = 1; step <= f->host_cfg.max_steps; ++step) {
    k_prep<<<grid_c, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
    k_chi2<<<std::max(grid_p, 1), kBlock, 0, st>>>(f->ev, f->d_cfg, step);
    k_clone<<<grid_w, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
    k_update<<<grid_c, kBlock, 0, st>>>(f->ev, f->d_cfg, step);
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
  const int n_work = 4 * (f->host_cfg.max_steps + 2);
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

static int run_plain(mkfg_context* ctx, Finder* f) {
  if (f->n_seeds == 0) return MKFG_OK;
  return enqueue_run(f, ctx->stream);
}

// Same sequence captured once into a CUDA graph and replayed: one launch
// for the whole batch of events and all layer steps.
static int run_graph(mkfg_context* ctx, Finder* f) {
  if (f->n_seeds == 0) return MKFG_OK;
  cudaStream_t st = ctx->stream;
  if (!f->graph) {
    cudaGraph_t g = nullptr;
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

static int download(mkfg_context* ctx, Finder* f, mkfg_find_out* out, int n_seeds_in) {
  const int S = f->n_seeds;
  const int m = f->host_cfg.max_cands;
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
  auto dn = [&](void* h, const void* d, size_t bytes) -> int {
    if (!h) return MKFG_OK;
    MKFG_CUDA_TRY(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st));
    return MKFG_OK;
  };
  const size_t ns = n_seeds_in;
  if ((rc = dn(out->n_cands, O.n_cands, 4 * ns))) return rc;
  if ((rc = dn(out->region, O.region, 4 * ns))) return rc;
  if ((rc = dn(out->par, O.par, 4 * 6 * ns * m))) return rc;
  if ((rc = dn(out->err, O.err, 4 * 21 * ns * m))) return rc;
  if ((rc = dn(out->chg, O.chg, 4 * ns * m))) return rc;
  if ((rc = dn(out->chi2, O.chi2, 4 * ns * m))) return rc;
  if ((rc = dn(out->score, O.score, 4 * ns * m))) return rc;
  if ((rc = dn(out->nfound, O.nfound, 4 * ns * m))) return rc;
  if ((rc = dn(out->ntot, O.ntot, 4 * ns * m))) return rc;
  if ((rc = dn(out->noverlap, O.noverlap, 4 * ns * m))) return rc;
  if ((rc = dn(out->ninside, O.ninside, 4 * ns * m))) return rc;
  if ((rc = dn(out->ntail, O.ntail, 4 * ns * m))) return rc;
  if ((rc = dn(out->hit_idx, O.hit_idx, 4 * ns * m * kExportHits))) return rc;
  if ((rc = dn(out->hit_lyr, O.hit_lyr, 4 * ns * m * kExportHits))) return rc;
  int flags = 0;
  MKFG_CUDA_TRY(cudaMemcpyAsync(&flags, f->ev.err_flags, 4, cudaMemcpyDeviceToHost, st));
  MKFG_CUDA_TRY(cudaStreamSynchronize(st));
  if (flags & kErrArena)
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

extern "C" int mkfg_find_work(mkfg_context* ctx, int64_t* active_cands, int64_t* hit_pairs,
                              int64_t* updates, int32_t* steps) {
  int rc = activate(ctx);
  if (rc) return rc;
  Finder* f = finder_of(ctx);
  MKFG_REQUIRE(f->events_loaded, "no event uploaded");
  const int ns = f->host_cfg.max_steps + 2;
  std::vector<int> work(4 * (size_t)ns), pairs(ns);
  MKFG_CUDA_TRY(cudaMemcpyAsync(work.data(), f->ev.work, 4 * work.size(), cudaMemcpyDeviceToHost, ctx->stream));
  MKFG_CUDA_TRY(cudaMemcpyAsync(pairs.data(), f->ev.pair_count, 4 * pairs.size(), cudaMemcpyDeviceToHost, ctx->stream));
  MKFG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  int64_t a = 0, p = 0, u = 0, p2 = 0, cs = 0;
  for (int i = 0; i < ns; ++i) {
    a += work[4 * i];
    u += work[4 * i + 1];
    p2 += work[4 * i + 2];
    cs += work[4 * i + 3];
    p += pairs[i];
  }
  f->last_chi2_evals = p2;
  f->last_seeds_cloned = cs;
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
  return download(ctx, f, out, n_seeds);
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
    SeedInput si{ev->n_seeds, ev->seed_par, ev->seed_chg, ev->seed_nhits, ev->seed_hit_layer,
                 ev->seed_hit_index};
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
