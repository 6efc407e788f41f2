// Oracle driver: plain-C entry points into the reference's own CPU Matriplex
// path (trackreco/mkFit), compiled in-process from the reference sources.
//
// TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py may load this library, and only as the
// checker or the timed CPU reference; the GPU product never routes through
// it.
//
// Every function builds the reference's own data structures from flat SoA
// arrays, calls the reference's public worker / builder API exactly as its
// drivers do, and copies the results back into flat arrays:
//   fit      : mkFit/fittestMPlex.cc:65-100 (InputTracksForFit ->
//              FitTracksWithInterSlurp -> OutputFittedTracks)
//   finding  : mkFit/buildtestMPlex.cc:320-366 (find_tracks_load_seeds ->
//              FindTracksCloneEngine) and mkFit/MkBuilder.cc:267-290
//              (export of the best / all comb candidates)
//   geometry : Geoms/CMS-2017.cc:717-859 (plugin creator, called directly)
#include "Config.h"
#include "Event.h"
#include "Hit.h"
#include "MaterialEffects.h"
#include "Track.h"
#include "TrackerInfo.h"
#include "mkFit/CandCloner.h"
#include "mkFit/FindingFoos.h"
#include "mkFit/HitStructures.h"
#include "mkFit/IterationConfig.h"
#include "mkFit/KalmanUtilsMPlex.h"
#include "mkFit/MkBuilder.h"
#include "mkFit/MkFinder.h"
#include "mkFit/MkFitter.h"
#include "mkFit/MkStdSeqs.h"
#include "mkFit/PropagationMPlex.h"
#include "tbb/parallel_for.h"
#include "tbb/shim_pool.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

using namespace mkfit;

// The CMS-2017 plugin exports its creator through this symbol
// (Geoms/CMS-2017.cc:862).
extern void* TrackerInfoCrator_ptr;

namespace {

double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

bool g_cms2017_loaded = false;
// ref_find runs MkBuilder::BackwardFit after the clone engine when set.
bool g_backward_fit = false;
bool g_backward_search = false;
// Row width of the seed-hit arrays the finding drivers take.
int g_seed_hit_stride = 4;
// CMS-2017 iteration whose configuration the geometry export and the
// finding drivers use (Config::ItrInfo index).
int g_iteration = 0;
// ref_find: hits masked by earlier iterations (one byte per hit in the
// event's layer order, 1 = masked), given to the builder through the
// reference's IterationMaskIfc; NULL = no mask.
const unsigned char* g_hit_mask = nullptr;
// When set, ref_find also runs the output selection of run_OneIteration
// (qfilter_nan_n_silly, export_best_comb_cands(.., true),
// find_and_remove_duplicates) and marks the surviving seeds here (by label).
int* g_keep_out = nullptr;
// Quality filters ref_find applies with MkBuilder::filter_comb_cands, as
// run_OneIteration does (mkFit/buildtestMPlex.cc:676-719): after the clone
// engine (g_qf_pre) and after the backward fit / search (g_qf_post); -1 =
// none; kinds in the order of qfilter_by_kind.
int g_qf_pre = -1, g_qf_post = -1, g_qf_min_hits = 0;
float g_bs_x = 0.f, g_bs_y = 0.f;
// Duplicate removal of the output selection (find_and_remove_duplicates,
// mkFit/MkStdSeqs.cc:605-630, by the branch it takes): 0
// find_duplicates_sharedhits_pixelseed, 1 find_duplicates_sharedhits,
// 2 find_duplicates + remove_duplicates, 3 none (do_remove_duplicates off).
int g_dup_mode = 0;
// Duplicate parameters of the selection replacing iteration 0's when >= 0:
// fracSharedHits, drth_central, drth_obarrel, drth_forward.
float g_dup_params[4] = {-1.f, -1.f, -1.f, -1.f};

void set_material(const float* rl_grid, const float* xi_grid) {
  if (rl_grid && xi_grid) {
    std::memcpy(Config::RlgridME, rl_grid, sizeof(Config::RlgridME));
    std::memcpy(Config::XigridME, xi_grid, sizeof(Config::XigridME));
  } else {
    fillZRgridME();
  }
}

Track make_track(int i, int n, const float* par, const float* err, const int* chg) {
  SVector6 p;
  SMatrixSym66 e;
  for (int k = 0; k < 6; ++k) p[k] = par[k * n + i];
  for (int k = 0; k < 21; ++k) e.Array()[k] = err[k * n + i];
  TrackState ts;
  ts.parameters = p;
  ts.errors = e;
  ts.charge = chg[i];
  Track t(ts, 0.f, i, 0, nullptr);
  return t;
}

Hit make_hit(int i, int n, const float* pos, const float* err) {
  SVector3 p(pos[0 * n + i], pos[1 * n + i], pos[2 * n + i]);
  SMatrixSym33 e;
  for (int k = 0; k < 6; ++k) e.Array()[k] = err[k * n + i];
  return Hit(p, e, -1);
}

}  // namespace

extern "C" {

// Number of host threads the reference's TBB loops run on.
void ref_set_threads(int n) { tbbshim::Pool::instance().resize(n); }
// The shim's cut of parallel_for ranges (tbb/parallel_for.h): 0 near-equal
// pieces of at most the grain, 1 recursive halving, 2 near-equal pieces of
// at most twice the grain, 3 one piece, 4 random pieces of half the grain
// to the grain.
void ref_set_task_split(int mode) { tbbshim::split_mode() = mode; }
// Seed of the random cut (mode 4).
void ref_set_task_split_seed(unsigned seed) { tbbshim::split_seed() = seed; }
int ref_get_threads() { return tbbshim::Pool::instance().concurrency(); }

// Matriplex width this build was compiled with (8 for AVX2, 16 for AVX-512).
int ref_matriplex_width() { return NN; }

//------------------------------------------------------------------------------
// Plain Kalman fit (reference MkFitter path).
//
// Inputs (lane-fastest SoA, n = n_tracks):
//   par[6][n], err[21][n] (packed lower triangle), chg[n]
//   hit_pos[n_layers][3][n], hit_err[n_layers][6][n]: hit of track i on layer l
//   rl_grid/xi_grid: material (z,r) grid [300][120] or null for the CMS map
//   pflags: PropagationFlags bits (1 = param B field, 2 = material)
// Outputs: out_par[6][n], out_err[21][n], out_chg[n].
// Runs the timed loop `repeat` times; *best_seconds = best wall time.
// The reference packs exactly Config::nLayers (=10) hits per track.
int ref_fit(int n_tracks, int n_layers, const float* par, const float* err, const int* chg,
            const float* hit_pos, const float* hit_err, const float* rl_grid,
            const float* xi_grid, int pflags, int repeat, float* out_par, float* out_err,
            int* out_chg, double* best_seconds) {
  if (n_layers != Config::nLayers || n_tracks <= 0) return -1;
  set_material(rl_grid, xi_grid);
  Config::forward_fit_pflags = PropagationFlags(pflags);

  std::vector<HitVec> layer_hits(n_layers);
  for (int l = 0; l < n_layers; ++l) {
    layer_hits[l].reserve(n_tracks);
    for (int i = 0; i < n_tracks; ++i)
      layer_hits[l].push_back(make_hit(i, n_tracks, hit_pos + size_t(l) * 3 * n_tracks,
                                       hit_err + size_t(l) * 6 * n_tracks));
  }
  std::vector<Track> sim(n_tracks);
  for (int i = 0; i < n_tracks; ++i) {
    sim[i] = make_track(i, n_tracks, par, err, chg);
    for (int l = 0; l < n_layers; ++l) sim[i].addHitIdx(i, l, 0.f);
  }
  std::vector<Track> rec(n_tracks);

  const int count = (n_tracks + NN - 1) / NN;
  double best = 1e30;
  for (int r = 0; r < std::max(1, repeat); ++r) {
    const double t0 = now_s();
    // Same loop structure as the reference's runFittingTestPlex.
    tbb::parallel_for(
        tbb::blocked_range<int>(0, count, std::max(1, Config::numSeedsPerTask / NN)),
        [&](const tbb::blocked_range<int>& rng) {
          std::unique_ptr<MkFitter> mkfp(new (_mm_malloc(sizeof(MkFitter), 64)) MkFitter);
          mkfp->SetNhits(n_layers);
          for (int it = rng.begin(); it < rng.end(); ++it) {
            const int beg = it * NN;
            const int end = std::min(beg + NN, n_tracks);
            mkfp->InputTracksForFit(sim, beg, end);
            mkfp->FitTracksWithInterSlurp(layer_hits, end - beg);
            mkfp->OutputFittedTracks(rec, beg, end);
          }
          MkFitter* raw = mkfp.release();
          raw->~MkFitter();
          _mm_free(raw);
        });
    best = std::min(best, now_s() - t0);
  }
  if (best_seconds) *best_seconds = best;

  for (int i = 0; i < n_tracks; ++i) {
    for (int k = 0; k < 6; ++k) out_par[k * n_tracks + i] = rec[i].parameters()[k];
    for (int k = 0; k < 21; ++k) out_err[k * n_tracks + i] = rec[i].errors().Array()[k];
    out_chg[i] = rec[i].charge();
  }
  return 0;
}

// Steered fit (MkFitter::FitTracksSteered, mkFit/MkFitter.cc:473-503):
// step l propagates to the hit's radius and runs the barrel update when
// is_barrel[l], else to the hit's z and the endcap update. Tracks enter
// through InputTracksAndHits (mkFit/MkFitter.cc:56-91), any number of
// steps up to Config::nMaxTrkHits - 1. Arrays as in ref_fit.
int ref_fit_steered(int n_tracks, int n_layers, const int* is_barrel, const float* par,
                    const float* err, const int* chg, const float* hit_pos, const float* hit_err,
                    const float* rl_grid, const float* xi_grid, int pflags, float* out_par,
                    float* out_err, int* out_chg) {
  if (n_layers <= 0 || n_layers > Config::nMaxTrkHits - 1 || n_tracks <= 0) return -1;
  set_material(rl_grid, xi_grid);
  std::vector<HitVec> layer_hits(n_layers);
  for (int l = 0; l < n_layers; ++l) {
    layer_hits[l].reserve(n_tracks);
    for (int i = 0; i < n_tracks; ++i)
      layer_hits[l].push_back(make_hit(i, n_tracks, hit_pos + size_t(l) * 3 * n_tracks,
                                       hit_err + size_t(l) * 6 * n_tracks));
  }
  std::vector<Track> sim(n_tracks);
  for (int i = 0; i < n_tracks; ++i) {
    sim[i] = make_track(i, n_tracks, par, err, chg);
    for (int l = 0; l < n_layers; ++l) sim[i].addHitIdx(i, l, 0.f);
  }
  std::vector<Track> rec(n_tracks);
  std::unique_ptr<bool[]> barrel(new bool[n_layers]);
  for (int l = 0; l < n_layers; ++l) barrel[l] = is_barrel[l] != 0;
  const int count = (n_tracks + NN - 1) / NN;
  tbb::parallel_for(
      tbb::blocked_range<int>(0, count, std::max(1, Config::numSeedsPerTask / NN)),
      [&](const tbb::blocked_range<int>& rng) {
        std::unique_ptr<MkFitter> mkfp(new (_mm_malloc(sizeof(MkFitter), 64)) MkFitter);
        mkfp->SetNhits(n_layers);
        for (int it = rng.begin(); it < rng.end(); ++it) {
          const int beg = it * NN;
          const int end = std::min(beg + NN, n_tracks);
          mkfp->InputTracksAndHits(sim, layer_hits, beg, end);
          mkfp->FitTracksSteered(barrel.get(), end - beg, nullptr, PropagationFlags(pflags));
          mkfp->OutputFittedTracks(rec, beg, end);
        }
        MkFitter* raw = mkfp.release();
        raw->~MkFitter();
        _mm_free(raw);
      });
  for (int i = 0; i < n_tracks; ++i) {
    for (int k = 0; k < 6; ++k) out_par[k * n_tracks + i] = rec[i].parameters()[k];
    for (int k = 0; k < 21; ++k) out_err[k * n_tracks + i] = rec[i].errors().Array()[k];
    out_chg[i] = rec[i].charge();
  }
  return 0;
}

}  // extern "C"

//==============================================================================
// CMS-2017 geometry and clone-engine finding
//==============================================================================

namespace {

// Exposes the builder's comb-candidate storage for export (the reference
// keeps it protected; MkBuilder.h:92-100).
struct RefBuilder : public MkBuilder {
  EventOfCombCandidates& eocc() { return m_event_of_comb_cands; }
};

constexpr int kLayerDescLen = 32;

void ensure_cms2017() {
  if (g_cms2017_loaded) return;
  Config::silent = true;
  auto creator = (TrackerInfoCreator_foo)TrackerInfoCrator_ptr;
  creator(Config::TrkInfo, Config::ItrInfo, false);
  fillZRgridME();
  g_cms2017_loaded = true;
}

// MkFinder::FindCandidatesCloneEngine's pixel same-layer check reads the
// first three hit-on-track nodes of the comb candidate
// (mkFit/MkFinder.cc:1195-1210); for a seed of two hits the third is
// storage the vector has reserved but not written, whose content depends on
// what earlier calls left on the heap. Writing nodes on no layer (-1) into
// that storage right after the seeds are loaded -- by growing the vector
// into its reserved capacity and shrinking it back, so no element is
// written outside the vector's size -- makes the read see the same nodes
// every time, so the reference's result no longer depends on call history.
// Runs outside the timed region (the reference times FindTracksCloneEngine
// only, mkFit/buildtestMPlex.cc:362-366).
void fill_unused_nodes(RefBuilder& b) {
  EventOfCombCandidates& eocc = b.eocc();
  HoTNode blank;
  blank.m_hot = HitOnTrack(-1, -1);
  blank.m_chi2 = 0.f;
  blank.m_prev_idx = -1;
  for (int i = 0; i < eocc.m_size; ++i) {
    std::vector<HoTNode>& v = eocc[i].m_hots;
    const size_t n = v.size();
    const size_t upto = std::min<size_t>(v.capacity(), 3);
    if (n < upto) {
      v.resize(upto, blank);  // within capacity: the storage does not move
      v.resize(n);
    }
  }
}

// The StdSeq quality filters (mkFit/MkStdSeqs.h:39-148) by code: 0
// qfilter_nan_n_silly, 1 qfilter_n_hits, 2 qfilter_n_hits_pixseed,
// 3 qfilter_n_layers, 4 qfilter_n_layers_pixelLess, 5 qfilter_pixelLessFwd,
// 6 qfilter_pixelLessBkwd.
bool qfilter_by_kind(const TrackCand& t, int kind, int min_hits, const BeamSpot& bs) {
  const TrackerInfo& ti = Config::TrkInfo;
  switch (kind) {
    case 0: return StdSeq::qfilter_nan_n_silly(t);
    case 1: return StdSeq::qfilter_n_hits(t, min_hits);
    case 2: return StdSeq::qfilter_n_hits_pixseed(t, min_hits);
    case 3: return StdSeq::qfilter_n_layers(t, bs, ti);
    case 4: return StdSeq::qfilter_n_layers_pixelLess(t, bs);
    case 5: return StdSeq::qfilter_pixelLessFwd(t, bs, ti);
    case 6: return StdSeq::qfilter_pixelLessBkwd(t, bs, ti);
  }
  return true;
}

// One event's hits into the reference's containers, as ref_find builds
// them (Hit::setupAsPixel / setupAsStrip, EventOfHits::SuckInHits).
// layer_hits must outlive eoh: LayerOfHits points into it.
void load_event_hits(int n_layers, const int* layer_begin, const float* hpos, const float* herr,
                     const int* detid, const int* cpcm, std::vector<HitVec>& layer_hits,
                     EventOfHits& eoh) {
  const int nh_tot = layer_begin[n_layers];
  layer_hits.assign(n_layers, HitVec());
  for (int l = 0; l < n_layers; ++l)
    for (int h = layer_begin[l]; h < layer_begin[l + 1]; ++h) {
      Hit hit = make_hit(h, nh_tot, hpos, herr);
      if (cpcm[h] < 0)
        hit.setupAsPixel(detid[h], 1, 1);
      else
        hit.setupAsStrip(detid[h], cpcm[h], 1);
      layer_hits[l].push_back(hit);
    }
  for (int l = 0; l < n_layers; ++l) eoh.SuckInHits(l, layer_hits[l]);
}

constexpr int kNumQFilters = 7;

// MkBuilder::filter_comb_cands with one of the filters. The reference reads
// front() of every comb candidate, so an empty one is refused (-3) rather
// than read.
int apply_qfilter(RefBuilder& b, int kind) {
  EventOfCombCandidates& eocc = b.eocc();
  for (int i = 0; i < eocc.m_size; ++i)
    if (eocc[i].empty()) return -3;
  BeamSpot bs;
  bs.x = g_bs_x;
  bs.y = g_bs_y;
  b.filter_comb_cands([&](const TrackCand& t) { return qfilter_by_kind(t, kind, g_qf_min_hits, bs); });
  return 0;
}

// find_and_remove_duplicates by branch (g_dup_mode codes).
void remove_dups(TrackVec& out, int mode, const IterationParams& p) {
  if (mode == 0)
    StdSeq::find_duplicates_sharedhits_pixelseed(out, p.fracSharedHits, p.drth_central, p.drth_obarrel,
                                                 p.drth_forward);
  else if (mode == 1)
    StdSeq::find_duplicates_sharedhits(out, p.fracSharedHits);
  else if (mode == 2) {
    StdSeq::find_duplicates(out);
    StdSeq::remove_duplicates(out);
  }
}

}  // namespace

extern "C" {

// ref_find: also run the backward fit (MkBuilder::BackwardFit,
// mkFit/MkBuilder.cc:2153-2253) on the best candidate of every seed, as
// run_OneIteration does with do_backward_fit (mkFit/buildtestMPlex.cc).
void ref_set_backward_fit(int on) { g_backward_fit = on != 0; }

// ref_find then runs the backward search as run_OneIteration does:
// CompactifyHitStorageForBestCand, BackwardFit, BeginBkwSearch,
// FindTracksCloneEngine(IT_BkwSearch), EndBkwSearch.
void ref_set_backward_search(int on) { g_backward_search = on != 0; }

// Iteration (0-9) whose configuration ref_cms2017_sizes / _export,
// ref_find, ref_event_prep and ref_find_batch use; -1 if out of range.
int ref_set_iteration(int it) {
  ensure_cms2017();
  if (it < 0 || it >= (int)Config::ItrInfo.m_iterations.size()) return -1;
  g_iteration = it;
  return 0;
}

// ref_find: per-hit mask of hits used by earlier iterations (see
// g_hit_mask); NULL switches it off.
void ref_set_hit_mask(const unsigned char* mask) { g_hit_mask = mask; }

// Row width of seed_hit_layer / seed_hit_index in ref_find, ref_event_prep
// and ref_find_batch (default 4).
void ref_set_seed_hit_stride(int w) { g_seed_hit_stride = w > 0 ? w : 4; }

// ref_find: keep[ns] (by seed label) receives 1 for the seeds whose best
// candidate survives run_OneIteration's output selection
// (mkFit/buildtestMPlex.cc:721-731), 0 otherwise; NULL switches it off.
void ref_set_select_output(int* keep) { g_keep_out = keep; }

// ref_find: quality filters applied with filter_comb_cands after the clone
// engine (pre) and after the backward fit / search (post), by
// qfilter_by_kind code (-1 none); min_hits for qfilter_n_hits*, the beam
// spot for the d0 cuts. dup_mode picks the duplicate removal of the output
// selection (0 pixelseed, 1 sharedhits, 2 find_duplicates, 3 none).
void ref_set_iteration_filters(int pre, int post, int min_hits, float bs_x, float bs_y, int dup_mode,
                               const float* dup_params) {
  for (int k = 0; k < 4; ++k) g_dup_params[k] = dup_params ? dup_params[k] : -1.f;
  g_qf_pre = pre;
  g_qf_post = post;
  g_qf_min_hits = min_hits;
  g_bs_x = bs_x;
  g_bs_y = bs_y;
  g_dup_mode = dup_mode;
}

// The quality filters on candidates given as exported hit lists (hits in
// chain order, oldest first, missing-hit entries included). Each one is
// rebuilt as the clone engine holds it: CombCandidate::ImportSeed of a seed
// made of the first nseed[i] entries (which sets the 4-bit seed-hit count),
// then TrackCand::addHitIdx for the rest. par[n][6], err[n][21], chg[n],
// ntot[n], hit_idx / hit_lyr[n][w]. out[i] bit k: filter k (qfilter_by_kind
// code) passes.
int ref_qfilters(int n, const float* par, const float* err, const int* chg, const int* nseed,
                 const int* ntot, const int* hit_idx, const int* hit_lyr, int w, int min_hits,
                 float bs_x, float bs_y, int* out) {
  ensure_cms2017();
  if (n <= 0) return 0;
  EventOfCombCandidates eocc;
  eocc.Reset(n, 1, 2 * w);
  BeamSpot bs;
  bs.x = bs_x;
  bs.y = bs_y;
  for (int i = 0; i < n; ++i) {
    if (nseed[i] > ntot[i] || ntot[i] > w) return -1;
    TrackState ts;
    for (int k = 0; k < 6; ++k) ts.parameters[k] = par[i * 6 + k];
    for (int k = 0; k < 21; ++k) ts.errors.Array()[k] = err[i * 21 + k];
    ts.charge = chg[i];
    Track seed(ts, 0.f, i, 0, nullptr);
    for (int k = 0; k < nseed[i]; ++k) seed.addHitIdx(hit_idx[i * w + k], hit_lyr[i * w + k], 0.f);
    eocc.InsertSeed(seed, 0);
    TrackCand& tc = eocc[i].front();
    for (int k = nseed[i]; k < ntot[i]; ++k) tc.addHitIdx(hit_idx[i * w + k], hit_lyr[i * w + k], 0.f);
    int m = 0;
    for (int q = 0; q < kNumQFilters; ++q)
      if (qfilter_by_kind(tc, q, min_hits, bs)) m |= 1 << q;
    out[i] = m;
  }
  return 0;
}

// Duplicate removal of run_OneIteration's output on exported tracks (hits
// without missing entries), by g_dup_mode code: par[n][6], chg, score,
// label, nfound, nh[n], hit_idx / hit_lyr[n][w]; every track has algorithm
// `algo`. The parameters are iteration 0's duplicate parameters with frac
// and the three dR thresholds replaced. keep[i]: 1 when track i survives.
int ref_dups(int mode, int n, const float* par, const int* chg, const float* score, const int* label,
             int algo, const int* nfound, const int* nh, const int* hit_idx, const int* hit_lyr, int w,
             float frac, float drth_c, float drth_ob, float drth_fw, int* keep) {
  ensure_cms2017();
  TrackVec tv;
  tv.reserve(n);
  for (int i = 0; i < n; ++i) {
    if (nh[i] > w) return -1;
    TrackState ts;
    for (int k = 0; k < 6; ++k) ts.parameters[k] = par[i * 6 + k];
    ts.charge = chg[i];
    Track t(ts, 0.f, label[i], 0, nullptr);
    t.resizeHits(nh[i], nfound[i]);
    for (int k = 0; k < nh[i]; ++k) t.setHitIdxAtPos(k, HitOnTrack{hit_idx[i * w + k], hit_lyr[i * w + k]});
    t.setScore(score[i]);
    t.setAlgoint(algo);
    // The position rides in chi2, which no duplicate test reads.
    t.setChi2((float)i);
    tv.push_back(t);
  }
  IterationParams p = Config::ItrInfo[0].m_params;
  p.fracSharedHits = frac;
  p.drth_central = drth_c;
  p.drth_obarrel = drth_ob;
  p.drth_forward = drth_fw;
  remove_dups(tv, mode, p);
  std::fill(keep, keep + n, 0);
  for (const Track& t : tv) keep[(int)t.chi2()] = 1;
  return 0;
}

// The selection settings of CMS-2017 iteration `it` (Geoms/CMS-2017.cc):
// iv = {track algorithm, requires_quality_filter, requires_dupclean_tight,
// minHitsQF, requires_seed_hit_sorting}, fv = {fracSharedHits, drth_central, drth_obarrel,
// drth_forward}.
int ref_cms2017_iteration(int it, int* iv, float* fv) {
  ensure_cms2017();
  if (it < 0 || it >= (int)Config::ItrInfo.m_iterations.size()) return -1;
  const IterationConfig& c = Config::ItrInfo[it];
  iv[0] = c.m_track_algorithm;
  iv[1] = c.m_requires_quality_filter;
  iv[2] = c.m_requires_dupclean_tight;
  iv[3] = c.m_params.minHitsQF;
  iv[4] = c.m_requires_seed_hit_sorting;
  fv[0] = c.m_params.fracSharedHits;
  fv[1] = c.m_params.drth_central;
  fv[2] = c.m_params.drth_obarrel;
  fv[3] = c.m_params.drth_forward;
  return 0;
}

// Geometry export sizes: n_layers, n_regions, max plan length.
int ref_cms2017_sizes(int* n_layers, int* n_regions, int* max_plan) {
  ensure_cms2017();
  const IterationConfig& ic = Config::ItrInfo[g_iteration];
  *n_layers = (int)Config::TrkInfo.m_layers.size();
  *n_regions = ic.m_n_regions;
  int mp = 0;
  for (auto& sp : ic.m_steering_params) mp = std::max(mp, (int)sp.m_layer_plan.size());
  *max_plan = mp;
  return 0;
}

// Exports the CMS-2017 detector description and iteration-0 configuration
// (Geoms/CMS-2017.cc:717-790 and the generated CMS-2017.acc tables).
//   layer_desc[n_layers][32]: see mkfit_b200/geometry.py LAYER_FIELDS
//   plans[n_regions][max_plan] (-1 padded), plan_len/pickup/bkfit_last/
//   bksearch_pickup[n_regions], region_order[n_regions]
//   iter_params[8]: maxCands, maxHoles, maxConsecHoles, chi2Cut_min,
//                   chi2CutOverlap, pTCutOverlap, nlayers_per_seed, -
//   flags[4]: requires_prop_to_hit, inter pflags, intra pflags, bkfit pflags
//   eta[3]: transition begin/end, endcap end
//   rl/xi[300*120]: material grid after fillZRgridME()
int ref_cms2017_export(float* layer_desc, int* plans, int* plan_len, int* pickup,
                       int* bkfit_last, int* bksearch_pickup, int* region_order,
                       float* iter_params, int* flags, float* eta, float* rl, float* xi) {
  ensure_cms2017();
  const TrackerInfo& ti = Config::TrkInfo;
  const IterationConfig& ic = Config::ItrInfo[g_iteration];
  int n_layers, n_regions, max_plan;
  ref_cms2017_sizes(&n_layers, &n_regions, &max_plan);
  for (int l = 0; l < n_layers; ++l) {
    const LayerInfo& L = ti.m_layers[l];
    const IterationLayerConfig& C = ic.m_layer_configs[l];
    float* d = layer_desc + l * kLayerDescLen;
    std::fill(d, d + kLayerDescLen, 0.f);
    d[0] = L.is_barrel();
    d[1] = L.m_rin;
    d[2] = L.m_rout;
    d[3] = L.m_zmin;
    d[4] = L.m_zmax;
    d[5] = L.m_propagate_to;
    d[6] = L.m_q_bin;
    d[7] = L.m_has_r_range_hole;
    d[8] = L.m_has_r_range_hole ? L.m_hole_r_min : 0.f;
    d[9] = L.m_has_r_range_hole ? L.m_hole_r_max : 0.f;
    d[10] = L.is_pix_lyr();
    d[11] = L.is_stereo_lyr();
    d[12] = C.m_select_min_dphi;
    d[13] = C.m_select_max_dphi;
    d[14] = C.m_select_min_dq;
    d[15] = C.m_select_max_dq;
    d[16] = C.c_dp_sf; d[17] = C.c_dp_0; d[18] = C.c_dp_1; d[19] = C.c_dp_2;
    d[20] = C.c_dq_sf; d[21] = C.c_dq_0; d[22] = C.c_dq_1; d[23] = C.c_dq_2;
    d[24] = C.c_c2_sf; d[25] = C.c_c2_0; d[26] = C.c_c2_1; d[27] = C.c_c2_2;
    d[28] = (float)L.m_layer_type;
    d[29] = L.is_seed_lyr();
    d[30] = L.is_tib_lyr() || L.is_tob_lyr() ? 1.f : (L.is_tid_lyr() || L.is_tec_lyr() ? 2.f : 0.f);
  }
  for (int r = 0; r < n_regions; ++r) {
    const SteeringParams& sp = ic.m_steering_params[r];
    plan_len[r] = (int)sp.m_layer_plan.size();
    pickup[r] = sp.m_fwd_search_pickup;
    bkfit_last[r] = sp.m_bkw_fit_last;
    bksearch_pickup[r] = sp.m_bkw_search_pickup;
    for (int i = 0; i < max_plan; ++i)
      plans[r * max_plan + i] = i < plan_len[r] ? sp.m_layer_plan[i].m_layer : -1;
    region_order[r] = ic.m_region_order[r];
  }
  const IterationParams& ip = ic.m_params;
  iter_params[0] = ip.maxCandsPerSeed;
  iter_params[1] = ip.maxHolesPerCand;
  iter_params[2] = ip.maxConsecHoles;
  iter_params[3] = ip.chi2Cut_min;
  iter_params[4] = ip.chi2CutOverlap;
  iter_params[5] = ip.pTCutOverlap;
  iter_params[6] = ip.nlayers_per_seed;
  iter_params[7] = 0;
  flags[0] = Config::finding_requires_propagation_to_hit_pos;
  flags[1] = Config::finding_inter_layer_pflags._raw_ & 3;
  flags[2] = Config::finding_intra_layer_pflags._raw_ & 3;
  flags[3] = Config::backward_fit_pflags._raw_ & 3;
  eta[0] = ti.m_eta_trans_beg;
  eta[1] = ti.m_eta_trans_end;
  eta[2] = ti.m_eta_ecap_end;
  std::memcpy(rl, Config::RlgridME, sizeof(Config::RlgridME));
  std::memcpy(xi, Config::XigridME, sizeof(Config::XigridME));
  return 0;
}

// MkFinder::SelectHitIndices on given states (taken as propagated to layer
// `layer`: Par[iP] / Err[iP]) against one event's hits, built as in
// ref_find; the selected iteration's windows. par[6][n], err[21][n]
// (lane-fastest), chg[n]. Out: xsize[n] (XHitSize), xidx[n][16] (XHitArr,
// -1 after the last hit).
int ref_select_hit_indices(int n_layers_in, const int* layer_begin, const float* hpos,
                           const float* herr, const int* detid, const int* cpcm, int layer, int n,
                           const float* par, const float* err, const int* chg, int* xsize, int* xidx) {
  ensure_cms2017();
  const int n_layers = (int)Config::TrkInfo.m_layers.size();
  if (n_layers_in != n_layers || layer < 0 || layer >= n_layers) return -1;
  std::vector<HitVec> layer_hits;
  EventOfHits eoh(Config::TrkInfo);
  load_event_hits(n_layers, layer_begin, hpos, herr, detid, cpcm, layer_hits, eoh);
  const IterationConfig& itconf = Config::ItrInfo[g_iteration];
  TrackVec tracks;
  tracks.reserve(n);
  for (int i = 0; i < n; ++i) tracks.push_back(make_track(i, n, par, err, chg));
  std::unique_ptr<MkFinder> mkf(new MkFinder);
  mkf->Setup(itconf.m_params, itconf.m_layer_configs[layer], nullptr);
  for (int beg = 0; beg < n; beg += NN) {
    const int end = std::min(beg + NN, n);
    mkf->InputTracksAndHitIdx(tracks, beg, end, true);
    mkf->SelectHitIndices(eoh.m_layers_of_hits[layer], end - beg);
    for (int i = beg; i < end; ++i) {
      const int x = mkf->XHitSize.At(i - beg, 0, 0);
      xsize[i] = x;
      for (int k = 0; k < 16; ++k) xidx[i * 16 + k] = k < x ? mkf->XHitArr.At(i - beg, k, 0) : -1;
    }
  }
  mkf->Release();
  return 0;
}

// Candidate i of a worker driver as comb candidate i of eocc, alone in it:
// state, counters and the given hit-on-track nodes (index, layer pairs;
// the candidate's last node is the last one given).
static void worker_cand(EventOfCombCandidates& eocc, int i, int n, const float* par, const float* err,
                 const int* chg, const HitOnTrack* nodes, int n_nodes) {
  CombCandidate& cc = eocc[i];
  int prev = -1;
  for (int j = 0; j < n_nodes; ++j) prev = cc.AddHit(nodes[j], 0.f, prev);
  cc.emplace_back(TrackCand(make_track(i, n, par, err, chg), &cc));
  cc.back().setLastCcIndex(prev);
  cc.m_state = CombCandidate::Finding;
}

// MkFinder::FindCandidatesCloneEngine (mkFit/MkFinder.cc:1116-1284) on
// given states (Par[iP], taken as propagated to `layer`) with the given
// counters, after the reference's own SelectHitIndices on them, as
// find_tracks_in_layers calls the two (mkFit/MkBuilder.cc:1960-1990). Each
// candidate is alone in a comb candidate whose first three nodes lie on
// hot_layers[i][0..2] (the pixel same-layer check reads them); the chi2
// cut set as ref_find sets it (chi2_cut, zero_c2). Out:
// xsize[n] (XHitSize), and the records the cloner received per candidate,
// in order: n_rec[n], r_hit / r_module / r_chi2 (chi2_hit) / r_score
// [n][17].
int ref_ce_records(int n_layers_in, const int* layer_begin, const float* hpos, const float* herr,
                   const int* detid, const int* cpcm, int layer, int n, const float* par,
                   const float* err, const int* chg, const int* nfound, const int* nover,
                   const int* ninside, const int* ntail, const float* cchi2, const int* hot_layers,
                   float chi2_cut, int zero_c2, int* xsize, int* n_rec, int* r_hit, int* r_module,
                   float* r_chi2, float* r_score) {
  ensure_cms2017();
  fillZRgridME();  // the fit entry may have replaced the material grid
  const int n_layers = (int)Config::TrkInfo.m_layers.size();
  if (n_layers_in != n_layers || layer < 0 || layer >= n_layers || n <= 0) return -1;
  std::vector<HitVec> layer_hits;
  EventOfHits eoh(Config::TrkInfo);
  load_event_hits(n_layers, layer_begin, hpos, herr, detid, cpcm, layer_hits, eoh);
  // The chi2 cut as ref_find sets it (chi2Cut_min, dynamic terms zeroed
  // when zero_c2).
  IterationConfig itconf = Config::ItrInfo[g_iteration];
  itconf.m_params.chi2Cut_min = chi2_cut;
  if (zero_c2)
    for (auto& lc : itconf.m_layer_configs) lc.c_c2_0 = lc.c_c2_1 = lc.c_c2_2 = 0.f;
  EventOfCombCandidates eocc;
  eocc.Reset(n, 1, 8);
  eocc.m_size = n;
  for (int i = 0; i < n; ++i) {
    HitOnTrack nodes[3];
    for (int j = 0; j < 3; ++j) nodes[j] = HitOnTrack{0, hot_layers[i * 3 + j]};
    worker_cand(eocc, i, n, par, err, chg, nodes, 3);
    TrackCand& t = eocc[i].back();
    t.setNFoundHits(nfound[i]);
    t.setNOverlapHits(nover[i]);
    t.setNInsideMinusOneHits(ninside[i]);
    t.setNTailMinusOneHits(ntail[i]);
    t.setChi2(cchi2[i]);
  }
  std::vector<std::pair<int, int>> idxs(n), upd_list;
  for (int i = 0; i < n; ++i) idxs[i] = {i, 0};
  std::vector<std::vector<TrackCand>> extras(n);
  CandCloner cloner;
  cloner.Setup(itconf.m_params);
  cloner.begin_eta_bin(&eocc, &upd_list, &extras, 0, n);
  cloner.begin_layer(layer);
  const LayerOfHits& loh = eoh.m_layers_of_hits[layer];
  const FindingFoos& ff = FindingFoos::get_finding_foos(loh.is_barrel());
  std::unique_ptr<MkFinder> mkf(new MkFinder);
  mkf->Setup(itconf.m_params, itconf.m_layer_configs[layer], nullptr);
  for (int beg = 0; beg < n; beg += NN) {
    const int end = std::min(beg + NN, n);
    mkf->InputTracksAndHitIdx(eocc.m_candidates, idxs, beg, end, true);
    mkf->SelectHitIndices(loh, end - beg);
    for (int i = beg; i < end; ++i) xsize[i] = mkf->XHitSize.At(i - beg, 0, 0);
    mkf->FindCandidatesCloneEngine(loh, cloner, 0, end - beg, ff);
  }
  for (int i = 0; i < n; ++i) {
    const std::vector<IdxChi2List>& v = cloner.m_hits_to_add[i];
    n_rec[i] = (int)std::min<size_t>(v.size(), 17);
    for (int k = 0; k < 17; ++k) {
      const bool live = k < n_rec[i];
      r_hit[i * 17 + k] = live ? v[k].hitIdx : 0;
      r_module[i * 17 + k] = live ? (int)v[k].module : 0;
      r_chi2[i * 17 + k] = live ? v[k].chi2_hit : 0.f;
      r_score[i * 17 + k] = live ? v[k].score : 0.f;
    }
  }
  mkf->Release();
  cloner.Release();
  return 0;
}

// MkFinder::UpdateWithLastHit + CopyOutParErr (mkFit/MkFinder.cc:
// 1291-1335) as find_tracks_in_layers calls them (InputTracksAndHitIdx
// with inputProp, mkFit/MkBuilder.cc:2020-2035): given states, each
// updated with hit hit_idx[i] of `layer` (its comb candidate's last node).
int ref_update_with_last_hit(int n_layers_in, const int* layer_begin, const float* hpos,
                             const float* herr, const int* detid, const int* cpcm, int layer, int n,
                             const float* par, const float* err, const int* chg,
                             const int* hit_idx, float* out_par, float* out_err, int* out_chg) {
  ensure_cms2017();
  fillZRgridME();  // the fit entry may have replaced the material grid
  const int n_layers = (int)Config::TrkInfo.m_layers.size();
  if (n_layers_in != n_layers || layer < 0 || layer >= n_layers || n <= 0) return -1;
  std::vector<HitVec> layer_hits;
  EventOfHits eoh(Config::TrkInfo);
  load_event_hits(n_layers, layer_begin, hpos, herr, detid, cpcm, layer_hits, eoh);
  const IterationConfig& itconf = Config::ItrInfo[g_iteration];
  EventOfCombCandidates eocc;
  eocc.Reset(n, 1, 2);
  eocc.m_size = n;
  for (int i = 0; i < n; ++i) {
    const HitOnTrack node{hit_idx[i], layer};
    worker_cand(eocc, i, n, par, err, chg, &node, 1);
  }
  std::vector<std::pair<int, int>> idxs(n);
  for (int i = 0; i < n; ++i) idxs[i] = {i, 0};
  const LayerOfHits& loh = eoh.m_layers_of_hits[layer];
  const FindingFoos& ff = FindingFoos::get_finding_foos(loh.is_barrel());
  std::unique_ptr<MkFinder> mkf(new MkFinder);
  mkf->Setup(itconf.m_params, itconf.m_layer_configs[layer], nullptr);
  for (int beg = 0; beg < n; beg += NN) {
    const int end = std::min(beg + NN, n);
    mkf->InputTracksAndHitIdx(eocc.m_candidates, idxs, beg, end, true);
    mkf->UpdateWithLastHit(loh, end - beg, ff);
    mkf->CopyOutParErr(eocc.m_candidates, end - beg, false);
  }
  for (int i = 0; i < n; ++i) {
    const TrackCand& t = eocc[i][0];
    for (int k = 0; k < 6; ++k) out_par[k * n + i] = t.parameters()[k];
    for (int k = 0; k < 21; ++k) out_err[k * n + i] = t.errors().Array()[k];
    out_chg[i] = t.charge();
  }
  mkf->Release();
  return 0;
}

// CandCloner::ProcessSeedRange (mkFit/CandCloner.cc:36-189) on given
// seeds at `layer`, through the cloner as find_tracks_in_layers drives it
// (begin_layer, add_cand, end_layer), with maxCandsPerSeed = max_cands
// and the selected iteration's overlap cuts. Candidate slot k = 8 s + c;
// par / err [6|21][8 n_seeds], records [8 n_seeds][17], held_back 0/1/2
// (2: a stop node added, as find_tracks_handle_missed_layers does). Each
// candidate starts from a node of its own (so its lineage can be traced);
// its overlap memory is filled from its hit records under the overlap
// chi2 cut, in record order, as FindCandidatesCloneEngine fills it. Out
// per new slot: state, counters, parent slot, the hit and overlap hit it
// added (-100000 / -1 for a held-back copy), the hit it takes the Kalman
// update with (-1: not on the update list); per seed the best short
// candidate.
int ref_clone_seeds(int layer, int n_seeds, int max_cands, const int* n_cands, const float* par,
                    const float* err, const int* chg, const float* chi2, const float* score,
                    const int* nfound, const int* nmiss, const int* nover, const int* ninside,
                    const int* ntail, const int* held_back, const int* n_rec, const int* rec_hit,
                    const int* rec_module, const float* rec_chi2, const float* rec_score,
                    const int* bshort_valid, const float* bshort_score, int* o_ncand,
                    float* o_par, float* o_err, int* o_chg, float* o_chi2, float* o_score,
                    int* o_nfound, int* o_nmiss, int* o_nover, int* o_ninside, int* o_ntail,
                    int* o_parent, int* o_hit, int* o_ovl, int* o_upd, int* o_bvalid,
                    float* o_bscore, int* o_bnfound, float* o_bchi2) {
  ensure_cms2017();
  if (n_seeds <= 0 || max_cands < 1 || max_cands > 8) return -1;
  IterationParams params = Config::ItrInfo[g_iteration].m_params;
  params.maxCandsPerSeed = max_cands;
  const int S = n_seeds, SC = 8 * n_seeds;
  EventOfCombCandidates eocc;
  eocc.Reset(S, max_cands, 64);
  eocc.m_size = S;
  std::vector<std::vector<TrackCand>> extras(S);
  std::vector<int> n_setup(S);
  for (int s = 0; s < S; ++s) {
    if (n_cands[s] < 1 || n_cands[s] > max_cands) return -2;
    CombCandidate& cc = eocc[s];
    cc.m_state = CombCandidate::Finding;
    for (int c = 0; c < n_cands[s]; ++c) cc.AddHit(HitOnTrack{0, layer - 1}, 0.f, -1);
    for (int c = 0; c < n_cands[s]; ++c) {
      const int k = 8 * s + c;
      cc.emplace_back(TrackCand(make_track(k, SC, par, err, chg), &cc));
      TrackCand& t = cc.back();
      t.setLastCcIndex(c);
      t.setNFoundHits(nfound[k]);
      t.setNMissingHits(nmiss[k]);
      t.setNOverlapHits(nover[k]);
      t.setNInsideMinusOneHits(ninside[k]);
      t.setNTailMinusOneHits(ntail[k]);
      t.setChi2(chi2[k]);
      t.setScore(score[k]);
      for (int j = 0; j < n_rec[k]; ++j) {
        const int r = k * 17 + j;
        if (rec_hit[r] >= 0 && rec_chi2[r] < params.chi2CutOverlap)
          t.considerHitForOverlap(rec_hit[r], rec_module[r], rec_chi2[r]);
      }
    }
    for (int c = 0; c < n_cands[s]; ++c) {
      const int k = 8 * s + c;
      if (held_back[k] == 0) continue;
      extras[s].push_back(cc[c]);
      if (held_back[k] == 2) extras[s].back().addHitIdx(-2, layer, 0.0f);
    }
    if (bshort_valid[s]) {
      cc.m_best_short_cand = cc[0];
      cc.m_best_short_cand.setScore(bshort_score[s]);
    } else {
      cc.m_best_short_cand.resetShortTrack();
    }
    n_setup[s] = (int)cc.m_hots.size();
  }
  std::vector<std::pair<int, int>> upd_list;
  CandCloner cloner;
  cloner.Setup(params);
  cloner.begin_eta_bin(&eocc, &upd_list, &extras, 0, S);
  cloner.begin_layer(layer);
  for (int s = 0; s < S; ++s)
    for (int c = 0; c < n_cands[s]; ++c) {
      const int k = 8 * s + c;
      for (int j = 0; j < n_rec[k]; ++j) {
        const int r = k * 17 + j;
        IdxChi2List h{};
        h.trkIdx = c;
        h.hitIdx = rec_hit[r];
        h.module = (unsigned)rec_module[r];
        h.chi2_hit = rec_chi2[r];
        h.score = rec_score[r];
        cloner.add_cand(s, h);
      }
    }
  cloner.end_layer();
  std::vector<int> upd_of(SC, -1);
  for (const auto& u : upd_list) upd_of[8 * u.first + u.second] = 1;
  for (int s = 0; s < S; ++s) {
    const CombCandidate& cc = eocc[s];
    o_ncand[s] = (int)cc.size();
    for (int c = 0; c < 8; ++c) {
      const int k = 8 * s + c;
      o_parent[k] = -1;
      o_hit[k] = -100000;
      o_ovl[k] = -1;
      o_upd[k] = -1;
      if (c >= (int)cc.size()) continue;
      const TrackCand& t = cc[c];
      for (int e = 0; e < 6; ++e) o_par[e * SC + k] = t.parameters()[e];
      for (int e = 0; e < 21; ++e) o_err[e * SC + k] = t.errors().Array()[e];
      o_chg[k] = t.charge();
      o_chi2[k] = t.chi2();
      o_score[k] = t.score();
      o_nfound[k] = t.nFoundHits();
      o_nmiss[k] = t.nMissingHits();
      o_nover[k] = t.nOverlapHits();
      o_ninside[k] = t.nInsideMinusOneHits();
      o_ntail[k] = t.nTailMinusOneHits();
      // Nodes added by the clone step (above the setup nodes), last first.
      int node = t.lastCcIndex(), added[2], n_added = 0;
      while (node >= n_setup[s] && n_added < 2) {
        added[n_added++] = node;
        node = cc.m_hots[node].m_prev_idx;
      }
      if (node >= n_cands[s]) node = cc.m_hots[node].m_prev_idx;  // a setup stop node
      o_parent[k] = node;
      if (n_added == 2) {
        o_hit[k] = cc.m_hots[added[1]].m_hot.index;
        o_ovl[k] = cc.m_hots[added[0]].m_hot.index;
      } else if (n_added == 1) {
        o_hit[k] = cc.m_hots[added[0]].m_hot.index;
      }
      if (upd_of[k] > 0) o_upd[k] = cc.m_hots[t.lastCcIndex()].m_hot.index;
    }
    const TrackCand& b = cc.m_best_short_cand;
    o_bvalid[s] = b.combCandidate() != nullptr;
    o_bscore[s] = b.score();
    o_bnfound[s] = b.nFoundHits();
    o_bchi2[s] = b.chi2();
  }
  cloner.Release();
  return 0;
}

// The backward search's IterationParams of the selected iteration
// (IterationConfig::m_backward_params, set by SetupBackwardSearch_*):
// bk[8] in the iter_params layout, and flags[2] = {m_backward_drop_seed_hits,
// m_backward_fit_min_hits}.
int ref_cms2017_backward_params(float* bk, int* flags) {
  ensure_cms2017();
  const IterationConfig& ic = Config::ItrInfo[g_iteration];
  const IterationParams& ip = ic.m_backward_params;
  bk[0] = ip.maxCandsPerSeed;
  bk[1] = ip.maxHolesPerCand;
  bk[2] = ip.maxConsecHoles;
  bk[3] = ip.chi2Cut_min;
  bk[4] = ip.chi2CutOverlap;
  bk[5] = ip.pTCutOverlap;
  bk[6] = ip.nlayers_per_seed;
  bk[7] = 0;
  flags[0] = ic.m_backward_drop_seed_hits;
  flags[1] = ic.m_backward_fit_min_hits;
  return 0;
}

// Clone-engine combinatorial finding on one event, CMS-2017 geometry,
// iteration 0 with overrides (the benchmark workloads' settings: max cands
// per seed, flat chi2 cut: the dynamic c2 parameters are zeroed when
// zero_c2 != 0).
//
// Hits: layer l occupies [layer_begin[l], layer_begin[l+1]) of pos[3][nh],
//   err[6][nh]; detid[nh] (12-bit module id), cpcm[nh] (< 0: pixel hit,
//   otherwise the strip charge per cm given to Hit::setupAsStrip).
// Seeds: par[6][ns], err[21][ns], chg[ns]; seed_nhits[ns] (<= w) hits given
//   as seed_hit_layer[ns][w], seed_hit_index[ns][w] (index within layer;
//   w = 4 unless ref_set_seed_hit_stride says otherwise).
// Outputs, indexed by input seed (label), m = max_cands:
//   n_cands[ns], region[ns], sorted_pos[ns] (position after the seed sort),
//   c_par[ns*m][6], c_err[ns*m][21], c_chg, c_chi2, c_score, c_nfound,
//   c_ntot, c_noverlap, c_ninside, c_ntail [ns*m],
//   c_hit_idx / c_hit_lyr [ns*m][64].
int ref_find(int n_layers_in, const int* layer_begin, const float* hpos, const float* herr,
             const int* detid, const int* cpcm, int ns, const float* spar, const float* serr,
             const int* schg, const int* seed_nhits, const int* seed_hit_layer,
             const int* seed_hit_index, int max_cands, float chi2_cut, int zero_c2, int repeat,
             int* n_cands, int* region, int* sorted_pos, float* c_par, float* c_err, int* c_chg,
             float* c_chi2, float* c_score, int* c_nfound, int* c_ntot, int* c_noverlap,
             int* c_ninside, int* c_ntail, int* c_hit_idx, int* c_hit_lyr, double* best_seconds) {
  ensure_cms2017();
  fillZRgridME();  // the fit entry may have replaced the material grid
  const int n_layers = (int)Config::TrkInfo.m_layers.size();
  if (n_layers_in != n_layers) return -1;

  IterationConfig itconf = Config::ItrInfo[g_iteration];
  itconf.m_params.maxCandsPerSeed = max_cands;
  itconf.m_backward_params.maxCandsPerSeed = max_cands;
  itconf.m_params.chi2Cut_min = chi2_cut;
  itconf.m_backward_params.chi2Cut_min = chi2_cut;
  if (zero_c2)
    for (auto& lc : itconf.m_layer_configs) lc.c_c2_0 = lc.c_c2_1 = lc.c_c2_2 = 0.f;

  const int nh_tot = layer_begin[n_layers];
  std::vector<HitVec> layer_hits(n_layers);
  for (int l = 0; l < n_layers; ++l) {
    for (int h = layer_begin[l]; h < layer_begin[l + 1]; ++h) {
      Hit hit = make_hit(h, nh_tot, hpos, herr);
      if (cpcm[h] < 0)
        hit.setupAsPixel(detid[h], 1, 1);
      else
        hit.setupAsStrip(detid[h], cpcm[h], 1);
      layer_hits[l].push_back(hit);
    }
  }
  EventOfHits eoh(Config::TrkInfo);
  for (int l = 0; l < n_layers; ++l) eoh.SuckInHits(l, layer_hits[l]);

  TrackVec seeds;
  seeds.reserve(ns);
  for (int s = 0; s < ns; ++s) {
    Track t = make_track(s, ns, spar, serr, schg);
    t.setLabel(s);
    for (int k = 0; k < seed_nhits[s]; ++k)
      t.addHitIdx(seed_hit_index[s * g_seed_hit_stride + k], seed_hit_layer[s * g_seed_hit_stride + k], 0.f);
    seeds.push_back(t);
  }
  // run_OneIteration drops seeds with NaN / silly covariances first, and
  // sorts the seeds' hits by layer for the iterations that ask for it.
  MkBuilder::seed_post_cleaning(seeds);
  if (itconf.m_requires_seed_hit_sorting)
    for (auto& t : seeds) t.sortHitsByLayer();

  IterationMaskIfc mask_ifc;
  if (g_hit_mask) {
    mask_ifc.m_mask_vector.resize(n_layers);
    for (int l = 0; l < n_layers; ++l)
      for (int h = layer_begin[l]; h < layer_begin[l + 1]; ++h)
        mask_ifc.m_mask_vector[l].push_back(g_hit_mask[h] != 0);
  }
  MkJob job({Config::TrkInfo, itconf, eoh, g_hit_mask ? &mask_ifc : nullptr});
  double best = 1e30;
  RefBuilder builder;
  for (int r = 0; r < std::max(1, repeat); ++r) {
    builder.begin_event(&job, nullptr, "ref_find");
    builder.find_tracks_load_seeds(seeds);
    fill_unused_nodes(builder);
    const double t0 = now_s();
    builder.FindTracksCloneEngine();
    if (g_qf_pre >= 0 && apply_qfilter(builder, g_qf_pre)) return -3;
    if (g_backward_search) {
      // run_OneIteration with m_backward_search (mkFit/buildtestMPlex.cc:700-714).
      builder.CompactifyHitStorageForBestCand(itconf.m_backward_drop_seed_hits,
                                              itconf.m_backward_fit_min_hits);
      builder.BackwardFit();
      builder.BeginBkwSearch();
      builder.FindTracksCloneEngine(SteeringParams::IT_BkwSearch);
      builder.EndBkwSearch();
    } else if (g_backward_fit) {
      builder.BackwardFit();
    }
    if (g_qf_post >= 0 && apply_qfilter(builder, g_qf_post)) return -3;
    best = std::min(best, now_s() - t0);
    if (r + 1 < std::max(1, repeat)) builder.end_event();
  }
  if (best_seconds) *best_seconds = best;

  if (g_keep_out) {
    // Output selection of run_OneIteration on a copy of the builder's
    // result, leaving the comb candidates themselves as exported below.
    EventOfCombCandidates& src = builder.eocc();
    std::fill(g_keep_out, g_keep_out + ns, 0);
    TrackVec out;
    out.reserve(src.m_size);
    for (int i = 0; i < src.m_size; ++i) {
      if (src[i].empty()) continue;
      const TrackCand& t = src[i].front();
      if (!StdSeq::qfilter_nan_n_silly(t)) continue;
      out.emplace_back(t.exportTrack(true));
    }
    IterationParams dp = itconf.m_params;
    if (g_dup_params[0] >= 0.f) dp.fracSharedHits = g_dup_params[0];
    if (g_dup_params[1] >= 0.f) dp.drth_central = g_dup_params[1];
    if (g_dup_params[2] >= 0.f) dp.drth_obarrel = g_dup_params[2];
    if (g_dup_params[3] >= 0.f) dp.drth_forward = g_dup_params[3];
    remove_dups(out, g_dup_mode, dp);
    for (const Track& t : out)
      if (t.label() >= 0 && t.label() < ns) g_keep_out[t.label()] = 1;
  }

  EventOfCombCandidates& eocc = builder.eocc();
  std::fill(n_cands, n_cands + ns, 0);
  for (int i = 0; i < eocc.m_size; ++i) {
    CombCandidate& cc = eocc[i];
    if (cc.empty()) continue;
    const int s = cc.front().label();
    if (s < 0 || s >= ns) return -2;
    sorted_pos[s] = i;
    region[s] = cc.front().getEtaRegion();
    n_cands[s] = std::min((int)cc.size(), max_cands);
    for (int c = 0; c < n_cands[s]; ++c) {
      const TrackCand& tc = cc[c];
      const int slot = s * max_cands + c;
      for (int k = 0; k < 6; ++k) c_par[slot * 6 + k] = tc.parameters()[k];
      for (int k = 0; k < 21; ++k) c_err[slot * 21 + k] = tc.errors().Array()[k];
      c_chg[slot] = tc.charge();
      c_chi2[slot] = tc.chi2();
      c_score[slot] = tc.score();
      c_nfound[slot] = tc.nFoundHits();
      c_ntot[slot] = tc.nTotalHits();
      c_noverlap[slot] = tc.nOverlapHits();
      c_ninside[slot] = tc.nInsideMinusOneHits();
      c_ntail[slot] = tc.nTailMinusOneHits();
      Track t = tc.exportTrack(false);
      const int nh = std::min(t.nTotalHits(), Config::nMaxTrkHits);
      for (int k = 0; k < Config::nMaxTrkHits; ++k) {
        c_hit_idx[slot * Config::nMaxTrkHits + k] = k < nh ? t.getHitIdx(k) : -100;
        c_hit_lyr[slot * Config::nMaxTrkHits + k] = k < nh ? t.getHitLyr(k) : -100;
      }
    }
  }
  builder.end_event();
  return 0;
}

}  // extern "C"

extern "C" {

// The reference's own hit index (LayerOfHits::SuckInHits) and seed order
// (MkBuilder::import_seeds) for one event, in the layout of
// mkfg_prepare_event_host: bins per layer (first | last << 16) over
// nq x 256, sorted-position -> index-within-layer, seed order and regions.
int ref_event_prep(int n_layers_in, const int* layer_begin, const float* hpos, const float* herr,
                   const int* detid, const int* cpcm, int ns, const float* spar,
                   const float* serr, const int* schg, const int* seed_nhits,
                   const int* seed_hit_layer, const int* seed_hit_index, unsigned* bins,
                   int* n_bins, int* srank, int* seed_order, int* seed_region) {
  ensure_cms2017();
  const int n_layers = (int)Config::TrkInfo.m_layers.size();
  if (n_layers_in != n_layers) return -1;
  const int nh_tot = layer_begin[n_layers];
  std::vector<HitVec> layer_hits(n_layers);
  for (int l = 0; l < n_layers; ++l)
    for (int h = layer_begin[l]; h < layer_begin[l + 1]; ++h) {
      Hit hit = make_hit(h, nh_tot, hpos, herr);
      if (cpcm[h] < 0) hit.setupAsPixel(detid[h], 1, 1);
      else hit.setupAsStrip(detid[h], cpcm[h], 1);
      layer_hits[l].push_back(hit);
    }
  EventOfHits eoh(Config::TrkInfo);
  for (int l = 0; l < n_layers; ++l) eoh.SuckInHits(l, layer_hits[l]);
  int off = 0;
  for (int l = 0; l < n_layers; ++l) {
    const LayerOfHits& L = eoh[l];
    if (bins)
      for (int q = 0; q < L.m_nq; ++q)
        for (int p = 0; p < Config::m_nphi; ++p) {
          auto b = L.m_phi_bin_infos[q][p];
          bins[off + q * Config::m_nphi + p] = unsigned(b.first) | (unsigned(b.second) << 16);
        }
    off += L.m_nq * Config::m_nphi;
    if (srank)
      for (int i = 0; i < layer_begin[l + 1] - layer_begin[l]; ++i)
        srank[layer_begin[l] + i] = L.GetOriginalHitIndex(i);
  }
  *n_bins = off;
  if (!seed_order) return 0;

  TrackVec seeds;
  for (int s = 0; s < ns; ++s) {
    Track t = make_track(s, ns, spar, serr, schg);
    t.setLabel(s);
    for (int k = 0; k < seed_nhits[s]; ++k)
      t.addHitIdx(seed_hit_index[s * g_seed_hit_stride + k], seed_hit_layer[s * g_seed_hit_stride + k], 0.f);
    seeds.push_back(t);
  }
  MkBuilder::seed_post_cleaning(seeds);
  IterationConfig itconf = Config::ItrInfo[g_iteration];
  MkJob job({Config::TrkInfo, itconf, eoh, nullptr});
  RefBuilder builder;
  builder.begin_event(&job, nullptr, "ref_event_prep");
  builder.find_tracks_load_seeds(seeds);
  EventOfCombCandidates& eocc = builder.eocc();
  for (int i = 0; i < eocc.m_size; ++i) {
    const TrackCand& tc = eocc[i].front();
    seed_order[i] = tc.label();
    seed_region[tc.label()] = tc.getEtaRegion();
  }
  builder.end_event();
  return 0;
}

}  // extern "C"

//------------------------------------------------------------------------------
// Several events "in flight" (mkFit/mkFit.cc:308-425): events are found
// concurrently on the shim thread pool, each with its own builder, while
// every event's FindTracksCloneEngine also parallelises over its regions
// and seed chunks. Inputs are the per-event arrays concatenated:
//   hit_off[n_ev+1], seed_off[n_ev+1] (prefix sums), layer_begin[n_ev][L+1]
//   (event-local), pos[3][NH], err[6][NH], detid[NH], cpcm[NH],
//   spar[6][NS], serr[21][NS], schg[NS], seed_nhits[NS], hit layer/index
//   [NS][4]. Outputs per concatenated seed as in ref_find. The timed region
//   (best of `repeat`) covers seed import + FindTracksCloneEngine of all
//   events; the hit-index build precedes it, as in the reference's own
//   timing (mkFit/buildtestMPlex.cc:342-366).
extern "C" int ref_find_batch(int n_ev, const int* hit_off, const int* seed_off,
                              const int* layer_begin, const float* hpos, const float* herr,
                              const int* detid, const int* cpcm, const float* spar,
                              const float* serr, const int* schg, const int* seed_nhits,
                              const int* seed_hit_layer, const int* seed_hit_index, int max_cands,
                              float chi2_cut, int zero_c2, int repeat, int* n_cands,
                              int* best_nfound, int* best_ntot, int* best_hit_idx,
                              int* best_hit_lyr, double* best_seconds) {
  ensure_cms2017();
  fillZRgridME();
  const int L = (int)Config::TrkInfo.m_layers.size();
  IterationConfig itconf = Config::ItrInfo[g_iteration];
  itconf.m_params.maxCandsPerSeed = max_cands;
  itconf.m_backward_params.maxCandsPerSeed = max_cands;
  itconf.m_params.chi2Cut_min = chi2_cut;
  itconf.m_backward_params.chi2Cut_min = chi2_cut;
  if (zero_c2)
    for (auto& lc : itconf.m_layer_configs) lc.c_c2_0 = lc.c_c2_1 = lc.c_c2_2 = 0.f;
  const int NH = hit_off[n_ev], NS = seed_off[n_ev];

  std::vector<std::vector<HitVec>> hits(n_ev, std::vector<HitVec>(L));
  std::vector<std::unique_ptr<EventOfHits>> eohs(n_ev);
  std::vector<TrackVec> seeds(n_ev);
  for (int e = 0; e < n_ev; ++e) {
    const int* lb = layer_begin + (size_t)e * (L + 1);
    for (int l = 0; l < L; ++l)
      for (int h = lb[l]; h < lb[l + 1]; ++h) {
        const int g = hit_off[e] + h;
        Hit hit = make_hit(g, NH, hpos, herr);
        if (cpcm[g] < 0) hit.setupAsPixel(detid[g], 1, 1);
        else hit.setupAsStrip(detid[g], cpcm[g], 1);
        hits[e][l].push_back(hit);
      }
    eohs[e].reset(new EventOfHits(Config::TrkInfo));
    for (int l = 0; l < L; ++l) eohs[e]->SuckInHits(l, hits[e][l]);
    for (int s = seed_off[e]; s < seed_off[e + 1]; ++s) {
      Track t = make_track(s, NS, spar, serr, schg);
      t.setLabel(s);
      for (int k = 0; k < seed_nhits[s]; ++k)
        t.addHitIdx(seed_hit_index[s * g_seed_hit_stride + k], seed_hit_layer[s * g_seed_hit_stride + k], 0.f);
      seeds[e].push_back(t);
    }
    MkBuilder::seed_post_cleaning(seeds[e]);
  }
  std::vector<std::unique_ptr<RefBuilder>> builders(n_ev);
  std::vector<std::unique_ptr<MkJob>> jobs(n_ev);
  for (int e = 0; e < n_ev; ++e) {
    builders[e].reset(new RefBuilder);
    jobs[e].reset(new MkJob({Config::TrkInfo, itconf, *eohs[e], nullptr}));
  }
  double best = 1e30;
  for (int r = 0; r < std::max(1, repeat); ++r) {
    // Seed loading outside the timed region, as the reference times it
    // (mkFit/buildtestMPlex.cc:353-366); every event then in flight.
    for (int e = 0; e < n_ev; ++e) {
      if (r > 0) builders[e]->end_event();
      builders[e]->begin_event(jobs[e].get(), nullptr, "ref_find_batch");
      builders[e]->find_tracks_load_seeds(seeds[e]);
      fill_unused_nodes(*builders[e]);
    }
    const double t0 = now_s();
    tbb::parallel_for(tbb::blocked_range<int>(0, n_ev, 1), [&](const tbb::blocked_range<int>& rg) {
      for (int e = rg.begin(); e < rg.end(); ++e) builders[e]->FindTracksCloneEngine();
    });
    best = std::min(best, now_s() - t0);
  }
  if (best_seconds) *best_seconds = best;
  std::fill(n_cands, n_cands + NS, 0);
  for (int e = 0; e < n_ev; ++e) {
    EventOfCombCandidates& eocc = builders[e]->eocc();
    for (int i = 0; i < eocc.m_size; ++i) {
      CombCandidate& cc = eocc[i];
      if (cc.empty()) continue;
      const int s = cc.front().label();
      n_cands[s] = std::min((int)cc.size(), max_cands);
      const TrackCand& tc = cc.front();
      best_nfound[s] = tc.nFoundHits();
      best_ntot[s] = tc.nTotalHits();
      Track t = tc.exportTrack(false);
      const int nh = std::min(t.nTotalHits(), Config::nMaxTrkHits);
      for (int k = 0; k < Config::nMaxTrkHits; ++k) {
        best_hit_idx[s * Config::nMaxTrkHits + k] = k < nh ? t.getHitIdx(k) : -100;
        best_hit_lyr[s * Config::nMaxTrkHits + k] = k < nh ? t.getHitLyr(k) : -100;
      }
    }
    builders[e]->end_event();
  }
  return 0;
}

// Seed cleaning by the reference (StdSeq::clean_cms_seedtracks_iter,
// mkFit/MkStdSeqs.cc:115-311) of one event's seeds: params = {pt_thr,
// dzmax_bh, drmax_bh, dzmax_bl, drmax_bl, dzmax_eh, drmax_eh, dzmax_el,
// drmax_el} in IterationConfig::set_seed_cleaning_params order. keep[ns]
// marks the surviving seeds; their hit lists go to out_* ([ns][max_hits]).
// Returns the number kept.
extern "C" int ref_clean_seeds(int ns, const float* spar, const float* serr, const int* schg,
                               const int* seed_nhits, const int* seed_hit_layer,
                               const int* seed_hit_index, int in_hits, const float* params,
                               float beam_x, float beam_y, int max_hits, int* keep,
                               int* out_nhits, int* out_hit_layer, int* out_hit_index) {
  IterationConfig itconf;
  itconf.set_seed_cleaning_params(params[0], params[1], params[2], params[3], params[4],
                                  params[5], params[6], params[7], params[8]);
  BeamSpot bs;
  bs.x = beam_x;
  bs.y = beam_y;
  TrackVec seeds;
  seeds.reserve(ns);
  for (int s = 0; s < ns; ++s) {
    Track t = make_track(s, ns, spar, serr, schg);
    t.setLabel(s);
    for (int k = 0; k < seed_nhits[s]; ++k)
      t.addHitIdx(seed_hit_index[s * in_hits + k], seed_hit_layer[s * in_hits + k], 0.f);
    seeds.push_back(t);
  }
  StdSeq::clean_cms_seedtracks_iter(&seeds, itconf, bs);
  for (int s = 0; s < ns; ++s) keep[s] = 0;
  for (const Track& t : seeds) {
    const int s = t.label();
    keep[s] = 1;
    const int n = std::min(t.nTotalHits(), max_hits);
    out_nhits[s] = n;
    for (int k = 0; k < n; ++k) {
      const HitOnTrack h = t.getHitOnTrack(k);
      out_hit_layer[s * max_hits + k] = h.layer;
      out_hit_index[s * max_hits + k] = h.index;
    }
  }
  return (int)seeds.size();
}

// ---- memoryFile round trips through the reference's own DataFile / Event
// (Event.cc:123-444, 866-1000). Track vectors are passed as flat arrays:
// par [6][n], err [21][n], charge, chi2, score, status, label, hits_begin
// [n+1], hit_index, hit_layer.
namespace {

TrackVec tracks_from(int n, const float* par, const float* err, const int* chg, const float* chi2,
                     const float* score, const unsigned* status, const int* label,
                     const int* hits_begin, const int* hit_index, const int* hit_layer) {
  TrackVec tv;
  tv.reserve(n);
  for (int i = 0; i < n; ++i) {
    Track t = make_track(i, n, par, err, chg);
    for (int h = hits_begin[i]; h < hits_begin[i + 1]; ++h) t.addHitIdx(hit_index[h], hit_layer[h], 0.f);
    t.setChi2(chi2[i]);
    t.setScore(score[i]);
    t.setRawStatus(status[i]);
    t.setLabel(label[i]);
    tv.push_back(t);
  }
  return tv;
}

int tracks_to(const TrackVec& tv, int cap, int hcap, float* par, float* err, int* chg, float* chi2,
              float* score, unsigned* status, int* label, int* nfound, int* hits_begin,
              int* hit_index, int* hit_layer) {
  const int n = (int)tv.size();
  if (n > cap) return -1;
  hits_begin[0] = 0;
  for (int i = 0; i < n; ++i) {
    const Track& t = tv[i];
    for (int k = 0; k < 6; ++k) par[k * cap + i] = t.parameters()[k];
    for (int k = 0; k < 21; ++k) err[k * cap + i] = t.errors().Array()[k];
    chg[i] = t.charge();
    chi2[i] = t.chi2();
    score[i] = t.score();
    status[i] = t.getRawStatus();
    label[i] = t.label();
    nfound[i] = t.nFoundHits();
    const int nh = t.nTotalHits();
    if (hits_begin[i] + nh > hcap) return -1;
    for (int h = 0; h < nh; ++h) {
      hit_index[hits_begin[i] + h] = t.getHitIdx(h);
      hit_layer[hits_begin[i] + h] = t.getHitLyr(h);
    }
    hits_begin[i + 1] = hits_begin[i] + nh;
  }
  return n;
}

DataFile g_wfile;
int g_written = 0;

}  // namespace

extern "C" int ref_mf_write_begin(const char* path, int n_events, int extra_sections) {
  ensure_cms2017();
  g_written = 0;
  g_wfile.f_header = DataFileHeader();  // takes Config::nTotalLayers as set by the geometry
  g_wfile.OpenWrite(path, n_events, extra_sections);
  return g_wfile.f_fp ? 0 : -1;
}

// One event: hits [3][NH] / [6][NH] with layer_begin[n_layers+1], mcHitID,
// packed bits; masks [NH] (ignored unless the section is on); mc [n_mc][4];
// sim, seed and cmssw track vectors; beam spot[8]; sim track states.
extern "C" int ref_mf_write_event(
    int n_layers, const int* layer_begin, const float* pos, const float* herr, const int* mcid,
    const unsigned* packed, const unsigned long long* masks, int n_mc, const int* mc,
    int ns, const float* s_par, const float* s_err, const int* s_chg, const float* s_chi2,
    const float* s_score, const unsigned* s_status, const int* s_label, const int* s_hb,
    const int* s_hi, const int* s_hl, int nd, const float* d_par, const float* d_err,
    const int* d_chg, const float* d_chi2, const float* d_score, const unsigned* d_status,
    const int* d_label, const int* d_hb, const int* d_hi, const int* d_hl, int nc,
    const float* c_par, const float* c_err, const int* c_chg, const float* c_chi2,
    const float* c_score, const unsigned* c_status, const int* c_label, const int* c_hb,
    const int* c_hi, const int* c_hl, const float* beam, int n_states, const float* st_par,
    const float* st_err, const int* st_chg) {
  Event ev(g_written);
  const int NH = layer_begin[n_layers];
  ev.layerHits_.assign(n_layers, HitVec());
  ev.layerHitMasks_.assign(n_layers, std::vector<uint64_t>());
  for (int l = 0; l < n_layers; ++l) {
    for (int h = layer_begin[l]; h < layer_begin[l + 1]; ++h) {
      // Hit is a plain 44-byte record: fill its bytes as the file holds them.
      Hit hit;
      float f[9];
      for (int k = 0; k < 3; ++k) f[k] = pos[k * NH + h];
      for (int k = 0; k < 6; ++k) f[3 + k] = herr[k * NH + h];
      unsigned char* b = reinterpret_cast<unsigned char*>(&hit);
      std::memcpy(b, f, 36);
      std::memcpy(b + 36, &mcid[h], 4);
      std::memcpy(b + 40, &packed[h], 4);
      ev.layerHits_[l].push_back(hit);
      ev.layerHitMasks_[l].push_back(masks ? masks[h] : 0ull);
    }
  }
  ev.simHitsInfo_.clear();
  for (int i = 0; i < n_mc; ++i)
    ev.simHitsInfo_.push_back(MCHitInfo(mc[4 * i], mc[4 * i + 1], mc[4 * i + 2], mc[4 * i + 3]));
  ev.simTracks_ = tracks_from(ns, s_par, s_err, s_chg, s_chi2, s_score, s_status, s_label, s_hb, s_hi, s_hl);
  ev.seedTracks_ = tracks_from(nd, d_par, d_err, d_chg, d_chi2, d_score, d_status, d_label, d_hb, d_hi, d_hl);
  ev.cmsswTracks_ = tracks_from(nc, c_par, c_err, c_chg, c_chi2, c_score, c_status, c_label, c_hb, c_hi, c_hl);
  if (beam) std::memcpy(&ev.beamSpot_, beam, sizeof(BeamSpot));
  ev.simTrackStates_.clear();
  for (int i = 0; i < n_states; ++i) {
    TrackState ts;
    for (int k = 0; k < 6; ++k) ts.parameters[k] = st_par[k * n_states + i];
    for (int k = 0; k < 21; ++k) ts.errors.Array()[k] = st_err[k * n_states + i];
    ts.charge = st_chg[i];
    ev.simTrackStates_.push_back(ts);
  }
  ev.write_out(g_wfile);
  ++g_written;
  return 0;
}

extern "C" int ref_mf_write_end() {
  g_wfile.CloseWrite(g_written);
  return g_written;
}

// Reads event `which` of a file with the reference. counts out: n_layers,
// n_hits, n_mc, n_sim, n_seeds, n_cmssw, n_states. Hit arrays sized by
// hit_cap, track arrays by trk_cap (hits hcap). Returns 0, or -1 when a
// capacity is exceeded.
extern "C" int ref_mf_read(const char* path, int which, int hit_cap, int trk_cap, int hcap,
                           int* counts, int* layer_begin, float* pos, float* herr, int* mcid,
                           unsigned* packed, unsigned long long* masks, int* mc, float* tpar,
                           float* terr, int* tchg, float* tchi2, float* tscore, unsigned* tstatus,
                           int* tlabel, int* tnfound, int* thb, int* thi, int* thl, float* beam,
                           float* st_par, float* st_err, int* st_chg) {
  ensure_cms2017();
  DataFile df;
  const auto saved_seed = Config::seedInput;
  const bool saved_cmssw = Config::readCmsswTracks;
  Config::seedInput = simSeeds;  // OpenRead exits if cmsswSeeds and no seed section
  Config::readCmsswTracks = false;
  df.OpenRead(path, false);
  if (df.HasSeeds()) Config::seedInput = cmsswSeeds;  // read_in reads seeds only then
  Config::readCmsswTracks = df.HasCmsswTracks();
  Event ev(0);
  df.SkipNEvents(which);
  ev.read_in(df);
  Config::seedInput = saved_seed;
  Config::readCmsswTracks = saved_cmssw;
  df.Close();
  const int nl = (int)ev.layerHits_.size();
  layer_begin[0] = 0;
  for (int l = 0; l < nl; ++l) layer_begin[l + 1] = layer_begin[l] + (int)ev.layerHits_[l].size();
  const int NH = layer_begin[nl];
  if (NH > hit_cap) return -1;
  for (int l = 0; l < nl; ++l)
    for (int h = layer_begin[l]; h < layer_begin[l + 1]; ++h) {
      const Hit& hit = ev.layerHits_[l][h - layer_begin[l]];
      const unsigned char* b = reinterpret_cast<const unsigned char*>(&hit);
      float f[9];
      std::memcpy(f, b, 36);
      for (int k = 0; k < 3; ++k) pos[k * hit_cap + h] = f[k];
      for (int k = 0; k < 6; ++k) herr[k * hit_cap + h] = f[3 + k];
      std::memcpy(&mcid[h], b + 36, 4);
      std::memcpy(&packed[h], b + 40, 4);
      masks[h] = ev.layerHitMasks_[l][h - layer_begin[l]];
    }
  const int nm = (int)ev.simHitsInfo_.size();
  for (int i = 0; i < nm && i < hit_cap; ++i) {
    mc[4 * i] = ev.simHitsInfo_[i].mcTrackID_;
    mc[4 * i + 1] = ev.simHitsInfo_[i].layer_;
    mc[4 * i + 2] = ev.simHitsInfo_[i].ithLayerHit_;
    mc[4 * i + 3] = ev.simHitsInfo_[i].mcHitID_;
  }
  counts[0] = nl;
  counts[1] = NH;
  counts[2] = nm;
  const TrackVec* tv[3] = {&ev.simTracks_, &ev.seedTracks_, &ev.cmsswTracks_};
  for (int k = 0; k < 3; ++k) {
    const size_t o = (size_t)k * trk_cap, oh = (size_t)k * hcap;
    const int n = tracks_to(*tv[k], trk_cap, hcap, tpar + 6 * o, terr + 21 * o, tchg + o, tchi2 + o,
                            tscore + o, tstatus + o, tlabel + o, tnfound + o,
                            thb + (size_t)k * (trk_cap + 1), thi + oh, thl + oh);
    if (n < 0) return -1;
    counts[3 + k] = n;
  }
  std::memcpy(beam, &ev.beamSpot_, sizeof(BeamSpot));
  const int nst = (int)ev.simTrackStates_.size();
  if (nst > trk_cap) return -1;
  for (int i = 0; i < nst; ++i) {
    for (int k = 0; k < 6; ++k) st_par[k * trk_cap + i] = ev.simTrackStates_[i].parameters[k];
    for (int k = 0; k < 21; ++k) st_err[k * trk_cap + i] = ev.simTrackStates_[i].errors.Array()[k];
    st_chg[i] = ev.simTrackStates_[i].charge;
  }
  counts[6] = nst;
  return 0;
}
