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
#include "Hit.h"
#include "MaterialEffects.h"
#include "Track.h"
#include "TrackerInfo.h"
#include "mkFit/FindingFoos.h"
#include "mkFit/HitStructures.h"
#include "mkFit/IterationConfig.h"
#include "mkFit/KalmanUtilsMPlex.h"
#include "mkFit/MkBuilder.h"
#include "mkFit/MkFinder.h"
#include "mkFit/MkFitter.h"
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

}  // extern "C"
