// Test driver of the MkFitterGpu adapter (mkfit_b200/shims/MkFitterGpu.h):
// the reference's own fitting loop (mkFit/fittestMPlex.cc:65-100,
// runFittingTestPlex: InputTracksForFit -> FitTracksWithInterSlurp ->
// OutputFittedTracks over chunks of tracks) and the steered seed fit
// (InputTracksAndHits -> FitTracksSteered -> OutputFittedTracks), with
// MkFitterGpu in place of MkFitter and the reference's own Track / Hit /
// Config types. TEST INFRASTRUCTURE ONLY: loaded by tests/ to show that
// the adapter drops into a reference call site.
//
// Flat inputs as oracle/ref_driver.cc ref_fit: par[6][n], err[21][n],
// chg[n], hit_pos[n_layers][3][n], hit_err[n_layers][6][n]; `chunk` tracks
// per MkFitterGpu call (the reference uses NN).
#include "Config.h"
#include "Hit.h"
#include "MaterialEffects.h"
#include "Track.h"
#include "shims/MkFitterGpu.h"

#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

using namespace mkfit;

namespace {

mkfg_context* g_ctx = nullptr;

int context() {
  if (!g_ctx && mkfg_context_create(0, &g_ctx) != MKFG_OK) return -1;
  return 0;
}

void setup(int n, int n_layers, const float* par, const float* err, const int* chg,
           const float* hit_pos, const float* hit_err, const float* rl, const float* xi,
           std::vector<HitVec>& layer_hits, std::vector<Track>& tracks) {
  if (rl && xi) {
    std::memcpy(Config::RlgridME, rl, sizeof(Config::RlgridME));
    std::memcpy(Config::XigridME, xi, sizeof(Config::XigridME));
  } else {
    fillZRgridME();
  }
  layer_hits.assign(n_layers, HitVec());
  for (int l = 0; l < n_layers; ++l)
    for (int i = 0; i < n; ++i) {
      const float* p = hit_pos + (size_t)l * 3 * n;
      const float* e = hit_err + (size_t)l * 6 * n;
      SVector3 pos(p[i], p[n + i], p[2 * n + i]);
      SMatrixSym33 cov;
      for (int k = 0; k < 6; ++k) cov.Array()[k] = e[k * n + i];
      layer_hits[l].push_back(Hit(pos, cov, -1));
    }
  tracks.assign(n, Track());
  for (int i = 0; i < n; ++i) {
    SVector6 pv;
    SMatrixSym66 ev;
    for (int k = 0; k < 6; ++k) pv[k] = par[k * n + i];
    for (int k = 0; k < 21; ++k) ev.Array()[k] = err[k * n + i];
    TrackState ts;
    ts.parameters = pv;
    ts.errors = ev;
    ts.charge = chg[i];
    tracks[i] = Track(ts, 0.f, i, 0, nullptr);
    for (int l = 0; l < n_layers; ++l) tracks[i].addHitIdx(i, l, 0.f);
  }
}

void output(const std::vector<Track>& rec, int n, float* out_par, float* out_err, int* out_chg) {
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 6; ++k) out_par[k * n + i] = rec[i].parameters()[k];
    for (int k = 0; k < 21; ++k) out_err[k * n + i] = rec[i].errors().Array()[k];
    out_chg[i] = rec[i].charge();
  }
}

}  // namespace

extern "C" {

// runFittingTestPlex's loop with MkFitterGpu; Config::forward_fit_pflags
// = pflags. Returns 0, -1 on bad arguments or context failure, -2 when
// the adapter threw.
int shim_fit(int n, int n_layers, const float* par, const float* err, const int* chg,
             const float* hit_pos, const float* hit_err, const float* rl, const float* xi,
             int pflags, int chunk, float* out_par, float* out_err, int* out_chg) {
  if (n <= 0 || n_layers != Config::nLayers || chunk <= 0 || context()) return -1;
  Config::forward_fit_pflags = PropagationFlags(pflags);
  std::vector<HitVec> layer_hits;
  std::vector<Track> sim, rec;
  setup(n, n_layers, par, err, chg, hit_pos, hit_err, rl, xi, layer_hits, sim);
  rec.resize(n);
  try {
    MkFitterGpu mkfp(g_ctx);
    mkfp.SetNhits(n_layers);
    for (int beg = 0; beg < n; beg += chunk) {
      const int end = std::min(beg + chunk, n);
      mkfp.InputTracksForFit(sim, beg, end);
      mkfp.FitTracksWithInterSlurp(layer_hits, end - beg);
      mkfp.OutputFittedTracks(rec, beg, end);
    }
  } catch (const std::exception&) {
    return -2;
  }
  output(rec, n, out_par, out_err, out_chg);
  return 0;
}

// The steered fit with MkFitterGpu: step l is an endcap step when
// is_barrel[l] is 0.
int shim_fit_steered(int n, int n_layers, const int* is_barrel, const float* par, const float* err,
                     const int* chg, const float* hit_pos, const float* hit_err, const float* rl,
                     const float* xi, int pflags, int chunk, float* out_par, float* out_err,
                     int* out_chg) {
  if (n <= 0 || n_layers <= 0 || n_layers > Config::nMaxTrkHits - 1 || chunk <= 0 || context())
    return -1;
  std::vector<HitVec> layer_hits;
  std::vector<Track> sim, rec;
  setup(n, n_layers, par, err, chg, hit_pos, hit_err, rl, xi, layer_hits, sim);
  rec.resize(n);
  std::unique_ptr<bool[]> barrel(new bool[n_layers]);
  for (int l = 0; l < n_layers; ++l) barrel[l] = is_barrel[l] != 0;
  try {
    MkFitterGpu mkfp(g_ctx);
    mkfp.SetNhits(n_layers);
    for (int beg = 0; beg < n; beg += chunk) {
      const int end = std::min(beg + chunk, n);
      mkfp.InputTracksAndHits(sim, layer_hits, beg, end);
      mkfp.FitTracksSteered(barrel.get(), end - beg, nullptr, PropagationFlags(pflags));
      mkfp.OutputFittedTracks(rec, beg, end);
    }
  } catch (const std::exception&) {
    return -2;
  }
  output(rec, n, out_par, out_err, out_chg);
  return 0;
}

}  // extern "C"
