// Test driver of the C++ adapters (mkfit_b200/shims/MkFitterGpu.h,
// FindingFoosGpu.h). MkFitterGpu:
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
#include "mkFit/KalmanUtilsMPlex.h"
#include "shims/FindingFoosGpu.h"
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

extern "C" {

// The finding operator table on n states, NN lanes per call as MkFinder
// calls it, through the reference's own FindingFoos (the CPU functions)
// and through FindingFoosGpu: propagation of the states to `target` (r on
// the barrel, z on the endcap), and propagation to the hits with the chi2
// and with the update. Inputs par[6][n], err[21][n], chg[n],
// hit_pos[3][n], hit_err[6][n]; outputs per side (0 reference, 1 GPU):
// prop_par[side][6][n], prop_err[side][21][n], chi2[side][n],
// chi2_par[side][6][n], upd_par[side][6][n], upd_err[side][21][n],
// upd_chg[side][n]. Material: the given (z, r) grids on both sides.
int shim_ops(int n, int endcap, const float* par, const float* err, const int* chg,
             const float* hit_pos, const float* hit_err, float target, const float* rl,
             const float* xi, int pflags, float* prop_par, float* prop_err, float* chi2,
             float* chi2_par, float* upd_par, float* upd_err, int* upd_chg) {
  if (n <= 0 || context()) return -1;
  std::memcpy(Config::RlgridME, rl, sizeof(Config::RlgridME));
  std::memcpy(Config::XigridME, xi, sizeof(Config::XigridME));
  if (mkfg_set_material(g_ctx, rl, xi) != MKFG_OK) return -1;
  Config::finding_requires_propagation_to_hit_pos = true;
  FindingFoosGpu::set_context(g_ctx);
  const PropagationFlags pf(pflags);
  const FindingFoos* foos[2] = {&FindingFoos::get_finding_foos(!endcap),
                                &FindingFoosGpu::get_finding_foos(!endcap)};
  try {
    for (int beg = 0; beg < n; beg += NN) {
      const int np = std::min(NN, n - beg);
      for (int side = 0; side < 2; ++side) {
        MkBase mb;
        MPlexHS msErr;
        MPlexHV msPar;
        for (int i = 0; i < np; ++i) {
          for (int k = 0; k < 6; ++k) mb.Par[MkBase::iC].fArray[k * NN + i] = par[k * n + beg + i];
          for (int k = 0; k < 21; ++k) mb.Err[MkBase::iC].fArray[k * NN + i] = err[k * n + beg + i];
          mb.Chg.fArray[i] = chg[beg + i];
          for (int k = 0; k < 3; ++k) msPar.fArray[k * NN + i] = hit_pos[k * n + beg + i];
          for (int k = 0; k < 6; ++k) msErr.fArray[k * NN + i] = hit_err[k * n + beg + i];
        }
        // Propagation to the layer: the reference's MkBase member on the
        // CPU side, FindingFoosGpu's form on the GPU side.
        if (side == 0)
          (mb.*(foos[0]->m_propagate_foo))(target, np, pf);
        else if (endcap)
          FindingFoosGpu::propagate_to_z(mb, target, np, pf);
        else
          FindingFoosGpu::propagate_to_r(mb, target, np, pf);
        MPlexQF outChi2;
        MPlexLV propPar, outPar;
        MPlexLS outErr;
        MPlexQI c = mb.Chg;
        (*foos[side]->m_compute_chi2_foo)(mb.Err[MkBase::iC], mb.Par[MkBase::iC], mb.Chg, msErr,
                                          msPar, outChi2, propPar, np, pf);
        (*foos[side]->m_update_param_foo)(mb.Err[MkBase::iC], mb.Par[MkBase::iC], c, msErr, msPar,
                                          outErr, outPar, np, pf);
        for (int i = 0; i < np; ++i) {
          const size_t o = beg + i;
          for (int k = 0; k < 6; ++k) {
            prop_par[(side * 6 + k) * (size_t)n + o] = mb.Par[MkBase::iP].fArray[k * NN + i];
            chi2_par[(side * 6 + k) * (size_t)n + o] = propPar.fArray[k * NN + i];
            upd_par[(side * 6 + k) * (size_t)n + o] = outPar.fArray[k * NN + i];
          }
          for (int k = 0; k < 21; ++k) {
            prop_err[(side * 21 + k) * (size_t)n + o] = mb.Err[MkBase::iP].fArray[k * NN + i];
            upd_err[(side * 21 + k) * (size_t)n + o] = outErr.fArray[k * NN + i];
          }
          chi2[side * (size_t)n + o] = outChi2.fArray[i];
          upd_chg[side * (size_t)n + o] = c.fArray[i];
        }
      }
    }
  } catch (const std::exception&) {
    return -2;
  }
  return 0;
}

}  // extern "C"
