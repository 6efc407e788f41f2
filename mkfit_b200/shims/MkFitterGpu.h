// MkFitterGpu: the reference's MkFitter worker interface (mkFit/MkFitter.h:
// 54-87) over this library's C ABI, so MkFitter call sites -- the fitting
// loop of mkFit/fittestMPlex.cc:65-100 (runFittingTestPlex) and the seed
// fit of FitTracks / FitTracksSteered -- run on the GPU unchanged except
// for the class name.
//
// Header-only; compile it against the reference's headers (Track.h, Hit.h,
// Config.h, Event.h) and link libmkfit_b200.so. The methods keep
// MkFitter's signatures and meaning:
//
//   SetNhits                  number of layer steps (capped at
//                             Config::nMaxTrkHits - 1, as MkFitter does)
//   InputTracksForFit         state, charge, chi2, label and the first
//                             Config::nLayers hits on track of tracks
//                             [beg, end) (mkFit/MkFitter.cc:286-321)
//   FitTracksWithInterSlurp   per step: each track's hit on its own layer
//                             (HitOnTrack index / layer), propagation to
//                             the hit's radius with Config::forward_fit_pflags
//                             and the barrel update (:323-363); a track
//                             without a hit on a step (index or layer < 0)
//                             gets hit 0 of layer `step`, as the
//                             reference's null packer input does
//   InputTracksAndHits        state and the hits layerHits[hi][hit index hi]
//                             (:56-91)
//   FitTracks                 all steps barrel (:430-448)
//   FitTracksSteered          step hi barrel when is_barrel[hi], else the
//                             propagation to the hit's z and the endcap
//                             update (:473-503)
//   OutputFittedTracks        updated state, charge, input chi2 and label
//                             back into tracks [beg, end) (:505-522)
//
// Unlike MkFitter, one object takes any number of tracks per call (the
// whole range, not NN); chunking the range as the reference's loop does
// gives the same results. The fit itself runs in Fit* through
// mkfg_fit_host (synchronous); the material map is the reference's
// Config::RlgridME / XigridME, uploaded when it changed since the last
// fit. Errors from the library throw std::runtime_error with its message
// (MkFitter has no error path). InputTracksAndHits with a negative hit
// index uses hit 0 of the layer, where MkFitter keeps whatever the
// previous call left in that lane.
#ifndef MKFIT_B200_SHIMS_MKFITTERGPU_H
#define MKFIT_B200_SHIMS_MKFITTERGPU_H

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "Config.h"
#include "Event.h"
#include "Hit.h"
#include "Track.h"
#include "mkfit_b200.h"

namespace mkfit {

class MkFitterGpu {
 public:
  // ctx: the library context the fits run on (owned by the caller).
  explicit MkFitterGpu(mkfg_context* ctx) : ctx_(ctx) {}

  void SetNhits(int newnhits) { Nhits = std::min(newnhits, Config::nMaxTrkHits - 1); }

  void InputTracksForFit(const std::vector<Track>& tracks, int beg, int end) {
    load_states(tracks, beg, end);
    const int n = end - beg, nl = Config::nLayers;
    hot_idx_.assign((size_t)nl * n, -1);
    hot_lyr_.assign((size_t)nl * n, -1);
    for (int i = 0; i < n; ++i) {
      const Track& t = tracks[beg + i];
      for (int l = 0; l < nl && l < t.nTotalHits(); ++l) {
        hot_idx_[(size_t)l * n + i] = t.getHitIdx(l);
        hot_lyr_[(size_t)l * n + i] = t.getHitLyr(l);
      }
    }
  }

  void FitTracksWithInterSlurp(const std::vector<HitVec>& layersohits, const int N_proc) {
    const int n = std::min(N_proc, n_);
    // All layers in one hit buffer: each track's hit is addressed by its
    // global index, so every track may take its hit from its own layer.
    std::vector<int> first(layersohits.size() + 1, 0);
    for (size_t l = 0; l < layersohits.size(); ++l)
      first[l + 1] = first[l] + (int)layersohits[l].size();
    pack_hits(layersohits, first);
    std::vector<int32_t> hot((size_t)Nhits * n);
    for (int s = 0; s < Nhits; ++s)
      for (int i = 0; i < n; ++i) {
        const int hidx = hot_idx_[(size_t)s * n_ + i], hlyr = hot_lyr_[(size_t)s * n_ + i];
        hot[(size_t)s * n + i] = (hidx < 0 || hlyr < 0) ? first[s] : first[hlyr] + hidx;
      }
    run(n, hot, std::vector<int32_t>(Nhits, 0), 0, pflag_bits(Config::forward_fit_pflags),
        {0, first.back()});
  }

  void InputTracksAndHits(const std::vector<Track>& tracks, const std::vector<HitVec>& layerHits,
                          int beg, int end) {
    load_states(tracks, beg, end);
    const int n = end - beg;
    hits_ = &layerHits;
    hot_idx_.assign((size_t)Nhits * n, 0);
    for (int i = 0; i < n; ++i)
      for (int hi = 0; hi < Nhits; ++hi) {
        const int h = tracks[beg + i].getHitIdx(hi);
        hot_idx_[(size_t)hi * n + i] = h < 0 ? 0 : h;
      }
  }

  void FitTracks(const int N_proc, const Event* /*ev*/, const PropagationFlags pflags) {
    fit_loaded(N_proc, 0, pflags);
  }

  void FitTracksSteered(const bool is_barrel[], const int N_proc, const Event* /*ev*/,
                        const PropagationFlags pflags) {
    uint64_t mask = 0;
    for (int hi = 0; hi < Nhits; ++hi)
      if (!is_barrel[hi]) mask |= 1ull << hi;
    fit_loaded(N_proc, mask, pflags);
  }

  void OutputFittedTracks(std::vector<Track>& tracks, int beg, int end) const {
    for (int i = beg, k = 0; i < end; ++i, ++k) {
      Track& t = tracks[i];
      for (int e = 0; e < 6; ++e) t.parameters_nc()[e] = out_par_[(size_t)e * n_ + k];
      for (int e = 0; e < 21; ++e) t.errors_nc().Array()[e] = out_err_[(size_t)e * n_ + k];
      t.setCharge(out_chg_[k]);
      t.setChi2(chi2_[k]);
      t.setLabel(label_[k]);
    }
  }

  int Nhits = 0;

 private:
  static uint32_t pflag_bits(const PropagationFlags& p) {
    return (p.use_param_b_field ? 1u : 0u) | (p.apply_material ? 2u : 0u);
  }

  void load_states(const std::vector<Track>& tracks, int beg, int end) {
    n_ = end - beg;
    par_.assign((size_t)6 * n_, 0.f);
    err_.assign((size_t)21 * n_, 0.f);
    chg_.assign(n_, 0);
    chi2_.assign(n_, 0.f);
    label_.assign(n_, 0);
    for (int i = 0; i < n_; ++i) {
      const Track& t = tracks[beg + i];
      for (int e = 0; e < 6; ++e) par_[(size_t)e * n_ + i] = t.parameters()[e];
      for (int e = 0; e < 21; ++e) err_[(size_t)e * n_ + i] = t.errors().Array()[e];
      chg_[i] = t.charge();
      chi2_[i] = t.chi2();
      label_[i] = t.label();
    }
  }

  // Hits of the given layers into the SoA buffers, layer l at
  // [first[l], first[l + 1]).
  void pack_hits(const std::vector<HitVec>& layers, const std::vector<int>& first) {
    const int nh = first.back();
    hpos_.assign((size_t)3 * nh, 0.f);
    herr_.assign((size_t)6 * nh, 0.f);
    for (size_t l = 0; l < layers.size(); ++l)
      for (size_t h = 0; h < layers[l].size(); ++h) {
        const size_t g = first[l] + h;
        const float* p = layers[l][h].posArray();
        const float* e = layers[l][h].errArray();
        for (int k = 0; k < 3; ++k) hpos_[(size_t)k * nh + g] = p[k];
        for (int k = 0; k < 6; ++k) herr_[(size_t)k * nh + g] = e[k];
      }
  }

  void fit_loaded(int N_proc, uint64_t endcap_mask, const PropagationFlags& pflags) {
    if (!hits_) throw std::runtime_error("MkFitterGpu: InputTracksAndHits was not called");
    if ((int)hits_->size() < Nhits) throw std::runtime_error("MkFitterGpu: fewer hit layers than Nhits");
    const int n = std::min(N_proc, n_);
    std::vector<int> first(Nhits + 1, 0);
    for (int hi = 0; hi < Nhits; ++hi) first[hi + 1] = first[hi] + (int)(*hits_)[hi].size();
    std::vector<HitVec> used(hits_->begin(), hits_->begin() + Nhits);
    pack_hits(used, first);
    std::vector<int32_t> hot((size_t)Nhits * n), layer(Nhits);
    for (int hi = 0; hi < Nhits; ++hi) {
      layer[hi] = hi;
      for (int i = 0; i < n; ++i) hot[(size_t)hi * n + i] = hot_idx_[(size_t)hi * n_ + i];
    }
    run(n, hot, layer, endcap_mask, pflag_bits(pflags), first);
  }

  void sync_material() {
    const size_t bytes = sizeof(Config::RlgridME);
    if (mat_rl_.size() == bytes / 4 &&
        !std::memcmp(mat_rl_.data(), &Config::RlgridME[0][0], bytes) &&
        !std::memcmp(mat_xi_.data(), &Config::XigridME[0][0], bytes))
      return;
    mat_rl_.assign(&Config::RlgridME[0][0], &Config::RlgridME[0][0] + bytes / 4);
    mat_xi_.assign(&Config::XigridME[0][0], &Config::XigridME[0][0] + bytes / 4);
    check(mkfg_set_material(ctx_, mat_rl_.data(), mat_xi_.data()));
  }

  // Fits the first n loaded tracks: hot[step][n] indices within layer
  // layer[step] of the packed hits (layer l at first[l]).
  void run(int n, const std::vector<int32_t>& hot, const std::vector<int32_t>& layer,
           uint64_t endcap_mask, uint32_t pflags, const std::vector<int>& first) {
    sync_material();
    out_par_.assign((size_t)6 * n_, 0.f);
    out_err_.assign((size_t)21 * n_, 0.f);
    out_chg_.assign(n_, 0);
    if (n <= 0) return;
    // The state arrays hold n_ tracks per row; the fit takes the first n.
    std::vector<float> par((size_t)6 * n), err((size_t)21 * n);
    for (int e = 0; e < 6; ++e) std::copy_n(&par_[(size_t)e * n_], n, &par[(size_t)e * n]);
    for (int e = 0; e < 21; ++e) std::copy_n(&err_[(size_t)e * n_], n, &err[(size_t)e * n]);
    std::vector<float> op((size_t)6 * n), oe((size_t)21 * n);
    std::vector<int32_t> chg(chg_.begin(), chg_.begin() + n), oc(n);
    std::vector<int32_t> lb(first.begin(), first.end());
    mkfg_fit_args a{};
    a.in = mkfg_tracks{par.data(), err.data(), chg.data(), n, n};
    a.out = mkfg_tracks{op.data(), oe.data(), oc.data(), n, n};
    a.hits = mkfg_hits{hpos_.data(), herr_.data(), lb.data(), (int32_t)lb.size() - 1,
                       (int32_t)(hpos_.size() / 3)};
    a.hot_index = hot.data();
    a.hot_stride = n;
    a.n_steps = (int32_t)layer.size();
    a.hit_layer = layer.data();
    a.endcap_mask = endcap_mask;
    a.pflags = pflags;
    a.out_chi2 = nullptr;
    check(mkfg_fit_host(ctx_, &a));
    for (int e = 0; e < 6; ++e) std::copy_n(&op[(size_t)e * n], n, &out_par_[(size_t)e * n_]);
    for (int e = 0; e < 21; ++e) std::copy_n(&oe[(size_t)e * n], n, &out_err_[(size_t)e * n_]);
    std::copy_n(oc.begin(), n, out_chg_.begin());
  }

  static void check(int rc) {
    if (rc == MKFG_OK) return;
    char msg[512];
    mkfg_last_error(msg, sizeof(msg));
    throw std::runtime_error(std::string("mkfit_b200: ") + msg);
  }

  mkfg_context* ctx_;
  int n_ = 0;
  const std::vector<HitVec>* hits_ = nullptr;
  std::vector<float> par_, err_, chi2_, out_par_, out_err_, hpos_, herr_, mat_rl_, mat_xi_;
  std::vector<int32_t> chg_, label_, out_chg_, hot_idx_, hot_lyr_;
};

}  // namespace mkfit

#endif
