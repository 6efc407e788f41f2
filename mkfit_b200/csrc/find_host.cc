// Host-side preparation for combinatorial finding (see find_host.h).
// Float arithmetic follows the cited reference routines operation by
// operation, because bin indices and seed ordering depend on it.
#include "find_host.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace mkfg {

namespace {
constexpr float kPIf = 3.14159265358979323846f;
constexpr float kTwoPIf = 6.28318530717958647692f;
constexpr float kSolf = 0.299792458f;
constexpr float kBfieldf = 3.8112f;
constexpr float kFphiFine = 1024 / kTwoPIf;  // LayerOfHits::m_fphi_fine
constexpr int kPhiFineXmask = ~((1 << 2) - 1);
}  // namespace

LayerBinning setup_layer_binning(const float* d) {
  LayerBinning b;
  b.barrel = d[LC_IS_BARREL] > 0.5f;
  const float qmin = b.barrel ? d[LC_ZMIN] : d[LC_RIN];
  const float qmax = b.barrel ? d[LC_ZMAX] : d[LC_ROUT];
  const float dq = d[LC_Q_BIN];
  if (dq < 0) {
    b.nq = (int)-dq;
    b.qmin = qmin;
    b.qmax = qmax;
  } else {
    const float extent = qmax - qmin;
    b.nq = (int)std::ceil(extent / dq);
    const float extra = 0.5f * (b.nq * dq - extent);
    b.qmin = qmin - extra;
    b.qmax = qmax + extra;
  }
  b.fq = b.nq / (qmax - qmin);
  return b;
}

uint32_t decoded_charge_pcm(int32_t cpcm) {
  uint32_t code;
  if (cpcm < 0)
    code = 0xff;  // setupAsPixel
  else if (cpcm < 1620)
    code = 0;
  else
    code = std::min(0xff, ((cpcm - 1620) >> 3) + 1);
  return code == 0 ? 0u : ((code - 1) << 3) + 1620;
}

void prepare_event_hits(const std::vector<LayerBinning>& lb, const int32_t* layer_begin,
                        int n_layers, const float* pos, int pos_stride, const int32_t* detid,
                        const int32_t* cpcm, EventHitsPrep& out) {
  const int nh = layer_begin[n_layers];
  int n_bins = 0;
  for (auto& b : lb) n_bins = std::max(n_bins, b.bin_offset + b.nq * kPhiBins);
  out.bins.assign(n_bins, 0u);
  out.sphi.resize(nh);
  out.sq.resize(nh);
  out.srank.resize(nh);
  out.hinfo.resize(nh);
  std::vector<uint32_t> key;
  std::vector<float> hphi, hq;
  std::vector<int32_t> idx;
  const float* X = pos;
  const float* Y = pos + pos_stride;
  const float* Z = pos + 2 * (size_t)pos_stride;
  for (int l = 0; l < n_layers; ++l) {
    const LayerBinning& b = lb[l];
    const int h0 = layer_begin[l], n = layer_begin[l + 1] - h0;
    key.resize(n);
    hphi.resize(n);
    hq.resize(n);
    for (int i = 0; i < n; ++i) {
      const int h = h0 + i;
      const float x = X[h], y = Y[h], z = Z[h];
      const float phi = std::atan2(y, x);                            // Hit::phi()
      const float q = b.barrel ? z : std::sqrt(x * x + y * y);       // Hit::z() / Hit::r()
      hphi[i] = phi;
      hq[i] = q;
      const int phi_fine = (int)std::floor(kFphiFine * (phi + kPIf));
      const int qb = std::clamp((int)((q - b.qmin) * b.fq), 0, b.nq - 1);
      key[i] = (uint32_t)(phi_fine + (qb << 16));
      out.hinfo[h] = (uint32_t(detid[h]) & 0xfffu) | (decoded_charge_pcm(cpcm[h]) << 12);
    }
    idx.resize(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int c) { return key[a] < key[c]; });
    int curr = -1;
    uint32_t* bins = out.bins.data() + b.bin_offset;
    for (int i = 0; i < n; ++i) {
      const int j = idx[i];
      out.sphi[h0 + i] = hphi[j];
      out.sq[h0 + i] = hq[j];
      out.srank[h0 + i] = j;
      const int jqphi = (int)key[j] & kPhiFineXmask;
      const int phi_bin = (jqphi & 0x3ff) >> 2;
      const int q_bin = jqphi >> 16;
      uint32_t& bin = bins[q_bin * kPhiBins + phi_bin];
      if (jqphi != curr) {
        bin = uint32_t(i) | (uint32_t(i) << 16);
        curr = jqphi;
      }
      bin += (1u << 16);
    }
  }
}

namespace {

// Track helix helpers of the reference (Track.cc:258-322, Track.h:110-118).
struct SeedTrack {
  float x, y, z, ipt, phi, theta;
  int chg;
  // The momentum, as TrackBase computes it on every call (Track.h), taken
  // once per seed: the same float operations on the same inputs.
  float pt_, px_, py_, pz_;
  SeedTrack(float x_, float y_, float z_, float ipt_, float phi_, float theta_, int chg_)
      : x(x_), y(y_), z(z_), ipt(ipt_), phi(phi_), theta(theta_), chg(chg_) {
    pt_ = std::abs(1.f / ipt);
    px_ = pt_ * std::cos(phi);
    py_ = pt_ * std::sin(phi);
    pz_ = pt_ / std::tan(theta);
  }
  float pT() const { return pt_; }
  float px() const { return px_; }
  float py() const { return py_; }
  float pz() const { return pz_; }

  float maxReachRadius() const {
    const float k = ((chg < 0) ? 100.0f : -100.0f) / (kSolf * kBfieldf);
    const float abs_ooc_half = std::abs(k * pT());
    const float x_center = x - k * py();
    const float y_center = y + k * px();
    return std::hypot(x_center, y_center) + abs_ooc_half;
  }

  float zAtR(float R) const {
    float xc = x, yc = y, pxc = px(), pyc = py();
    const float kinv = ((chg < 0) ? 0.01f : -0.01f) * kSolf * kBfieldf;
    const float k = 1.0f / kinv;
    const float c = 0.5f * kinv * ipt;
    const float ooc = 1.0f / c;
    const float lambda = pz() * ipt;
    float D = 0;
    for (int i = 0; i < 5; ++i) {
      const float r0 = std::hypot(xc, yc);
      const float td = (R - r0) * c;
      const float id = ooc * td * (1.0f + 0.16666666f * td * td);
      D += id;
      const float cosa = std::cos(id * ipt * kinv);
      const float sina = std::sin(id * ipt * kinv);
      xc += k * (pxc * sina - pyc * (1.0f - cosa));
      yc += k * (pyc * sina + pxc * (1.0f - cosa));
      const float pxo = pxc;
      pxc = pxc * cosa - pyc * sina;
      pyc = pyc * cosa + pxo * sina;
    }
    return z + lambda * D;
  }
};

}  // namespace

RegionCuts region_cuts_cms2017(const float* L) {
  auto col = [&](int l, int c) { return L[l * LC_COUNT + c]; };
  RegionCuts r;
  r.tib1_rin = col(4, LC_RIN);
  r.tib1_zmax = col(4, LC_ZMAX);
  r.tib1_zmin = col(4, LC_ZMIN);
  r.tob1_rin = col(10, LC_RIN);
  r.tob1_zmax = col(10, LC_ZMAX);
  r.tob1_zmin = col(10, LC_ZMIN);
  r.tidp1_zmin = col(21, LC_ZMIN);
  r.tidn1_zmax = col(48, LC_ZMAX);
  r.tecp1_zmin = col(27, LC_ZMIN);
  r.tecn1_zmax = col(54, LC_ZMAX);
  r.tidp_rin = std::min(col(21, LC_RIN), col(22, LC_RIN));
  r.tidp_rout = std::max(col(21, LC_ROUT), col(22, LC_ROUT));
  r.tecp_rin = std::min(col(27, LC_RIN), col(28, LC_RIN));
  r.tecp_rout = std::max(col(27, LC_ROUT), col(28, LC_ROUT));
  r.tidn_rin = std::min(col(48, LC_RIN), col(49, LC_RIN));
  r.tidn_rout = std::max(col(48, LC_ROUT), col(49, LC_ROUT));
  r.tecn_rin = std::min(col(54, LC_RIN), col(55, LC_RIN));
  r.tecn_rout = std::max(col(54, LC_ROUT), col(55, LC_ROUT));
  return r;
}

void partition_seeds_cms2017(const float* L, int n_layers, const SeedInput& s,
                             const int32_t* layer_begin, const float* hit_pos, int hit_stride,
                             SeedOrder& out) {
  const RegionCuts r = region_cuts_cms2017(L);
  const float tib1_rin = r.tib1_rin, tib1_zmax = r.tib1_zmax, tib1_zmin = r.tib1_zmin;
  const float tob1_rin = r.tob1_rin, tob1_zmax = r.tob1_zmax, tob1_zmin = r.tob1_zmin;
  const float tidp1_zmin = r.tidp1_zmin, tidn1_zmax = r.tidn1_zmax;
  const float tecp1_zmin = r.tecp1_zmin, tecn1_zmax = r.tecn1_zmax;
  const float tidp_rin = r.tidp_rin, tidp_rout = r.tidp_rout;
  const float tecp_rin = r.tecp_rin, tecp_rout = r.tecp_rout;
  const float tidn_rin = r.tidn_rin, tidn_rout = r.tidn_rout;
  const float tecn_rin = r.tecn_rin, tecn_rout = r.tecn_rout;
  (void)n_layers;

  auto barrel_pos = [](const SeedTrack& S, float maxR, float rin, float zmax) {
    return maxR > rin && S.zAtR(rin) < zmax;
  };
  auto barrel_neg = [](const SeedTrack& S, float maxR, float rin, float zmin) {
    return maxR > rin && S.zAtR(rin) > zmin;
  };
  auto endcap_pos = [](const SeedTrack& S, float maxR, float rout, float rin, float zmin) {
    return maxR > rout ? S.zAtR(rout) > zmin : (maxR > rin && S.zAtR(maxR) > zmin);
  };
  auto endcap_neg = [](const SeedTrack& S, float maxR, float rout, float rin, float zmax) {
    return maxR > rout ? S.zAtR(rout) < zmax : (maxR > rin && S.zAtR(maxR) < zmax);
  };

  const int n = s.n;
  std::vector<float> score(n);
  out.region.assign(n, 2);
  for (int i = 0; i < n; ++i) {
    const SeedTrack S(s.par[0 * n + i], s.par[1 * n + i], s.par[2 * n + i], s.par[3 * n + i],
                      s.par[4 * n + i], s.par[5 * n + i], s.chg[i]);
    // Eta of the seed's last hit (Hit::eta, Hit.h:82-87).
    const int last = s.nhits[i] - 1;
    const int hl = s.hit_layer[i * s.stride + last], hi = s.hit_index[i * s.stride + last];
    const int h = layer_begin[hl] + hi;
    const float hx = hit_pos[h], hy = hit_pos[hit_stride + h], hz = hit_pos[2 * (size_t)hit_stride + h];
    const float theta = std::atan2(std::sqrt(hx * hx + hy * hy), hz);
    const float eta = -1.0f * std::log(std::tan(theta / 2.0f));

    int reg;
    const bool z_dir_pos = S.pz() > 0;
    const float maxR = S.maxReachRadius();
    // The tests are pure, so each pair is evaluated with a short circuit:
    // the second only when the first fails (same regions, fewer helix
    // steps).
    if (z_dir_pos) {
      const bool in_barrel = barrel_pos(S, maxR, tib1_rin, tib1_zmax) ||
                             barrel_pos(S, maxR, tob1_rin, tob1_zmax);
      if (!in_barrel) {
        reg = 4;  // Reg_Endcap_Pos
      } else {
        const bool in_endcap = endcap_pos(S, maxR, tidp_rout, tidp_rin, tidp1_zmin) ||
                               endcap_pos(S, maxR, tecp_rout, tecp_rin, tecp1_zmin);
        reg = in_endcap ? 3 : 2;  // Transition_Pos : Barrel
      }
    } else {
      const bool in_barrel = barrel_neg(S, maxR, tib1_rin, tib1_zmin) ||
                             barrel_neg(S, maxR, tob1_rin, tob1_zmin);
      if (!in_barrel) {
        reg = 0;  // Reg_Endcap_Neg
      } else {
        const bool in_endcap = endcap_neg(S, maxR, tidn_rout, tidn_rin, tidn1_zmax) ||
                               endcap_neg(S, maxR, tecn_rout, tecn_rin, tecn1_zmax);
        reg = in_endcap ? 1 : 2;  // Transition_Neg : Barrel
      }
    }
    out.region[i] = reg;
    score[i] = 7.0f * (reg - 2) + eta;
  }
  out.order.resize(n);
  std::iota(out.order.begin(), out.order.end(), 0);
  std::stable_sort(out.order.begin(), out.order.end(),
                   [&](int a, int b) { return score[a] < score[b]; });
}

}  // namespace mkfg
