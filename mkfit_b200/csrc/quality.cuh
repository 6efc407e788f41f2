// Quality filters of run_OneIteration (StdSeq::qfilter_*,
// mkFit/MkStdSeqs.h:39-148) on a seed's best candidate, read from its
// hit-on-track chain the way the TrackCand hit walks read it
// (mkFit/HitStructures.h:732-859).
#pragma once

#include "find_steps.cuh"

namespace mkfg {

// Filter codes, in the order of the MKFG_QF_* values of the C ABI.
enum QFilterKind {
  kQfNanNSilly = 0,      // qfilter_nan_n_silly
  kQfNHits,              // qfilter_n_hits(min_hits)
  kQfNHitsPixseed,       // qfilter_n_hits_pixseed(min_hits)
  kQfNLayers,            // qfilter_n_layers
  kQfNLayersPixelLess,   // qfilter_n_layers_pixelLess
  kQfPixelLessFwd,       // qfilter_pixelLessFwd
  kQfPixelLessBkwd,      // qfilter_pixelLessBkwd
  kQfCount
};

// The hit counts the filters read, from one walk of the chain newest hit
// first (the walk of every TrackCand counter):
//   last_lyr   getLastFoundHitLyr: newest hit with index >= 0;
//   last_pix   getLastFoundPixelHitLyr: the same on layers 0-3, 18-20, 45-47;
//   n_unique   nUniqueLayers: found hits (index >= 0 or -9) on a layer other
//              than the previous counted one;
//   enc_hits   nHitsByTypeEncoded: pixel + 100 stereo + 10^4 mono + 10^6
//              matched over found hits, a mono hit matching when a stereo
//              hit has been seen so far (the reference's 'previous stereo'
//              flag holds the stereo count) and it lies one layer below the
//              previous hit, or on the previous hit's layer when that is one
//              below a doubly hit stereo layer;
//   enc_layers nLayersByTypeEncoded: the same over the n_unique layers.
struct ChainCounts {
  int last_lyr, last_pix, n_unique, enc_hits, enc_layers;
};

__device__ __forceinline__ bool in_pix_ranges(int l) {
  return (0 <= l && l <= 3) || (18 <= l && l <= 20) || (45 <= l && l <= 47);
}

__device__ inline ChainCounts chain_counts(const EventDev& E, const FindConfigDev& C, int s, int last,
                                           int ntot) {
  ChainCounts R{-1, -1, 0, 0, 0};
  int h_pix = 0, h_st = 0, h_mono = 0, h_mat = 0, h_prev = -1, h_prev_st = 0, dbl = -1;
  int l_pix = 0, l_st = 0, l_mono = 0, l_mat = 0, l_prev = -1, l_prev_st = 0;
  bool got_last = false;
  int node = last;
  for (int k = ntot - 1; k >= 0 && node >= 0; --k) {
    const int hv = node_hot_of(E, s, node);
    const int idx = hot_index(hv), lyr = hot_layer(hv);
    if (idx >= 0 && !got_last) {
      R.last_lyr = lyr;
      got_last = true;
    }
    if (idx >= 0 && R.last_pix == -1 && in_pix_ranges(lyr)) R.last_pix = lyr;
    if (lyr >= 0 && lyr < C.n_layers && (idx >= 0 || idx == -9)) {
      const LayerDev& L = C.layer[lyr];
      if (L.is_pix) {
        ++h_pix;
      } else if (L.is_stereo) {
        ++h_st;
        if (lyr == h_prev) dbl = lyr;
      } else {
        ++h_mono;
        if (h_prev_st && lyr == h_prev - 1) ++h_mat;
        else if (lyr == h_prev && lyr == dbl - 1) ++h_mat;
      }
      h_prev = lyr;
      h_prev_st = h_st;
      if (lyr != l_prev) {
        ++R.n_unique;
        if (L.is_pix) {
          ++l_pix;
        } else if (L.is_stereo) {
          ++l_st;
        } else {
          ++l_mono;
          if (l_prev_st && lyr == l_prev - 1) ++l_mat;
        }
        l_prev = lyr;
        l_prev_st = l_st;
      }
    }
    node = E.node_prev[(size_t)s * E.hot_cap + node];
  }
  R.enc_hits = h_pix + 100 * h_st + 10000 * h_mono + 1000000 * h_mat;
  R.enc_layers = l_pix + 100 * l_st + 10000 * l_mono + 1000000 * l_mat;
  return R;
}

// TrackCand::nPixelDecoded / nTotMatchDecoded.
__device__ __forceinline__ int enc_pixel(int e) { return e % 100; }
__device__ __forceinline__ int enc_tot_match(int e) {
  return e % 100 + (e / 100) % 100 + (e / 10000) % 100 - e / 1000000;
}

// TrackBase::hasNanNSillyValues (Track.cc:177-192): a negative diagonal or a
// non-finite element of the packed covariance.
__device__ __forceinline__ bool silly_errors(const CandSoA& B, int slot) {
  bool silly = false;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      const float v = B.err[sidx(i, j) * B.cap + slot];
      if ((i == j && v < 0.f) || !isfinite(v)) silly = true;
    }
  return silly;
}

struct QFilterParams {
  int kind;
  int min_hits;
  float beam_x, beam_y;
};

// One filter on candidate `slot` of seed s (the verdict of
// MkStdSeqs.h:39-148 for the TrackCand).
__device__ inline bool qfilter_pass(const EventDev& E, const FindConfigDev& C, const CandSoA& B, int s,
                                    int slot, const QFilterParams& P) {
  if (P.kind == kQfNanNSilly) return !silly_errors(B, slot);
  const int nfound = B.nfound[slot];
  // TrackBase::getNSeedHits: the seed's hit count in a 4-bit field.
  const int seed_reduction = (E.init_hot[s] & 15) <= 5 ? 2 : 3;
  if (P.kind == kQfNHits) return nfound - seed_reduction >= P.min_hits;
  if (P.kind == kQfNHitsPixseed) return nfound >= P.min_hits;
  const ChainCounts K = chain_counts(E, C, s, B.last[slot], nfound + B.nmiss[slot]);
  const float invpt = B.par[3 * B.cap + slot];
  const float d0 = fabsf(d0_beam_spot(B.par[0 * B.cap + slot], B.par[1 * B.cap + slot], invpt,
                                      B.par[4 * B.cap + slot], B.chg[slot], P.beam_x, P.beam_y));
  // std::abs(theta - Config::PIOver2).
  const float thetasym = fabsf(__fsub_rn(B.par[5 * B.cap + slot], kPIOver2));
  switch (P.kind) {
    case kQfNLayers: {
      const int npixhits = enc_pixel(K.enc_hits), npixlyrs = enc_pixel(K.enc_layers);
      const int nmatlyrs = enc_tot_match(K.enc_layers);
      const int llyr = K.last_lyr, lplyr = K.last_pix;
      const float invptmin = 1.43f, d0_max = 0.1f;
      const bool ends_inside_pix = llyr == 2 || llyr == 18 || llyr == 45;
      const bool last_inside_pix = (0 <= lplyr && lplyr < 3) || (18 <= lplyr && lplyr < 20) ||
                                   (45 <= lplyr && lplyr < 47);
      return !(((npixhits <= 3 || npixlyrs <= 3) && ends_inside_pix &&
                (invpt < invptmin || (invpt >= invptmin && d0 > d0_max))) ||
               ((npixlyrs <= 3 && nmatlyrs <= 6) && last_inside_pix && llyr != lplyr && d0 > d0_max));
    }
    case kQfNLayersPixelLess:
      return !((nfound <= 6 || K.n_unique <= 6) && d0 > 0.1f);
    case kQfPixelLessFwd: {
      const int nlyrs = enc_tot_match(K.enc_layers), nhits = enc_tot_match(K.enc_hits);
      const float invptmin = 1.11f, thetasymmin = 1.11f;
      const int nf = nfound - seed_reduction;
      return ((nf >= 4 && invpt < invptmin) || (nf >= 3 && invpt > invptmin && thetasym <= thetasymmin) ||
              (nf >= 4 && invpt > invptmin && thetasym > thetasymmin)) &&
             !((nlyrs <= 4 || nhits <= 4) && d0 > 0.05f && invpt < invptmin);
    }
    case kQfPixelLessBkwd: {
      const int nlyrs = enc_tot_match(K.enc_layers), nhits = enc_tot_match(K.enc_hits);
      const float invptmin = 1.11f, d0_max = 0.1f;
      const float thetasymmin_l = 0.80f, thetasymmin_h = 1.11f;
      return !((nlyrs <= 3 || nhits <= 3) ||
               ((nlyrs <= 4 || nhits <= 4) && (invpt < invptmin || (thetasym > thetasymmin_l && d0 > d0_max))) ||
               ((nlyrs <= 6 || nhits <= 6) && (invpt > invptmin && thetasym > thetasymmin_h && d0 > d0_max)));
    }
  }
  return true;
}

}  // namespace mkfg
