// Host-side preparation for combinatorial finding: per-layer hit bins and
// seed import. Plain C++; the device side lives in find.cu.
#pragma once

#include <cstdint>
#include <vector>

namespace mkfg {

// Columns of the layer descriptor rows (same order as the C ABI's
// mkfg_find_config.layer_desc, documented in include/mkfit_b200.h).
enum LayerCol {
  LC_IS_BARREL = 0, LC_RIN, LC_ROUT, LC_ZMIN, LC_ZMAX, LC_PROPAGATE_TO, LC_Q_BIN,
  LC_HAS_HOLE, LC_HOLE_MIN, LC_HOLE_MAX, LC_IS_PIX, LC_IS_STEREO,
  LC_MIN_DPHI, LC_MAX_DPHI, LC_MIN_DQ, LC_MAX_DQ,
  LC_C_DP_SF, LC_C_DP_0, LC_C_DP_1, LC_C_DP_2,
  LC_C_DQ_SF, LC_C_DQ_0, LC_C_DQ_1, LC_C_DQ_2,
  LC_C_C2_SF, LC_C_C2_0, LC_C_C2_1, LC_C_C2_2,
  LC_LAYER_TYPE, LC_IS_SEED, LC_SUBDET, LC_PAD, LC_COUNT
};

constexpr int kPhiBins = 256;  // Config::m_nphi

// q-binning of one layer: LayerOfHits::setup_bins (mkFit/HitStructures.cc:11-35).
struct LayerBinning {
  int nq = 0;
  float qmin = 0.f, qmax = 0.f, fq = 0.f;
  int bin_offset = 0;  // offset of this layer's nq * 256 bins in the event bin table
  bool barrel = true;
};

LayerBinning setup_layer_binning(const float* desc);

// Hit-side per-event preparation, mirroring LayerOfHits::SuckInHits
// (mkFit/HitStructures.cc:77-182): hits of each layer sorted (stably) by
// the packed key phi_fine(10 bit) + (q_bin << 16); per (q bin, phi bin) the
// [first, last) range of sorted positions; per sorted position the hit's
// phi, q and its index within the layer.
struct EventHitsPrep {
  std::vector<uint32_t> bins;   // (first | last << 16) per bin, all layers
  std::vector<float> sphi, sq;  // per sorted hit (global sorted position)
  std::vector<int32_t> srank;   // index within layer of the sorted hit
  std::vector<uint32_t> hinfo;  // per original hit: detid (12 bit) | decoded charge/cm << 12
};

void prepare_event_hits(const std::vector<LayerBinning>& lb, const int32_t* layer_begin,
                        int n_layers, const float* pos, int pos_stride, const int32_t* detid,
                        const int32_t* cpcm, EventHitsPrep& out);

// Hit::chargePerCM() of a hit set up with setupAsStrip(id, cpcm, rows)
// (Hit.h:260-282); pixel hits (cpcm < 0) store the saturated code.
uint32_t decoded_charge_pcm(int32_t cpcm);

// Seed partition into eta regions and sort by (region, eta): restates
// partitionSeeds1 (Geoms/CMS-2017.cc:436-549) and MkBuilder::import_seeds
// (mkFit/MkBuilder.cc:214-275). Returns for each sorted position the input
// seed index, and per input seed its region.
struct SeedOrder {
  std::vector<int32_t> order;   // sorted position -> input seed
  std::vector<int32_t> region;  // input seed -> region
};

struct SeedInput {
  int n;
  const float* par;  // [6][n]
  const int32_t* chg;
  const int32_t* nhits;
  const int32_t* hit_layer;  // [n][stride]
  const int32_t* hit_index;  // [n][stride]
  int stride;
};

// The layer limits partitionSeeds1 tests seeds against (Geoms/CMS-2017.cc:
// 440-470): first TIB and TOB layers, first TID and TEC disks each side,
// and the radial extent of the first two disks of each.
struct RegionCuts {
  float tib1_rin, tib1_zmax, tib1_zmin, tob1_rin, tob1_zmax, tob1_zmin;
  float tidp1_zmin, tidn1_zmax, tecp1_zmin, tecn1_zmax;
  float tidp_rin, tidp_rout, tecp_rin, tecp_rout, tidn_rin, tidn_rout, tecn_rin, tecn_rout;
};
RegionCuts region_cuts_cms2017(const float* layer_desc);

void partition_seeds_cms2017(const float* layer_desc, int n_layers, const SeedInput& s,
                             const int32_t* layer_begin, const float* hit_pos, int hit_stride,
                             SeedOrder& out);

}  // namespace mkfg
