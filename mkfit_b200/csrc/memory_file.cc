// mkFit "memoryFile" event files (DataFile / Event::write_out / read_in,
// Event.cc:123-444, DataFileHeader Event.h:74-89), read into and written
// from this library's structure-of-arrays layout. Host code only.
//
// The format is the reference's raw struct dump on x86-64:
//   header: 8 int32 (magic 0xBEEF, version 6, sizeof Track / Hit /
//           HitOnTrack, n_layers, n_events, extra-section bits);
//   per event: int32 size of the event record (itself included), then
//     tracks(sim)         [n, data_size, n x Track (160 B), hits of each]
//     [sim track states]  [n, n x TrackState (112 B)]     (ES_SimTrackStates)
//     n_layers, per layer [n_hits, n_hits x Hit (44 B)]
//     [hit masks]         per layer n_hits x uint64        (ES_HitIterMasks)
//     n_mc, n_mc x MCHitInfo (4 x int32)
//     [tracks(seeds)]                                      (ES_Seeds)
//     [tracks(cmssw)]                                      (ES_CmsswTracks)
//     [BeamSpot]          8 float32                        (ES_BeamSpot)
// Track (160 B): TrackState {params 6 f32, errors 21 f32, charge int16,
// valid bool, pad} @0, chi2 f32 @112, score f32 @116, lastHitIdx int16
// @120, nFoundHits int16 @122, status uint32 @124, label int32 @128, pad,
// std::vector<HitOnTrack> @136 (pointers; meaningless on file, written as
// zeros here). Hit (44 B): pos 3 f32, err 6 f32 (packed sym 3x3), mcHitID
// int32, packed uint32 (detid 12 bits | charge-per-cm code 8 | span rows 3
// | span cols 3). HitOnTrack: int32 with index in the low 24 bits (signed),
// layer in the high 8.
#include "../../include/mkfit_b200.h"

#include <algorithm>
#include <cerrno>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace mkfg {
int set_error(int code, const char* fmt, ...);
}

namespace {

constexpr int kMagic = 0xBEEF;
constexpr int kVersion = 6;
constexpr int kMinVersion = 4;
constexpr int kSizeTrack = 160;
constexpr int kSizeTrackState = 112;
constexpr int kSizeHit = 44;
constexpr int kSizeHot = 4;
constexpr int kSizeMc = 16;
constexpr int kSizeBeamSpot = 32;

struct TrackArrays {
  std::vector<float> par, err, chi2, score;
  std::vector<int32_t> charge, label, nfound, hits_begin, hit_index, hit_layer;
  std::vector<uint32_t> status;
  std::vector<uint8_t> valid;
  void fill(mkfg_mf_tracks* t) const {
    t->n = (int32_t)charge.size();
    t->par = par.data();
    t->err = err.data();
    t->charge = charge.data();
    t->valid = valid.data();
    t->chi2 = chi2.data();
    t->score = score.data();
    t->status = status.data();
    t->label = label.data();
    t->nfound = nfound.data();
    t->hits_begin = hits_begin.data();
    t->hit_index = hit_index.data();
    t->hit_layer = hit_layer.data();
  }
};

template <typename T>
T load(const uint8_t* p) {
  T v;
  std::memcpy(&v, p, sizeof(T));
  return v;
}
template <typename T>
void store(uint8_t* p, T v) {
  std::memcpy(p, &v, sizeof(T));
}

struct Cursor {
  const uint8_t* p;
  const uint8_t* end;
  bool ok = true;
  bool need(size_t n) {
    if (!ok || (size_t)(end - p) < n) ok = false;
    return ok;
  }
  int32_t i32() {
    if (!need(4)) return 0;
    const int32_t v = load<int32_t>(p);
    p += 4;
    return v;
  }
};

// TrackState fields from 112 bytes, into column n of [6][cap] / [21][cap].
void unpack_state(const uint8_t* s, int i, int cap, float* par, float* err, int32_t* charge,
                  uint8_t* valid) {
  for (int k = 0; k < 6; ++k) par[k * cap + i] = load<float>(s + 4 * k);
  for (int k = 0; k < 21; ++k) err[k * cap + i] = load<float>(s + 24 + 4 * k);
  charge[i] = load<int16_t>(s + 108);
  valid[i] = load<uint8_t>(s + 110);
}

bool read_tracks(Cursor& c, TrackArrays& t) {
  const int n = c.i32();
  const int data_size = c.i32();
  if (!c.ok || n < 0 || data_size < 8) return false;
  if (!c.need((size_t)n * kSizeTrack)) return false;
  t.par.assign(6 * (size_t)n, 0.f);
  t.err.assign(21 * (size_t)n, 0.f);
  t.charge.assign(n, 0);
  t.valid.assign(n, 0);
  t.chi2.assign(n, 0.f);
  t.score.assign(n, 0.f);
  t.status.assign(n, 0);
  t.label.assign(n, 0);
  t.nfound.assign(n, 0);
  t.hits_begin.assign(n + 1, 0);
  std::vector<int> nh(n);
  for (int i = 0; i < n; ++i) {
    const uint8_t* r = c.p + (size_t)i * kSizeTrack;
    unpack_state(r, i, n, t.par.data(), t.err.data(), t.charge.data(), t.valid.data());
    t.chi2[i] = load<float>(r + 112);
    t.score[i] = load<float>(r + 116);
    nh[i] = load<int16_t>(r + 120) + 1;  // lastHitIdx + 1
    t.nfound[i] = load<int16_t>(r + 122);
    t.status[i] = load<uint32_t>(r + 124);
    t.label[i] = load<int32_t>(r + 128);
    if (nh[i] < 0) return false;
    t.hits_begin[i + 1] = t.hits_begin[i] + nh[i];
  }
  c.p += (size_t)n * kSizeTrack;
  const int total = t.hits_begin[n];
  if (!c.need((size_t)total * kSizeHot)) return false;
  if (8 + (size_t)n * kSizeTrack + (size_t)total * kSizeHot != (size_t)data_size) return false;
  t.hit_index.resize(total);
  t.hit_layer.resize(total);
  for (int h = 0; h < total; ++h) {
    const uint32_t w = load<uint32_t>(c.p + 4 * (size_t)h);
    t.hit_index[h] = (int32_t)(w << 8) >> 8;  // signed 24-bit
    t.hit_layer[h] = (int32_t)w >> 24;        // signed 8-bit
  }
  c.p += (size_t)total * kSizeHot;
  return true;
}

}  // namespace

struct mkfg_mf_reader {
  FILE* fp = nullptr;
  mkfg_mf_header hdr{};
  std::vector<long> ev_pos;  // file offset of each event record
  std::vector<uint8_t> buf;
  // Current event, in SoA.
  std::vector<int32_t> layer_begin, hit_mcid, mc;
  std::vector<float> hit_pos, hit_err, beam;
  std::vector<uint32_t> hit_packed;
  std::vector<uint64_t> hit_masks;
  std::vector<float> state_par, state_err;
  std::vector<int32_t> state_charge;
  std::vector<uint8_t> state_valid;
  TrackArrays sim, seeds, cmssw;
};

extern "C" int mkfg_mf_open(const char* path, mkfg_mf_reader** out, mkfg_mf_header* hdr) {
  using mkfg::set_error;
  if (!path || !out) return set_error(MKFG_ERR_BAD_INPUT, "null argument");
  *out = nullptr;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return set_error(MKFG_ERR_BAD_INPUT, "cannot open %s: %s", path, std::strerror(errno));
  int32_t h[8];
  if (std::fread(h, 4, 8, fp) != 8) {
    std::fclose(fp);
    return set_error(MKFG_ERR_BAD_INPUT, "%s: short header", path);
  }
  auto fail = [&](const char* what, int got, int want) {
    std::fclose(fp);
    return set_error(MKFG_ERR_BAD_INPUT, "%s: %s is %d, expected %d", path, what, got, want);
  };
  if (h[0] != kMagic) return fail("magic", h[0], kMagic);
  if (h[1] < kMinVersion || h[1] > kVersion) return fail("format version", h[1], kVersion);
  if (h[2] != kSizeTrack) return fail("sizeof(Track)", h[2], kSizeTrack);
  if (h[3] != kSizeHit) return fail("sizeof(Hit)", h[3], kSizeHit);
  if (h[4] != kSizeHot) return fail("sizeof(HitOnTrack)", h[4], kSizeHot);
  if (h[5] <= 0 || h[5] > 127) return fail("n_layers", h[5], 72);
  auto* r = new mkfg_mf_reader;
  r->fp = fp;
  r->hdr.format_version = h[1];
  r->hdr.n_layers = h[5];
  r->hdr.n_events = h[6];
  r->hdr.extra_sections = h[7];
  // Index the event records: each starts with its own size.
  std::fseek(fp, 0, SEEK_END);
  const long size = std::ftell(fp);
  long pos = 32;
  while (pos + 4 <= size && (int)r->ev_pos.size() < std::max(h[6], 0)) {
    int32_t ev_size = 0;
    std::fseek(fp, pos, SEEK_SET);
    if (std::fread(&ev_size, 4, 1, fp) != 1 || ev_size < 4 || pos + ev_size > size) break;
    r->ev_pos.push_back(pos);
    pos += ev_size;
  }
  r->hdr.n_events = (int32_t)r->ev_pos.size();
  *out = r;
  if (hdr) *hdr = r->hdr;
  if ((int)r->ev_pos.size() != h[6])
    return set_error(MKFG_ERR_BAD_INPUT, "%s: header promises %d events, %d complete records found",
                     path, h[6], (int)r->ev_pos.size());
  return MKFG_OK;
}

extern "C" int mkfg_mf_read_event(mkfg_mf_reader* r, int32_t event, mkfg_mf_event* out) {
  using mkfg::set_error;
  if (!r || !out) return set_error(MKFG_ERR_BAD_INPUT, "null argument");
  if (event < 0 || event >= (int)r->ev_pos.size())
    return set_error(MKFG_ERR_BAD_INPUT, "event %d out of range (%d events)", event, (int)r->ev_pos.size());
  int32_t ev_size = 0;
  std::fseek(r->fp, r->ev_pos[event], SEEK_SET);
  if (std::fread(&ev_size, 4, 1, r->fp) != 1) return set_error(MKFG_ERR_BAD_INPUT, "read error");
  r->buf.resize((size_t)ev_size - 4);
  if (std::fread(r->buf.data(), 1, r->buf.size(), r->fp) != r->buf.size())
    return set_error(MKFG_ERR_BAD_INPUT, "event %d: short record", event);
  Cursor c{r->buf.data(), r->buf.data() + r->buf.size()};
  const int es = r->hdr.extra_sections;
  auto bad = [&](const char* what) {
    return set_error(MKFG_ERR_BAD_INPUT, "event %d: malformed %s", event, what);
  };
  if (!read_tracks(c, r->sim)) return bad("sim tracks");
  int n_states = 0;
  if (es & MKFG_MF_SIM_TRACK_STATES) {
    n_states = c.i32();
    if (n_states < 0 || !c.need((size_t)n_states * kSizeTrackState)) return bad("sim track states");
    r->state_par.assign(6 * (size_t)n_states, 0.f);
    r->state_err.assign(21 * (size_t)n_states, 0.f);
    r->state_charge.assign(n_states, 0);
    r->state_valid.assign(n_states, 0);
    for (int i = 0; i < n_states; ++i)
      unpack_state(c.p + (size_t)i * kSizeTrackState, i, n_states, r->state_par.data(),
                   r->state_err.data(), r->state_charge.data(), r->state_valid.data());
    c.p += (size_t)n_states * kSizeTrackState;
  }
  const int nl = c.i32();
  if (!c.ok || nl < 0 || nl > 127) return bad("layer count");
  r->layer_begin.assign(nl + 1, 0);
  std::vector<const uint8_t*> lay(nl);
  for (int l = 0; l < nl; ++l) {
    const int nh = c.i32();
    if (nh < 0 || !c.need((size_t)nh * kSizeHit)) return bad("layer hits");
    lay[l] = c.p;
    c.p += (size_t)nh * kSizeHit;
    r->layer_begin[l + 1] = r->layer_begin[l] + nh;
  }
  const int NH = r->layer_begin[nl];
  r->hit_pos.assign(3 * (size_t)NH, 0.f);
  r->hit_err.assign(6 * (size_t)NH, 0.f);
  r->hit_mcid.assign(NH, 0);
  r->hit_packed.assign(NH, 0);
  for (int l = 0; l < nl; ++l)
    for (int h = r->layer_begin[l]; h < r->layer_begin[l + 1]; ++h) {
      const uint8_t* p = lay[l] + (size_t)(h - r->layer_begin[l]) * kSizeHit;
      for (int k = 0; k < 3; ++k) r->hit_pos[k * (size_t)NH + h] = load<float>(p + 4 * k);
      for (int k = 0; k < 6; ++k) r->hit_err[k * (size_t)NH + h] = load<float>(p + 12 + 4 * k);
      r->hit_mcid[h] = load<int32_t>(p + 36);
      r->hit_packed[h] = load<uint32_t>(p + 40);
    }
  r->hit_masks.clear();
  if (es & MKFG_MF_HIT_ITER_MASKS) {
    if (!c.need((size_t)NH * 8)) return bad("hit masks");
    r->hit_masks.resize(NH);
    std::memcpy(r->hit_masks.data(), c.p, (size_t)NH * 8);
    c.p += (size_t)NH * 8;
  }
  const int nm = c.i32();
  if (nm < 0 || !c.need((size_t)nm * kSizeMc)) return bad("MC hit info");
  r->mc.resize(4 * (size_t)nm);
  std::memcpy(r->mc.data(), c.p, (size_t)nm * kSizeMc);
  c.p += (size_t)nm * kSizeMc;
  TrackArrays empty;
  if (es & MKFG_MF_SEEDS) {
    if (!read_tracks(c, r->seeds)) return bad("seeds");
  } else {
    r->seeds = empty;
    r->seeds.hits_begin.assign(1, 0);
  }
  if (es & MKFG_MF_CMSSW_TRACKS) {
    if (!read_tracks(c, r->cmssw)) return bad("CMSSW tracks");
  } else {
    r->cmssw = empty;
    r->cmssw.hits_begin.assign(1, 0);
  }
  r->beam.assign(8, 0.f);
  if (es & MKFG_MF_BEAM_SPOT) {
    if (!c.need(kSizeBeamSpot)) return bad("beam spot");
    std::memcpy(r->beam.data(), c.p, kSizeBeamSpot);
    c.p += kSizeBeamSpot;
  }
  if (!c.ok) return bad("record");
  if (c.p != c.end) return bad("record size");

  std::memset(out, 0, sizeof(*out));
  out->n_layers = nl;
  out->layer_begin = r->layer_begin.data();
  out->hit_pos = r->hit_pos.data();
  out->hit_err = r->hit_err.data();
  out->hit_mcid = r->hit_mcid.data();
  out->hit_packed = r->hit_packed.data();
  out->hit_masks = r->hit_masks.empty() ? nullptr : r->hit_masks.data();
  out->n_mc = nm;
  out->mc_info = r->mc.data();
  r->sim.fill(&out->sim);
  r->seeds.fill(&out->seeds);
  r->cmssw.fill(&out->cmssw);
  out->n_sim_states = n_states;
  out->sim_state_par = r->state_par.data();
  out->sim_state_err = r->state_err.data();
  out->sim_state_charge = r->state_charge.data();
  out->beam_spot = r->beam.data();
  return MKFG_OK;
}

extern "C" void mkfg_mf_close(mkfg_mf_reader* r) {
  if (!r) return;
  if (r->fp) std::fclose(r->fp);
  delete r;
}

namespace {

void put_i32(std::vector<uint8_t>& b, int32_t v) {
  const size_t at = b.size();
  b.resize(at + 4);
  store(b.data() + at, v);
}

void pack_state(uint8_t* s, const float* par, const float* err, int i, int n, int charge,
                uint8_t valid) {
  for (int k = 0; k < 6; ++k) store(s + 4 * k, par[k * (size_t)n + i]);
  for (int k = 0; k < 21; ++k) store(s + 24 + 4 * k, err[k * (size_t)n + i]);
  store<int16_t>(s + 108, (int16_t)charge);
  store<uint8_t>(s + 110, valid);
}

int put_tracks(std::vector<uint8_t>& b, const mkfg_mf_tracks& t, const char* what) {
  using mkfg::set_error;
  const int n = t.n;
  if (n < 0) return set_error(MKFG_ERR_BAD_INPUT, "%s: negative count", what);
  if (n > 0 && (!t.par || !t.err || !t.charge || !t.hits_begin))
    return set_error(MKFG_ERR_BAD_INPUT, "%s: null array", what);
  const int total = n ? t.hits_begin[n] - t.hits_begin[0] : 0;
  if (total > 0 && (!t.hit_index || !t.hit_layer)) return set_error(MKFG_ERR_BAD_INPUT, "%s: null hits", what);
  put_i32(b, n);
  put_i32(b, 8 + n * kSizeTrack + total * kSizeHot);
  const size_t at = b.size();
  b.resize(at + (size_t)n * kSizeTrack, 0);
  for (int i = 0; i < n; ++i) {
    uint8_t* r = b.data() + at + (size_t)i * kSizeTrack;
    const int nh = t.hits_begin[i + 1] - t.hits_begin[i];
    if (nh < 0 || nh > 32767) return set_error(MKFG_ERR_BAD_INPUT, "%s %d: bad hit count", what, i);
    pack_state(r, t.par, t.err, i, n, t.charge[i], t.valid ? t.valid[i] : 1);
    store(r + 112, t.chi2 ? t.chi2[i] : 0.f);
    store(r + 116, t.score ? t.score[i] : 0.f);
    store<int16_t>(r + 120, (int16_t)(nh - 1));
    int nf = 0;
    if (t.nfound) {
      nf = t.nfound[i];
    } else {
      for (int h = t.hits_begin[i]; h < t.hits_begin[i + 1]; ++h)
        if (t.hit_index[h] >= 0 || t.hit_index[h] == -9) ++nf;  // Track::addHitIdx
    }
    store<int16_t>(r + 122, (int16_t)nf);
    store<uint32_t>(r + 124, t.status ? t.status[i] : 0u);
    store<int32_t>(r + 128, t.label ? t.label[i] : -1);
  }
  for (int h = t.hits_begin[0]; h < t.hits_begin[0] + total; ++h) {
    const int idx = t.hit_index[h], lay = t.hit_layer[h];
    if (idx < -(1 << 23) || idx >= (1 << 23) || lay < -128 || lay > 127)
      return set_error(MKFG_ERR_BAD_INPUT, "%s: hit (%d, %d) does not fit HitOnTrack", what, idx, lay);
    put_i32(b, (int32_t)(((uint32_t)idx & 0xffffffu) | ((uint32_t)lay << 24)));
  }
  return MKFG_OK;
}

}  // namespace

extern "C" int mkfg_mf_write(const char* path, int32_t n_layers, int32_t extra_sections,
                             int32_t n_events, const mkfg_mf_event* events) {
  using mkfg::set_error;
  if (!path || (n_events > 0 && !events)) return set_error(MKFG_ERR_BAD_INPUT, "null argument");
  if (n_layers <= 0 || n_layers > 127) return set_error(MKFG_ERR_BAD_INPUT, "bad n_layers %d", n_layers);
  if (extra_sections & ~0x1f) return set_error(MKFG_ERR_BAD_INPUT, "unknown extra sections 0x%x", extra_sections);
  std::vector<uint8_t> b;
  const int32_t hdr[8] = {kMagic, kVersion, kSizeTrack, kSizeHit, kSizeHot, n_layers, n_events,
                          extra_sections};
  for (int k = 0; k < 8; ++k) put_i32(b, hdr[k]);
  for (int e = 0; e < n_events; ++e) {
    const mkfg_mf_event& ev = events[e];
    if (ev.n_layers != n_layers) return set_error(MKFG_ERR_BAD_INPUT, "event %d: n_layers %d", e, ev.n_layers);
    const size_t start = b.size();
    put_i32(b, 0);  // record size, set below
    int rc = put_tracks(b, ev.sim, "sim tracks");
    if (rc) return rc;
    if (extra_sections & MKFG_MF_SIM_TRACK_STATES) {
      const int n = ev.n_sim_states;
      if (n < 0 || (n > 0 && (!ev.sim_state_par || !ev.sim_state_err || !ev.sim_state_charge)))
        return set_error(MKFG_ERR_BAD_INPUT, "event %d: sim track states", e);
      put_i32(b, n);
      const size_t at = b.size();
      b.resize(at + (size_t)n * kSizeTrackState, 0);
      for (int i = 0; i < n; ++i)
        pack_state(b.data() + at + (size_t)i * kSizeTrackState, ev.sim_state_par, ev.sim_state_err, i,
                   n, ev.sim_state_charge[i], 1);
    }
    const int NH = ev.layer_begin ? ev.layer_begin[n_layers] : 0;
    if (!ev.layer_begin || ev.layer_begin[0] != 0 || (NH > 0 && (!ev.hit_pos || !ev.hit_err)))
      return set_error(MKFG_ERR_BAD_INPUT, "event %d: hits", e);
    put_i32(b, n_layers);
    for (int l = 0; l < n_layers; ++l) {
      const int h0 = ev.layer_begin[l], h1 = ev.layer_begin[l + 1];
      if (h1 < h0) return set_error(MKFG_ERR_BAD_INPUT, "event %d: layer_begin not sorted", e);
      put_i32(b, h1 - h0);
      const size_t at = b.size();
      b.resize(at + (size_t)(h1 - h0) * kSizeHit, 0);
      for (int h = h0; h < h1; ++h) {
        uint8_t* p = b.data() + at + (size_t)(h - h0) * kSizeHit;
        for (int k = 0; k < 3; ++k) store(p + 4 * k, ev.hit_pos[k * (size_t)NH + h]);
        for (int k = 0; k < 6; ++k) store(p + 12 + 4 * k, ev.hit_err[k * (size_t)NH + h]);
        store<int32_t>(p + 36, ev.hit_mcid ? ev.hit_mcid[h] : -1);
        store<uint32_t>(p + 40, ev.hit_packed ? ev.hit_packed[h] : 0u);
      }
    }
    if (extra_sections & MKFG_MF_HIT_ITER_MASKS) {
      const size_t at = b.size();
      b.resize(at + (size_t)NH * 8, 0);
      if (ev.hit_masks) std::memcpy(b.data() + at, ev.hit_masks, (size_t)NH * 8);
    }
    if (ev.n_mc < 0 || (ev.n_mc > 0 && !ev.mc_info)) return set_error(MKFG_ERR_BAD_INPUT, "event %d: MC info", e);
    put_i32(b, ev.n_mc);
    {
      const size_t at = b.size();
      b.resize(at + (size_t)ev.n_mc * kSizeMc);
      if (ev.n_mc) std::memcpy(b.data() + at, ev.mc_info, (size_t)ev.n_mc * kSizeMc);
    }
    if (extra_sections & MKFG_MF_SEEDS)
      if ((rc = put_tracks(b, ev.seeds, "seeds"))) return rc;
    if (extra_sections & MKFG_MF_CMSSW_TRACKS)
      if ((rc = put_tracks(b, ev.cmssw, "CMSSW tracks"))) return rc;
    if (extra_sections & MKFG_MF_BEAM_SPOT) {
      const size_t at = b.size();
      b.resize(at + kSizeBeamSpot, 0);
      if (ev.beam_spot) {
        std::memcpy(b.data() + at, ev.beam_spot, kSizeBeamSpot);
      } else {
        const float def[8] = {0.f, 0.f, 0.f, 5.f, 5e-4f, 5e-4f, 0.f, 0.f};  // BeamSpot() defaults
        std::memcpy(b.data() + at, def, kSizeBeamSpot);
      }
    }
    store<int32_t>(b.data() + start, (int32_t)(b.size() - start));
  }
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return set_error(MKFG_ERR_BAD_INPUT, "cannot create %s: %s", path, std::strerror(errno));
  const bool ok = std::fwrite(b.data(), 1, b.size(), fp) == b.size();
  if (std::fclose(fp) != 0 || !ok) return set_error(MKFG_ERR_BAD_INPUT, "write to %s failed", path);
  return MKFG_OK;
}

extern "C" int mkfg_mf_finder_event(const mkfg_mf_event* ev, int32_t* detid, int32_t* cpcm,
                                    int32_t max_seed_hits, int32_t* seed_nhits,
                                    int32_t* seed_hit_layer, int32_t* seed_hit_index) {
  using mkfg::set_error;
  if (!ev || (!detid && !cpcm && !seed_nhits)) return set_error(MKFG_ERR_BAD_INPUT, "null argument");
  const int NH = ev->layer_begin ? ev->layer_begin[ev->n_layers] : 0;
  for (int h = 0; h < NH; ++h) {
    const uint32_t w = ev->hit_packed ? ev->hit_packed[h] : 0u;
    if (detid) detid[h] = (int32_t)(w & 0xfffu);
    if (cpcm) {
      // A charge-per-cm value whose Hit::setupAsStrip code is the stored
      // code; 0xff (pixels, or the top strip code) becomes -1, which codes
      // to 0xff as well.
      const int code = (int)((w >> 12) & 0xffu);
      cpcm[h] = code == 0xff ? -1 : code == 0 ? 0 : ((code - 1) << 3) + 1620;
    }
  }
  if (seed_nhits) {
    if (!seed_hit_layer || !seed_hit_index || max_seed_hits <= 0)
      return set_error(MKFG_ERR_BAD_INPUT, "null seed-hit arrays");
    const mkfg_mf_tracks& s = ev->seeds;
    for (int i = 0; i < s.n; ++i) {
      const int h0 = s.hits_begin[i], n = s.hits_begin[i + 1] - h0;
      if (n > max_seed_hits)
        return set_error(MKFG_ERR_OVERFLOW, "seed %d has %d hits (> %d)", i, n, max_seed_hits);
      seed_nhits[i] = n;
      for (int k = 0; k < max_seed_hits; ++k) {
        seed_hit_layer[(size_t)i * max_seed_hits + k] = k < n ? s.hit_layer[h0 + k] : -1;
        seed_hit_index[(size_t)i * max_seed_hits + k] = k < n ? s.hit_index[h0 + k] : -1;
      }
    }
  }
  return MKFG_OK;
}
