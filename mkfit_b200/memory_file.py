"""mkFit memoryFile event files (DataFile / Event::write_out / read_in,
Event.cc:123-444): the host side of mkfg_mf_open / _read_event / _write.

    hdr, events = memory_file.read("events.bin")       # list of dicts
    memory_file.write("out.bin", events, n_layers=72, sections=SEEDS | BEAM_SPOT)
    ev = memory_file.to_cms_event(events[0])            # finder input

Event dicts hold numpy arrays in this library's SoA layout: layer_begin,
hit_pos [3][n], hit_err [6][n], hit_mcid, hit_packed, hit_masks (or None),
mc_info [n_mc][4], sim / seeds / cmssw track dicts (par [6][n], err [21][n],
charge, valid, chi2, score, status, label, nfound, hits_begin, hit_index,
hit_layer), sim_states (par, err, charge), beam_spot [8]."""
import ctypes

import numpy as np

from . import capi

SIM_TRACK_STATES, SEEDS, CMSSW_TRACKS, HIT_ITER_MASKS, BEAM_SPOT = 0x1, 0x2, 0x4, 0x8, 0x10

_vp = ctypes.c_void_p


class MkfgMfHeader(ctypes.Structure):
    _fields_ = [("format_version", ctypes.c_int32), ("n_layers", ctypes.c_int32),
                ("n_events", ctypes.c_int32), ("extra_sections", ctypes.c_int32)]


class MkfgMfTracks(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32)] + [(k, _vp) for k in (
        "par", "err", "charge", "valid", "chi2", "score", "status", "label", "nfound",
        "hits_begin", "hit_index", "hit_layer")]


class MkfgMfEvent(ctypes.Structure):
    _fields_ = [("n_layers", ctypes.c_int32)] + [(k, _vp) for k in (
        "layer_begin", "hit_pos", "hit_err", "hit_mcid", "hit_packed", "hit_masks")] + [
        ("n_mc", ctypes.c_int32), ("mc_info", _vp), ("sim", MkfgMfTracks),
        ("seeds", MkfgMfTracks), ("cmssw", MkfgMfTracks), ("n_sim_states", ctypes.c_int32),
        ("sim_state_par", _vp), ("sim_state_err", _vp), ("sim_state_charge", _vp),
        ("beam_spot", _vp)]


TRACK_FIELDS = (("par", np.float32), ("err", np.float32), ("charge", np.int32),
                ("valid", np.uint8), ("chi2", np.float32), ("score", np.float32),
                ("status", np.uint32), ("label", np.int32), ("nfound", np.int32),
                ("hits_begin", np.int32), ("hit_index", np.int32), ("hit_layer", np.int32))


def _lib():
    lib = capi.load()
    if not getattr(lib, "_mf_bound", False):
        lib.mkfg_mf_open.argtypes = [ctypes.c_char_p, ctypes.POINTER(_vp), ctypes.POINTER(MkfgMfHeader)]
        lib.mkfg_mf_read_event.argtypes = [_vp, ctypes.c_int32, ctypes.POINTER(MkfgMfEvent)]
        lib.mkfg_mf_close.argtypes = [_vp]
        lib.mkfg_mf_close.restype = None
        lib.mkfg_mf_write.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.POINTER(MkfgMfEvent)]
        lib.mkfg_mf_finder_event.argtypes = [ctypes.POINTER(MkfgMfEvent), _vp, _vp, ctypes.c_int32,
                                             _vp, _vp, _vp]
        lib._mf_bound = True
    return lib


def _copy(ptr, n, dtype):
    if n == 0 or not ptr:
        return np.zeros(n, dtype)
    buf = (ctypes.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(buf, dtype).copy()


def _tracks_out(t):
    n = t.n
    hb = _copy(t.hits_begin, n + 1, np.int32)
    nh = int(hb[-1]) if n >= 0 else 0
    return dict(par=_copy(t.par, 6 * n, np.float32).reshape(6, n),
                err=_copy(t.err, 21 * n, np.float32).reshape(21, n),
                charge=_copy(t.charge, n, np.int32), valid=_copy(t.valid, n, np.uint8),
                chi2=_copy(t.chi2, n, np.float32), score=_copy(t.score, n, np.float32),
                status=_copy(t.status, n, np.uint32), label=_copy(t.label, n, np.int32),
                nfound=_copy(t.nfound, n, np.int32), hits_begin=hb,
                hit_index=_copy(t.hit_index, nh, np.int32), hit_layer=_copy(t.hit_layer, nh, np.int32))


def _event_out(e):
    nl = e.n_layers
    lb = _copy(e.layer_begin, nl + 1, np.int32)
    nh = int(lb[-1])
    st = e.n_sim_states
    return dict(
        n_layers=nl, layer_begin=lb,
        hit_pos=_copy(e.hit_pos, 3 * nh, np.float32).reshape(3, nh),
        hit_err=_copy(e.hit_err, 6 * nh, np.float32).reshape(6, nh),
        hit_mcid=_copy(e.hit_mcid, nh, np.int32), hit_packed=_copy(e.hit_packed, nh, np.uint32),
        hit_masks=_copy(e.hit_masks, nh, np.uint64) if e.hit_masks else None,
        mc_info=_copy(e.mc_info, 4 * e.n_mc, np.int32).reshape(e.n_mc, 4),
        sim=_tracks_out(e.sim), seeds=_tracks_out(e.seeds), cmssw=_tracks_out(e.cmssw),
        sim_states=dict(par=_copy(e.sim_state_par, 6 * st, np.float32).reshape(6, st),
                        err=_copy(e.sim_state_err, 21 * st, np.float32).reshape(21, st),
                        charge=_copy(e.sim_state_charge, st, np.int32)),
        beam_spot=_copy(e.beam_spot, 8, np.float32))


class Reader:
    """DataFile opened for reading; events by index (reader[i]), len()."""

    def __init__(self, path):
        self.lib = _lib()
        self.handle = _vp()
        h = MkfgMfHeader()
        rc = self.lib.mkfg_mf_open(str(path).encode(), ctypes.byref(self.handle), ctypes.byref(h))
        if rc != capi.MKFG_OK:
            msg = capi.last_error()
            if self.handle:
                self.lib.mkfg_mf_close(self.handle)
                self.handle = _vp()
            raise capi.MkfgError(rc, msg)
        self.header = dict(format_version=h.format_version, n_layers=h.n_layers,
                           n_events=h.n_events, extra_sections=h.extra_sections)

    def __len__(self):
        return self.header["n_events"]

    def __getitem__(self, i):
        e = MkfgMfEvent()
        capi.check(self.lib.mkfg_mf_read_event(self.handle, int(i), ctypes.byref(e)))
        return _event_out(e)

    def close(self):
        if self.handle:
            self.lib.mkfg_mf_close(self.handle)
            self.handle = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        self.close()


def read(path):
    """(header dict, list of event dicts) of a whole file."""
    with Reader(path) as r:
        return r.header, [r[i] for i in range(len(r))]


def _tracks_in(t, keep):
    t = t or {}
    n = len(t.get("charge", ()))
    s = MkfgMfTracks()
    s.n = n
    for k, dt in TRACK_FIELDS:
        v = t.get(k)
        if v is None:
            if k == "hits_begin":
                v = np.zeros(n + 1, np.int32)
            elif k in ("par", "err", "charge"):
                v = np.zeros(((6 if k == "par" else 21), n) if k != "charge" else n, dt)
            else:
                setattr(s, k, None)
                continue
        a = np.ascontiguousarray(v, dt)
        keep.append(a)
        setattr(s, k, a.ctypes.data)
    return s


def _event_in(ev, keep):
    e = MkfgMfEvent()
    e.n_layers = int(ev["n_layers"])
    for k, dt in (("layer_begin", np.int32), ("hit_pos", np.float32), ("hit_err", np.float32),
                  ("hit_mcid", np.int32), ("hit_packed", np.uint32), ("hit_masks", np.uint64)):
        v = ev.get(k)
        if v is None:
            setattr(e, k, None)
            continue
        a = np.ascontiguousarray(v, dt)
        keep.append(a)
        setattr(e, k, a.ctypes.data)
    mc = np.ascontiguousarray(ev.get("mc_info", np.zeros((0, 4))), np.int32).reshape(-1, 4)
    keep.append(mc)
    e.n_mc = mc.shape[0]
    e.mc_info = mc.ctypes.data
    e.sim = _tracks_in(ev.get("sim"), keep)
    e.seeds = _tracks_in(ev.get("seeds"), keep)
    e.cmssw = _tracks_in(ev.get("cmssw"), keep)
    st = ev.get("sim_states") or {}
    n = len(st.get("charge", ()))
    e.n_sim_states = n
    for k, f, dt in (("par", "sim_state_par", np.float32), ("err", "sim_state_err", np.float32),
                     ("charge", "sim_state_charge", np.int32)):
        if n:
            a = np.ascontiguousarray(st[k], dt)
            keep.append(a)
            setattr(e, f, a.ctypes.data)
    if ev.get("beam_spot") is not None:
        b = np.ascontiguousarray(ev["beam_spot"], np.float32)
        keep.append(b)
        e.beam_spot = b.ctypes.data
    return e


def write(path, events, n_layers, sections=0):
    """DataFile::OpenWrite + Event::write_out of each event + CloseWrite."""
    keep = []
    arr = (MkfgMfEvent * max(len(events), 1))()
    for i, ev in enumerate(events):
        arr[i] = _event_in(ev, keep)
    capi.check(_lib().mkfg_mf_write(str(path).encode(), int(n_layers), int(sections), len(events), arr))


def packed_hits(detid, cpcm):
    """Hit::PackedData bits of hits given as the finder's (detid, cpcm):
    setupAsPixel (cpcm < 0: code 0xff) or setupAsStrip (Hit.h:285-300);
    the cluster spans, which the finder does not use, are left 0."""
    detid = np.asarray(detid, np.int64)
    cpcm = np.asarray(cpcm, np.int64)
    code = np.where(cpcm < 0, 0xff, np.where(cpcm < 1620, 0, np.minimum(0xff, ((cpcm - 1620) >> 3) + 1)))
    return ((detid & 0xfff) | (code << 12)).astype(np.uint32)


def from_cms_event(ev, with_seeds=True):
    """Event dict of a synthetic CmsEvent (hits, MC hit info, seeds)."""
    n = ev.n_hits
    mcid = np.arange(n, dtype=np.int32)
    mc = np.zeros((n, 4), np.int32)
    mc[:, 0] = ev.hit_mc
    for l in range(ev.n_layers):
        a, b = ev.layer_begin[l], ev.layer_begin[l + 1]
        mc[a:b, 1] = l
        mc[a:b, 2] = np.arange(b - a)
    mc[:, 3] = mcid
    out = dict(n_layers=ev.n_layers, layer_begin=ev.layer_begin, hit_pos=ev.hit_pos,
               hit_err=ev.hit_err, hit_mcid=mcid, hit_packed=packed_hits(ev.hit_detid, ev.hit_cpcm),
               hit_masks=None, mc_info=mc, beam_spot=None)
    if with_seeds:
        ns = ev.n_seeds
        hb = np.concatenate([[0], np.cumsum(ev.seed_nhits)]).astype(np.int32)
        hi = np.concatenate([ev.seed_hit_index[i, :ev.seed_nhits[i]] for i in range(ns)] or
                            [np.zeros(0, np.int32)])
        hl = np.concatenate([ev.seed_hit_layer[i, :ev.seed_nhits[i]] for i in range(ns)] or
                            [np.zeros(0, np.int32)])
        out["seeds"] = dict(par=ev.seed_par, err=ev.seed_err, charge=ev.seed_chg,
                            label=np.arange(ns, dtype=np.int32), hits_begin=hb,
                            hit_index=hi, hit_layer=hl)
    return out


def to_cms_event(ev, max_seed_hits=16):
    """The finder's input (a CmsEvent: hits with detid / cpcm and seeds with
    up to max_seed_hits hits) from a read event dict."""
    from .synth import CmsEvent
    lib = _lib()
    keep = []
    e = _event_in(ev, keep)
    nh = int(ev["layer_begin"][-1])
    ns = len(ev["seeds"]["charge"])
    detid = np.zeros(nh, np.int32)
    cpcm = np.zeros(nh, np.int32)
    snh = np.zeros(ns, np.int32)
    shl = np.zeros((ns, max_seed_hits), np.int32)
    shi = np.zeros((ns, max_seed_hits), np.int32)
    capi.check(lib.mkfg_mf_finder_event(ctypes.byref(e), detid.ctypes.data, cpcm.ctypes.data,
                                        max_seed_hits, snh.ctypes.data, shl.ctypes.data,
                                        shi.ctypes.data))
    s = ev["seeds"]
    return CmsEvent(n_layers=int(ev["n_layers"]), layer_begin=np.asarray(ev["layer_begin"], np.int32),
                    hit_pos=np.ascontiguousarray(ev["hit_pos"], np.float32),
                    hit_err=np.ascontiguousarray(ev["hit_err"], np.float32),
                    hit_detid=detid, hit_cpcm=cpcm,
                    hit_mc=np.asarray(ev["mc_info"][:, 0] if len(ev["mc_info"]) == nh else
                                      np.full(nh, -1), np.int32),
                    seed_par=np.ascontiguousarray(s["par"], np.float32),
                    seed_err=np.ascontiguousarray(s["err"], np.float32),
                    seed_chg=np.asarray(s["charge"], np.int32), seed_nhits=snh,
                    seed_hit_layer=shl, seed_hit_index=shi,
                    seed_mc=np.asarray(s["label"], np.int32), n_tracks=ns, seed=0,
                    n_signal_hits=0)
