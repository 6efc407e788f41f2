"""Seed cleaning of an iteration's seeds on the GPU (the host side of
mkfg_clean_seeds): StdSeq::clean_cms_seedtracks_iter
(mkFit/MkStdSeqs.cc:115-311), as MkBuilder's run_OneIteration calls it
before finding (mkFit/buildtestMPlex.cc:660-665)."""
import ctypes

import numpy as np

from . import capi

MAX_HITS = 16  # output row width: a merge stops at 15 hits


class MkfgSeedCleanParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_float) for k in (
        "pt_thr", "dzmax_bh", "drmax_bh", "dzmax_bl", "drmax_bl", "dzmax_eh", "drmax_eh",
        "dzmax_el", "drmax_el", "beam_x", "beam_y")]


# IterationParams defaults (mkFit/IterationConfig.h:107-116): what the
# CMS-2017 initialStep uses (it sets no cleaning parameters of its own).
SEED_CLEAN_ITER0 = dict(pt_thr=2.0, dzmax_bh=0.005, drmax_bh=0.010, dzmax_bl=0.005, drmax_bl=0.010,
                        dzmax_eh=0.020, drmax_eh=0.020, dzmax_el=0.030, drmax_el=0.030)
PARAM_ORDER = ("pt_thr", "dzmax_bh", "drmax_bh", "dzmax_bl", "drmax_bl", "dzmax_eh", "drmax_eh",
               "dzmax_el", "drmax_el")


def _bind(lib):
    if getattr(lib, "_seed_clean_bound", False):
        return lib
    vp = ctypes.c_void_p
    lib.mkfg_clean_seeds.argtypes = [vp, ctypes.POINTER(MkfgSeedCleanParams), ctypes.c_int32,
                                     vp, vp, vp, vp, vp, vp, ctypes.c_int32, ctypes.c_int32,
                                     vp, vp, vp, vp]
    lib._seed_clean_bound = True
    return lib


def clean_seeds(ctx, event_seed_begin, par, chg, nhits, hit_layer, hit_index, beam=(0.0, 0.0),
                **params):
    """Cleans the seeds of a batch of events. par [6][n] float32, chg [n],
    nhits [n], hit_layer / hit_index [n][k]; event e's seeds at
    [event_seed_begin[e], event_seed_begin[e+1]). Returns (keep [n],
    nhits [n], hit_layer [n][16], hit_index [n][16])."""
    lib = _bind(capi.load())
    p = {**SEED_CLEAN_ITER0, **params}
    c = MkfgSeedCleanParams(**p, beam_x=float(beam[0]), beam_y=float(beam[1]))
    eb = np.ascontiguousarray(event_seed_begin, np.int32)
    n = int(eb[-1]) if len(eb) else 0
    par = np.ascontiguousarray(par, np.float32)
    chg = np.ascontiguousarray(chg, np.int32)
    nh = np.ascontiguousarray(nhits, np.int32)
    hl = np.ascontiguousarray(hit_layer, np.int32)
    hx = np.ascontiguousarray(hit_index, np.int32)
    if par.shape != (6, n) or chg.shape != (n,) or nh.shape != (n,) or hl.shape != hx.shape \
            or hl.shape[0] != n:
        raise ValueError("seed arrays do not match event_seed_begin")
    keep = np.zeros(n, np.int32)
    onh = np.zeros(n, np.int32)
    ohl = np.zeros((n, MAX_HITS), np.int32)
    ohx = np.zeros((n, MAX_HITS), np.int32)
    d = lambda a: a.ctypes.data  # noqa: E731
    capi.check(lib.mkfg_clean_seeds(ctx.handle, ctypes.byref(c), len(eb) - 1, d(eb), d(par),
                                    d(chg), d(nh), d(hl), d(hx), hl.shape[1], MAX_HITS,
                                    d(keep), d(onh), d(ohl), d(ohx)))
    return keep, onh, ohl, ohx


def cleaned_event(ev, seeds, result):
    """The finder's input after cleaning: event `ev`'s hits with the kept
    seeds of `seeds` (a dict par [6][n], err [21][n], chg, ...) in their
    order, with the merged hit lists of `result` (clean_seeds' output for
    this event) as [k][MAX_HITS] rows."""
    from .synth import CmsEvent
    keep, nh, hl, hx = result
    k = np.nonzero(keep == 1)[0]
    return CmsEvent(
        n_layers=ev.n_layers, layer_begin=ev.layer_begin, hit_pos=ev.hit_pos, hit_err=ev.hit_err,
        hit_detid=ev.hit_detid, hit_cpcm=ev.hit_cpcm, hit_mc=ev.hit_mc,
        seed_par=np.ascontiguousarray(seeds["par"][:, k], np.float32),
        seed_err=np.ascontiguousarray(seeds["err"][:, k], np.float32),
        seed_chg=np.ascontiguousarray(seeds["chg"][k], np.int32),
        seed_nhits=np.ascontiguousarray(nh[k], np.int32),
        seed_hit_layer=np.ascontiguousarray(hl[k], np.int32),
        seed_hit_index=np.ascontiguousarray(hx[k], np.int32),
        seed_mc=np.asarray(seeds.get("src", k), np.int32)[k] if "src" in seeds else k.astype(np.int32),
        n_tracks=ev.n_tracks, seed=ev.seed, n_signal_hits=ev.n_signal_hits)
