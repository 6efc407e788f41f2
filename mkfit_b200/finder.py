"""Host mirror of the reference's finding interface (MkBuilder /
MkFinder clone engine) over the C ABI: configuration from the CMS-2017
geometry, event upload, run and export."""
import ctypes

import numpy as np

from . import capi
from .geometry import LAYER_FIELDS, cms2017

vp = ctypes.c_void_p


class MkfgFindConfig(ctypes.Structure):
    _fields_ = [("n_layers", ctypes.c_int32), ("layer_desc", vp), ("n_regions", ctypes.c_int32),
                ("max_plan", ctypes.c_int32), ("plans", vp), ("plan_len", vp), ("pickup", vp),
                ("max_cands_per_seed", ctypes.c_int32), ("max_holes_per_cand", ctypes.c_int32),
                ("max_consec_holes", ctypes.c_int32), ("chi2_cut_min", ctypes.c_float),
                ("chi2_cut_overlap", ctypes.c_float), ("pt_cut_overlap", ctypes.c_float),
                ("inter_layer_pflags", ctypes.c_uint32), ("intra_layer_pflags", ctypes.c_uint32),
                ("requires_prop_to_hit", ctypes.c_int32), ("sort_seed_hits", ctypes.c_int32)]


class MkfgSelectConfig(ctypes.Structure):
    _fields_ = [(k, ctypes.c_float) for k in (
        "frac_shared_hits", "drth_central", "drth_obarrel", "drth_forward", "max_d_invpt",
        "max_d_phi", "max_d_cottheta", "max_cottheta_obarrel", "max_cottheta_forward")] + [
        ("mode", ctypes.c_int32), ("algorithm", ctypes.c_int32)] + [
        (k, ctypes.c_float) for k in ("ep_max_d_pt", "ep_max_d_phi", "ep_max_d_eta", "ep_max_dr",
                                      "ep_min_frac_hits_shared")] + [
        ("ep_use_hits", ctypes.c_int32)]


class MkfgSearchParams(ctypes.Structure):
    _fields_ = [("max_cands_per_seed", ctypes.c_int32), ("max_holes_per_cand", ctypes.c_int32),
                ("max_consec_holes", ctypes.c_int32), ("chi2_cut_min", ctypes.c_float),
                ("chi2_cut_overlap", ctypes.c_float), ("pt_cut_overlap", ctypes.c_float)]


class MkfgQFilterConfig(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("min_hits", ctypes.c_int32),
                ("beam_spot_x", ctypes.c_float), ("beam_spot_y", ctypes.c_float)]


class MkfgGraphTuning(ctypes.Structure):
    _fields_ = [("grid_mult", ctypes.c_int32 * 4), ("stage_bins", ctypes.c_int32),
                ("ms_before", ctypes.c_float), ("ms_after", ctypes.c_float)]


class MkfgCandCounts(ctypes.Structure):
    _fields_ = [(k, vp) for k in ("nfound", "nover", "ninside", "ntail", "chi2")]


class MkfgCeRecords(ctypes.Structure):
    _fields_ = [(k, vp) for k in ("n", "hit", "module", "chi2", "score")]


# Input and output fields of mkfg_find_clone_seeds with their dtypes and
# per-slot widths (0 = one per seed).
CLONE_IN_FIELDS = [("n_cands", np.int32, 0), ("par", np.float32, 6), ("err", np.float32, 21),
                   ("chg", np.int32, 1), ("chi2", np.float32, 1), ("score", np.float32, 1),
                   ("nfound", np.int32, 1), ("nmiss", np.int32, 1), ("nover", np.int32, 1),
                   ("ninside", np.int32, 1), ("ntail", np.int32, 1), ("held_back", np.int32, 1),
                   ("n_rec", np.int32, 1), ("rec_hit", np.int32, 17), ("rec_module", np.int32, 17),
                   ("rec_chi2", np.float32, 17), ("rec_score", np.float32, 17),
                   ("bshort_valid", np.int32, 0), ("bshort_score", np.float32, 0)]
CLONE_OUT_FIELDS = [("n_cands", np.int32, 0), ("par", np.float32, 6), ("err", np.float32, 21),
                    ("chg", np.int32, 1), ("chi2", np.float32, 1), ("score", np.float32, 1),
                    ("nfound", np.int32, 1), ("nmiss", np.int32, 1), ("nover", np.int32, 1),
                    ("ninside", np.int32, 1), ("ntail", np.int32, 1), ("parent", np.int32, 1),
                    ("hit", np.int32, 1), ("overlap_hit", np.int32, 1),
                    ("update_hit", np.int32, 1), ("bshort_valid", np.int32, 0),
                    ("bshort_score", np.float32, 0), ("bshort_nfound", np.int32, 0),
                    ("bshort_chi2", np.float32, 0)]


class MkfgCloneIn(ctypes.Structure):
    _fields_ = [("n_seeds", ctypes.c_int32)] + [(k, vp) for k, _, _ in CLONE_IN_FIELDS]


class MkfgCloneOut(ctypes.Structure):
    _fields_ = [(k, vp) for k, _, _ in CLONE_OUT_FIELDS]


# Records per candidate (MKFG_REC_PER_CAND) and the hit code of a
# held-back copy (MKFG_NO_HIT).
REC_PER_CAND = 17
NO_HIT = -100000


def clone_arrays(fields, n_seeds, given=None):
    """Arrays of mkfg_clone_in / mkfg_clone_out for n_seeds seeds: the
    given ones made contiguous with the field's dtype, the rest zero.
    Per-slot arrays are [width][8 n_seeds] for par / err, [8 n_seeds][17]
    for records, [8 n_seeds] otherwise."""
    out = {}
    for k, dt, w in fields:
        shape = (n_seeds,) if w == 0 else ((w, 8 * n_seeds) if w in (6, 21) else
                                           ((8 * n_seeds, w) if w == 17 else (8 * n_seeds,)))
        if given is not None and k in given:
            a = np.ascontiguousarray(given[k], dt)
            if a.shape != shape:
                raise ValueError(f"{k}: shape {a.shape}, expected {shape}")
        else:
            a = np.zeros(shape, dt)
        out[k] = a
    return out


# Duplicate removal modes of mkfg_find_select (MKFG_DUP_*).
DUP_PIXELSEED, DUP_SHAREDHITS, DUP_ETA_PHI, DUP_NONE = range(4)
# Quality filters of mkfg_find_filter (MKFG_QF_*), StdSeq::qfilter_*.
(QF_NAN_N_SILLY, QF_N_HITS, QF_N_HITS_PIXSEED, QF_N_LAYERS, QF_N_LAYERS_PIXELLESS,
 QF_PIXELLESS_FWD, QF_PIXELLESS_BKWD) = range(7)

# Iteration 0 of CMS-2017: set_dupl_params(0.24, 0.002, 0.004, 0.008)
# (Geoms/CMS-2017.cc:750), the window constants of Config.cc:93-97 and the
# find_duplicates constants of Config.cc:86-91.
SELECT_ITER0 = dict(frac_shared_hits=0.24, drth_central=0.002, drth_obarrel=0.004,
                    drth_forward=0.008, max_d_invpt=1.8, max_d_phi=0.37, max_d_cottheta=0.37,
                    max_cottheta_obarrel=1.99, max_cottheta_forward=6.05, mode=DUP_PIXELSEED,
                    algorithm=4, ep_max_d_pt=0.5, ep_max_d_phi=0.25, ep_max_d_eta=0.05,
                    ep_max_dr=0.0025, ep_min_frac_hits_shared=0.75, ep_use_hits=1)


def _iteration_selection():
    """run_OneIteration's filters and duplicate removal for the ten CMS-2017
    iterations (Geoms/CMS-2017.cc:740-845; mkFit/buildtestMPlex.cc:676-731):
    (TrackBase algorithm, filter after finding, filter after the backward
    fit, min hits, duplicate mode, frac_shared_hits, (drth central,
    obarrel, forward)). None = no filter."""
    rows = {
        # index: (algorithm, requires_quality_filter, dupclean_tight, minHitsQF, frac, drth)
        0: (4, False, True, 4, 0.24, (0.002, 0.004, 0.008)),
        1: (22, False, True, 4, 0.24, (0.03, 0.05, 0.08)),
        2: (23, False, True, 4, 0.5, (0.01, 0.03, 0.05)),
        3: (5, False, True, 4, 0.33, (0.018, 0.05, 0.018)),
        4: (24, False, True, 4, 0.24, (0.018, 0.05, 0.05)),
        5: (7, True, True, 4, 0.24, (0.01, 0.01, 0.1)),
        6: (8, False, True, 4, 0.2, (0.05, 0.05, 0.05)),
        7: (9, True, False, 3, 0.14, (0.001, 0.001, 0.001)),
        8: (10, True, False, 4, 0.25, (0.001, 0.001, 0.001)),
        9: (6, True, True, 4, 0.5, (0.03, 0.05, 0.05)),
    }
    out = {}
    for it, (algo, qf, tight, min_hits, frac, drth) in rows.items():
        pre = post = None
        if qf and algo != 7:
            pre = {6: QF_N_HITS_PIXSEED, 9: QF_PIXELLESS_FWD}.get(algo, QF_N_HITS)
        if qf and algo in (7, 9):
            post = QF_N_LAYERS if algo == 7 else QF_PIXELLESS_BKWD
        if qf and not tight:
            mode = DUP_SHAREDHITS
        elif tight:
            mode = DUP_PIXELSEED
        else:
            mode = DUP_ETA_PHI
        out[it] = dict(algorithm=algo, pre=pre, post=post, sort_seed_hits=qf and not tight,
                       min_hits=3 if algo == 6 else min_hits, mode=mode, frac_shared_hits=frac,
                       drth=drth)
    return out


ITERATION_SELECTION = _iteration_selection()


class MkfgEvent(ctypes.Structure):
    _fields_ = [("n_layers", ctypes.c_int32), ("layer_begin", vp), ("pos", vp), ("err", vp),
                ("detid", vp), ("cpcm", vp), ("n_seeds", ctypes.c_int32), ("seed_par", vp),
                ("seed_err", vp), ("seed_chg", vp), ("seed_nhits", vp), ("seed_hit_layer", vp),
                ("seed_hit_index", vp), ("seed_hit_stride", ctypes.c_int32), ("hit_mask", vp)]


class MkfgFindOut(ctypes.Structure):
    _fields_ = [(k, vp) for k in ("n_cands", "region", "par", "err", "chg", "chi2", "score",
                                  "nfound", "ntot", "noverlap", "ninside", "ntail", "hit_idx",
                                  "hit_lyr")]


def _bind(lib):
    if getattr(lib, "_finder_bound", False):
        return
    lib.mkfg_finder_setup.argtypes = [vp, ctypes.POINTER(MkfgFindConfig)]
    lib.mkfg_find_upload.argtypes = [vp, ctypes.POINTER(MkfgEvent)]
    lib.mkfg_find_upload_batch.argtypes = [vp, ctypes.POINTER(MkfgEvent), ctypes.c_int32]
    lib.mkfg_find_run.argtypes = [vp]
    lib.mkfg_find_run_graph.argtypes = [vp]
    lib.mkfg_find_backward_fit.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_int32]
    lib.mkfg_find_hit_index.argtypes = [vp, ctypes.c_int32, vp, vp]
    lib.mkfg_find_run_timed.argtypes = [vp, vp]
    lib.mkfg_find_backward_search.argtypes = [vp, vp]
    lib.mkfg_find_backward_search_with.argtypes = [vp, vp, ctypes.POINTER(MkfgSearchParams)]
    lib.mkfg_find_step_profile.argtypes = [vp, vp, vp]
    lib.mkfg_find_select.argtypes = [vp, ctypes.POINTER(MkfgSelectConfig), ctypes.c_int32, vp]
    lib.mkfg_find_filter.argtypes = [vp, ctypes.POINTER(MkfgQFilterConfig), ctypes.c_int32,
                                     ctypes.c_int32, vp]
    lib.mkfg_find_select_hit_indices.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                 vp, vp, vp, vp, vp]
    lib.mkfg_find_candidates_clone_engine.argtypes = [
        vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp, vp, vp,
        ctypes.POINTER(MkfgCandCounts), vp, vp, vp, vp, ctypes.POINTER(MkfgCeRecords)]
    lib.mkfg_find_update_with_last_hit.argtypes = [vp, ctypes.c_int32, ctypes.c_int32,
                                                   ctypes.c_int32, vp, vp, vp, vp, vp, vp, vp]
    lib.mkfg_find_clone_seeds.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(MkfgCloneIn),
                                          ctypes.POINTER(MkfgCloneOut)]
    lib.mkfg_find_run_fused.argtypes = [vp, ctypes.c_int32]
    lib.mkfg_find_autotune.argtypes = [vp, ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_float)]
    i64p = ctypes.POINTER(ctypes.c_int64)
    lib.mkfg_find_work.argtypes = [vp, i64p, i64p, i64p, ctypes.POINTER(ctypes.c_int32)]
    lib.mkfg_find_work_detail.argtypes = [vp, i64p, i64p]
    lib.mkfg_find_work_clone.argtypes = [vp, i64p, i64p]
    lib.mkfg_find_set_arena_capacity.argtypes = [vp, ctypes.c_int32]
    lib.mkfg_find_set_seed_import.argtypes = [vp, ctypes.c_int32]
    lib.mkfg_find_set_bin_staging.argtypes = [vp, ctypes.c_int32]
    lib.mkfg_find_autotune_graph.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(MkfgGraphTuning)]
    lib.mkfg_find_set_graph_tuning.argtypes = [vp, ctypes.POINTER(MkfgGraphTuning)]
    lib.mkfg_find_get_graph_tuning.argtypes = [vp, ctypes.POINTER(MkfgGraphTuning)]
    lib.mkfg_find_download.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(MkfgFindOut)]
    lib.mkfg_find_download_best.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(MkfgFindOut)]
    lib.mkfg_find_event.argtypes = [vp, ctypes.POINTER(MkfgEvent), ctypes.POINTER(MkfgFindOut)]
    lib.mkfg_prepare_event_host.argtypes = [ctypes.POINTER(MkfgFindConfig),
                                            ctypes.POINTER(MkfgEvent), vp,
                                            ctypes.POINTER(ctypes.c_int32), vp, vp, vp]
    lib._finder_bound = True


class FindConfig:
    """CMS-2017 finding configuration of one iteration (default
    initialStep) with the workload's overrides: maxCandsPerSeed,
    chi2Cut_min (None: the iteration's own) and (zero_c2) a flat chi2
    cut."""

    def __init__(self, geom=None, max_cands=6, chi2_cut=30.0, zero_c2=True, iteration=0):
        g = geom or cms2017(iteration)
        self.geom = g
        desc = g.layer_desc.copy()
        if zero_c2:
            for k in ("c_c2_0", "c_c2_1", "c_c2_2"):
                desc[:, LAYER_FIELDS.index(k)] = 0.0
        self.layer_desc = np.ascontiguousarray(desc, np.float32)
        self.plans = np.ascontiguousarray(g.plans, np.int32)
        self.plan_len = np.ascontiguousarray(g.plan_len, np.int32)
        self.pickup = np.ascontiguousarray(g.pickup, np.int32)
        ip = g.iter_params
        if max_cands is None:
            max_cands = int(ip[0])
        if chi2_cut is None:
            chi2_cut = float(ip[3])
        self.chi2_cut = float(chi2_cut)
        self.max_cands = int(max_cands)
        c = MkfgFindConfig()
        c.n_layers = g.n_layers
        c.layer_desc = self.layer_desc.ctypes.data
        c.n_regions = self.plans.shape[0]
        c.max_plan = self.plans.shape[1]
        c.plans = self.plans.ctypes.data
        c.plan_len = self.plan_len.ctypes.data
        c.pickup = self.pickup.ctypes.data
        c.max_cands_per_seed = self.max_cands
        c.max_holes_per_cand = int(ip[1])
        c.max_consec_holes = int(ip[2])
        c.chi2_cut_min = float(chi2_cut)
        c.chi2_cut_overlap = float(ip[4])
        c.pt_cut_overlap = float(ip[5])
        c.inter_layer_pflags = int(g.flags[1])
        c.intra_layer_pflags = int(g.flags[2])
        c.requires_prop_to_hit = int(g.flags[0])
        # m_requires_seed_hit_sorting (set_qf_flags: pixelLessStep, tobTecStep).
        c.sort_seed_hits = int(ITERATION_SELECTION[g.iteration]["sort_seed_hits"])
        self.c = c

    @property
    def max_steps(self):
        """Layer-plan steps of a run: the longest plan after its pickup layer."""
        return int(np.max(self.plan_len - self.pickup - 1))


def event_struct(ev):
    """ctypes view of a synth.CmsEvent (keeps references to the arrays)."""
    keep = {}

    def p(name, arr, dt):
        a = np.ascontiguousarray(arr, dt)
        keep[name] = a
        return a.ctypes.data

    e = MkfgEvent()
    e.n_layers = ev.n_layers
    e.layer_begin = p("lb", ev.layer_begin, np.int32)
    e.pos = p("pos", ev.hit_pos, np.float32)
    e.err = p("err", ev.hit_err, np.float32)
    e.detid = p("det", ev.hit_detid, np.int32)
    e.cpcm = p("cpcm", ev.hit_cpcm, np.int32)
    e.n_seeds = ev.n_seeds
    e.seed_par = p("spar", ev.seed_par, np.float32)
    e.seed_err = p("serr", ev.seed_err, np.float32)
    e.seed_chg = p("schg", ev.seed_chg, np.int32)
    e.seed_nhits = p("snh", ev.seed_nhits, np.int32)
    e.seed_hit_layer = p("shl", ev.seed_hit_layer, np.int32)
    e.seed_hit_index = p("shi", ev.seed_hit_index, np.int32)
    shl = np.asarray(ev.seed_hit_layer)
    e.seed_hit_stride = int(shl.shape[1]) if shl.ndim == 2 else 4
    mask = getattr(ev, "hit_mask", None)
    e.hit_mask = None if mask is None else p("mask", mask, np.uint8)
    e._keep = keep
    return e


def output_arrays(n_seeds, m):
    no = n_seeds * m
    return dict(n_cands=np.zeros(n_seeds, np.int32), region=np.zeros(n_seeds, np.int32),
                par=np.zeros((no, 6), np.float32), err=np.zeros((no, 21), np.float32),
                chg=np.zeros(no, np.int32), chi2=np.zeros(no, np.float32),
                score=np.zeros(no, np.float32), nfound=np.zeros(no, np.int32),
                ntot=np.zeros(no, np.int32), noverlap=np.zeros(no, np.int32),
                ninside=np.zeros(no, np.int32), ntail=np.zeros(no, np.int32),
                hit_idx=np.zeros((no, 64), np.int32), hit_lyr=np.zeros((no, 64), np.int32))


def out_struct(o):
    s = MkfgFindOut()
    for k, _ in MkfgFindOut._fields_:
        setattr(s, k, o[k].ctypes.data if o.get(k) is not None else None)
    return s


class Finder:
    """Clone-engine finding on one context (plain form)."""

    def __init__(self, ctx, cfg=None):
        self.ctx = ctx
        self.lib = ctx.lib
        _bind(self.lib)
        self.cfg = cfg or FindConfig()
        g = self.cfg.geom
        ctx.set_material(g.rl, g.xi)
        capi.check(self.lib.mkfg_finder_setup(ctx.handle, ctypes.byref(self.cfg.c)))

    def upload(self, ev):
        self._ev = event_struct(ev)
        capi.check(self.lib.mkfg_find_upload(self.ctx.handle, ctypes.byref(self._ev)))

    def upload_batch(self, events):
        arr = (MkfgEvent * len(events))()
        self._evs = [event_struct(ev) for ev in events]
        for i, e in enumerate(self._evs):
            arr[i] = e
        self._arr = arr
        capi.check(self.lib.mkfg_find_upload_batch(self.ctx.handle, arr, len(events)))
        return sum(ev.n_seeds for ev in events)

    def run(self):
        capi.check(self.lib.mkfg_find_run(self.ctx.handle))

    def run_graph(self):
        capi.check(self.lib.mkfg_find_run_graph(self.ctx.handle))

    def backward_fit(self, group_width=8):
        """Backward fit of every seed's best candidate (MkBuilder::BackwardFit)
        with the geometry's bkfit_last and backward-fit propagation flags."""
        g = self.cfg.geom
        self._bk_last = np.ascontiguousarray(g.bkfit_last, np.int32)
        capi.check(self.lib.mkfg_find_backward_fit(self.ctx.handle, self._bk_last.ctypes.data,
                                                   int(g.flags[3]), int(group_width)))

    def backward_search(self):
        """Backward search of every seed's backward-fitted best candidate
        through the iteration's backward plans with its backward-search
        parameters (m_backward_params; maxCandsPerSeed and the chi2 cut
        follow this configuration's overrides, as the reference driver's
        do) — mkfg_find_backward_search_with."""
        g = self.cfg.geom
        if int(g.bk_flags[0]):
            raise NotImplementedError("backward search that drops the seed hits")
        bk = g.bk_iter_params
        self._bks_params = MkfgSearchParams(self.cfg.max_cands, int(bk[1]), int(bk[2]),
                                            self.cfg.chi2_cut, float(bk[4]), float(bk[5]))
        self._bks_pickup = np.ascontiguousarray(g.bksearch_pickup, np.int32)
        capi.check(self.lib.mkfg_find_backward_search_with(
            self.ctx.handle, self._bks_pickup.ctypes.data, ctypes.byref(self._bks_params)))

    KERNELS = ("reset", "activate", "propagate", "chi2", "clone", "update", "merge")

    def run_timed(self):
        """Plain run with per-kernel CUDA-event timing: {kernel: ms}."""
        ms = np.zeros(len(self.KERNELS), np.float32)
        capi.check(self.lib.mkfg_find_run_timed(self.ctx.handle, ms.ctypes.data))
        return dict(zip(self.KERNELS, ms.tolist()))

    STEP_COUNTS = ("act_barrel", "act_endcap", "pairs_barrel", "pairs_endcap", "upd_barrel",
                   "upd_endcap", "finding_seeds")

    def step_profile(self, timed=True):
        """Per layer-plan step: {kernel: ms[max_steps]} of the last run_timed
        (when timed) and {counter: int[max_steps]} of the last run."""
        ns = self.cfg.max_steps
        ms = np.zeros((ns, 5), np.float32)
        cnt = np.zeros((ns, len(self.STEP_COUNTS)), np.int32)
        capi.check(self.lib.mkfg_find_step_profile(self.ctx.handle,
                                                   ms.ctypes.data if timed else None,
                                                   cnt.ctypes.data))
        out = {k: cnt[:, i] for i, k in enumerate(self.STEP_COUNTS)}
        if timed:
            out.update({k: ms[:, i] for i, k in enumerate(self.KERNELS[1:6])})
        return out

    def run_fused(self, seeds_per_block=0):
        """One launch for all layer steps; seeds_per_block 0 = tuned value."""
        capi.check(self.lib.mkfg_find_run_fused(self.ctx.handle, seeds_per_block))

    def autotune(self):
        """Picks the fastest seeds_per_block on the uploaded events;
        returns (seeds_per_block, ms per run)."""
        w, ms = ctypes.c_int32(), ctypes.c_float()
        capi.check(self.lib.mkfg_find_autotune(self.ctx.handle, ctypes.byref(w), ctypes.byref(ms)))
        return w.value, ms.value

    def work(self):
        a, p, u = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        st = ctypes.c_int32()
        capi.check(self.lib.mkfg_find_work(self.ctx.handle, ctypes.byref(a), ctypes.byref(p),
                                           ctypes.byref(u), ctypes.byref(st)))
        e, c = ctypes.c_int64(), ctypes.c_int64()
        capi.check(self.lib.mkfg_find_work_detail(self.ctx.handle, ctypes.byref(e), ctypes.byref(c)))
        r, n = ctypes.c_int64(), ctypes.c_int64()
        capi.check(self.lib.mkfg_find_work_clone(self.ctx.handle, ctypes.byref(r), ctypes.byref(n)))
        return dict(active_cands=a.value, hit_pairs=p.value, updates=u.value, steps=st.value,
                    chi2_evals=e.value, seed_steps=c.value, records=r.value, new_cands=n.value)

    def select(self, n_seeds, **params):
        """Output selection of run_OneIteration (NaN/silly filter + duplicate
        removal, `mode` one of DUP_*) on the current results: keep[n_seeds]
        by input seed."""
        c = MkfgSelectConfig(**{**SELECT_ITER0, **params})
        keep = np.zeros(n_seeds, np.int32)
        capi.check(self.lib.mkfg_find_select(self.ctx.handle, ctypes.byref(c), n_seeds,
                                             keep.ctypes.data))
        return keep

    def filter(self, n_seeds, kind, min_hits=4, beam_spot=(0.0, 0.0), remove=False):
        """A quality filter (QF_*) on every seed's best candidate, as
        MkBuilder::filter_comb_cands applies it: pass[n_seeds] by input seed
        (1 pass, 0 fail, -1 no candidate); with remove, failing seeds lose
        their comb candidate until the next run."""
        c = MkfgQFilterConfig(kind, min_hits, beam_spot[0], beam_spot[1])
        out = np.zeros(n_seeds, np.int32)
        capi.check(self.lib.mkfg_find_filter(self.ctx.handle, ctypes.byref(c), n_seeds,
                                             1 if remove else 0, out.ctypes.data))
        return out

    def run_iteration_selection(self, n_seeds, iteration=0, beam_spot=(0.0, 0.0), backward_fit=True,
                                remove_duplicates=True):
        """The steps of run_OneIteration after the clone engine for CMS-2017
        iteration `iteration` (mkFit/buildtestMPlex.cc:676-731): its
        quality filter with removal, the backward fit, the filter after it,
        then the NaN/silly filter and duplicate removal. Returns keep by
        input seed. The backward search is not part of it (backward_search
        runs it on its own)."""
        sel = ITERATION_SELECTION[iteration]
        if sel["pre"] is not None:
            self.filter(n_seeds, sel["pre"], sel["min_hits"], beam_spot, remove=True)
        if backward_fit:
            self.backward_fit()
            if sel["post"] is not None:
                self.filter(n_seeds, sel["post"], sel["min_hits"], beam_spot, remove=True)
        d = sel["drth"]
        return self.select(n_seeds, mode=sel["mode"] if remove_duplicates else DUP_NONE,
                           algorithm=sel["algorithm"], frac_shared_hits=sel["frac_shared_hits"],
                           drth_central=d[0], drth_obarrel=d[1], drth_forward=d[2])

    def select_hit_indices(self, event, layer, par, err):
        """MkFinder::SelectHitIndices on states par [6][n], err [21][n]
        propagated to `layer` of uploaded event `event`: (xhit_size [n],
        xhit_idx [n][16], wsr [n])."""
        par = np.ascontiguousarray(par, np.float32)
        err = np.ascontiguousarray(err, np.float32)
        n = par.shape[1]
        size = np.zeros(n, np.int32)
        idx = np.zeros((n, 16), np.int32)
        wsr = np.zeros(n, np.int32)
        capi.check(self.lib.mkfg_find_select_hit_indices(
            self.ctx.handle, int(event), int(layer), n, par.ctypes.data, err.ctypes.data,
            size.ctypes.data, idx.ctypes.data, wsr.ctypes.data))
        return size, idx, wsr

    def candidates_clone_engine(self, event, layer, par, err, chg, counts, xhit_size, xhit_idx,
                                wsr, seed_hot_layers=None):
        """MkFinder::FindCandidatesCloneEngine on states par [6][n], err
        [21][n], chg [n] propagated to `layer` of uploaded event `event`, with
        counters `counts` (dict of nfound, nover, ninside, ntail, chi2 [n])
        and the SelectHitIndices lists: dict of n [n] and hit, module, chi2,
        score [n][17] (the records in hand-over order)."""
        c = np.ascontiguousarray
        par, err = c(par, np.float32), c(err, np.float32)
        n = par.shape[1]
        cnt = {k: c(counts[k], np.float32 if k == "chi2" else np.int32)
               for k in ("nfound", "nover", "ninside", "ntail", "chi2")}
        cc = MkfgCandCounts(**{k: v.ctypes.data for k, v in cnt.items()})
        out = dict(n=np.zeros(n, np.int32), hit=np.zeros((n, 17), np.int32),
                   module=np.zeros((n, 17), np.int32), chi2=np.zeros((n, 17), np.float32),
                   score=np.zeros((n, 17), np.float32))
        rec = MkfgCeRecords(**{k: v.ctypes.data for k, v in out.items()})
        hl = None if seed_hot_layers is None else c(seed_hot_layers, np.int32)
        xs, xi, w = c(xhit_size, np.int32), c(xhit_idx, np.int32), c(wsr, np.int32)
        ch = c(chg, np.int32)
        capi.check(self.lib.mkfg_find_candidates_clone_engine(
            self.ctx.handle, int(event), int(layer), n, par.ctypes.data, err.ctypes.data,
            ch.ctypes.data, ctypes.byref(cc), hl.ctypes.data if hl is not None else None,
            xs.ctypes.data, xi.ctypes.data, w.ctypes.data, ctypes.byref(rec)))
        return out

    def update_with_last_hit(self, event, layer, par, err, chg, hit_idx):
        """MkFinder::UpdateWithLastHit + CopyOutParErr: states par [6][n],
        err [21][n], chg [n] updated with hit hit_idx[i] of `layer` of
        uploaded event `event`. Returns (par, err, chg)."""
        c = np.ascontiguousarray
        par, err = c(par, np.float32).copy(), c(err, np.float32).copy()
        chg, hit = c(chg, np.int32).copy(), c(hit_idx, np.int32)
        n = par.shape[1]
        capi.check(self.lib.mkfg_find_update_with_last_hit(
            self.ctx.handle, int(event), int(layer), n, par.ctypes.data, err.ctypes.data,
            chg.ctypes.data, hit.ctypes.data, par.ctypes.data, err.ctypes.data, chg.ctypes.data))
        return par, err, chg

    def clone_seeds(self, layer, inp):
        """CandCloner::ProcessSeedRange for the seeds of `inp` (the
        mkfg_clone_in fields, see clone_arrays) at `layer`. Returns the
        mkfg_clone_out fields as a dict."""
        n_seeds = len(inp["n_cands"])
        a = clone_arrays(CLONE_IN_FIELDS, n_seeds, inp)
        o = clone_arrays(CLONE_OUT_FIELDS, n_seeds)
        ci = MkfgCloneIn(n_seeds=n_seeds, **{k: v.ctypes.data for k, v in a.items()})
        co = MkfgCloneOut(**{k: v.ctypes.data for k, v in o.items()})
        capi.check(self.lib.mkfg_find_clone_seeds(self.ctx.handle, int(layer), ctypes.byref(ci),
                                                  ctypes.byref(co)))
        return o

    def autotune_graph(self, reps=2):
        """Tunes the graph form's launch configuration on the uploaded
        batch (mkfg_find_autotune_graph); returns it as a dict with the
        step time before and after."""
        t = MkfgGraphTuning()
        capi.check(self.lib.mkfg_find_autotune_graph(self.ctx.handle, int(reps), ctypes.byref(t)))
        return dict(grid_mult=list(t.grid_mult), stage_bins=int(t.stage_bins),
                    ms_before=float(t.ms_before), ms_after=float(t.ms_after))

    def graph_tuning(self):
        t = MkfgGraphTuning()
        capi.check(self.lib.mkfg_find_get_graph_tuning(self.ctx.handle, ctypes.byref(t)))
        return dict(grid_mult=list(t.grid_mult), stage_bins=int(t.stage_bins))

    def set_graph_tuning(self, tuning):
        t = MkfgGraphTuning()
        t.grid_mult[:] = [int(x) for x in tuning["grid_mult"]]
        t.stage_bins = int(tuning["stage_bins"])
        capi.check(self.lib.mkfg_find_set_graph_tuning(self.ctx.handle, ctypes.byref(t)))

    def set_bin_staging(self, on):
        """Bin tables staged in shared memory by the propagation kernel of
        the following runs (mkfg_find_set_bin_staging)."""
        capi.check(self.lib.mkfg_find_set_bin_staging(self.ctx.handle, int(bool(on))))

    def set_seed_import(self, on_host):
        """Seed import of the following uploads on the host (True) or on the
        device (False, the default); see mkfg_find_set_seed_import."""
        capi.check(self.lib.mkfg_find_set_seed_import(self.ctx.handle, int(bool(on_host))))

    def hit_index(self, event, n_bins, n_hits):
        """The device-built hit index of uploaded event `event`:
        (bins[n_bins], srank[n_hits])."""
        bins = np.zeros(n_bins, np.uint32)
        srank = np.zeros(n_hits, np.int32)
        capi.check(self.lib.mkfg_find_hit_index(self.ctx.handle, int(event), bins.ctypes.data,
                                                srank.ctypes.data))
        return bins, srank

    def download_best(self, n_seeds, out=None):
        """Best candidate per seed only (mkfg_find_download_best). `out`: the
        arrays of an earlier call with the same seed count, reused."""
        o = out if out is not None and len(out["n_cands"]) == n_seeds else output_arrays(n_seeds, 1)
        capi.check(self.lib.mkfg_find_download_best(self.ctx.handle, n_seeds,
                                                    ctypes.byref(out_struct(o))))
        return o

    def download(self, n_seeds):
        o = output_arrays(n_seeds, self.cfg.max_cands)
        capi.check(self.lib.mkfg_find_download(self.ctx.handle, n_seeds,
                                               ctypes.byref(out_struct(o))))
        return o

    def find_event(self, ev):
        e = event_struct(ev)
        o = output_arrays(ev.n_seeds, self.cfg.max_cands)
        capi.check(self.lib.mkfg_find_event(self.ctx.handle, ctypes.byref(e),
                                            ctypes.byref(out_struct(o))))
        return o


def prepare_event_host(ev, cfg=None):
    """Host-side hit index + seed order of the library (no GPU needed)."""
    lib = capi.load()
    _bind(lib)
    cfg = cfg or FindConfig()
    e = event_struct(ev)
    nb = ctypes.c_int32(0)
    capi.check(lib.mkfg_prepare_event_host(ctypes.byref(cfg.c), ctypes.byref(e), None,
                                           ctypes.byref(nb), None, None, None))
    bins = np.zeros(nb.value, np.uint32)
    srank = np.zeros(ev.n_hits, np.int32)
    order = np.zeros(ev.n_seeds, np.int32)
    region = np.zeros(ev.n_seeds, np.int32)
    capi.check(lib.mkfg_prepare_event_host(ctypes.byref(cfg.c), ctypes.byref(e),
                                           bins.ctypes.data, ctypes.byref(nb), srank.ctypes.data,
                                           order.ctypes.data, region.ctypes.data))
    return dict(bins=bins, srank=srank, seed_order=order, seed_region=region)
