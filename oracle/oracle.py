"""ctypes front end of the oracle.

TEST INFRASTRUCTURE ONLY. Loads
  * oracle/_ref/libmkfit_ref_<flavour>.so -- the reference's own CPU code
    (trackreco/mkFit) compiled from its sources by oracle/Makefile, with the
    C driver oracle/ref_driver.cc;
  * oracle/_ref/librestate.so -- the FP64 restatement (oracle/restate.c).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def ref_lib_path(flavour="avx2"):
    return os.path.join(REF_DIR, f"libmkfit_ref_{flavour}.so")


def restate_lib_path():
    return os.path.join(REF_DIR, "librestate.so")


def shims_lib_path(flavour="avx2"):
    return os.path.join(REF_DIR, f"libmkfit_shims_{flavour}.so")


def have_shims(flavour="avx2"):
    return os.path.exists(shims_lib_path(flavour))


def have_ref(flavour="avx2"):
    return os.path.exists(ref_lib_path(flavour))


def have_restate():
    return os.path.exists(restate_lib_path())


def _opt(arr, dtype):
    if arr is None:
        return None
    return np.ascontiguousarray(arr, dtype=dtype)


class RefLib:
    """The reference CPU Matriplex path (compiled reference sources)."""

    def __init__(self, flavour="avx2"):
        self.lib = ctypes.CDLL(ref_lib_path(flavour))
        L = self.lib
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_get_threads.restype = ctypes.c_int
        L.ref_matriplex_width.restype = ctypes.c_int
        L.ref_fit.restype = ctypes.c_int
        L.ref_fit.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p, _i32p, _f32p, _f32p,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                              _f32p, _f32p, _i32p, ctypes.POINTER(ctypes.c_double)]

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def set_task_split(self, mode, seed=1):
        """How the TBB shim cuts parallel_for ranges into tasks: 0 near-equal
        pieces of at most the grain size (default), 1 recursive halving as
        TBB's simple_partitioner cuts them, 2 near-equal pieces of at most
        twice the grain, 3 the whole range (cuts TBB's auto_partitioner
        makes), 4 pieces of random sizes from half the grain to the grain
        (seeded by `seed`; TBB's proportional splits)."""
        self.lib.ref_set_task_split.argtypes = [ctypes.c_int]
        self.lib.ref_set_task_split_seed.argtypes = [ctypes.c_uint]
        self.lib.ref_set_task_split_seed(int(seed))
        self.lib.ref_set_task_split(int(mode))

    def threads(self):
        return self.lib.ref_get_threads()

    def width(self):
        return self.lib.ref_matriplex_width()

    def fit(self, par, err, chg, hit_pos, hit_err, rl_grid=None, xi_grid=None, pflags=2, repeat=1):
        """MkFitter fit (InputTracksForFit -> FitTracksWithInterSlurp ->
        OutputFittedTracks). Returns (par, err, chg, best_seconds)."""
        n = chg.shape[0]
        nl = hit_pos.shape[0]
        out_par = np.zeros((6, n), np.float32)
        out_err = np.zeros((21, n), np.float32)
        out_chg = np.zeros(n, np.int32)
        secs = ctypes.c_double(0)
        rl = _opt(rl_grid, np.float32)
        xi = _opt(xi_grid, np.float32)
        rc = self.lib.ref_fit(n, nl, np.ascontiguousarray(par, np.float32),
                              np.ascontiguousarray(err, np.float32),
                              np.ascontiguousarray(chg, np.int32),
                              np.ascontiguousarray(hit_pos, np.float32),
                              np.ascontiguousarray(hit_err, np.float32),
                              rl.ctypes.data if rl is not None else None,
                              xi.ctypes.data if xi is not None else None,
                              int(pflags), int(repeat), out_par, out_err, out_chg,
                              ctypes.byref(secs))
        if rc != 0:
            raise RuntimeError(f"ref_fit failed rc={rc}")
        return out_par, out_err, out_chg, secs.value

    def fit_steered(self, par, err, chg, hit_pos, hit_err, endcap_mask, rl_grid=None,
                    xi_grid=None, pflags=2):
        """MkFitter steered fit (InputTracksAndHits -> FitTracksSteered ->
        OutputFittedTracks): step l is an endcap step when bit l of
        endcap_mask is set. Returns (par, err, chg)."""
        L = self.lib
        L.ref_fit_steered.restype = ctypes.c_int
        L.ref_fit_steered.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _f32p, _f32p, _i32p,
                                      _f32p, _f32p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int, _f32p, _f32p, _i32p]
        n = chg.shape[0]
        nl = hit_pos.shape[0]
        barrel = np.array([0 if (int(endcap_mask) >> l) & 1 else 1 for l in range(nl)], np.int32)
        out_par = np.zeros((6, n), np.float32)
        out_err = np.zeros((21, n), np.float32)
        out_chg = np.zeros(n, np.int32)
        rl = _opt(rl_grid, np.float32)
        xi = _opt(xi_grid, np.float32)
        rc = L.ref_fit_steered(n, nl, barrel, np.ascontiguousarray(par, np.float32),
                               np.ascontiguousarray(err, np.float32),
                               np.ascontiguousarray(chg, np.int32),
                               np.ascontiguousarray(hit_pos, np.float32),
                               np.ascontiguousarray(hit_err, np.float32),
                               rl.ctypes.data if rl is not None else None,
                               xi.ctypes.data if xi is not None else None, int(pflags),
                               out_par, out_err, out_chg)
        if rc != 0:
            raise RuntimeError(f"ref_fit_steered failed rc={rc}")
        return out_par, out_err, out_chg


class RsMaterial(ctypes.Structure):
    _fields_ = [("rl", ctypes.c_void_p), ("xi", ctypes.c_void_p)]


class Restate:
    """FP64 restatement of the fit arithmetic (oracle/restate.c)."""

    def __init__(self):
        self.lib = ctypes.CDLL(restate_lib_path())
        L = self.lib
        L.rs_fit.restype = None
        L.rs_fit.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p, _i32p, _f32p, _f32p,
                             ctypes.c_ulonglong, ctypes.c_uint, ctypes.POINTER(RsMaterial),
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                             _f64p, _f64p, ctypes.c_void_p]

    def fit(self, par, err, chg, hit_pos, hit_err, rl_grid=None, xi_grid=None, pflags=2,
            endcap_mask=0, shift_rphi=None, shift_z=None, mat_scale=None, want_chi2=True):
        n = chg.shape[0]
        nl = hit_pos.shape[0]
        rl = _opt(rl_grid, np.float32)
        xi = _opt(xi_grid, np.float32)
        mat = RsMaterial(rl.ctypes.data if rl is not None else None,
                         xi.ctypes.data if xi is not None else None)
        out_par = np.zeros((6, n), np.float64)
        out_err = np.zeros((21, n), np.float64)
        chi2 = np.zeros(n, np.float64) if want_chi2 else None
        sr = _opt(shift_rphi, np.float64)
        sz = _opt(shift_z, np.float64)
        ms = _opt(mat_scale, np.float64)
        self.lib.rs_fit(n, nl, np.ascontiguousarray(par, np.float32),
                        np.ascontiguousarray(err, np.float32), np.ascontiguousarray(chg, np.int32),
                        np.ascontiguousarray(hit_pos, np.float32),
                        np.ascontiguousarray(hit_err, np.float32), int(endcap_mask), int(pflags),
                        ctypes.byref(mat),
                        sr.ctypes.data if sr is not None else None,
                        sz.ctypes.data if sz is not None else None,
                        ms.ctypes.data if ms is not None else None,
                        out_par, out_err, chi2.ctypes.data if chi2 is not None else None)
        return out_par, out_err, chi2


def restate_replay_cands(rs, ev, out, m, slots, geom=None):
    """FP64 replay (oracle/restate.c rs_replay_cands) of the finding
    candidates `slots` (indices seed * m + c into a finding result `out`,
    by input seed) of event `ev` from their seeds along their hit lists.
    Returns (par[n][6], err[n][21], chg[n], chi2[n]) in double."""
    from mkfit_b200.geometry import cms2017
    g = geom or cms2017()
    slots = np.asarray(slots, np.int64)
    n = len(slots)
    seeds = slots // m
    L = rs.lib
    L.rs_replay_cands.restype = None
    L.rs_replay_cands.argtypes = ([ctypes.c_int, _f32p, _f32p, _i32p, _i32p, _i32p, _i32p,
                                   ctypes.c_int, _i32p, _f32p, _f32p, ctypes.c_int, _i32p, _i32p,
                                   _f32p, ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(RsMaterial),
                                   _f64p, _f64p, _i32p, _f64p])
    c = lambda a, t: np.ascontiguousarray(a, t)  # noqa: E731
    sp = c(ev.seed_par.T[seeds], np.float32)
    se = c(ev.seed_err.T[seeds], np.float32)
    sc = c(ev.seed_chg[seeds], np.int32)
    rl = c(g.rl, np.float32)
    xi = c(g.xi, np.float32)
    mat = RsMaterial(rl.ctypes.data, xi.ctypes.data)
    par = np.zeros((n, 6), np.float64)
    err = np.zeros((n, 21), np.float64)
    chg = np.zeros(n, np.int32)
    chi2 = np.zeros(n, np.float64)
    hi = c(out["hit_idx"][slots], np.int32)
    L.rs_replay_cands(n, sp, se, sc, c(out["ntot"][slots], np.int32), hi,
                      c(out["hit_lyr"][slots], np.int32), hi.shape[1],
                      c(ev.seed_nhits[seeds], np.int32), c(ev.hit_pos, np.float32),
                      c(ev.hit_err, np.float32), ev.hit_pos.shape[1],
                      c(ev.layer_begin, np.int32), c(g.field("is_barrel"), np.int32),
                      c(g.field("propagate_to"), np.float32), int(g.flags[1]), int(g.flags[2]),
                      ctypes.byref(mat), par, err, chg, chi2)
    return par, err, chg, chi2


def adjoint_f64_lib_path():
    return os.path.join(REF_DIR, "libadjoint_f64.so")


def adj_f64_grad(par, err, chg, hit_pos, hit_err, theta, rl_grid=None, xi_grid=None, material=True):
    """FP64 host evaluation of the product's generated fit-step adjoint
    (oracle/adjoint_f64.cc): returns (sum chi2, gradient [n_steps][3])."""
    lib = ctypes.CDLL(adjoint_f64_lib_path())
    f = lib.adj_f64_fit_grad
    f.restype = None
    n = chg.shape[0]
    ns = hit_pos.shape[0]
    th = np.ascontiguousarray(theta, np.float64).reshape(ns, 3)
    rl = np.ascontiguousarray(rl_grid, np.float32) if rl_grid is not None else None
    xi = np.ascontiguousarray(xi_grid, np.float32) if xi_grid is not None else None
    total = ctypes.c_double()
    grad = np.zeros((ns, 3), np.float64)
    args = [np.ascontiguousarray(par, np.float32), np.ascontiguousarray(err, np.float32),
            np.ascontiguousarray(chg, np.int32), np.ascontiguousarray(hit_pos, np.float32),
            np.ascontiguousarray(hit_err, np.float32), th]
    f(ctypes.c_int(n), ctypes.c_int(ns), *[a.ctypes.data_as(ctypes.c_void_p) for a in args],
      rl.ctypes.data_as(ctypes.c_void_p) if rl is not None else None,
      xi.ctypes.data_as(ctypes.c_void_p) if xi is not None else None,
      ctypes.c_int(1 if material else 0), ctypes.byref(total),
      grad.ctypes.data_as(ctypes.c_void_p))
    return total.value, grad


def restate_chi2_sum(rs, ev, theta, material=True):
    """Sum over tracks of the FP64 restatement's fit chi2 at parameters
    theta [n_steps][3] (r-phi shift, z shift, material scale)."""
    th = np.asarray(theta, np.float64).reshape(-1, 3)
    _, _, chi2 = rs.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid, ev.xi_grid,
                        pflags=2 if material else 0, shift_rphi=th[:, 0].copy(),
                        shift_z=th[:, 1].copy(), mat_scale=th[:, 2].copy())
    return float(np.sum(chi2))


def restate_fd_grad(rs, ev, theta, h_shift=1e-4, h_scale=1e-3, material=True):
    """Central finite differences of restate_chi2_sum in every parameter."""
    th = np.asarray(theta, np.float64).reshape(-1, 3)
    g = np.zeros_like(th)
    for s in range(th.shape[0]):
        for j in range(3):
            h = h_scale if j == 2 else h_shift
            tp, tm = th.copy(), th.copy()
            tp[s, j] += h
            tm[s, j] -= h
            g[s, j] = (restate_chi2_sum(rs, ev, tp, material) -
                       restate_chi2_sum(rs, ev, tm, material)) / (2 * h)
    return g


def backward_fit_groups(region_sorted, nn=8):
    """Seed groups of MkBuilder::BackwardFit (mkFit/MkBuilder.cc:2153-2190)
    for one event, as lists of sorted positions: per eta region, the seed
    range is cut into tasks with grain clamp(n_seeds + 1, 4, 32) -- as the
    oracle's task pool cuts a blocked_range: ceil(n / grain) near-equal
    pieces -- and fit_cands takes groups of nn from each task's start."""
    ns = len(region_sorted)
    grain = min(max(ns + 1, 4), 32)
    groups = []
    b = 0
    while b < ns:
        e = b
        while e < ns and region_sorted[e] == region_sorted[b]:
            e += 1
        n = e - b
        pieces = (n + grain - 1) // grain
        base, extra = divmod(n, pieces)
        t0 = b
        for i in range(pieces):
            t1 = t0 + base + (1 if i < extra else 0)
            for g0 in range(t0, t1, nn):
                groups.append(list(range(g0, min(g0 + nn, t1))))
            t0 = t1
        b = e
    return groups


def restate_backward_fit(rs, ev, found, geom, m, nn=8):
    """FP64 restatement of the backward fit of every seed's best candidate
    (MkFinder::BkFitInputTracks / BkFitFitTracks / BkFitOutputTracks,
    mkFit/MkFinder.cc:1368-1452, 1573-1742, driven as MkBuilder::BackwardFit)
    from a finding result `found` (ref_find output before the backward fit):
    covariance scaled by 100, reverse layer plan down to bkfit_last, hits
    taken from the candidate's hit list backwards (first node of a layer,
    holes skipped), NN-wide groups sharing layer skips, stand-in
    measurements (own position, variance 666, no material) for members
    without a hit. Returns par [ns][6], err [ns][21], chi2 [ns] (float64),
    indexed by seed label."""
    L = rs.lib
    d6 = ctypes.c_double * 6
    d21 = ctypes.c_double * 21
    d3 = ctypes.c_double * 3
    L.rs_propagate_to_r.restype = ctypes.c_int
    L.rs_kalman_barrel.restype = ctypes.c_double
    L.rs_kalman_endcap.restype = ctypes.c_double
    rl = np.ascontiguousarray(geom.rl, np.float32)
    xi = np.ascontiguousarray(geom.xi, np.float32)
    mat = RsMaterial(rl.ctypes.data, xi.ctypes.data)
    pflags = int(geom.flags[3])
    barrel = geom.field("is_barrel") > 0.5
    ns = ev.n_seeds
    label_at = np.empty(ns, np.int64)
    label_at[found["sorted_pos"]] = np.arange(ns)
    hp = np.asarray(ev.hit_pos, np.float64)
    he = np.asarray(ev.hit_err, np.float64)
    lb = np.asarray(ev.layer_begin)
    out_par = np.zeros((ns, 6))
    out_err = np.zeros((ns, 21))
    out_chi2 = np.zeros(ns)
    for grp in backward_fit_groups(found["region"][label_at], nn):
        labels = [int(label_at[p]) for p in grp]
        reg = int(found["region"][labels[0]])
        st = []
        for s in labels:
            slot = s * m
            ntot = int(found["ntot"][slot])
            st.append(dict(p=found["par"][slot].astype(np.float64).copy(),
                           e=found["err"][slot].astype(np.float64) * 100.0,
                           chg=int(found["chg"][slot]), k=ntot - 1,
                           idx=found["hit_idx"][slot][:ntot], lyr=found["hit_lyr"][slot][:ntot],
                           chi2=0.0))
        for li in range(int(geom.plan_len[reg]) - 1, int(geom.bkfit_last[reg]) - 1, -1):
            layer = int(geom.plans[reg][li])
            meas = []
            for t in st:
                while t["k"] >= 0 and t["idx"][t["k"]] < 0:
                    t["k"] -= 1
                done = t["k"] < 0
                here = (not done) and t["lyr"][t["k"]] == layer
                if here:
                    while t["k"] - 1 >= 0 and t["lyr"][t["k"] - 1] == layer:
                        t["k"] -= 1
                    g = lb[layer] + t["idx"][t["k"]]
                    t["k"] -= 1
                    meas.append((done, here, hp[:, g].copy(), he[:, g].copy()))
                else:
                    meas.append((done, here, t["p"][:3].copy(),
                                 np.array([666.0, 0.0, 666.0, 0.0, 0.0, 666.0])))
            if all(mm[0] for mm in meas):
                break
            if not any(mm[1] for mm in meas):
                continue
            for t, (done, here, mpos, merr) in zip(st, meas):
                pin, ein = d6(*t["p"]), d21(*t["e"])
                pp, pe = d6(), d21()
                pf = pflags if here else (pflags & ~2)
                if barrel[layer]:
                    L.rs_propagate_to_r(pin, ein, t["chg"], ctypes.c_double(float(np.hypot(mpos[0], mpos[1]))),
                                        pf, ctypes.byref(mat), pp, pe)
                    op, oe = d6(), d21()
                    c2 = L.rs_kalman_barrel(pp, pe, d3(*mpos), d6(*merr), op, oe)
                else:
                    L.rs_propagate_to_z(pin, ein, t["chg"], ctypes.c_double(float(mpos[2])), pf,
                                        ctypes.byref(mat), pp, pe)
                    op, oe = d6(), d21()
                    c2 = L.rs_kalman_endcap(pp, pe, d3(*mpos), d6(*merr), op, oe)
                t["p"] = np.array(op[:])
                t["e"] = np.array(oe[:])
                if t["p"][3] < 0:
                    t["chg"] = -t["chg"]
                    t["p"][3] = -t["p"][3]
                t["chi2"] += c2
        for s, t in zip(labels, st):
            out_par[s] = t["p"]
            out_err[s] = t["e"]
            out_chi2[s] = t["chi2"]
    return out_par, out_err, out_chi2


def _load_find_api(lib):
    c_int_p = ctypes.POINTER(ctypes.c_int)
    lib.ref_cms2017_sizes.argtypes = [c_int_p, c_int_p, c_int_p]
    lib.ref_cms2017_export.argtypes = [_f32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _f32p,
                                       _i32p, _f32p, _f32p, _f32p]
    lib.ref_find.restype = ctypes.c_int
    lib.ref_find.argtypes = ([ctypes.c_int, _i32p, _f32p, _f32p, _i32p, _i32p, ctypes.c_int,
                              _f32p, _f32p, _i32p, _i32p, _i32p, _i32p, ctypes.c_int,
                              ctypes.c_float, ctypes.c_int, ctypes.c_int] +
                             [_i32p, _i32p, _i32p, _f32p, _f32p, _i32p, _f32p, _f32p] +
                             [_i32p] * 5 + [_i32p, _i32p, ctypes.POINTER(ctypes.c_double)])


def _set_iteration(lib, it):
    lib.ref_set_iteration.restype = ctypes.c_int
    lib.ref_set_iteration.argtypes = [ctypes.c_int]
    if lib.ref_set_iteration(int(it)) != 0:
        raise IndexError(f"no iteration {it}")


def cms2017_export(reflib, iteration=0):
    """CMS-2017 geometry + the configuration of one iteration (layer plans,
    search windows, iteration parameters) from the reference's own plugin
    (Geoms/CMS-2017.cc), as numpy arrays."""
    lib = reflib.lib
    _load_find_api(lib)
    _set_iteration(lib, iteration)
    try:
        return _cms2017_export(lib)
    finally:
        _set_iteration(lib, 0)


def _cms2017_export(lib):
    nl, nr, mp = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib.ref_cms2017_sizes(ctypes.byref(nl), ctypes.byref(nr), ctypes.byref(mp))
    nl, nr, mp = nl.value, nr.value, mp.value
    out = dict(layer_desc=np.zeros((nl, 32), np.float32), plans=np.zeros((nr, mp), np.int32),
               plan_len=np.zeros(nr, np.int32), pickup=np.zeros(nr, np.int32),
               bkfit_last=np.zeros(nr, np.int32), bksearch_pickup=np.zeros(nr, np.int32),
               region_order=np.zeros(nr, np.int32), iter_params=np.zeros(8, np.float32),
               flags=np.zeros(4, np.int32), eta=np.zeros(3, np.float32),
               rl=np.zeros((300, 120), np.float32), xi=np.zeros((300, 120), np.float32))
    lib.ref_cms2017_export(out["layer_desc"], out["plans"], out["plan_len"], out["pickup"],
                           out["bkfit_last"], out["bksearch_pickup"], out["region_order"],
                           out["iter_params"], out["flags"], out["eta"], out["rl"], out["xi"])
    out["bk_iter_params"] = np.zeros(8, np.float32)
    out["bk_flags"] = np.zeros(2, np.int32)
    lib.ref_cms2017_backward_params.argtypes = [_f32p, _i32p]
    lib.ref_cms2017_backward_params(out["bk_iter_params"], out["bk_flags"])
    return out


def _set_seed_stride(lib, seed_hit_layer):
    lib.ref_set_seed_hit_stride.argtypes = [ctypes.c_int]
    a = np.asarray(seed_hit_layer)
    lib.ref_set_seed_hit_stride(int(a.shape[1]) if a.ndim == 2 else 4)


def ref_find(reflib, ev, max_cands=6, chi2_cut=30.0, zero_c2=True, repeat=1, backward_fit=False,
             select=False, backward_search=False, qf_pre=-1, qf_post=-1, qf_min_hits=0,
             beam=(0.0, 0.0), dup_mode=0, dup_params=None, iteration=0, hit_mask=None):
    """Reference clone-engine finding (find_tracks_load_seeds +
    FindTracksCloneEngine, then MkBuilder::BackwardFit when backward_fit,
    or CompactifyHitStorageForBestCand + BackwardFit + the backward search
    when backward_search) on a synth.CmsEvent. Returns a dict of per-seed candidate arrays (see
    oracle/ref_driver.cc ref_find); with select, also keep[ns]: 1 for the
    seeds whose best candidate survives run_OneIteration's output selection
    (NaN/silly filter, best-candidate export, duplicate removal).
    qf_pre / qf_post: quality filter (QF_KINDS index, -1 none) applied with
    MkBuilder::filter_comb_cands after the clone engine / after the backward
    fit or search, as run_OneIteration does; dup_mode: the duplicate removal
    of the selection (DUP_MODES index) with dup_params (fracSharedHits,
    drth central, obarrel, forward) replacing the iteration's. iteration:
    the CMS-2017 iteration whose steering and parameters the finding uses
    (max_cands, chi2_cut and zero_c2 still override). hit_mask: one flag per
    hit in the event's layer order, hits used by earlier iterations
    (IterationMaskIfc)."""
    lib = reflib.lib
    _load_find_api(lib)
    _set_iteration(lib, iteration)
    lib.ref_set_hit_mask.argtypes = [ctypes.c_void_p]
    hm = None if hit_mask is None else np.ascontiguousarray(hit_mask, np.uint8)
    lib.ref_set_hit_mask(None if hm is None else hm.ctypes.data)
    lib.ref_set_iteration_filters.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                              ctypes.c_void_p]
    dp = None if dup_params is None else np.ascontiguousarray(dup_params, np.float32)
    lib.ref_set_iteration_filters(int(qf_pre), int(qf_post), int(qf_min_hits), float(beam[0]),
                                  float(beam[1]), int(dup_mode),
                                  None if dp is None else dp.ctypes.data)
    lib.ref_set_backward_fit.argtypes = [ctypes.c_int]
    lib.ref_set_backward_fit(1 if backward_fit else 0)
    lib.ref_set_backward_search.argtypes = [ctypes.c_int]
    lib.ref_set_backward_search(1 if backward_search else 0)
    _set_seed_stride(lib, ev.seed_hit_layer)
    lib.ref_set_select_output.argtypes = [ctypes.c_void_p]
    keep = np.zeros(ev.n_seeds, np.int32) if select else None
    lib.ref_set_select_output(keep.ctypes.data if select else None)
    ns = ev.n_seeds
    m = max_cands
    o = dict(n_cands=np.zeros(ns, np.int32), region=np.zeros(ns, np.int32),
             sorted_pos=np.zeros(ns, np.int32), par=np.zeros((ns * m, 6), np.float32),
             err=np.zeros((ns * m, 21), np.float32), chg=np.zeros(ns * m, np.int32),
             chi2=np.zeros(ns * m, np.float32), score=np.zeros(ns * m, np.float32),
             nfound=np.zeros(ns * m, np.int32), ntot=np.zeros(ns * m, np.int32),
             noverlap=np.zeros(ns * m, np.int32), ninside=np.zeros(ns * m, np.int32),
             ntail=np.zeros(ns * m, np.int32), hit_idx=np.zeros((ns * m, 64), np.int32),
             hit_lyr=np.zeros((ns * m, 64), np.int32))
    secs = ctypes.c_double(0)
    c = lambda a, t: np.ascontiguousarray(a, t)
    rc = lib.ref_find(ev.n_layers, c(ev.layer_begin, np.int32), c(ev.hit_pos, np.float32),
                      c(ev.hit_err, np.float32), c(ev.hit_detid, np.int32),
                      c(ev.hit_cpcm, np.int32), ns, c(ev.seed_par, np.float32),
                      c(ev.seed_err, np.float32), c(ev.seed_chg, np.int32),
                      c(ev.seed_nhits, np.int32), c(ev.seed_hit_layer, np.int32),
                      c(ev.seed_hit_index, np.int32), m, float(chi2_cut), int(zero_c2),
                      int(repeat), o["n_cands"], o["region"], o["sorted_pos"], o["par"], o["err"],
                      o["chg"], o["chi2"], o["score"], o["nfound"], o["ntot"], o["noverlap"],
                      o["ninside"], o["ntail"], o["hit_idx"], o["hit_lyr"], ctypes.byref(secs))
    lib.ref_set_backward_fit(0)
    lib.ref_set_backward_search(0)
    lib.ref_set_select_output(None)
    lib.ref_set_iteration_filters(-1, -1, 0, 0.0, 0.0, 0, None)
    _set_iteration(lib, 0)
    lib.ref_set_hit_mask(None)
    if rc != 0:
        raise RuntimeError(f"ref_find failed rc={rc}")
    o["seconds"] = secs.value
    if select:
        o["keep"] = keep
    return o


def ref_event_prep(reflib, ev):
    """The reference's hit index bins / sorted ranks and seed order for an
    event (oracle/ref_driver.cc ref_event_prep)."""
    lib = reflib.lib
    lib.ref_event_prep.restype = ctypes.c_int
    lib.ref_event_prep.argtypes = [ctypes.c_int, _i32p, _f32p, _f32p, _i32p, _i32p, ctypes.c_int,
                                   _f32p, _f32p, _i32p, _i32p, _i32p, _i32p, ctypes.c_void_p,
                                   ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p]
    _set_seed_stride(lib, ev.seed_hit_layer)
    c = lambda a, t: np.ascontiguousarray(a, t)
    args = [ev.n_layers, c(ev.layer_begin, np.int32), c(ev.hit_pos, np.float32),
            c(ev.hit_err, np.float32), c(ev.hit_detid, np.int32), c(ev.hit_cpcm, np.int32),
            ev.n_seeds, c(ev.seed_par, np.float32), c(ev.seed_err, np.float32),
            c(ev.seed_chg, np.int32), c(ev.seed_nhits, np.int32), c(ev.seed_hit_layer, np.int32),
            c(ev.seed_hit_index, np.int32)]
    nb = ctypes.c_int(0)
    lib.ref_event_prep(*args, None, ctypes.byref(nb), None, None, None)
    bins = np.zeros(nb.value, np.uint32)
    srank = np.zeros(ev.n_hits, np.int32)
    order = np.zeros(ev.n_seeds, np.int32)
    region = np.zeros(ev.n_seeds, np.int32)
    rc = lib.ref_event_prep(*args, bins.ctypes.data, ctypes.byref(nb), srank.ctypes.data,
                            order.ctypes.data, region.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ref_event_prep failed rc={rc}")
    return dict(bins=bins, srank=srank, seed_order=order, seed_region=region)


def ref_find_batch(reflib, events, max_cands=6, chi2_cut=30.0, zero_c2=True, repeat=1):
    """Reference clone-engine finding of several events in flight
    (oracle/ref_driver.cc ref_find_batch). Returns best-candidate summaries
    per concatenated seed and the best timed-region seconds."""
    lib = reflib.lib
    L = events[0].n_layers
    hit_off = np.zeros(len(events) + 1, np.int32)
    seed_off = np.zeros(len(events) + 1, np.int32)
    for i, ev in enumerate(events):
        hit_off[i + 1] = hit_off[i] + ev.n_hits
        seed_off[i + 1] = seed_off[i] + ev.n_seeds
    cat = lambda k, ax, t: np.ascontiguousarray(np.concatenate([getattr(e, k) for e in events], axis=ax), t)
    lb = np.ascontiguousarray(np.stack([ev.layer_begin for ev in events]), np.int32)
    NS = int(seed_off[-1])
    _set_seed_stride(lib, events[0].seed_hit_layer if events else np.zeros((0, 4)))
    lib.ref_find_batch.restype = ctypes.c_int
    lib.ref_find_batch.argtypes = ([ctypes.c_int, _i32p, _i32p, _i32p, _f32p, _f32p, _i32p, _i32p,
                                    _f32p, _f32p, _i32p, _i32p, _i32p, _i32p, ctypes.c_int,
                                    ctypes.c_float, ctypes.c_int, ctypes.c_int] +
                                   [_i32p] * 5 + [ctypes.POINTER(ctypes.c_double)])
    o = dict(n_cands=np.zeros(NS, np.int32), nfound=np.zeros(NS, np.int32),
             ntot=np.zeros(NS, np.int32), hit_idx=np.zeros((NS, 64), np.int32),
             hit_lyr=np.zeros((NS, 64), np.int32))
    secs = ctypes.c_double(0)
    rc = lib.ref_find_batch(len(events), hit_off, seed_off, lb, cat("hit_pos", 1, np.float32),
                            cat("hit_err", 1, np.float32), cat("hit_detid", 0, np.int32),
                            cat("hit_cpcm", 0, np.int32), cat("seed_par", 1, np.float32),
                            cat("seed_err", 1, np.float32), cat("seed_chg", 0, np.int32),
                            cat("seed_nhits", 0, np.int32), cat("seed_hit_layer", 0, np.int32),
                            cat("seed_hit_index", 0, np.int32), int(max_cands), float(chi2_cut),
                            int(zero_c2), int(repeat), o["n_cands"], o["nfound"], o["ntot"],
                            o["hit_idx"], o["hit_lyr"], ctypes.byref(secs))
    if rc != 0:
        raise RuntimeError(f"ref_find_batch failed rc={rc}")
    o["seconds"] = secs.value
    return o


def ref_clean_seeds(reflib, seeds, params, beam=(0.0, 0.0), max_hits=16):
    """Seed cleaning of one event's seeds by the reference
    (StdSeq::clean_cms_seedtracks_iter via oracle/ref_driver.cc
    ref_clean_seeds). seeds: dict par [6][n], err [21][n], chg, nhits,
    hit_layer / hit_index [n][k]; params in set_seed_cleaning_params order.
    Returns (keep, nhits, hit_layer, hit_index); rows of dropped seeds 0."""
    lib = reflib.lib
    lib.ref_clean_seeds.restype = ctypes.c_int
    lib.ref_clean_seeds.argtypes = [ctypes.c_int, _f32p, _f32p, _i32p, _i32p, _i32p, _i32p,
                                    ctypes.c_int, _f32p, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_int, _i32p, _i32p, _i32p, _i32p]
    n = int(seeds["chg"].shape[0])
    c = np.ascontiguousarray
    hl = c(seeds["hit_layer"], np.int32)
    keep = np.zeros(n, np.int32)
    onh = np.zeros(n, np.int32)
    ohl = np.zeros((n, max_hits), np.int32)
    ohx = np.zeros((n, max_hits), np.int32)
    lib.ref_clean_seeds(n, c(seeds["par"], np.float32), c(seeds["err"], np.float32),
                        c(seeds["chg"], np.int32), c(seeds["nhits"], np.int32), hl,
                        c(seeds["hit_index"], np.int32), hl.shape[1],
                        np.ascontiguousarray(params, np.float32), float(beam[0]), float(beam[1]),
                        max_hits, keep, onh, ohl, ohx)
    return keep, onh, ohl, ohx


# dz2*dzi + dr2*dri < 1 (MkStdSeqs.cc:247-254) as GCC contracts it: the
# first product fused with the second as addend.
WINDOW_SUM = lambda dz2, dzi, dr2, dri: _fma32(dz2, dzi, np.float32(dr2 * dri))  # noqa: E731


def _fma32(a, b, c):
    """Single-rounding a*b + c of float32 values (the float64 product is
    exact; the sum is rounded twice, which differs from one rounding only in
    rare ties)."""
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


_LIBM = None


def _libm_f32(name, v):
    """The host C library's float function `name` (sinf, cosf, tanf, logf)
    applied elementwise: the functions the reference's float calls reach."""
    global _LIBM
    if _LIBM is None:
        _LIBM = ctypes.CDLL("libm.so.6")
        for fn in ("sinf", "cosf", "tanf", "logf"):
            getattr(_LIBM, fn).restype = ctypes.c_float
            getattr(_LIBM, fn).argtypes = [ctypes.c_float]
    f = getattr(_LIBM, name)
    return np.array([f(float(x)) for x in np.asarray(v, np.float32).ravel()], np.float32)


def clean_seed_features(seeds, beam=(0.0, 0.0)):
    """Per-seed quantities of the seed cleaning (MkStdSeqs.cc:166-180) in
    float32 with the host C library's float functions: pt, eta, pos2,
    ctheta, invptq, d0 (Track::d0BeamSpot, Track.cc:195-210, with x - k*py
    and y + k*px contracted into FMAs as the reference build does) and the
    helix radius |k pt| that d0 is a difference against."""
    f = np.float32
    par = np.asarray(seeds["par"], np.float32)
    chg = np.asarray(seeds["chg"], np.int32)
    n = chg.shape[0]
    x, y = par[0], par[1]
    ipt, phi, theta = par[3], par[4], par[5]
    pt = np.abs(f(1.0) / ipt)
    eta = f(-1.0) * _libm_f32("logf", _libm_f32("tanf", theta / f(2.0)))
    pos2 = (x.astype(np.float64) ** 2 + y.astype(np.float64) ** 2).astype(np.float32)
    ctheta = f(1.0) / _libm_f32("tanf", theta)
    invptq = chg.astype(np.float32) * ipt
    d0, radius = d0_beam_spot(par, chg, beam)
    return dict(pt=pt, eta=eta, pos2=pos2, ctheta=ctheta, invptq=invptq, d0=d0, radius=radius)


def d0_beam_spot(par, chg, beam=(0.0, 0.0)):
    """TrackBase::d0BeamSpot, not linearised (Track.cc:195-210), in float32
    with the host C library's sinf / cosf and x - k*py, y + k*px contracted
    into FMAs as the reference build does. par [6][n]. Returns (d0, |k pt|),
    the second being the helix radius d0 is a difference against."""
    f = np.float32
    par = np.asarray(par, np.float32)
    chg = np.asarray(chg, np.int32)
    n = chg.shape[0]
    x, y, ipt, phi = par[0], par[1], par[3], par[4]
    pt = np.abs(f(1.0) / ipt)
    sb = f(0.299792458) * f(3.8112)
    k = np.where(chg < 0, f(100.0) / sb, f(-100.0) / sb).astype(np.float32)
    px, py = pt * _libm_f32("cosf", phi), pt * _libm_f32("sinf", phi)
    xc = np.array([_fma32(-k[i], py[i], x[i]) for i in range(n)], np.float32)
    yc = np.array([_fma32(k[i], px[i], y[i]) for i in range(n)], np.float32)
    radius = np.abs(k * pt)
    d0 = (np.hypot((xc - f(beam[0])).astype(np.float64), (yc - f(beam[1])).astype(np.float64))
          .astype(np.float32) - radius)
    return d0, radius


def restate_clean_seeds(seeds, params, beam=(0.0, 0.0), max_hits=16):
    """Pure-Python restatement of StdSeq::clean_cms_seedtracks_iter
    (mkFit/MkStdSeqs.cc:115-311) in float32 arithmetic, for small n: the
    per-seed quantities (:166-180, Track::d0BeamSpot Track.cc:195-210), the
    ordered pair loop with its skip of already-dropped seeds (:182-186), the
    window (:196-256), the drop of the larger-d0 seed (:258-270) and the hit
    merge with its 15-hit cap and layer sort (:271-305)."""
    f = np.float32
    par = np.asarray(seeds["par"], np.float32)
    chg = np.asarray(seeds["chg"], np.int32)
    n = chg.shape[0]
    ptthr, dz_bh, dr_bh, dz_bl, dr_bl, dz_eh, dr_eh, dz_el, dr_el = [f(v) for v in params]
    inv2 = lambda v: f(1.0) / (v * v)  # noqa: E731
    dzi = dict(bh=inv2(dz_bh), bl=inv2(dz_bl), eh=inv2(dz_eh), el=inv2(dz_el))
    dri = dict(bh=inv2(dr_bh), bl=inv2(dr_bl), eh=inv2(dr_eh), el=inv2(dr_el))
    F = clean_seed_features(seeds, beam)
    x, y, z, phi = par[0], par[1], par[2], par[4]
    pt, eta, pos2, ctheta, invptq, d0 = (F[k] for k in ("pt", "eta", "pos2", "ctheta", "invptq",
                                                          "d0"))
    hits = [[(int(seeds["hit_index"][i][j]), int(seeds["hit_layer"][i][j]))
             for j in range(int(seeds["nhits"][i]))] for i in range(n)]
    write = [True] * n
    inv_r1 = f(1.0) / f(87.6)
    for ts in range(n):
        if not write[ts]:
            continue
        added = 0
        for tss in range(ts + 1, n):
            if chg[tss] != chg[ts]:
                continue
            if abs(pt[tss] - pt[ts]) > f(0.25) * pt[ts]:
                continue
            deta2 = f((eta[ts] - eta[tss]) ** 2)
            sign = f(-0.5) if pos2[tss] > pos2[ts] else f(0.5)
            dx, dy = f(x[ts] - x[tss]), f(y[ts] - y[tss])
            dxy = f(float(sign) * np.sqrt(float(dx) ** 2 + float(dy) ** 2))
            t = dxy * inv_r1
            # Contracted as the reference build does: phi -/+ t*invptq,
            # deta2 + dphi^2, (z1 - z2) - dxy*(ct1 + ct2), and the window sum.
            nphi1 = _fma32(-t, invptq[ts], phi[ts])
            nphi2 = _fma32(t, invptq[tss], phi[tss])
            dphi = abs(f(nphi1 - nphi2))
            if dphi > f(np.pi):
                dphi = f(2 * np.pi) - dphi
            dr2 = _fma32(dphi, dphi, deta2)
            dz = _fma32(-dxy, f(ctheta[ts] + ctheta[tss]), f(z[ts] - z[tss]))
            dz2 = dz * dz
            key = ("b" if abs(eta[ts]) < f(0.9) else "e") + ("h" if pt[ts] > ptthr else "l")
            if not WINDOW_SUM(dz2, dzi[key], dr2, dri[key]) < f(1.0):
                continue
            if d0[tss] > d0[ts]:
                write[tss] = False
                i1, i2 = ts, tss
            else:
                write[ts] = False
                i1, i2 = tss, ts
            if len(hits[i1]) < 15:
                for h in hits[i2]:
                    if h[0] >= 0 and h not in hits[i1]:
                        hits[i1].append(h)
                        added += 1
                        if len(hits[i1]) >= 15:
                            break
            if added > 0:
                hits[i1].sort(key=lambda h: h[1])  # stable, by layer
    keep = np.array(write, np.int32)
    onh = np.zeros(n, np.int32)
    ohl = np.zeros((n, max_hits), np.int32)
    ohx = np.zeros((n, max_hits), np.int32)
    for i in range(n):
        if keep[i]:
            onh[i] = len(hits[i])
            for j, (hx, hly) in enumerate(hits[i][:max_hits]):
                ohl[i, j], ohx[i, j] = hly, hx
    return keep, onh, ohl, ohx


def _mf_tracks_args(t):
    t = t or {}
    n = len(t.get("charge", ()))
    c = np.ascontiguousarray
    z = lambda dt, *s: np.zeros(s, dt)  # noqa: E731
    return [n, c(t.get("par", z(np.float32, 6, n)), np.float32).ravel(),
            c(t.get("err", z(np.float32, 21, n)), np.float32).ravel(),
            c(t.get("charge", z(np.int32, n)), np.int32),
            c(t.get("chi2", z(np.float32, n)), np.float32),
            c(t.get("score", z(np.float32, n)), np.float32),
            c(t.get("status", z(np.uint32, n)), np.uint32),
            c(t.get("label", np.full(n, -1)), np.int32),
            c(t.get("hits_begin", z(np.int32, n + 1)), np.int32),
            c(t.get("hit_index", z(np.int32, 1)), np.int32),
            c(t.get("hit_layer", z(np.int32, 1)), np.int32)]


def ref_mf_write(reflib, path, events, sections):
    """Writes events (memory_file event dicts, 72 layers) with the
    reference's DataFile::OpenWrite + Event::write_out + CloseWrite."""
    lib = reflib.lib
    vp = ctypes.c_void_p
    lib.ref_mf_write_begin.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
    lib.ref_mf_write_event.argtypes = [ctypes.c_int] + [vp] * 6 + [ctypes.c_int, vp] + \
        ([ctypes.c_int] + [vp] * 10) * 3 + [vp, ctypes.c_int, vp, vp, vp]
    keep = []

    def p(a):
        if a is None:
            return None
        keep.append(a)
        return a.ctypes.data

    if lib.ref_mf_write_begin(str(path).encode(), len(events), sections) != 0:
        raise RuntimeError("ref_mf_write_begin failed")
    c = np.ascontiguousarray
    for ev in events:
        mc = c(ev.get("mc_info", np.zeros((0, 4))), np.int32)
        args = [int(ev["n_layers"]), p(c(ev["layer_begin"], np.int32)),
                p(c(ev["hit_pos"], np.float32)), p(c(ev["hit_err"], np.float32)),
                p(c(ev["hit_mcid"], np.int32)), p(c(ev["hit_packed"], np.uint32)),
                p(None if ev.get("hit_masks") is None else c(ev["hit_masks"], np.uint64)),
                mc.shape[0], p(mc)]
        for key in ("sim", "seeds", "cmssw"):
            ta = _mf_tracks_args(ev.get(key))
            args += [ta[0]] + [p(a) for a in ta[1:]]
        st = ev.get("sim_states") or {}
        ns = len(st.get("charge", ()))
        bs = ev.get("beam_spot")
        args += [p(None if bs is None else c(bs, np.float32)), ns,
                 p(c(st["par"], np.float32)) if ns else None,
                 p(c(st["err"], np.float32)) if ns else None,
                 p(c(st["charge"], np.int32)) if ns else None]
        lib.ref_mf_write_event(*args)
    return lib.ref_mf_write_end()


def ref_mf_read(reflib, path, which, hit_cap=1 << 20, trk_cap=1 << 15, hcap=1 << 18):
    """Event `which` of a memoryFile as the reference's Event::read_in sees
    it, as a memory_file-style event dict."""
    lib = reflib.lib
    vp = ctypes.c_void_p
    lib.ref_mf_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int] + [vp] * 23
    counts = np.zeros(8, np.int32)
    lb = np.zeros(129, np.int32)
    pos = np.zeros((3, hit_cap), np.float32)
    herr = np.zeros((6, hit_cap), np.float32)
    mcid = np.zeros(hit_cap, np.int32)
    packed = np.zeros(hit_cap, np.uint32)
    masks = np.zeros(hit_cap, np.uint64)
    mc = np.zeros((hit_cap, 4), np.int32)
    T = 3
    tpar = np.zeros((T, 6, trk_cap), np.float32)
    terr = np.zeros((T, 21, trk_cap), np.float32)
    ti = {k: np.zeros((T, trk_cap), dt) for k, dt in (("charge", np.int32), ("chi2", np.float32),
                                                       ("score", np.float32), ("status", np.uint32),
                                                       ("label", np.int32), ("nfound", np.int32))}
    thb = np.zeros((T, trk_cap + 1), np.int32)
    thi = np.zeros((T, hcap), np.int32)
    thl = np.zeros((T, hcap), np.int32)
    beam = np.zeros(8, np.float32)
    stp = np.zeros((6, trk_cap), np.float32)
    ste = np.zeros((21, trk_cap), np.float32)
    stc = np.zeros(trk_cap, np.int32)
    d = lambda a: a.ctypes.data  # noqa: E731
    rc = lib.ref_mf_read(str(path).encode(), which, hit_cap, trk_cap, hcap, d(counts), d(lb),
                         d(pos), d(herr), d(mcid), d(packed), d(masks), d(mc), d(tpar), d(terr),
                         d(ti["charge"]), d(ti["chi2"]), d(ti["score"]), d(ti["status"]),
                         d(ti["label"]), d(ti["nfound"]), d(thb), d(thi), d(thl), d(beam),
                         d(stp), d(ste), d(stc))
    if rc != 0:
        raise RuntimeError("ref_mf_read: capacity exceeded")
    nl, nh, nm = counts[0], counts[1], counts[2]
    out = dict(n_layers=int(nl), layer_begin=lb[:nl + 1].copy(), hit_pos=pos[:, :nh].copy(),
               hit_err=herr[:, :nh].copy(), hit_mcid=mcid[:nh].copy(), hit_packed=packed[:nh].copy(),
               hit_masks=masks[:nh].copy(), mc_info=mc[:nm].copy(), beam_spot=beam.copy())
    for k, key in enumerate(("sim", "seeds", "cmssw")):
        n = counts[3 + k]
        nh_t = thb[k, n]
        out[key] = dict(par=tpar[k, :, :n].copy(), err=terr[k, :, :n].copy(),
                        hits_begin=thb[k, :n + 1].copy(), hit_index=thi[k, :nh_t].copy(),
                        hit_layer=thl[k, :nh_t].copy(),
                        **{f: ti[f][k, :n].copy() for f in ti})
    ns = counts[6]
    out["sim_states"] = dict(par=stp[:, :ns].copy(), err=ste[:, :ns].copy(), charge=stc[:ns].copy())
    return out


# ---------------------------------------------------------------------------
# Quality filters and duplicate removal of run_OneIteration
# ---------------------------------------------------------------------------

# StdSeq quality filters (mkFit/MkStdSeqs.h:39-148) in the order of their
# codes (the bits of ref_qfilters / restate_qfilters).
QF_KINDS = ("nan_n_silly", "n_hits", "n_hits_pixseed", "n_layers", "n_layers_pixelless",
            "pixelless_fwd", "pixelless_bkwd")
# Duplicate removal by the branch of find_and_remove_duplicates
# (mkFit/MkStdSeqs.cc:605-630), plus "none" (do_remove_duplicates off).
DUP_MODES = ("pixelseed", "sharedhits", "eta_phi", "none")


def ref_qfilters(reflib, cands, nseed, min_hits=4, beam=(0.0, 0.0)):
    """Every quality filter on candidates given as exported hit lists (chain
    order, missing-hit entries included), by the reference (oracle/ref_driver.cc
    ref_qfilters: each candidate rebuilt as a TrackCand). cands: par [n][6],
    err [n][21], chg, ntot [n], hit_idx / hit_lyr [n][w]; nseed [n]: hits of
    the seed. Returns int32 [n], bit k = QF_KINDS[k] passes."""
    lib = reflib.lib
    lib.ref_qfilters.restype = ctypes.c_int
    lib.ref_qfilters.argtypes = [ctypes.c_int, _f32p, _f32p, _i32p, _i32p, _i32p, _i32p, _i32p,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, _i32p]
    c = np.ascontiguousarray
    n = int(len(cands["chg"]))
    hi = c(cands["hit_idx"], np.int32)
    out = np.zeros(n, np.int32)
    rc = lib.ref_qfilters(n, c(cands["par"], np.float32).reshape(n, 6),
                          c(cands["err"], np.float32).reshape(n, 21), c(cands["chg"], np.int32),
                          c(nseed, np.int32), c(cands["ntot"], np.int32), hi,
                          c(cands["hit_lyr"], np.int32), hi.shape[1], int(min_hits),
                          float(beam[0]), float(beam[1]), out)
    if rc != 0:
        raise RuntimeError(f"ref_qfilters failed rc={rc}")
    return out


def ref_dups(reflib, mode, tracks, algo=0, frac=0.24, drth=(0.002, 0.004, 0.008)):
    """Duplicate removal (DUP_MODES[mode]) by the reference on exported
    tracks (oracle/ref_driver.cc ref_dups). tracks: par [n][6], chg, score,
    label, nfound, nh [n], hit_idx / hit_lyr [n][w] (no missing-hit
    entries). Returns keep [n]."""
    lib = reflib.lib
    lib.ref_dups.restype = ctypes.c_int
    lib.ref_dups.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _i32p, _f32p, _i32p, ctypes.c_int,
                             _i32p, _i32p, _i32p, _i32p, ctypes.c_int, ctypes.c_float,
                             ctypes.c_float, ctypes.c_float, ctypes.c_float, _i32p]
    c = np.ascontiguousarray
    n = int(len(tracks["chg"]))
    hi = c(tracks["hit_idx"], np.int32)
    keep = np.zeros(n, np.int32)
    rc = lib.ref_dups(int(mode), n, c(tracks["par"], np.float32).reshape(n, 6),
                      c(tracks["chg"], np.int32), c(tracks["score"], np.float32),
                      c(tracks["label"], np.int32), int(algo), c(tracks["nfound"], np.int32),
                      c(tracks["nh"], np.int32), hi, c(tracks["hit_lyr"], np.int32), hi.shape[1],
                      float(frac), float(drth[0]), float(drth[1]), float(drth[2]), keep)
    if rc != 0:
        raise RuntimeError(f"ref_dups failed rc={rc}")
    return keep


def _in_pix_ranges(lyr):
    """The pixel layers TrackCand::getLastFoundPixelHitLyr names
    (HitStructures.h:753-773): 0-3, 18-20, 45-47."""
    return 0 <= lyr <= 3 or 18 <= lyr <= 20 or 45 <= lyr <= 47


def restate_qfilters(cands, nseed, is_pix, is_stereo, min_hits=4, beam=(0.0, 0.0)):
    """Pure-Python restatement of the quality filters on the same inputs as
    ref_qfilters: the TrackCand hit walks (HitStructures.h:732-859, newest
    hit first, with their quirks: the 'previous stereo' flag holds the
    stereo count so far, a double stereo layer matches the mono layer
    below it), TrackBase::d0BeamSpot and the cuts of MkStdSeqs.h:39-148 in
    float32. is_pix / is_stereo: per-layer flags of the geometry."""
    f = np.float32
    n = len(cands["chg"])
    par = np.asarray(cands["par"], np.float32).reshape(n, 6)
    err = np.asarray(cands["err"], np.float32).reshape(n, 21)
    chg = np.asarray(cands["chg"], np.int32)
    d0, _ = d0_beam_spot(par.T, chg, beam)
    pi_over_2 = f(f(3.14159265358979323846) / f(2.0))
    out = np.zeros(n, np.int32)
    for i in range(n):
        nt = int(cands["ntot"][i])
        hots = [(int(cands["hit_idx"][i][k]), int(cands["hit_lyr"][i][k])) for k in range(nt)]
        found = lambda h: h[0] >= 0 or h[0] == -9  # noqa: E731
        nfound = sum(1 for h in hots if found(h))
        nseed4 = int(nseed[i]) & 15
        back = hots[::-1]
        # getLastFoundHitLyr / getLastFoundPixelHitLyr
        llyr = next((h[1] for h in back if h[0] >= 0), -1)
        lplyr = next((h[1] for h in back if h[0] >= 0 and _in_pix_ranges(h[1])), -1)
        # nUniqueLayers
        nul, prev = 0, -1
        for idx, lyr in back:
            if lyr >= 0 and (idx >= 0 or idx == -9) and lyr != prev:
                nul += 1
                prev = lyr
        # nHitsByTypeEncoded
        pix = stereo = mono = matched = 0
        prev, prev_stereo, double_stereo = -1, 0, -1
        for idx, lyr in back:
            if lyr >= 0 and (idx >= 0 or idx == -9):
                if is_pix[lyr]:
                    pix += 1
                elif is_stereo[lyr]:
                    stereo += 1
                    if lyr == prev:
                        double_stereo = lyr
                else:
                    mono += 1
                    if prev_stereo and lyr == prev - 1:
                        matched += 1
                    elif lyr == prev and lyr == double_stereo - 1:
                        matched += 1
                prev = lyr
                prev_stereo = stereo
        enhits = pix + 100 * stereo + 10000 * mono + 1000000 * matched
        # nLayersByTypeEncoded
        pix = stereo = mono = matched = 0
        prev, prev_stereo = -1, 0
        for idx, lyr in back:
            if lyr >= 0 and (idx >= 0 or idx == -9) and lyr != prev:
                if is_pix[lyr]:
                    pix += 1
                elif is_stereo[lyr]:
                    stereo += 1
                else:
                    mono += 1
                    if prev_stereo and lyr == prev - 1:
                        matched += 1
                prev = lyr
                prev_stereo = stereo
        enlyrs = pix + 100 * stereo + 10000 * mono + 1000000 * matched

        def tot_match(e):
            return e % 100 + (e // 100) % 100 + (e // 10000) % 100 - e // 1000000

        invpt = par[i, 3]
        ad0 = abs(d0[i])
        theta = par[i, 5]
        thetasym = abs(f(theta - pi_over_2))
        red = 2 if nseed4 <= 5 else 3
        m = 0
        # qfilter_nan_n_silly: hasNanNSillyValues over the packed lower triangle.
        silly = False
        k = 0
        for a in range(6):
            for b in range(a + 1):
                v = err[i, k]
                if (a == b and v < 0) or not np.isfinite(v):
                    silly = True
                k += 1
        m |= (not silly) << 0
        m |= (nfound - red >= min_hits) << 1
        m |= (nfound >= min_hits) << 2
        npixhits, npixlyrs, nmatlyrs = enhits % 100, enlyrs % 100, tot_match(enlyrs)
        ends_pix = llyr in (2, 18, 45)
        last_pix = (0 <= lplyr < 3) or (18 <= lplyr < 20) or (45 <= lplyr < 47)
        invptmin = f(1.43)
        d0max = f(0.1)
        fail = (((npixhits <= 3 or npixlyrs <= 3) and ends_pix
                 and (invpt < invptmin or (invpt >= invptmin and ad0 > d0max)))
                or ((npixlyrs <= 3 and nmatlyrs <= 6) and last_pix and llyr != lplyr
                    and ad0 > d0max))
        m |= (not fail) << 3
        m |= (not ((nfound <= 6 or nul <= 6) and ad0 > d0max)) << 4
        nlyrs, nhits = tot_match(enlyrs), tot_match(enhits)
        iptm = f(1.11)
        fwd = (((nfound - red >= 4 and invpt < iptm)
                or (nfound - red >= 3 and invpt > iptm and thetasym <= f(1.11))
                or (nfound - red >= 4 and invpt > iptm and thetasym > f(1.11)))
               and not ((nlyrs <= 4 or nhits <= 4) and ad0 > f(0.05) and invpt < iptm))
        m |= fwd << 5
        bkwd = not ((nlyrs <= 3 or nhits <= 3)
                    or ((nlyrs <= 4 or nhits <= 4)
                        and (invpt < iptm or (thetasym > f(0.80) and ad0 > d0max)))
                    or ((nlyrs <= 6 or nhits <= 6)
                        and (invpt > iptm and thetasym > f(1.11) and ad0 > d0max)))
        m |= bkwd << 6
        out[i] = m
    return out


def _squash_phi_minimal(phi):
    f = np.float32
    two_pi, pi = f(2.0 * np.pi), f(np.pi)
    return f(phi - two_pi) if phi >= pi else (f(phi + two_pi) if phi < -pi else phi)


DR2_SUM = lambda a, b: _fma32(a, a, np.float32(b * b))  # noqa: E731


def restate_dups(mode, tracks, algo=0, frac=0.24, drth=(0.002, 0.004, 0.008)):
    """Pure-Python restatement of the duplicate removal on the same inputs as
    ref_dups: find_duplicates_sharedhits_pixelseed (MkStdSeqs.cc:510-603),
    find_duplicates_sharedhits (:456-508) or find_duplicates (:334-423), in
    float32; every pair i < j is tested (a flag set earlier does not stop a
    track from marking others) and of a duplicate pair the lower score loses
    (the first track on a tie). dphi^2 + d^2 is formed as the reference
    build contracts it: the first product fused, the second as addend."""
    f = np.float32
    n = len(tracks["chg"])
    par = np.asarray(tracks["par"], np.float32).reshape(n, 6)
    score = np.asarray(tracks["score"], np.float32)
    label = np.asarray(tracks["label"], np.int32)
    nfound = np.asarray(tracks["nfound"], np.int32)
    hits = [[(int(tracks["hit_idx"][i][k]), int(tracks["hit_lyr"][i][k]))
             for k in range(int(tracks["nh"][i]))] for i in range(n)]
    tan = lambda v: _libm_f32("tanf", [v])[0]  # noqa: E731
    log = lambda v: _libm_f32("logf", [v])[0]  # noqa: E731
    cth = [f(f(1.0) / tan(par[i, 5])) for i in range(n)]
    dup = np.zeros(n, bool)
    if mode == 3:
        return np.ones(n, np.int32)

    def mark(i, j):
        dup[j if score[i] > score[j] else i] = True

    def shared(i, j):
        cnt = first = 0
        for a, (ia, la) in enumerate(hits[i]):
            if ia < 0:
                continue
            for b, (ib, lb) in enumerate(hits[j]):
                if ib < 0:
                    continue
                if la == lb and ia == ib:
                    cnt += 1
                    if a == 0 and b == 0:
                        first += 1
        return cnt, first

    if mode in (0, 1):
        dc, do, dfw = (f(v) for v in drth)
        for i in range(n):
            phi1, ipt1, c1 = par[i, 4], par[i, 3], cth[i]
            for j in range(i + 1, n):
                if mode == 0 and label[i] == label[j]:
                    continue
                dcth = abs(f(cth[j] - c1))
                dphi = abs(_squash_phi_minimal(f(phi1 - par[j, 4])))
                if mode == 1:
                    if dcth > 1.0 or dphi > 1.0:
                        continue
                else:
                    if dcth > f(0.37) or dphi > f(0.37):
                        continue
                    max_dr2 = f(dc * dc)
                    if abs(c1) > f(6.05):
                        max_dr2 = f(dfw * dfw)
                    elif abs(c1) > f(1.99):
                        max_dr2 = f(do * do)
                    if DR2_SUM(dphi, dcth) < max_dr2:
                        mark(i, j)
                        continue
                    if abs(f(par[j, 3] - ipt1)) > f(1.8):
                        continue
                cnt, first = shared(i, j)
                mf = min(nfound[i], nfound[j])
                if f(cnt - first) >= f(f(mf - first) * f(frac)):
                    mark(i, j)
    else:
        eta = [f(f(-1.0) * log(tan(f(par[i, 5] / f(2.0))))) for i in range(n)]
        pt = [abs(f(f(1.0) / par[i, 3])) for i in range(n)]
        for i in range(n - 1):
            if algo in (9, 10):
                continue
            for j in range(i + 1, n):
                if label[i] == label[j]:
                    continue
                deta = abs(f(eta[j] - eta[i]))
                if deta > f(0.05):
                    continue
                dphi = abs(_squash_phi_minimal(f(par[i, 4] - par[j, 4])))
                if dphi > f(0.25):
                    continue
                max_dr2 = f(f(0.0025) * f(0.0025))
                if abs(eta[i]) > f(2.5):
                    max_dr2 = f(max_dr2 * f(16.0))
                elif abs(eta[i]) > f(1.44):
                    max_dr2 = f(max_dr2 * f(9.0))
                if DR2_SUM(dphi, deta) < max_dr2:
                    mark(i, j)
                    continue
                if pt[i] == 0 or pt[j] == 0:
                    continue
                if abs(f(f(f(1.0) / pt[j]) - f(f(1.0) / pt[i]))) < f(0.5):
                    mine = set(hits[i])
                    nsh = sum(1 for h in hits[j] if h[0] >= 0 and h in mine)
                    mf = min(nfound[i], nfound[j])
                    with np.errstate(divide="ignore", invalid="ignore"):
                        fr = f(f(nsh) / f(mf))
                    if fr < f(0.75):
                        continue
                    mark(i, j)
    return (~dup).astype(np.int32)


def ref_cms2017_iteration(reflib, it):
    """The selection settings of CMS-2017 iteration `it` as the reference's
    geometry plugin sets them: dict algorithm, quality_filter,
    dupclean_tight, min_hits_qf, frac_shared_hits, drth (3)."""
    lib = reflib.lib
    lib.ref_cms2017_iteration.restype = ctypes.c_int
    lib.ref_cms2017_iteration.argtypes = [ctypes.c_int, _i32p, _f32p]
    iv = np.zeros(5, np.int32)
    fv = np.zeros(4, np.float32)
    if lib.ref_cms2017_iteration(int(it), iv, fv) != 0:
        raise IndexError(it)
    return dict(algorithm=int(iv[0]), quality_filter=bool(iv[1]), dupclean_tight=bool(iv[2]),
                min_hits_qf=int(iv[3]), sort_seed_hits=bool(iv[4]), frac_shared_hits=float(fv[0]),
                drth=tuple(float(x) for x in fv[1:]))


def ref_select_hit_indices(reflib, ev, layer, par, err, chg, iteration=0):
    """MkFinder::SelectHitIndices of the reference on states par [6][n],
    err [21][n], chg [n] taken as propagated to `layer`, against the hits of
    event `ev` (oracle/ref_driver.cc ref_select_hit_indices). Returns
    (xsize [n], xidx [n][16])."""
    lib = reflib.lib
    lib.ref_select_hit_indices.restype = ctypes.c_int
    lib.ref_select_hit_indices.argtypes = [ctypes.c_int, _i32p, _f32p, _f32p, _i32p, _i32p,
                                           ctypes.c_int, ctypes.c_int, _f32p, _f32p, _i32p, _i32p,
                                           _i32p]
    _set_iteration(reflib.lib, iteration)
    c = np.ascontiguousarray
    n = int(len(chg))
    xs = np.zeros(n, np.int32)
    xi = np.zeros((n, 16), np.int32)
    try:
        rc = lib.ref_select_hit_indices(ev.n_layers, c(ev.layer_begin, np.int32),
                                        c(ev.hit_pos, np.float32), c(ev.hit_err, np.float32),
                                        c(ev.hit_detid, np.int32), c(ev.hit_cpcm, np.int32),
                                        int(layer), n, c(par, np.float32), c(err, np.float32),
                                        c(chg, np.int32), xs, xi)
    finally:
        _set_iteration(reflib.lib, 0)
    if rc != 0:
        raise RuntimeError(f"ref_select_hit_indices failed rc={rc}")
    return xs, xi


def _event_hit_args(ev):
    c = np.ascontiguousarray
    return (ev.n_layers, c(ev.layer_begin, np.int32), c(ev.hit_pos, np.float32),
            c(ev.hit_err, np.float32), c(ev.hit_detid, np.int32), c(ev.hit_cpcm, np.int32))


_EV_TYPES = [ctypes.c_int, _i32p, _f32p, _f32p, _i32p, _i32p]


def ref_ce_records(reflib, ev, layer, par, err, chg, counts, hot_layers, chi2_cut=30.0,
                   zero_c2=True):
    """The reference's SelectHitIndices + FindCandidatesCloneEngine on
    states par [6][n], err [21][n], chg [n] taken as propagated to `layer`
    of event `ev`, with counters `counts` (dict of nfound, nover, ninside,
    ntail, chi2 [n]) and each comb candidate's first three node layers
    hot_layers [n][3], the chi2 cut set as ref_find sets it
    (oracle/ref_driver.cc ref_ce_records). Returns
    (xsize [n], records: dict of n [n] and hit, module, chi2, score
    [n][17])."""
    lib = reflib.lib
    lib.ref_ce_records.restype = ctypes.c_int
    lib.ref_ce_records.argtypes = _EV_TYPES + [ctypes.c_int, ctypes.c_int, _f32p, _f32p, _i32p,
                                               _i32p, _i32p, _i32p, _i32p, _f32p, _i32p,
                                               ctypes.c_float, ctypes.c_int, _i32p,
                                               _i32p, _i32p, _i32p, _f32p, _f32p]
    c = np.ascontiguousarray
    n = int(len(chg))
    xs = np.zeros(n, np.int32)
    out = dict(n=np.zeros(n, np.int32), hit=np.zeros((n, 17), np.int32),
               module=np.zeros((n, 17), np.int32), chi2=np.zeros((n, 17), np.float32),
               score=np.zeros((n, 17), np.float32))
    rc = lib.ref_ce_records(*_event_hit_args(ev), int(layer), n, c(par, np.float32),
                            c(err, np.float32), c(chg, np.int32), c(counts["nfound"], np.int32),
                            c(counts["nover"], np.int32), c(counts["ninside"], np.int32),
                            c(counts["ntail"], np.int32), c(counts["chi2"], np.float32),
                            c(hot_layers, np.int32), float(chi2_cut), int(bool(zero_c2)), xs,
                            out["n"], out["hit"], out["module"],
                            out["chi2"], out["score"])
    if rc != 0:
        raise RuntimeError(f"ref_ce_records failed rc={rc}")
    return xs, out


def ref_update_with_last_hit(reflib, ev, layer, par, err, chg, hit_idx):
    """The reference's InputTracksAndHitIdx + UpdateWithLastHit +
    CopyOutParErr (oracle/ref_driver.cc ref_update_with_last_hit): returns
    (par, err, chg) updated."""
    lib = reflib.lib
    lib.ref_update_with_last_hit.restype = ctypes.c_int
    lib.ref_update_with_last_hit.argtypes = _EV_TYPES + [ctypes.c_int, ctypes.c_int, _f32p, _f32p,
                                                         _i32p, _i32p, _f32p, _f32p, _i32p]
    n = int(len(chg))
    c = np.ascontiguousarray
    op = np.zeros((6, n), np.float32)
    oe = np.zeros((21, n), np.float32)
    oc = np.zeros(n, np.int32)
    rc = lib.ref_update_with_last_hit(*_event_hit_args(ev), int(layer), n, c(par, np.float32),
                                      c(err, np.float32), c(chg, np.int32),
                                      c(hit_idx, np.int32), op, oe, oc)
    if rc != 0:
        raise RuntimeError(f"ref_update_with_last_hit failed rc={rc}")
    return op, oe, oc


def ref_clone_seeds(reflib, layer, inp, max_cands):
    """CandCloner::ProcessSeedRange of the reference on the seeds of `inp`
    (the fields of mkfg_clone_in, mkfit_b200.finder.clone_arrays layout) at
    `layer` with maxCandsPerSeed = max_cands (oracle/ref_driver.cc
    ref_clone_seeds). Returns the fields of mkfg_clone_out as a dict."""
    from mkfit_b200.finder import CLONE_IN_FIELDS, CLONE_OUT_FIELDS, clone_arrays
    n_seeds = len(inp["n_cands"])
    a = clone_arrays(CLONE_IN_FIELDS, n_seeds, inp)
    o = clone_arrays(CLONE_OUT_FIELDS, n_seeds)
    lib = reflib.lib
    lib.ref_clone_seeds.restype = ctypes.c_int
    lib.ref_clone_seeds.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * (
        len(CLONE_IN_FIELDS) + len(CLONE_OUT_FIELDS))
    args = [a[k].ctypes.data for k, _, _ in CLONE_IN_FIELDS]
    args += [o[k].ctypes.data for k, _, _ in CLONE_OUT_FIELDS]
    rc = lib.ref_clone_seeds(int(layer), n_seeds, int(max_cands), *args)
    if rc != 0:
        raise RuntimeError(f"ref_clone_seeds failed rc={rc}")
    return o


_shims_lib = None


def _shims():
    global _shims_lib
    if _shims_lib is None:
        L = ctypes.CDLL(shims_lib_path())
        common = [_f32p, _f32p, _i32p, _f32p, _f32p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_int, _f32p, _f32p, _i32p]
        L.shim_fit.restype = ctypes.c_int
        L.shim_fit.argtypes = [ctypes.c_int, ctypes.c_int] + common
        L.shim_fit_steered.restype = ctypes.c_int
        L.shim_fit_steered.argtypes = [ctypes.c_int, ctypes.c_int, _i32p] + common
        _shims_lib = L
    return _shims_lib


def _shim_call(fn, ev, pflags, chunk, *lead):
    c = np.ascontiguousarray
    n, nl = ev.n, ev.hit_pos.shape[0]
    out = (np.zeros((6, n), np.float32), np.zeros((21, n), np.float32), np.zeros(n, np.int32))
    rl, xi = c(ev.rl_grid, np.float32), c(ev.xi_grid, np.float32)
    rc = fn(n, nl, *lead, c(ev.par, np.float32), c(ev.err, np.float32), c(ev.chg, np.int32),
            c(ev.hit_pos, np.float32), c(ev.hit_err, np.float32), rl.ctypes.data, xi.ctypes.data,
            int(pflags), int(chunk), *out)
    if rc != 0:
        raise RuntimeError(f"{fn.__name__} failed rc={rc}")
    return out


def shim_fit(ev, pflags=2, chunk=8):
    """The reference's fitting loop (runFittingTestPlex) with the
    MkFitterGpu adapter in place of MkFitter, `chunk` tracks per call
    (oracle/shim_driver.cc). Returns (par, err, chg)."""
    return _shim_call(_shims().shim_fit, ev, pflags, chunk)


def shim_fit_steered(ev, pflags=2, chunk=8):
    """InputTracksAndHits -> FitTracksSteered -> OutputFittedTracks with
    MkFitterGpu, steps steered by ev.endcap_mask. Returns (par, err, chg)."""
    nl = ev.hit_pos.shape[0]
    barrel = np.array([0 if (int(ev.endcap_mask) >> l) & 1 else 1 for l in range(nl)], np.int32)
    return _shim_call(_shims().shim_fit_steered, ev, pflags, chunk, barrel)


def shim_ops(par, err, chg, hit_pos, hit_err, target, endcap, rl_grid, xi_grid, pflags=2):
    """The finding operator table on n states through the reference's
    FindingFoos and through FindingFoosGpu (oracle/shim_driver.cc
    shim_ops): propagation to `target`, propagation to the hits with the
    chi2 and with the update. Returns a dict of [2][...] arrays (0 the
    reference, 1 the GPU): prop_par, prop_err, chi2, chi2_par, upd_par,
    upd_err, upd_chg."""
    L = ctypes.CDLL(shims_lib_path())
    L.shim_ops.restype = ctypes.c_int
    L.shim_ops.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p, _i32p, _f32p, _f32p,
                           ctypes.c_float, _f32p, _f32p, ctypes.c_int, _f32p, _f32p, _f32p,
                           _f32p, _f32p, _f32p, _i32p]
    c = np.ascontiguousarray
    n = int(len(chg))
    o = dict(prop_par=np.zeros((2, 6, n), np.float32), prop_err=np.zeros((2, 21, n), np.float32),
             chi2=np.zeros((2, n), np.float32), chi2_par=np.zeros((2, 6, n), np.float32),
             upd_par=np.zeros((2, 6, n), np.float32), upd_err=np.zeros((2, 21, n), np.float32),
             upd_chg=np.zeros((2, n), np.int32))
    rc = L.shim_ops(n, int(endcap), c(par, np.float32), c(err, np.float32), c(chg, np.int32),
                    c(hit_pos, np.float32), c(hit_err, np.float32), float(target),
                    c(rl_grid, np.float32), c(xi_grid, np.float32), int(pflags), o["prop_par"],
                    o["prop_err"], o["chi2"], o["chi2_par"], o["upd_par"], o["upd_err"],
                    o["upd_chg"])
    if rc != 0:
        raise RuntimeError(f"shim_ops failed rc={rc}")
    return o
