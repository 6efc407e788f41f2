"""Quality filters and duplicate removal of run_OneIteration.

CPU: the oracle's restatements (oracle.restate_qfilters, restate_dups)
against the reference's own StdSeq functions (oracle/_ref through
ref_qfilters / ref_dups) on synthetic candidates built to reach every branch
of the cuts: hit lists with holes (-1, -2, -3, -7), -9 hits, overlap hits on
one layer, stereo / mono layer pairs, seeds of 2 to 16 hits (the 4-bit seed
hit count), parameters on the 1/pT and theta thresholds, d0 around the 0.5
and 1 mm cuts, NaN / negative covariances; duplicate families that share hits
and sit inside or outside the (dphi, dcot theta) and (dphi, deta) windows,
score ties, repeated labels, tracks without hits.

GPU: the device filters (mkfg_find_filter) and duplicate removal modes
(mkfg_find_select) on the device's own candidates against the reference
evaluated on the same candidates, and run_OneIteration's order (finding,
filter with removal, backward fit, filter, selection) against the reference's
whole sequence.

Bar: bit-exact (every verdict is an integer function of float32 inputs that
both sides compute with the same operations and contractions)."""
import numpy as np
import pytest

from mkfit_b200.geometry import cms2017
from oracle.oracle import (DUP_MODES, QF_KINDS, ref_dups, ref_qfilters, restate_dups,
                           restate_qfilters)

f32 = np.float32
W = 64
PI_OVER_2 = f32(f32(3.14159265358979323846) / f32(2.0))


def layer_flags():
    g = cms2017()
    return g.field("is_pix") > 0.5, g.field("is_stereo") > 0.5


def synthetic_cands(n, seed):
    """Candidates as exported hit lists (chain order, seed hits first)."""
    rng = np.random.default_rng(seed)
    is_pix, _ = layer_flags()
    pix_layers = np.nonzero(is_pix)[0]
    par = np.zeros((n, 6), f32)
    par[:, 0] = rng.normal(0, 0.08, n)
    par[:, 1] = rng.normal(0, 0.08, n)
    par[:, 2] = rng.normal(0, 5, n)
    ipt = rng.uniform(0.05, 3.0, n).astype(f32)
    pick = rng.random(n)
    ipt[pick < 0.1] = f32(1.11)
    ipt[(pick >= 0.1) & (pick < 0.2)] = f32(1.43)
    par[:, 3] = ipt
    par[:, 4] = rng.uniform(-np.pi, np.pi, n)
    theta = rng.uniform(0.15, 3.0, n).astype(f32)
    pick = rng.random(n)
    for lo, v in ((0.0, 1.11), (0.05, -1.11), (0.1, 0.80), (0.15, -0.80)):
        sel = (pick >= lo) & (pick < lo + 0.05)
        theta[sel] = f32(PI_OVER_2 + f32(v))
    par[:, 5] = theta
    err = np.zeros((n, 21), f32)
    diag = [0, 2, 5, 9, 14, 20]
    err[:, diag] = rng.uniform(1e-4, 1e-2, (n, 6))
    off = [k for k in range(21) if k not in diag]
    err[:, off] = rng.normal(0, 1e-5, (n, len(off)))
    pick = rng.random(n)
    err[pick < 0.03, 9] = -1e-3
    err[(pick >= 0.03) & (pick < 0.06), 4] = np.nan
    err[(pick >= 0.06) & (pick < 0.08), 13] = np.inf
    chg = rng.choice([-1, 1], n).astype(np.int32)
    nseed = rng.choice([2, 3, 3, 4, 4, 4, 5, 6, 8, 15, 16], n).astype(np.int32)
    ntot = np.zeros(n, np.int32)
    hit_idx = np.full((n, W), -100, np.int32)
    hit_lyr = np.full((n, W), -100, np.int32)
    for i in range(n):
        if rng.random() < 0.2:
            lay = sorted(rng.choice([0, 1, 2, 18, 19, 45, 46], min(nseed[i], 3), replace=False))
            lay = (lay + list(rng.choice(pix_layers, nseed[i])))[:nseed[i]]
        else:
            lay = sorted(rng.choice(pix_layers, nseed[i]))
        hits = [(int(rng.integers(0, 5000)), int(l_)) for l_ in lay]
        more = 0 if rng.random() < 0.15 else int(rng.integers(1, 26))
        prev = max(lay)
        for _ in range(more):
            r = rng.random()
            if r < 0.1:
                lyr = prev
            elif r < 0.2:
                lyr = int(rng.integers(0, 72))
            else:
                lyr = min(prev + int(rng.choice([1, 1, 1, 2, 3])), 71)
            idx = int(rng.integers(0, 5000)) if rng.random() < 0.75 else int(
                rng.choice([-1, -1, -1, -2, -3, -7, -9]))
            hits.append((idx, lyr))
            prev = lyr
        hits = hits[:W]
        ntot[i] = len(hits)
        hit_idx[i, :len(hits)] = [h[0] for h in hits]
        hit_lyr[i, :len(hits)] = [h[1] for h in hits]
    return dict(par=par, err=err, chg=chg, ntot=ntot, hit_idx=hit_idx, hit_lyr=hit_lyr), nseed


def synthetic_tracks(n_fam, seed):
    """Exported tracks in duplicate families (hits without missing entries)."""
    rng = np.random.default_rng(seed)
    rows = []
    for fam in range(n_fam):
        size = 1 if rng.random() < 0.3 else int(rng.integers(2, 5))
        phi = rng.uniform(-np.pi, np.pi)
        if rng.random() < 0.1:
            phi = np.pi - 1e-3
        theta = rng.uniform(0.1, 3.0)
        ipt = rng.uniform(0.1, 3.0)
        nb = int(rng.integers(3, 16))
        base = [(int(rng.integers(0, 3000)), lyr) for lyr in sorted(rng.choice(72, nb, replace=False))]
        for m in range(size):
            spread = rng.choice([1e-4, 1e-3, 5e-3, 3e-2, 0.5])
            p = np.array([0, 0, 0, ipt + rng.choice([0.0, 0.01, 0.6, 2.0]) * (m > 0),
                          phi + rng.normal(0, spread) * (m > 0),
                          theta + rng.normal(0, spread) * (m > 0)], np.float64)
            p[4] = (p[4] + np.pi) % (2 * np.pi) - np.pi
            keep = rng.random(nb) < rng.choice([0.1, 0.5, 0.9, 1.0])
            hits = [h for h, k in zip(base, keep) if k or m == 0]
            hits += [(int(rng.integers(3000, 6000)), int(rng.integers(0, 72)))
                     for _ in range(int(rng.integers(0, 5)))]
            if rng.random() < 0.03:
                hits = []
            rows.append((p, hits, fam))
    order = rng.permutation(len(rows))
    rows = [rows[i] for i in order]
    n = len(rows)
    par = np.array([r[0] for r in rows], f32)
    nh = np.array([len(r[1]) for r in rows], np.int32)
    hit_idx = np.full((n, W), -100, np.int32)
    hit_lyr = np.full((n, W), -100, np.int32)
    for i, r in enumerate(rows):
        hit_idx[i, :nh[i]] = [h[0] for h in r[1]]
        hit_lyr[i, :nh[i]] = [h[1] for h in r[1]]
    score = rng.normal(0, 10, n).astype(f32)
    tie = rng.random(n) < 0.1
    score[tie] = f32(5.0)
    label = np.arange(n, dtype=np.int32)
    rep = np.nonzero(rng.random(n) < 0.05)[0]
    label[rep] = label[np.maximum(rep - 1, 0)]
    return dict(par=par, chg=rng.choice([-1, 1], n).astype(np.int32), score=score, label=label,
                nfound=nh.copy(), nh=nh, hit_idx=hit_idx, hit_lyr=hit_lyr)


@pytest.mark.parametrize("min_hits,beam", [(4, (0.0, 0.0)), (3, (0.03, -0.02))])
def test_qfilter_restatement_matches_reference(reflib, min_hits, beam):
    cands, nseed = synthetic_cands(3000, 7 + min_hits)
    is_pix, is_stereo = layer_flags()
    ref = ref_qfilters(reflib, cands, nseed, min_hits, beam)
    got = restate_qfilters(cands, nseed, is_pix, is_stereo, min_hits, beam)
    for k, name in enumerate(QF_KINDS):
        r, g = (ref >> k) & 1, (got >> k) & 1
        bad = np.nonzero(r != g)[0]
        assert len(bad) == 0, f"{name}: {len(bad)} differ, first {bad[:5]}"
        # Each filter both passes and fails some candidates.
        assert 0 < r.sum() < len(r), name


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_dup_restatement_matches_reference(reflib, mode):
    tracks = synthetic_tracks(250, 30 + mode)
    frac, drth = (0.24, (0.002, 0.004, 0.008)) if mode != 1 else (0.14, (0.0, 0.0, 0.0))
    ref = ref_dups(reflib, mode, tracks, frac=frac, drth=drth)
    got = restate_dups(mode, tracks, frac=frac, drth=drth)
    np.testing.assert_array_equal(got, ref, err_msg=DUP_MODES[mode])
    assert 0 < ref.sum() < len(ref)


def _pair(ph, th, hits=((1, 4), (2, 4))):
    par = np.zeros((2, 6), f32)
    par[:, 3] = 1.0
    par[:, 4] = ph
    par[:, 5] = th
    return dict(par=par, chg=np.array([1, 1], np.int32), score=np.array([2.0, 1.0], f32),
                label=np.array([0, 1], np.int32), nfound=np.array([5, 5], np.int32),
                nh=np.array([1, 1], np.int32), hit_idx=np.array([[hits[0][0]], [hits[1][0]]], np.int32),
                hit_lyr=np.array([[hits[0][1]], [hits[1][1]]], np.int32))


def test_dup_window_contraction(reflib):
    """Pairs whose dphi^2 + d^2 lands on the window edge differently with and
    without an FMA: the reference decides them as fma(dphi, dphi, d*d), and
    so do the restatement and the device. pixelseed: threshold tuned to the
    pair; find_duplicates: fixed maxdR, the pair's dphi scanned to the edge
    (phi near 0, where float steps are fine)."""
    from oracle.oracle import _fma32, _libm_f32, _squash_phi_minimal
    rng = np.random.default_rng(5)
    tan = lambda v: _libm_f32("tanf", [v])[0]  # noqa: E731
    log = lambda v: _libm_f32("logf", [v])[0]  # noqa: E731
    split = lambda a, b: (f32(f32(a * a) + f32(b * b)), _fma32(a, a, f32(b * b)))  # noqa: E731
    found = 0
    while found < 8:
        th1 = f32(rng.uniform(1.2, 1.9))
        ph1 = f32(rng.uniform(-3, 3))
        th2 = f32(th1 + f32(rng.uniform(-0.002, 0.002)))
        ph2 = f32(ph1 + f32(rng.uniform(-0.002, 0.002)))
        a = abs(_squash_phi_minimal(f32(ph1 - ph2)))
        b = abs(f32(f32(f32(1.0) / tan(th2)) - f32(f32(1.0) / tan(th1))))
        plain, fused = split(a, b)
        if plain == fused:
            continue
        v = max(plain, fused)
        d = f32(np.sqrt(np.float64(v)))
        ds = [x for x in (np.nextafter(d, f32(0)), d, np.nextafter(d, f32(1))) if f32(x * x) == v]
        if not ds:
            continue
        tr = _pair([ph1, ph2], [th1, th2])
        drth = (float(ds[0]),) * 3
        ref = ref_dups(reflib, 0, tr, frac=100.0, drth=drth)
        assert ref[1] == (0 if fused < v else 1)
        np.testing.assert_array_equal(restate_dups(0, tr, frac=100.0, drth=drth), ref)
        found += 1
    eta_of = lambda th: f32(f32(-1.0) * log(tan(f32(th / f32(2.0)))))  # noqa: E731
    found = 0
    while found < 4:
        th1 = f32(rng.uniform(0.3, 2.8))
        e1 = eta_of(th1)
        mult = f32(16.0) if abs(e1) > 2.5 else (f32(9.0) if abs(e1) > 1.44 else f32(1.0))
        thr = f32(f32(f32(0.0025) * f32(0.0025)) * mult)
        th2 = f32(th1 - rng.uniform(0.2, 0.8) * np.sqrt(thr) * np.sin(th1))
        b = abs(f32(eta_of(th2) - e1))
        ph1 = f32(-np.sqrt(float(thr) - float(b) ** 2) / 2)
        p2 = f32(ph1 + np.sqrt(float(thr) - float(b) ** 2))
        for k in range(2000):
            a = abs(_squash_phi_minimal(f32(ph1 - p2)))
            plain, fused = split(a, b)
            if (plain < thr) != (fused < thr):
                tr = _pair([ph1, p2], [th1, th2])
                ref = ref_dups(reflib, 2, tr)
                assert ref[1] == (0 if fused < thr else 1)
                np.testing.assert_array_equal(restate_dups(2, tr), ref)
                found += 1
                break
            # One float step of the second phi towards the window edge.
            p2 = np.nextafter(p2, f32(-10) if plain >= thr else f32(10))


def test_dup_edge_cases(reflib):
    """find_duplicates does nothing for pixelLess / tobTec tracks (algorithm
    9, 10); 'none' keeps everything; an empty input is fine."""
    tracks = synthetic_tracks(60, 41)
    n = len(tracks["chg"])
    for algo in (9, 10):
        assert ref_dups(reflib, 2, tracks, algo=algo).sum() == n
        assert restate_dups(2, tracks, algo=algo).sum() == n
    assert ref_dups(reflib, 3, tracks).sum() == n
    empty = {k: v[:0] for k, v in tracks.items()}
    for mode in range(4):
        assert len(ref_dups(reflib, mode, empty)) == 0


def test_iteration_table_matches_reference(reflib):
    """The per-iteration selection table of the host mirror follows the
    reference's CMS-2017 iteration settings through run_OneIteration's
    branches."""
    from mkfit_b200.finder import (DUP_PIXELSEED, DUP_SHAREDHITS, ITERATION_SELECTION, QF_N_HITS,
                                   QF_N_HITS_PIXSEED, QF_N_LAYERS, QF_PIXELLESS_BKWD,
                                   QF_PIXELLESS_FWD)
    from oracle.oracle import ref_cms2017_iteration
    for it, sel in ITERATION_SELECTION.items():
        r = ref_cms2017_iteration(reflib, it)
        algo, qf, tight = r["algorithm"], r["quality_filter"], r["dupclean_tight"]
        assert sel["algorithm"] == algo, it
        pre = None
        if qf and algo != 7:
            pre = QF_N_HITS_PIXSEED if algo == 6 else (QF_PIXELLESS_FWD if algo == 9 else QF_N_HITS)
        post = (QF_N_LAYERS if algo == 7 else QF_PIXELLESS_BKWD) if qf and algo in (7, 9) else None
        assert (sel["pre"], sel["post"]) == (pre, post), it
        assert sel["min_hits"] == (3 if algo == 6 else r["min_hits_qf"]), it
        assert sel["mode"] == (DUP_SHAREDHITS if qf and not tight else DUP_PIXELSEED), it
        assert sel["sort_seed_hits"] == r["sort_seed_hits"], it
        assert np.float32(sel["frac_shared_hits"]) == np.float32(r["frac_shared_hits"]), it
        assert tuple(np.float32(sel["drth"])) == tuple(np.float32(r["drth"])), it


# ---------------------------------------------------------------------------
# Device
# ---------------------------------------------------------------------------

M = 6
QF_D0_CUTS = (0.05, 0.1)


def _finder(gpu_ctx):
    from mkfit_b200.finder import FindConfig, Finder
    return Finder(gpu_ctx, FindConfig(max_cands=M, chi2_cut=30.0, zero_c2=True))


def _take(c, sel):
    return {k: v[sel] for k, v in c.items() if k != "n_cands"}


@pytest.mark.gpu
@pytest.mark.parametrize("stage", ["found", "bkfit", "bksearch"])
def test_device_filters_match_reference(gpu_ctx, reflib, stage):
    """Every filter on the device's best candidates equals the reference's
    filter on the same candidates (rebuilt as TrackCands), after the clone
    engine, after the backward fit and after the backward search. A verdict
    may differ only where |d0| lies within 2e-6 of the helix radius of a d0
    cut (the device's sin / cos are correctly rounded, the host's sinf /
    cosf are off by one ulp for ~1% of angles)."""
    from mkfit_b200 import synth
    from oracle.oracle import d0_beam_spot
    ev = synth.thinned(synth.gen_cms_event(2500, seed=81, noise_frac=0.02), 0.6, 81)
    fnd = _finder(gpu_ctx)
    fnd.upload(ev)
    fnd.run()
    if stage != "found":
        fnd.backward_fit()
    if stage == "bksearch":
        fnd.backward_search()
    c = fnd.download_best(ev.n_seeds)
    has = c["n_cands"] > 0
    cands = _take(c, has)
    nseed = ev.seed_nhits[has]
    fails = np.zeros(len(QF_KINDS), int)
    for beam in ((0.0, 0.0), (0.08, -0.05), (0.3, 0.2)):
        d0, radius = d0_beam_spot(cands["par"].T, cands["chg"], beam)
        gap = np.min([np.abs(np.abs(d0) - np.float32(cut)) for cut in QF_D0_CUTS], axis=0)
        near = gap < 2e-6 * radius + 1e-6
        for min_hits in (3, 4):
            ref = ref_qfilters(reflib, cands, nseed, min_hits, beam)
            for k, name in enumerate(QF_KINDS):
                got = fnd.filter(ev.n_seeds, k, min_hits, beam)
                assert (got[~has] == -1).all(), name
                g, r = got[has], (ref >> k) & 1
                bad = np.nonzero(g != r)[0]
                assert near[bad].all(), f"{name} beam {beam} min_hits {min_hits}: {len(bad)} differ"
                fails[k] += int((r == 0).sum())
    print(f"\nfilters ({stage}): failing candidates per filter {dict(zip(QF_KINDS, fails))}")
    # Every filter but the NaN / silly one fails some candidates.
    assert fails[1:].min() > 0


def _sorted_exports(c, begin, order, silly_ok=False):
    """Exported tracks (export_best_comb_cands(.., true)) of one event in the
    seed order: candidates that exist and pass the NaN / silly filter, hits
    without missing entries. Returns (tracks, input indices)."""
    idx = begin + np.asarray(order)
    err = c["err"][idx]
    diag = err[:, [0, 2, 5, 9, 14, 20]]
    silly = (diag < 0).any(axis=1) | ~np.isfinite(err).all(axis=1)
    idx = idx[(c["n_cands"][idx] > 0) & ~silly]
    n = len(idx)
    hi = np.full((n, 64), -100, np.int32)
    hl = np.full((n, 64), -100, np.int32)
    nh = np.zeros(n, np.int32)
    for r, s in enumerate(idx):
        m = c["hit_idx"][s, :c["ntot"][s]] >= 0
        h = c["hit_idx"][s, :c["ntot"][s]][m]
        nh[r] = len(h)
        hi[r, :len(h)] = h
        hl[r, :len(h)] = c["hit_lyr"][s, :c["ntot"][s]][m]
    return dict(par=c["par"][idx], chg=c["chg"][idx], score=c["score"][idx],
                label=(idx - begin).astype(np.int32), nfound=c["nfound"][idx], nh=nh, hit_idx=hi,
                hit_lyr=hl), idx


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_device_dup_modes_match_reference(gpu_ctx, reflib, mode):
    """The device's duplicate removal (mkfg_find_select, each mode) on a
    batch of two events whose seeds include near-duplicates equals the
    reference's function run on the device's own exported tracks, per
    event in the seed order: bit-exact."""
    from mkfit_b200 import synth
    from mkfit_b200.seed_clean import cleaned_event
    from mkfit_b200.finder import SELECT_ITER0
    from oracle.oracle import ref_event_prep
    evs = []
    for i, n in enumerate((1800, 900)):
        ev = synth.gen_cms_event(n, seed=91 + i, noise_frac=0.02)
        sd = synth.with_duplicate_seeds(ev, frac=0.3, seed=91 + i)
        k = len(sd["chg"])
        evs.append(cleaned_event(ev, sd, (np.ones(k, np.int32), sd["nhits"], sd["hit_layer"],
                                          sd["hit_index"])))
    frac, drth = (0.14, (0.001, 0.001, 0.001)) if mode == 1 else (0.24, (0.002, 0.004, 0.008))
    fnd = _finder(gpu_ctx)
    fnd.upload_batch(evs)
    fnd.run()
    N = sum(e.n_seeds for e in evs)
    keep = fnd.select(N, mode=mode, algorithm=4, frac_shared_hits=frac, drth_central=drth[0],
                      drth_obarrel=drth[1], drth_forward=drth[2])
    c = fnd.download_best(N)
    exp = np.zeros(N, np.int32)
    begin = 0
    for e in evs:
        tracks, idx = _sorted_exports(c, begin, ref_event_prep(reflib, e)["seed_order"])
        exp[idx] = ref_dups(reflib, mode, tracks, algo=4, frac=frac, drth=drth)
        begin += e.n_seeds
    np.testing.assert_array_equal(keep, exp)
    removed = int((c["n_cands"] > 0).sum() - keep.sum())
    print(f"\n{DUP_MODES[mode]}: {N} seeds, {removed} removed")
    if mode != 3:
        assert removed > 0


@pytest.mark.gpu
@pytest.mark.parametrize("it", [5, 7, 8, 9])
def test_iteration_selection_matches_reference(gpu_ctx, reflib, it):
    """run_OneIteration's steps after the clone engine with the selection of
    CMS-2017 iteration `it` (its filter with removal after the finding, the
    backward fit over the remaining seeds, its filter after the backward
    fit, duplicate removal) on the iteration-0 finding of an event with half
    its strip hits removed (short candidates, which the filters drop),
    against the same
    sequence run by the reference: the same seeds removed and kept for
    >= 99% of the seeds (the rest are finding near-ties)."""
    from mkfit_b200 import synth
    from mkfit_b200.finder import ITERATION_SELECTION
    from oracle.oracle import ref_find
    sel = ITERATION_SELECTION[it]
    beam = (0.02, -0.01)
    ev = synth.thinned(synth.gen_cms_event(1500, seed=100 + it, noise_frac=0.02), 0.5, 100 + it)
    if it == 9:
        # pixelPairStep seeds are hit pairs: qfilter_n_hits_pixseed(3) drops
        # the ones that found nothing.
        ev = synth.without_first_seed_hit(ev)
    ref = ref_find(reflib, ev, max_cands=M, chi2_cut=30.0, zero_c2=True, backward_fit=True,
                   select=True, qf_pre=-1 if sel["pre"] is None else sel["pre"],
                   qf_post=-1 if sel["post"] is None else sel["post"], qf_min_hits=sel["min_hits"],
                   beam=beam, dup_mode=sel["mode"], dup_params=[sel["frac_shared_hits"], *sel["drth"]])
    fnd = _finder(gpu_ctx)
    fnd.upload(ev)
    fnd.run()
    keep = fnd.run_iteration_selection(ev.n_seeds, it, beam_spot=beam)
    c = fnd.download_best(ev.n_seeds)
    present = c["n_cands"] > 0
    ref_present = ref["n_cands"] > 0
    removed = int((~ref_present).sum())
    agree_removed = float((present == ref_present).mean())
    agree_keep = float((keep == ref["keep"]).mean())
    print(f"\niteration {it}: {ev.n_seeds} seeds, removed by filters {removed} "
          f"(device {int((~present).sum())}), agree {agree_removed:.4f}, kept {int(keep.sum())}, "
          f"selection agree {agree_keep:.4f}")
    assert agree_removed >= 0.99
    assert agree_keep >= 0.99
    if sel["pre"] is not None or sel["post"] is not None:
        assert removed > 0
