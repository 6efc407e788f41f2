"""Pins the oracle: the FP64 restatement against the reference's own CPU
Matriplex fit (compiled from the reference sources) and against the golden
fixtures that reference produced."""
import glob
import os

import numpy as np
import pytest

from mkfit_b200 import synth
from tests.tolerances import par_scaled_err, cov_scaled_err

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "fit_*.npz")))


def _grids(g):
    return synth.toy_material_grid(g["radii"])


@pytest.mark.parametrize("path", GOLDEN, ids=os.path.basename)
def test_reference_reproduces_golden(reflib, path):
    """The in-process reference build reproduces the committed fixtures
    bit for bit (same Matriplex width)."""
    g = np.load(path)
    if reflib.width() != int(g["matriplex_width"]):
        pytest.skip("fixture made with another Matriplex width")
    rl, xi = _grids(g)
    par, err, chg, _ = reflib.fit(g["par"], g["err"], g["chg"], g["hit_pos"], g["hit_err"], rl, xi,
                                  pflags=int(g["pflags"]))
    np.testing.assert_array_equal(par, g["ref_par"])
    np.testing.assert_array_equal(err, g["ref_err"])
    np.testing.assert_array_equal(chg, g["ref_chg"])


@pytest.mark.parametrize("path", GOLDEN, ids=os.path.basename)
def test_restatement_matches_golden(restate, path):
    """FP64 restatement vs the reference's FP32 outputs: agreement at the
    level of FP32 rounding of the same algorithm."""
    g = np.load(path)
    rl, xi = _grids(g)
    par, err, _ = restate.fit(g["par"], g["err"], g["chg"], g["hit_pos"], g["hit_err"], rl, xi,
                              pflags=int(g["pflags"]))
    ep = par_scaled_err(g["ref_par"], par, err)
    ec = cov_scaled_err(g["ref_err"], err)
    assert np.median(ep) < 1e-6
    assert ep.max() < 1e-3
    assert np.median(ec) < 1e-5
    assert ec.max() < 5e-3


def test_restatement_matches_reference_fresh(reflib, restate):
    """Same check on a fresh 2000-track toy event run through the reference
    build (not only the fixtures)."""
    ev = synth.gen_fit_event(2000, seed=77)
    par, err, _, _ = reflib.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                ev.xi_grid, pflags=2)
    dpar, derr, chi2 = restate.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                   ev.xi_grid, pflags=2)
    ep = par_scaled_err(par, dpar, derr)
    ec = cov_scaled_err(err, derr)
    assert np.percentile(ep, 99.9) < 1e-4
    assert np.percentile(ec, 99.9) < 1e-3
    # Physics sanity of the synthetic event + fit: chi2/ndf of order 1.
    assert 0.3 < np.median(chi2) / 20 < 2.0


def test_reference_threads_deterministic(reflib):
    """The reference's results do not depend on the shim's thread count."""
    ev = synth.gen_fit_event(1000, seed=5)
    reflib.set_threads(1)
    a = reflib.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid, ev.xi_grid)
    reflib.set_threads(4)
    b = reflib.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid, ev.xi_grid)
    reflib.set_threads(1)
    for x, y in zip(a[:3], b[:3]):
        np.testing.assert_array_equal(x, y)


def test_restated_backward_fit_matches_reference(reflib, restate):
    """The FP64 restatement of the backward fit (oracle.restate_backward_fit,
    with the reference's NN-wide seed groups) reproduces the reference's own
    MkBuilder::BackwardFit from the same finding result, within the FP32
    error of the reference's fit (median at rounding level)."""
    import numpy as np
    from mkfit_b200 import synth
    from mkfit_b200.geometry import cms2017
    from oracle.oracle import ref_find, restate_backward_fit
    ev = synth.gen_cms_event(400, seed=7, noise_frac=0.01)
    m = 6
    ref0 = ref_find(reflib, ev, max_cands=m)
    ref = ref_find(reflib, ev, max_cands=m, backward_fit=True)
    par, err, chi2 = restate_backward_fit(restate, ev, ref0, cms2017(), m)
    slots = np.arange(ev.n_seeds) * m
    r = ref["chi2"][slots]
    ok = np.isfinite(r) & np.isfinite(chi2) & (chi2 < 1e6)
    assert ok.mean() > 0.99
    rel = np.abs(r[ok] - chi2[ok]) / np.maximum(np.abs(chi2[ok]), 1e-3)
    assert np.median(rel) < 1e-4, np.median(rel)
    assert np.percentile(rel, 99) < 1e-2, np.percentile(rel, 99)
    dpar = np.abs(ref["par"][slots][ok] - par[ok]) / np.sqrt(np.maximum(err[ok][:, [0, 2, 5, 9, 14, 20]], 1e-30))
    assert np.median(dpar) < 1e-3


def test_reference_steered_fit_matches_restatement(reflib, restate):
    """The reference's steered fit (MkFitter::FitTracksSteered: barrel steps,
    then endcap steps) agrees with the FP64 restatement given the same
    endcap mask, within the reference's FP32 error."""
    import numpy as np
    from mkfit_b200 import synth
    from tests.tolerances import PAR_RTOL, par_scaled_err
    ev = synth.gen_fit_event_steered(2000, seed=21)
    par, err, chg = reflib.fit_steered(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err,
                                       ev.endcap_mask, ev.rl_grid, ev.xi_grid, pflags=2)
    dpar, derr, _ = restate.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                ev.xi_grid, pflags=2, endcap_mask=ev.endcap_mask)
    ep = par_scaled_err(par, dpar, derr)
    assert np.median(ep) < 1e-6
    assert np.percentile(ep, 99.9) < PAR_RTOL
    # Fitting the disks as barrel layers is far off: the mask matters.
    bpar, _, _ = reflib.fit_steered(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, 0,
                                    ev.rl_grid, ev.xi_grid, pflags=2)
    assert np.median(par_scaled_err(bpar, dpar, derr)) > 1e-3


def test_restated_candidate_replay_matches_reference(reflib, restate):
    """The FP64 replay of clone-engine candidates (restate_replay_cands)
    reproduces the reference's own FP32 candidates: bulk at FP32 rounding,
    the same charges; the tails are the reference's FP32 accumulation."""
    from mkfit_b200 import synth
    from oracle.oracle import ref_find, restate_replay_cands
    from tests.tolerances import cov_scaled_err, par_scaled_err
    m = 6
    ev = synth.gen_cms_event(600, seed=21, noise_frac=0.05)
    o = ref_find(reflib, ev, max_cands=m, chi2_cut=30.0, zero_c2=True)
    slots = np.array([s * m + c for s in range(ev.n_seeds) for c in range(o["n_cands"][s])])
    par, err, chg, chi2 = restate_replay_cands(restate, ev, o, m, slots)
    ep = par_scaled_err(o["par"][slots].T, par.T, err.T)
    ec = cov_scaled_err(o["err"][slots].T, err.T)
    rc = np.abs(o["chi2"][slots] - chi2) / np.maximum(np.abs(chi2), 1e-3)
    np.testing.assert_array_equal(chg, o["chg"][slots])
    assert np.median(ep) < 1e-6 and np.percentile(ep, 99.9) < 1e-3
    assert np.median(ec) < 1e-5 and np.percentile(ec, 99) < 1e-3
    assert np.median(rc) < 1e-4 and np.percentile(rc, 99.9) < 1e-2
