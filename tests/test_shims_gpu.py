"""The MkFitterGpu adapter (mkfit_b200/shims/MkFitterGpu.h) at a reference
call site: the reference's own fitting loop (runFittingTestPlex,
mkFit/fittestMPlex.cc:65-100) and the steered seed fit, compiled against
the reference's Track / Hit / Config types with MkFitterGpu in place of
MkFitter (oracle/shim_driver.cc). Its results equal the library's direct
fit bit for bit, whether the loop hands the adapter NN tracks or the whole
range, and match the reference's MkFitter within the fit tolerances."""
import numpy as np
import pytest

from mkfit_b200 import synth
from oracle.oracle import have_shims, shim_fit, shim_fit_steered
from tests.test_fit_gpu import assert_parity, gpu_fit

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_shims(), reason="adapter driver not built")]


def _same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_fit_loop_through_mkfitter_adapter(gpu_ctx, reflib):
    ev = synth.gen_fit_event(5003, seed=77)
    chunked = shim_fit(ev, pflags=2, chunk=reflib.width())
    whole = shim_fit(ev, pflags=2, chunk=ev.n)
    _same(chunked, whole)
    direct = gpu_fit(gpu_ctx, ev, pflags=2)
    _same(chunked, (direct["par"], direct["err"], direct["chg"]))
    par, err, chg, _ = reflib.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                  ev.xi_grid, pflags=2)
    assert_parity(chunked[0], chunked[1], par, err, "MkFitterGpu loop")
    np.testing.assert_array_equal(chunked[2], chg)


def test_steered_fit_through_mkfitter_adapter(gpu_ctx, reflib):
    ev = synth.gen_fit_event_steered(4001, seed=78)
    chunked = shim_fit_steered(ev, pflags=2, chunk=reflib.width())
    whole = shim_fit_steered(ev, pflags=2, chunk=ev.n)
    _same(chunked, whole)
    direct = gpu_fit(gpu_ctx, ev, pflags=2)
    _same(chunked, (direct["par"], direct["err"], direct["chg"]))
    par, err, chg = reflib.fit_steered(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err,
                                       ev.endcap_mask, ev.rl_grid, ev.xi_grid, pflags=2)
    assert_parity(chunked[0], chunked[1], par, err, "MkFitterGpu steered")
    np.testing.assert_array_equal(chunked[2], chg)


@pytest.mark.parametrize("endcap", [0, 1])
def test_finding_operator_table_through_adapter(gpu_ctx, endcap):
    """The finding operator table (FindingFoos) with the GPU operators of
    FindingFoosGpu against the reference's own table on the same Matriplex
    inputs, NN lanes per call as MkFinder calls them: propagation to a
    layer, propagation to the hit with the chi2, and with the update, for
    the barrel (r) and the endcap (z) member."""
    from oracle.oracle import Restate, shim_ops
    from tests.tolerances import CHI2_RTOL, COV_RTOL, PAR_RTOL, cov_scaled_err, par_scaled_err
    if endcap:
        ev = synth.gen_fit_event_steered(3000, seed=79)
        keep = ev.hit_pos[2, 2] > 0      # forward side: one target z for all
        step, target = 2, float(ev.disks_z[0])
    else:
        ev = synth.gen_fit_event(3001, seed=80)
        keep = np.ones(ev.n, bool)
        step, target = 0, float(ev.radii[0])
    sel = lambda a: np.ascontiguousarray(a[..., keep])  # noqa: E731
    par, err, chg = sel(ev.par), sel(ev.err), sel(ev.chg)
    hp, he = sel(ev.hit_pos[step]), sel(ev.hit_err[step])
    o = shim_ops(par, err, chg, hp, he, target, endcap, ev.rl_grid, ev.xi_grid, pflags=2)
    n = len(chg)
    for k in ("prop", "upd"):
        ep = par_scaled_err(o[k + "_par"][1], o[k + "_par"][0], o[k + "_err"][0])
        ec = cov_scaled_err(o[k + "_err"][1], o[k + "_err"][0])
        print(f"\n{k} ({n} states, endcap={endcap}): par p999 {np.percentile(ep, 99.9):.3g} "
              f"cov p999 {np.percentile(ec, 99.9):.3g}")
        assert np.percentile(ep, 99.9) < PAR_RTOL
        if k == "prop":
            assert np.percentile(ec, 99.9) < COV_RTOL
    # The update's C - K H C cancels for these loose states on a disk (a
    # 1 cm-wide start propagated 35 cm to a 0.01 cm hit): both FP32 results
    # are held against the FP64 restatement of the same step, the GPU at
    # most 1.5 x as far from it as the reference.
    rs = Restate()
    dp, de, _ = rs.fit(par, err, chg, hp[None], he[None], ev.rl_grid, ev.xi_grid, pflags=2,
                       endcap_mask=endcap)
    ok = dp[3] > 0
    g64 = cov_scaled_err(o["upd_err"][1][:, ok], de[:, ok])
    r64 = cov_scaled_err(o["upd_err"][0][:, ok], de[:, ok])
    print(f"upd vs FP64 cov p999: GPU {np.percentile(g64, 99.9):.3g} reference "
          f"{np.percentile(r64, 99.9):.3g}")
    assert np.percentile(g64, 99.9) <= 1.5 * np.percentile(r64, 99.9) + 1e-6
    ep = par_scaled_err(o["chi2_par"][1], o["chi2_par"][0], err)
    rc = np.abs(o["chi2"][1] - o["chi2"][0]) / np.maximum(np.abs(o["chi2"][0]), 1e-3)
    print(f"chi2: rel p999 {np.percentile(rc, 99.9):.3g}; propagated parameters p999 "
          f"{np.percentile(ep, 99.9):.3g}")
    assert np.percentile(rc, 99.9) < CHI2_RTOL
    assert np.percentile(ep, 99.9) < PAR_RTOL
    np.testing.assert_array_equal(o["upd_chg"][1], o["upd_chg"][0])
