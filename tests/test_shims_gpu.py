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
