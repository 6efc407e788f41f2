"""The fit entry point that allocates nothing (mkfg_fit_host_static) against
the host-buffer entry point it mirrors (mkfg_fit_host): same inputs, two
calls in a row, outputs equal within the fit tolerances; oversize inputs
are rejected with an error that names the limit.

Collected last (file name) so that it also runs after every other GPU test
has used the device; it passes alone as well."""
import numpy as np
import pytest

from mkfit_b200 import capi, synth
from tests.tolerances import cov_scaled_err, par_scaled_err

pytestmark = pytest.mark.gpu


def _compare(a, b):
    ep = par_scaled_err(a["par"], b["par"], b["err"])
    ec = cov_scaled_err(a["err"], b["err"])
    assert ep.max() < 1e-5 and ec.max() < 1e-4, (ep.max(), ec.max())
    np.testing.assert_array_equal(a["chg"], b["chg"])
    np.testing.assert_allclose(a["chi2"], b["chi2"], rtol=1e-5, atol=1e-6)


def test_static_fit_matches_host_fit_twice(gpu_ctx):
    ev = synth.gen_fit_event(2500, seed=77)
    gpu_ctx.set_material(ev.rl_grid, ev.xi_grid)
    ref = gpu_ctx.fit_host(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2,
                           with_chi2=True)
    for _ in range(2):
        out = gpu_ctx.fit_host_static(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2,
                                      with_chi2=True)
        _compare(out, ref)
    # A smaller batch after a larger one: no stale data from the earlier call.
    small = synth.gen_fit_event(33, seed=78)
    ref_s = gpu_ctx.fit_host(small.par, small.err, small.chg, small.hit_pos, small.hit_err,
                             pflags=2, with_chi2=True)
    out_s = gpu_ctx.fit_host_static(small.par, small.err, small.chg, small.hit_pos,
                                    small.hit_err, pflags=2, with_chi2=True)
    _compare(out_s, ref_s)


def test_static_fit_rejects_oversize(gpu_ctx):
    ev = synth.gen_fit_event(40000, seed=79)
    with pytest.raises(capi.MkfgError) as e:
        gpu_ctx.fit_host_static(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2)
    assert e.value.code == 1  # MKFG_ERR_BAD_INPUT
    assert "fixed device array holds" in str(e.value)
