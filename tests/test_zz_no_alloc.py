"""The fit entry point that allocates nothing (mkfg_fit_host_static) against
the host-buffer entry point it mirrors (mkfg_fit_host): same inputs, two
calls in a row, outputs bit-identical (both launch the same kernel on the
same compacted inputs); the static calls leave the device's free memory
unchanged; oversize inputs are rejected with an error that names the limit.

Collected last (file name) so that it also runs after every other GPU test
has used the device; it passes alone as well."""
import numpy as np
import pytest

from mkfit_b200 import Context, capi, synth

pytestmark = pytest.mark.gpu


def _same(a, b):
    for k in ("par", "err", "chg", "chi2"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_static_fit_matches_host_fit_twice(gpu_ctx):
    ev = synth.gen_fit_event(2500, seed=77)
    gpu_ctx.set_material(ev.rl_grid, ev.xi_grid)
    ref = gpu_ctx.fit_host(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2,
                           with_chi2=True)
    for _ in range(2):
        out = gpu_ctx.fit_host_static(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2,
                                      with_chi2=True)
        _same(out, ref)
    # A smaller batch after a larger one: no stale data from the earlier call.
    small = synth.gen_fit_event(33, seed=78)
    ref_s = gpu_ctx.fit_host(small.par, small.err, small.chg, small.hit_pos, small.hit_err,
                             pflags=2, with_chi2=True)
    out_s = gpu_ctx.fit_host_static(small.par, small.err, small.chg, small.hit_pos,
                                    small.hit_err, pflags=2, with_chi2=True)
    _same(out_s, ref_s)


def test_static_fit_allocates_nothing():
    """On a fresh context: after a first call (which resolves the array's
    address on the device), further static calls leave cudaMemGetInfo's
    free memory unchanged, while the allocating entry point on the same
    context visibly takes device memory for its scratch."""
    import torch
    ev = synth.gen_fit_event(8000, seed=80)
    torch.cuda.mem_get_info(0)  # torch's own set-up happens before the counts
    ctx = Context(0)
    try:
        ctx.set_material(ev.rl_grid, ev.xi_grid)
        first = ctx.fit_host_static(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2,
                                    with_chi2=True)
        free0 = torch.cuda.mem_get_info(0)[0]
        for _ in range(2):
            out = ctx.fit_host_static(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2,
                                      with_chi2=True)
            _same(out, first)
        free1 = torch.cuda.mem_get_info(0)[0]
        assert free1 == free0, (free0, free1)
        ref = ctx.fit_host(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2,
                           with_chi2=True)
        free2 = torch.cuda.mem_get_info(0)[0]
        assert free2 < free1, "the allocating entry point's scratch should show in free memory"
        _same(first, ref)
    finally:
        ctx.close()


def test_static_fit_rejects_oversize(gpu_ctx):
    ev = synth.gen_fit_event(40000, seed=79)
    with pytest.raises(capi.MkfgError) as e:
        gpu_ctx.fit_host_static(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2)
    assert e.value.code == 1  # MKFG_ERR_BAD_INPUT
    assert "fixed device array holds" in str(e.value)
