"""GPU parity of the Kalman fit (mkfg_fit / mkfg_fit_host through the C ABI)
against the reference's own CPU MkFitter fit on identical inputs, and error
against the FP64 restatement of the same algorithm."""
import glob
import os

import numpy as np
import pytest
import torch

from mkfit_b200 import FitBuffers, synth
from tests.tolerances import (CHI2_RTOL, COV_RTOL, PAR_RTOL, cov_scaled_err, par_scaled_err,
                              summarize)

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "fit_*.npz")))


def gpu_fit(ctx, ev, pflags=2, with_chi2=False, grids=None):
    rl, xi = grids if grids is not None else (ev.rl_grid, ev.xi_grid)
    ctx.set_material(rl, xi)
    dev = FitBuffers.upload(ev)
    out = FitBuffers.outputs(ev.n)
    ctx.fit_device(dev, out, pflags=pflags, endcap_mask=getattr(ev, "endcap_mask", 0),
                   with_chi2=with_chi2)
    ctx.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def assert_parity(par, err, ref_par, ref_err, label):
    ep = par_scaled_err(par, ref_par, ref_err)
    ec = cov_scaled_err(err, ref_err)
    sp, sc = summarize(ep), summarize(ec)
    print(f"{label}: par {sp}  cov {sc}")
    # Bulk at FP32 rounding level; every element within the stated
    # tolerance except rare cancellation-dominated covariance terms.
    assert sp["median"] < 1e-6
    assert sp["p999"] < PAR_RTOL
    assert sp["max"] < 1e-2
    assert sc["median"] < 1e-5
    assert sc["p999"] < COV_RTOL
    assert sc["max"] < 1e-1


@pytest.mark.parametrize("path", GOLDEN, ids=os.path.basename)
def test_fit_matches_golden(gpu_ctx, path):
    g = np.load(path)
    ev = synth.FitEvent(par=g["par"], err=g["err"], chg=g["chg"], hit_pos=g["hit_pos"],
                        hit_err=g["hit_err"])
    out = gpu_fit(gpu_ctx, ev, pflags=int(g["pflags"]), grids=synth.toy_material_grid(g["radii"]))
    assert_parity(out["par"], out["err"], g["ref_par"], g["ref_err"], os.path.basename(path))
    np.testing.assert_array_equal(out["chg"], g["ref_chg"])


@pytest.mark.parametrize("pflags", [0, 2, 3])
def test_fit_matches_reference_20k(gpu_ctx, reflib, pflags):
    ev = synth.gen_fit_event(20000, seed=0xC0FFEE)
    out = gpu_fit(gpu_ctx, ev, pflags=pflags)
    par, err, chg, _ = reflib.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                  ev.xi_grid, pflags=pflags)
    assert_parity(out["par"], out["err"], par, err, f"20k pflags={pflags}")
    np.testing.assert_array_equal(out["chg"], chg)


@pytest.mark.parametrize("pflags", [0, 2, 3])
def test_steered_fit_matches_reference(gpu_ctx, reflib, restate, pflags):
    """Steered fit (MkFitter::FitTracksSteered): two barrel steps, then
    eight endcap steps (propagation to the hit's z and the endcap update)
    selected by endcap_mask, against the reference's own steered fit on the
    same tracks, and both against the FP64 restatement."""
    ev = synth.gen_fit_event_steered(20000, seed=0x57EE)
    out = gpu_fit(gpu_ctx, ev, pflags=pflags)
    par, err, chg = reflib.fit_steered(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err,
                                       ev.endcap_mask, ev.rl_grid, ev.xi_grid, pflags=pflags)
    assert_parity(out["par"], out["err"], par, err, f"steered 20k pflags={pflags}")
    np.testing.assert_array_equal(out["chg"], chg)
    dpar, derr, _ = restate.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                ev.xi_grid, pflags=pflags, endcap_mask=ev.endcap_mask)
    g = cov_scaled_err(out["err"], derr)
    r = cov_scaled_err(err, derr)
    gp = par_scaled_err(out["par"], dpar, derr)
    rp = par_scaled_err(par, dpar, derr)
    print(f"  vs FP64: GPU par {summarize(gp)} cov {summarize(g)}; reference par "
          f"{summarize(rp)} cov {summarize(r)}")
    assert np.percentile(gp, 99.9) <= 1.5 * np.percentile(rp, 99.9) + 1e-7
    assert np.percentile(g, 99.9) <= 1.5 * np.percentile(r, 99.9) + 1e-7


def test_fit_error_vs_fp64(gpu_ctx, restate):
    """Error of the FP32 GPU fit against the FP64 restatement, and chi2."""
    ev = synth.gen_fit_event(4000, seed=99)
    out = gpu_fit(gpu_ctx, ev, with_chi2=True)
    dpar, derr, dchi2 = restate.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                    ev.xi_grid, pflags=2)
    ep = par_scaled_err(out["par"], dpar, derr)
    ec = cov_scaled_err(out["err"], derr)
    rc = np.abs(out["chi2"] - dchi2) / np.maximum(np.abs(dchi2), 1e-6)
    print("vs FP64: par", summarize(ep), "cov", summarize(ec), "chi2", summarize(rc))
    assert np.percentile(ep, 99.9) < PAR_RTOL
    # chi2 summed over 10 updates in FP32: within the 1e-3 relative bound.
    assert np.median(rc) < 1e-4
    assert np.percentile(rc, 99.9) < CHI2_RTOL


def test_fit_host_entry_equals_device_entry(gpu_ctx):
    ev = synth.gen_fit_event(3001, seed=3)
    dev_out = gpu_fit(gpu_ctx, ev, with_chi2=True)
    host = gpu_ctx.fit_host(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, pflags=2,
                            with_chi2=True)
    for k in ("par", "err", "chg", "chi2"):
        np.testing.assert_array_equal(host[k], dev_out[k])


@pytest.mark.parametrize("n", [1, 31, 129])
def test_fit_ragged_sizes(gpu_ctx, reflib, n):
    ev = synth.gen_fit_event(n, seed=n)
    out = gpu_fit(gpu_ctx, ev)
    par, err, _, _ = reflib.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                ev.xi_grid, pflags=2)
    ep = par_scaled_err(out["par"], par, err)
    assert ep.max() < 1e-3


def test_fit_empty_batch(gpu_ctx):
    ev = synth.gen_fit_event(1, seed=1)
    ev0 = synth.FitEvent(par=ev.par[:, :0], err=ev.err[:, :0], chg=ev.chg[:0],
                         hit_pos=ev.hit_pos[:, :, :0], hit_err=ev.hit_err[:, :, :0])
    out = gpu_ctx.fit_host(ev0.par, ev0.err, ev0.chg, ev0.hit_pos, ev0.hit_err)
    assert out["par"].shape == (6, 0)


def test_failed_propagation_resets_like_reference(gpu_ctx, reflib):
    """Tracks starting near r=0 with momentum pointing inward fail the
    reference's iterative propagation; the output is then reset to the
    input (mkFit/PropagationMPlex.cc:497-504). The GPU must do the same."""
    ev = synth.gen_fit_event(512, seed=11, r_start=0.0)  # start at the vertex
    out = gpu_fit(gpu_ctx, ev)
    par, err, _, _ = reflib.fit(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, ev.rl_grid,
                                ev.xi_grid, pflags=2)
    ep = par_scaled_err(out["par"], par, err)
    # Failed tracks carry huge, ill-conditioned states: compare the bulk.
    assert np.median(ep) < 1e-5
    assert np.mean(ep < 1e-3) > 0.95


@pytest.mark.parametrize("entry", ["mkfg_fit_host", "mkfg_fit_host_static"])
def test_fit_host_rejects_hit_index_outside_layer(gpu_ctx, entry):
    """A hit index at or past its layer's size is refused with
    MKFG_ERR_BAD_INPUT before anything is copied; a negative index (the
    reference packer's null input, hit 0 of the layer) is accepted."""
    from mkfit_b200 import capi
    import ctypes
    ev = synth.gen_fit_event(64, seed=5)
    n, nl = ev.n, ev.hit_pos.shape[0]
    hp = np.ascontiguousarray(ev.hit_pos.transpose(1, 0, 2).reshape(3, nl * n), np.float32)
    he = np.ascontiguousarray(ev.hit_err.transpose(1, 0, 2).reshape(6, nl * n), np.float32)
    lb = np.arange(nl + 1, dtype=np.int32) * n
    out = dict(par=np.zeros((6, n), np.float32), err=np.zeros((21, n), np.float32),
               chg=np.zeros(n, np.int32))
    fn = getattr(gpu_ctx.lib, entry)
    for bad, ok in ((n, False), (-1, True), (n - 1, True)):
        hot = np.ascontiguousarray(np.broadcast_to(np.arange(n, dtype=np.int32), (nl, n)))
        hot[nl - 1, 7] = bad
        a = gpu_ctx._fit_args(ev.par, ev.err, ev.chg, out["par"], out["err"], out["chg"], hp, he,
                              lb, hot, np.arange(nl), n, n, nl * n, nl, 0, 2, None)
        rc = fn(gpu_ctx.handle, ctypes.byref(a))
        if ok:
            assert rc == 0, capi.last_error()
        else:
            assert rc == 1
            assert "outside layer" in capi.last_error()


def test_fit_on_caller_stream(gpu_ctx):
    """mkfg_context_set_stream: the fit enqueued on the caller's stream gives
    the same result as on the context's own stream, and the context goes
    back to its own stream on NULL."""
    own = gpu_ctx.stream_ptr
    ev = synth.gen_fit_event(2001, seed=31)
    base = gpu_fit(gpu_ctx, ev, with_chi2=True)
    s = torch.cuda.Stream()
    gpu_ctx.set_stream(s)
    try:
        assert gpu_ctx.stream_ptr == s.cuda_stream
        got = gpu_fit(gpu_ctx, ev, with_chi2=True)
    finally:
        gpu_ctx.set_stream(None)
    assert gpu_ctx.stream_ptr == own
    for k in base:
        np.testing.assert_array_equal(got[k], base[k], err_msg=k)
