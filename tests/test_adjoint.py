"""Differentiable fit (host side, no GPU): the product's generated fit-step
adjoint, evaluated in FP64 on the host (oracle/adjoint_f64.cc), against
central finite differences of the independent FP64 restatement of the fit
(oracle/restate.c) on a misaligned toy detector. This pins the derivation;
the GPU tests pin the FP32 device kernels against the same differences."""
import os

import numpy as np
import pytest

from mkfit_b200 import synth
from oracle.oracle import adj_f64_grad, adjoint_f64_lib_path, restate_chi2_sum, restate_fd_grad

NL = 10


def misaligned_event(n, seed):
    rng = np.random.default_rng(seed)
    ar = rng.normal(0, 0.002, NL)
    az = rng.normal(0, 0.002, NL)
    ms = 1 + rng.uniform(-0.1, 0.1, NL)
    return synth.gen_fit_event(n, seed=seed, align_rphi=ar, align_z=az, mat_scale=ms)


def nominal():
    th = np.zeros((NL, 3))
    th[:, 2] = 1.0
    return th


@pytest.fixture(scope="module")
def adj64():
    if not os.path.exists(adjoint_f64_lib_path()):
        pytest.fail("oracle/_ref/libadjoint_f64.so missing (run make -C oracle restate)")


@pytest.mark.parametrize("material", [False, True])
def test_adjoint_f64_matches_restate_fd(adj64, restate, material):
    ev = misaligned_event(200, seed=21)
    th = nominal()
    total, g = adj_f64_grad(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, th, ev.rl_grid,
                            ev.xi_grid, material=material)
    ref = restate_chi2_sum(restate, ev, th, material)
    assert abs(total - ref) <= 1e-9 * abs(ref)
    fd = restate_fd_grad(restate, ev, th, material=material)
    # Relative error per component; floor at 1e-3 of the largest component
    # of the same kind (shift or scale).
    for j in range(3):
        floor = 1e-3 * max(np.abs(fd[:, j]).max(), 1e-12)
        rel = np.abs(g[:, j] - fd[:, j]) / np.maximum(np.abs(fd[:, j]), floor)
        assert rel.max() < 1e-5, (j, rel)
    if not material:
        np.testing.assert_array_equal(g[:, 2], 0.0)


def test_adjoint_f64_off_nominal(adj64, restate):
    """Away from the nominal point (shifted layers, scaled material)."""
    ev = misaligned_event(150, seed=22)
    rng = np.random.default_rng(3)
    th = nominal()
    th[:, 0] = rng.normal(0, 0.003, NL)
    th[:, 1] = rng.normal(0, 0.003, NL)
    th[:, 2] = 1 + rng.uniform(-0.2, 0.2, NL)
    _, g = adj_f64_grad(ev.par, ev.err, ev.chg, ev.hit_pos, ev.hit_err, th, ev.rl_grid,
                        ev.xi_grid, material=True)
    fd = restate_fd_grad(restate, ev, th, material=True)
    floor = 1e-3 * np.abs(fd).max(axis=0)
    rel = np.abs(g - fd) / np.maximum(np.abs(fd), floor)
    assert rel.max() < 1e-5, rel


def test_misaligned_generator_points_gradient_at_truth(restate):
    """With hits recorded under a known r-phi misalignment, the gradient of
    the summed chi2 at the nominal point has the sign of -offset for the
    large offsets (chi2 decreases towards the truth)."""
    ar = np.zeros(NL)
    ar[3] = 0.01
    ar[6] = -0.01
    ev = synth.gen_fit_event(400, seed=23, align_rphi=ar)
    fd = restate_fd_grad(restate, ev, nominal(), material=True)
    assert fd[3, 0] < 0 and fd[6, 0] > 0


def test_torch_extension_loads():
    """The compiled PyTorch extension (autograd Function over the C ABI)
    imports without a GPU and exposes the differentiable entry."""
    from mkfit_b200.align import load_ext
    ext = load_ext()
    assert hasattr(ext, "align_chi2")
