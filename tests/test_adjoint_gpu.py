"""Differentiable fit on the GPU: the FP32 forward + adjoint kernels
(mkfg_align_chi2_forward / _backward) and their torch.autograd binding,
against the FP64 restatement: summed chi2 within 1e-4 relative, gradient
within 1e-3 relative of FP64 central finite differences (per component,
floored at 1e-3 of the largest component of the same kind)."""
import numpy as np
import pytest
import torch

from mkfit_b200 import synth
from mkfit_b200.align import AlignedFit
from oracle.oracle import restate_chi2_sum, restate_fd_grad

pytestmark = pytest.mark.gpu

NL = 10
GRAD_RTOL = 1e-3


def misaligned_event(n, seed):
    rng = np.random.default_rng(seed)
    return synth.gen_fit_event(n, seed=seed, align_rphi=rng.normal(0, 0.002, NL),
                               align_z=rng.normal(0, 0.002, NL),
                               mat_scale=1 + rng.uniform(-0.1, 0.1, NL))


def grad_rel(g, fd):
    floor = 1e-3 * np.maximum(np.abs(fd).max(axis=0), 1e-12)
    return np.abs(g - fd) / np.maximum(np.abs(fd), floor)


@pytest.mark.parametrize("material", [True, False])
def test_gradient_matches_fp64_fd(gpu_ctx, restate, material):
    ev = misaligned_event(4000, seed=31)
    fit = AlignedFit(gpu_ctx, ev, material=material)
    th = fit.nominal()
    total, g = fit.forward_backward(th)
    thn = th.cpu().numpy().astype(np.float64)
    ref = restate_chi2_sum(restate, ev, thn, material)
    fd = restate_fd_grad(restate, ev, thn, material=material)
    g = g.cpu().numpy()
    rel = grad_rel(g, fd)
    print(f"\nmaterial={material}: chi2 {total:.6g} vs FP64 {ref:.6g} "
          f"(rel {abs(total - ref) / ref:.2e}); gradient rel err max {rel.max():.2e} "
          f"median {np.median(rel):.2e}")
    assert abs(total - ref) < 1e-4 * ref
    assert rel.max() < GRAD_RTOL, rel


def test_autograd_function(gpu_ctx):
    ev = misaligned_event(3000, seed=32)
    fit = AlignedFit(gpu_ctx, ev, material=True)
    theta = fit.nominal()
    theta[:, 0] = 0.001
    theta.requires_grad_()
    loss = fit.chi2(theta)
    assert loss.dim() == 0 and loss.dtype == torch.float32
    (2.0 * loss).backward()
    total, g = fit.forward_backward(theta.detach())
    assert abs(loss.item() - total) <= 1e-6 * total
    np.testing.assert_allclose(theta.grad.cpu().numpy(), 2.0 * g.cpu().numpy(), rtol=1e-5,
                               atol=1e-6 * float(g.abs().max()))
    # Repeatable: the same forward/backward twice gives identical results.
    _, g2 = fit.forward_backward(theta.detach())
    torch.testing.assert_close(g, g2, rtol=0, atol=0)


def test_gradient_descent_moves_towards_truth(gpu_ctx):
    """A few gradient steps on the r-phi shifts reduce the summed chi2 and
    move the shifts towards the generated misalignment."""
    ar = np.zeros(NL)
    ar[2], ar[5], ar[8] = 0.01, -0.008, 0.006
    ev = synth.gen_fit_event(5000, seed=33, align_rphi=ar)
    fit = AlignedFit(gpu_ctx, ev, material=True)
    theta = fit.nominal().requires_grad_()
    opt = torch.optim.Adam([theta], lr=5e-4)
    first = None
    for _ in range(60):
        opt.zero_grad()
        loss = fit.chi2(theta)
        loss.backward()
        with torch.no_grad():
            theta.grad[:, 1:] = 0
        opt.step()
        first = first if first is not None else loss.item()
    final = fit.chi2(theta.detach()).item()
    est = theta.detach().cpu().numpy()[:, 0]
    assert final < first
    for l in (2, 5, 8):
        assert abs(est[l] - ar[l]) < 0.5 * abs(ar[l]), (l, est[l], ar[l])
