"""Differentiable fit: summed track chi2 as a function of per-layer alignment
and material parameters, with its gradient from the library's hand-derived
adjoint (mkfg_align_chi2_forward / mkfg_align_chi2_backward).

    fit = AlignedFit(ctx, event)              # synth.FitEvent, barrel layers
    theta = fit.nominal().requires_grad_()    # [n_layers][3]: r-phi, z, scale
    loss = fit.chi2(theta)                    # torch autograd.Function (C++)
    loss.backward()                           # theta.grad = dL/dtheta

`chi2` goes through the compiled PyTorch extension (_lib/_align_ext*.so);
`forward_backward` calls the C ABI directly (no autograd).
`distributed_chi2_grad` splits the tracks over the ranks of a process
group and sums the ranks' results with one all-reduce.
"""
import ctypes
import importlib.machinery
import importlib.util
import os

import numpy as np

from . import capi
from .build import ext_path


class MkfgAlignArgs(ctypes.Structure):
    _fields_ = [("fit", capi.MkfgFitArgs), ("theta", ctypes.c_void_p),
                ("checkpoint", ctypes.c_void_p), ("chi2_sum", ctypes.c_void_p)]


def _bind(lib):
    if getattr(lib, "_align_bound", False):
        return
    lib.mkfg_align_chi2_forward.argtypes = [ctypes.c_void_p, ctypes.POINTER(MkfgAlignArgs)]
    lib.mkfg_align_chi2_backward.argtypes = [ctypes.c_void_p, ctypes.POINTER(MkfgAlignArgs),
                                             ctypes.c_void_p, ctypes.c_void_p]
    lib._align_bound = True


_ext = None


def load_ext():
    """Imports the compiled PyTorch extension (raises if it was not built)."""
    global _ext
    if _ext is not None:
        return _ext
    import torch  # noqa: F401  (libtorch must be loaded first)
    path = ext_path()
    if not os.path.exists(path):
        raise RuntimeError(f"PyTorch extension not built: {path} "
                           "(run python -m mkfit_b200.build)")
    capi.load()  # libmkfit_b200.so, which the extension links
    loader = importlib.machinery.ExtensionFileLoader("_align_ext", path)
    spec = importlib.util.spec_from_file_location("_align_ext", path, loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    _ext = mod
    return mod


class AlignedFit:
    """A barrel fit workload resident on the context's device."""

    def __init__(self, ctx, ev, material=True):
        from . import FitBuffers
        self.ctx = ctx
        self.ev = ev
        self.material = material
        if material:
            ctx.set_material(ev.rl_grid, ev.xi_grid)
        self.dev = FitBuffers.upload(ev)
        self.n_steps = int(self.dev["n_layers"])
        self.pflags = capi.PF_MATERIAL if material else capi.PF_NONE

    def nominal(self):
        import torch
        t = torch.zeros((self.n_steps, 3), dtype=torch.float32, device=self.dev["par"].device)
        t[:, 2] = 1.0
        return t

    def chi2(self, theta):
        """Summed chi2 (0-dim tensor), differentiable in theta [n_steps][3]."""
        ext = load_ext()
        d = self.dev
        return ext.align_chi2(theta, int(self.ctx.handle.value), d["par"], d["err"], d["chg"],
                              d["hit_pos"], d["hit_err"], d["layer_begin"], d["hot"],
                              [int(x) for x in d["hit_layer"]], int(self.pflags))

    def forward_backward(self, theta, grad_out=1.0):
        """C-ABI path: returns (sum chi2, dL/dtheta as a float64 tensor)."""
        import torch
        lib = self.ctx.lib
        _bind(lib)
        d = self.dev
        n = d["n"]
        th = theta.detach().to(torch.float32).contiguous()
        dev = th.device
        ckpt = torch.empty((self.n_steps, 27, n), dtype=torch.float32, device=dev)
        total = torch.empty((), dtype=torch.float64, device=dev)
        grad = torch.empty((self.n_steps, 3), dtype=torch.float64, device=dev)
        gout = torch.full((), float(grad_out), dtype=torch.float32, device=dev)
        a = self._args(th, ckpt, total)
        torch.cuda.synchronize()
        capi.check(lib.mkfg_align_chi2_forward(self.ctx.handle, ctypes.byref(a)))
        capi.check(lib.mkfg_align_chi2_backward(self.ctx.handle, ctypes.byref(a),
                                                gout.data_ptr(), grad.data_ptr()))
        self.ctx.synchronize()
        return float(total.item()), grad

    def _args(self, th, ckpt, total):
        d = self.dev
        n = d["n"]
        a = MkfgAlignArgs()
        a.fit.in_ = capi.MkfgTracks(d["par"].data_ptr(), d["err"].data_ptr(),
                                    d["chg"].data_ptr(), n, n)
        a.fit.out = capi.MkfgTracks(None, None, None, n, n)
        a.fit.hits = capi.MkfgHits(d["hit_pos"].data_ptr(), d["hit_err"].data_ptr(),
                                   d["layer_begin"].data_ptr(), d["n_layers"], d["n_hits"])
        a.fit.hot_index = d["hot"].data_ptr()
        a.fit.hot_stride = n
        a.fit.n_steps = self.n_steps
        a._hl = np.ascontiguousarray(d["hit_layer"], np.int32)
        a.fit.hit_layer = a._hl.ctypes.data
        a.fit.endcap_mask = 0
        a.fit.pflags = self.pflags
        a.fit.out_chi2 = None
        a.theta = th.data_ptr()
        a.checkpoint = ckpt.data_ptr()
        a.chi2_sum = total.data_ptr()
        return a


def distributed_chi2_grad(ctx, ev, theta, world, rank, material=True, grad_fn=None):
    """Summed chi2 and its gradient over all tracks of `ev`, with the tracks
    split into one contiguous share per rank (mkfit_b200.dist.track_share)
    and the ranks' (chi2, gradient) summed by one all-reduce of
    1 + 3 * n_layers float64 numbers. grad_fn(share_event, theta) ->
    (chi2, grad [n_layers][3]) computes a share; by default the CUDA adjoint
    (AlignedFit.forward_backward) on `ctx`. Returns (chi2, grad) as float64,
    the same on every rank."""
    from . import dist
    begin, end = dist.track_share(ev.n, world, rank)
    share = ev.tracks(begin, end)
    if grad_fn is None:
        def grad_fn(e, th):
            c2, g = AlignedFit(ctx, e, material=material).forward_backward(th)
            return c2, g.cpu().numpy()
    c2, g = grad_fn(share, theta)
    g = np.asarray(g, np.float64)
    tot = dist.allreduce_sum(np.concatenate([[c2], g.ravel()]), world)
    return float(tot[0]), tot[1:].reshape(g.shape)
