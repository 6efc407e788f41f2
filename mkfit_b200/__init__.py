"""mkfit_b200: B200-native (sm_100a) Kalman-filter tracking hot path.

The compute path is the CUDA library behind the C ABI declared in
include/mkfit_b200.h; this package holds its ctypes front end, the
host-side mirror of the reference's worker interface used by the tests and
the benchmark, and the synthetic input generators. PyTorch is used only for
device memory and streams.
"""
import ctypes

import numpy as np

from . import capi

__all__ = ["Context", "capi"]


def _ptr(t):
    """Device/host address of a torch tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


class Context:
    """One CUDA device + stream with the library's device-side state.
    Mirrors the role of the reference's per-thread MkFitter / MkFinder
    pools (mkFit/Pool.h, mkFit/MkBuilder.h:34-49)."""

    def __init__(self, device=0):
        self.lib = capi.load()
        h = ctypes.c_void_p()
        capi.check(self.lib.mkfg_context_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            self.lib.mkfg_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_ptr(self):
        return self.lib.mkfg_context_stream(self.handle)

    def set_stream(self, stream):
        """Enqueue the context's work on `stream` (a torch.cuda.Stream, a
        raw cudaStream_t as an int, or None for the context's own stream):
        mkfg_context_set_stream."""
        import ctypes
        ptr = getattr(stream, "cuda_stream", stream)
        self.lib.mkfg_context_set_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        capi.check(self.lib.mkfg_context_set_stream(self.handle, ptr))

    def torch_stream(self):
        import torch
        return torch.cuda.ExternalStream(self.stream_ptr, device=torch.device("cuda", self.device))

    def synchronize(self):
        capi.check(self.lib.mkfg_context_synchronize(self.handle))

    def set_material(self, rl_grid, xi_grid):
        rl = np.ascontiguousarray(rl_grid, np.float32)
        xi = np.ascontiguousarray(xi_grid, np.float32)
        assert rl.size == 300 * 120 and xi.size == 300 * 120
        capi.check(self.lib.mkfg_set_material(self.handle, rl.ctypes.data, xi.ctypes.data))

    # ------------------------------------------------------------------ fit
    @staticmethod
    def _fit_args(par, err, chg, out_par, out_err, out_chg, hit_pos, hit_err, layer_begin,
                  hot, hit_layer, n, stride, hstride, n_layers, endcap_mask, pflags, out_chi2,
                  out_stride=None):
        a = capi.MkfgFitArgs()
        a.in_ = capi.MkfgTracks(_ptr(par), _ptr(err), _ptr(chg), n, stride)
        a.out = capi.MkfgTracks(_ptr(out_par), _ptr(out_err), _ptr(out_chg), n,
                                out_stride if out_stride is not None else stride)
        a.hits = capi.MkfgHits(_ptr(hit_pos), _ptr(hit_err), _ptr(layer_begin), n_layers, hstride)
        a.hot_index = _ptr(hot)
        a.hot_stride = stride
        a.n_steps = len(hit_layer)
        a._hit_layer = np.ascontiguousarray(hit_layer, np.int32)
        a.hit_layer = a._hit_layer.ctypes.data
        a.endcap_mask = int(endcap_mask)
        a.pflags = int(pflags)
        a.out_chi2 = _ptr(out_chi2)
        return a

    def fit_device(self, dev, out, pflags=capi.PF_MATERIAL, endcap_mask=0, with_chi2=False):
        """Fit with device-resident inputs (dict of torch CUDA tensors, see
        FitBuffers). Enqueues on the context stream; does not synchronize."""
        a = self._fit_args(dev["par"], dev["err"], dev["chg"], out["par"], out["err"], out["chg"],
                           dev["hit_pos"], dev["hit_err"], dev["layer_begin"], dev["hot"],
                           dev["hit_layer"], dev["n"], dev["n"], dev["n_hits"], dev["n_layers"],
                           endcap_mask, pflags, out["chi2"] if with_chi2 else None)
        capi.check(self.lib.mkfg_fit(self.handle, ctypes.byref(a)))

    def fit_host(self, par, err, chg, hit_pos, hit_err, pflags=capi.PF_MATERIAL, endcap_mask=0,
                 with_chi2=False, out=None):
        """Fit from host (numpy, ideally pinned) buffers through mkfg_fit_host:
        copies in, fits, copies out, synchronizes. hit_pos/hit_err are
        [n_layers][3|6][n] with track i's hit of layer l at index i."""
        n = chg.shape[0]
        nl = hit_pos.shape[0]
        hp = np.ascontiguousarray(hit_pos.transpose(1, 0, 2).reshape(3, nl * n), np.float32) \
            if hit_pos.ndim == 3 else hit_pos
        he = np.ascontiguousarray(hit_err.transpose(1, 0, 2).reshape(6, nl * n), np.float32) \
            if hit_err.ndim == 3 else hit_err
        lb = np.arange(nl + 1, dtype=np.int32) * n
        hot = np.ascontiguousarray(np.broadcast_to(np.arange(n, dtype=np.int32), (nl, n)))
        if out is None:
            out = dict(par=np.zeros((6, n), np.float32), err=np.zeros((21, n), np.float32),
                       chg=np.zeros(n, np.int32), chi2=np.zeros(n, np.float32))
        a = self._fit_args(par, err, chg, out["par"], out["err"], out["chg"], hp, he, lb, hot,
                           np.arange(nl), n, n, nl * n, nl, endcap_mask, pflags,
                           out["chi2"] if with_chi2 else None)
        capi.check(self.lib.mkfg_fit_host(self.handle, ctypes.byref(a)))
        return out


    def fit_host_static(self, par, err, chg, hit_pos, hit_err, pflags=capi.PF_MATERIAL,
                        endcap_mask=0, with_chi2=False, out=None):
        """fit_host through mkfg_fit_host_static: staging in the library's
        fixed device array, no allocation; same arguments and outputs."""
        n = chg.shape[0]
        nl = hit_pos.shape[0]
        hp = np.ascontiguousarray(hit_pos.transpose(1, 0, 2).reshape(3, nl * n), np.float32) \
            if hit_pos.ndim == 3 else hit_pos
        he = np.ascontiguousarray(hit_err.transpose(1, 0, 2).reshape(6, nl * n), np.float32) \
            if hit_err.ndim == 3 else hit_err
        lb = np.arange(nl + 1, dtype=np.int32) * n
        hot = np.ascontiguousarray(np.broadcast_to(np.arange(n, dtype=np.int32), (nl, n)))
        if out is None:
            out = dict(par=np.zeros((6, n), np.float32), err=np.zeros((21, n), np.float32),
                       chg=np.zeros(n, np.int32), chi2=np.zeros(n, np.float32))
        a = self._fit_args(par, err, chg, out["par"], out["err"], out["chg"], hp, he, lb, hot,
                           np.arange(nl), n, n, nl * n, nl, endcap_mask, pflags,
                           out["chi2"] if with_chi2 else None)
        capi.check(self.lib.mkfg_fit_host_static(self.handle, ctypes.byref(a)))
        return out


class FitBuffers:
    """Device-resident fit inputs in the C-ABI layout, built from a
    synth.FitEvent (hits of all layers concatenated, track i's hit on layer
    l at index i of that layer)."""

    @staticmethod
    def upload(ev, device="cuda"):
        import torch
        n = ev.n
        nl = ev.hit_pos.shape[0]
        hp = ev.hit_pos.transpose(1, 0, 2).reshape(3, nl * n)
        he = ev.hit_err.transpose(1, 0, 2).reshape(6, nl * n)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        dev = dict(par=t(ev.par), err=t(ev.err), chg=t(ev.chg), hit_pos=t(hp), hit_err=t(he),
                   layer_begin=t(np.arange(nl + 1, dtype=np.int32) * n),
                   hot=t(np.broadcast_to(np.arange(n, dtype=np.int32), (nl, n))),
                   hit_layer=np.arange(nl, dtype=np.int32), n=n, n_hits=nl * n, n_layers=nl)
        return dev

    @staticmethod
    def outputs(n, device="cuda"):
        import torch
        return dict(par=torch.zeros((6, n), dtype=torch.float32, device=device),
                    err=torch.zeros((21, n), dtype=torch.float32, device=device),
                    chg=torch.zeros(n, dtype=torch.int32, device=device),
                    chi2=torch.zeros(n, dtype=torch.float32, device=device))
