"""ctypes front end of the oracle.

TEST INFRASTRUCTURE ONLY. Loads
  * oracle/_ref/libmkfit_ref_<flavour>.so -- the reference's own CPU code
    (trackreco/mkFit) compiled from its sources by oracle/Makefile, with the
    C driver oracle/ref_driver.cc;
  * oracle/_ref/librestate.so -- the FP64 restatement (oracle/restate.c).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def ref_lib_path(flavour="avx2"):
    return os.path.join(REF_DIR, f"libmkfit_ref_{flavour}.so")


def restate_lib_path():
    return os.path.join(REF_DIR, "librestate.so")


def have_ref(flavour="avx2"):
    return os.path.exists(ref_lib_path(flavour))


def have_restate():
    return os.path.exists(restate_lib_path())


def _opt(arr, dtype):
    if arr is None:
        return None
    return np.ascontiguousarray(arr, dtype=dtype)


class RefLib:
    """The reference CPU Matriplex path (compiled reference sources)."""

    def __init__(self, flavour="avx2"):
        self.lib = ctypes.CDLL(ref_lib_path(flavour))
        L = self.lib
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_get_threads.restype = ctypes.c_int
        L.ref_matriplex_width.restype = ctypes.c_int
        L.ref_fit.restype = ctypes.c_int
        L.ref_fit.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p, _i32p, _f32p, _f32p,
                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                              _f32p, _f32p, _i32p, ctypes.POINTER(ctypes.c_double)]

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def threads(self):
        return self.lib.ref_get_threads()

    def width(self):
        return self.lib.ref_matriplex_width()

    def fit(self, par, err, chg, hit_pos, hit_err, rl_grid=None, xi_grid=None, pflags=2, repeat=1):
        """MkFitter fit (InputTracksForFit -> FitTracksWithInterSlurp ->
        OutputFittedTracks). Returns (par, err, chg, best_seconds)."""
        n = chg.shape[0]
        nl = hit_pos.shape[0]
        out_par = np.zeros((6, n), np.float32)
        out_err = np.zeros((21, n), np.float32)
        out_chg = np.zeros(n, np.int32)
        secs = ctypes.c_double(0)
        rl = _opt(rl_grid, np.float32)
        xi = _opt(xi_grid, np.float32)
        rc = self.lib.ref_fit(n, nl, np.ascontiguousarray(par, np.float32),
                              np.ascontiguousarray(err, np.float32),
                              np.ascontiguousarray(chg, np.int32),
                              np.ascontiguousarray(hit_pos, np.float32),
                              np.ascontiguousarray(hit_err, np.float32),
                              rl.ctypes.data if rl is not None else None,
                              xi.ctypes.data if xi is not None else None,
                              int(pflags), int(repeat), out_par, out_err, out_chg,
                              ctypes.byref(secs))
        if rc != 0:
            raise RuntimeError(f"ref_fit failed rc={rc}")
        return out_par, out_err, out_chg, secs.value


class RsMaterial(ctypes.Structure):
    _fields_ = [("rl", ctypes.c_void_p), ("xi", ctypes.c_void_p)]


class Restate:
    """FP64 restatement of the fit arithmetic (oracle/restate.c)."""

    def __init__(self):
        self.lib = ctypes.CDLL(restate_lib_path())
        L = self.lib
        L.rs_fit.restype = None
        L.rs_fit.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f32p, _i32p, _f32p, _f32p,
                             ctypes.c_ulonglong, ctypes.c_uint, ctypes.POINTER(RsMaterial),
                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                             _f64p, _f64p, ctypes.c_void_p]

    def fit(self, par, err, chg, hit_pos, hit_err, rl_grid=None, xi_grid=None, pflags=2,
            endcap_mask=0, shift_rphi=None, shift_z=None, mat_scale=None, want_chi2=True):
        n = chg.shape[0]
        nl = hit_pos.shape[0]
        rl = _opt(rl_grid, np.float32)
        xi = _opt(xi_grid, np.float32)
        mat = RsMaterial(rl.ctypes.data if rl is not None else None,
                         xi.ctypes.data if xi is not None else None)
        out_par = np.zeros((6, n), np.float64)
        out_err = np.zeros((21, n), np.float64)
        chi2 = np.zeros(n, np.float64) if want_chi2 else None
        sr = _opt(shift_rphi, np.float64)
        sz = _opt(shift_z, np.float64)
        ms = _opt(mat_scale, np.float64)
        self.lib.rs_fit(n, nl, np.ascontiguousarray(par, np.float32),
                        np.ascontiguousarray(err, np.float32), np.ascontiguousarray(chg, np.int32),
                        np.ascontiguousarray(hit_pos, np.float32),
                        np.ascontiguousarray(hit_err, np.float32), int(endcap_mask), int(pflags),
                        ctypes.byref(mat),
                        sr.ctypes.data if sr is not None else None,
                        sz.ctypes.data if sz is not None else None,
                        ms.ctypes.data if ms is not None else None,
                        out_par, out_err, chi2.ctypes.data if chi2 is not None else None)
        return out_par, out_err, chi2
