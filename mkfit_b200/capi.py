"""ctypes bindings of the C ABI in include/mkfit_b200.h.

The CUDA library is built in-tree (python -m mkfit_b200.build) and loaded
from mkfit_b200/_lib/libmkfit_b200.so. There is no fallback: if the library
is missing or no sm_100 device is present, calls raise.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MKFIT_B200_LIB", os.path.join(HERE, "_lib", "libmkfit_b200.so"))
HEADER_PATH = os.path.join(HERE, "..", "include", "mkfit_b200.h")

MKFG_OK, MKFG_ERR_BAD_INPUT, MKFG_ERR_CUDA, MKFG_ERR_OVERFLOW, MKFG_ERR_TIMEOUT = 0, 1, 2, 3, 4
STATUS_NAMES = {0: "OK", 1: "BAD_INPUT", 2: "CUDA", 3: "OVERFLOW", 4: "TIMEOUT", 5: "NO_DEVICE"}

PF_NONE, PF_PARAM_BFIELD, PF_MATERIAL = 0, 1, 2

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int32)


class MkfgTracks(ctypes.Structure):
    _fields_ = [("par", ctypes.c_void_p), ("err", ctypes.c_void_p), ("chg", ctypes.c_void_p),
                ("n", ctypes.c_int32), ("stride", ctypes.c_int32)]


class MkfgHits(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_void_p), ("err", ctypes.c_void_p),
                ("layer_begin", ctypes.c_void_p), ("n_layers", ctypes.c_int32),
                ("stride", ctypes.c_int32)]


class MkfgFitArgs(ctypes.Structure):
    _fields_ = [("in_", MkfgTracks), ("out", MkfgTracks), ("hits", MkfgHits),
                ("hot_index", ctypes.c_void_p), ("hot_stride", ctypes.c_int32),
                ("n_steps", ctypes.c_int32), ("hit_layer", ctypes.c_void_p),
                ("endcap_mask", ctypes.c_uint64), ("pflags", ctypes.c_uint32),
                ("out_chi2", ctypes.c_void_p)]


class MkfgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mkfit_b200 error {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load():
    """Loads the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run python -m mkfit_b200.build)")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    lib.mkfg_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    lib.mkfg_last_error.restype = None
    lib.mkfg_version.restype = ctypes.c_char_p
    lib.mkfg_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    lib.mkfg_context_destroy.argtypes = [vp]
    lib.mkfg_context_stream.argtypes = [vp]
    lib.mkfg_context_stream.restype = vp
    lib.mkfg_context_synchronize.argtypes = [vp]
    lib.mkfg_set_material.argtypes = [vp, vp, vp]
    lib.mkfg_probe_fp32_peak.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.mkfg_fit.argtypes = [vp, ctypes.POINTER(MkfgFitArgs)]
    lib.mkfg_fit_host.argtypes = [vp, ctypes.POINTER(MkfgFitArgs)]
    lib.mkfg_fit_host_static.argtypes = [vp, ctypes.POINTER(MkfgFitArgs)]
    _lib = lib
    return lib


def last_error():
    buf = ctypes.create_string_buffer(1024)
    load().mkfg_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != MKFG_OK:
        raise MkfgError(rc, last_error())
    return rc


def header_symbols():
    """Function names declared in include/mkfit_b200.h."""
    import re
    text = open(HEADER_PATH).read()
    return sorted(set(re.findall(r"\b(mkfg_[a-z0-9_]+)\s*\(", text)))
