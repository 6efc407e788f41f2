"""Parity tolerances and comparison helpers shared by the tests.

FP32 results of two implementations of the same algorithm are compared
element-wise with a relative tolerance whose floor is the element's natural
scale: a track parameter p_k against max(|p_k|, sqrt(C_kk)), a covariance
element C_ij against sqrt(C_ii * C_jj).
"""
import numpy as np

PAR_RTOL = 1e-4   # track parameters (FP32 vs FP32 reference)
COV_RTOL = 1e-4   # covariance elements
CHI2_RTOL = 1e-3  # chi2

DIAG = [0, 2, 5, 9, 14, 20]
SYM = [(i, j) for i in range(6) for j in range(i + 1)]


def par_scaled_err(a, ref, ref_err):
    sig = np.sqrt(np.abs(ref_err[DIAG]))
    scale = np.maximum(np.abs(ref), sig)
    return np.abs(a - ref) / np.maximum(scale, 1e-30)


def cov_scaled_err(a, ref):
    d = np.abs(ref[DIAG])
    scale = np.stack([np.sqrt(d[i] * d[j]) for (i, j) in SYM])
    return np.abs(a - ref) / np.maximum(scale, 1e-30)


def summarize(x):
    x = np.asarray(x).ravel()
    return dict(max=float(x.max()), p999=float(np.percentile(x, 99.9)),
                median=float(np.median(x)))
