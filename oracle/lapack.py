"""LAPACK oracle and CPU baseline: DGESVJ (one-sided Jacobi SVD) from the
OpenBLAS 0.3.30 that SciPy bundles (symbol scipy_dgesvj_), through ctypes.

TEST INFRASTRUCTURE ONLY: used by tests/ (accuracy oracle for the SVD
configurations) and by bench.py's CPU-baseline leg (timed on the host cores).
"""

from __future__ import annotations

import ctypes
import glob
import os
import time

import numpy as np

_lib = None


def _openblas():
    global _lib
    if _lib is None:
        import scipy
        d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
        cands = glob.glob(os.path.join(d, "libscipy_openblas*.so"))
        if not cands:
            raise RuntimeError("SciPy's bundled OpenBLAS not found")
        _lib = ctypes.CDLL(cands[0])
    return _lib


def set_threads(n: int) -> None:
    _openblas().scipy_openblas_set_num_threads(int(n))


def dgesvj(A: np.ndarray, jobv: str = "V", threads: int | None = None):
    """SVD of A (m >= n) by DGESVJ with JOBA='G', JOBU='U'.

    Returns (sigma descending, U (m x n), V (n x n) or None, info, seconds).
    """
    L = _openblas()
    if threads:
        set_threads(threads)
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    m, n = a.shape
    sva = np.zeros(n)
    v = np.zeros((n, n), order="F") if jobv == "V" else np.zeros((1, 1), order="F")
    lwork = max(6, m + n)
    work = np.zeros(lwork)
    info = ctypes.c_int(0)
    ci = ctypes.c_int
    pd = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    one = ctypes.c_size_t(1)
    t0 = time.perf_counter()
    L.scipy_dgesvj_(ctypes.c_char_p(b"G"), ctypes.c_char_p(b"U"), ctypes.c_char_p(jobv.encode()),
                    ctypes.byref(ci(m)), ctypes.byref(ci(n)), pd(a), ctypes.byref(ci(m)), pd(sva),
                    ctypes.byref(ci(0)), pd(v), ctypes.byref(ci(max(1, n if jobv == "V" else 1))), pd(work),
                    ctypes.byref(ci(lwork)), ctypes.byref(info), one, one, one)
    dt = time.perf_counter() - t0
    sig = sva * work[0]
    order = np.argsort(-sig)
    return sig[order], a[:, order], (v[:, order] if jobv == "V" else None), info.value, dt
