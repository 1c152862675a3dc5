"""HDF5 datasets through libgjx.so's own reader/writer (csrc/h5mini.cpp; no
libhdf5 or h5py needed).  Shapes are C order, as H5LT's dims are.

    h5.write("in.h5", "2048", {"IDADIM": np.array([M, M, N, P], np.int32), "G": G.T}, mode=0)
    U = h5.read("out.h5", "2048/G").T          # back to M x N (Fortran view)
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import GjxError, lib

_bound = False


def _bind():
    global _bound
    if not _bound:
        L = lib()
        L.gjx_h5_read.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_ulonglong,
                                  ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_int)]
        L.gjx_h5_read.restype = ctypes.c_int
        L.gjx_h5_write.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_void_p)]
        L.gjx_h5_write.restype = ctypes.c_int
        _bound = True
    return lib()


def shape(file: str, path: str) -> tuple:
    L = _bind()
    dims = (ctypes.c_ulonglong * 8)()
    rank = ctypes.c_int()
    r = L.gjx_h5_read(file.encode(), path.encode(), 1, None, 0, dims, ctypes.byref(rank))
    if r:
        raise GjxError(r, L.gjx_last_error().decode())
    return tuple(int(dims[i]) for i in range(rank.value))


def read(file: str, path: str, as_float: bool | None = None) -> np.ndarray:
    """The dataset at path ("group/name"), as float64 (default for floating
    datasets) or int32 (as_float=False)."""
    L = _bind()
    shp = shape(file, path)
    want_float = True if as_float is None else as_float
    out = np.zeros(shp, dtype=np.float64 if want_float else np.int32)
    dims = (ctypes.c_ulonglong * 8)()
    rank = ctypes.c_int()
    r = L.gjx_h5_read(file.encode(), path.encode(), int(want_float), out.ctypes.data, out.size, dims,
                      ctypes.byref(rank))
    if r:
        raise GjxError(r, L.gjx_last_error().decode())
    return out


def write(file: str, group: str, datasets: dict, mode: int = 0) -> None:
    """Write datasets (name -> array; float arrays as double, integer arrays
    as int32) into group.  mode 0: new file; 1: new group in an existing
    file; 2: existing file, group created if absent, same-shaped datasets
    overwritten."""
    L = _bind()
    names, arrs = [], []
    for k, v in datasets.items():
        a = np.asarray(v)
        a = np.ascontiguousarray(a, dtype=np.float64 if a.dtype.kind == "f" else np.int32)
        if a.ndim > 8:
            raise ValueError("rank above 8")
        names.append(k.encode())
        arrs.append(a)
    n = len(arrs)
    c_names = (ctypes.c_char_p * max(1, n))(*names)
    ranks = (ctypes.c_int * max(1, n))(*[a.ndim for a in arrs])
    dims = (ctypes.c_ulonglong * (8 * max(1, n)))()
    for i, a in enumerate(arrs):
        for j, d in enumerate(a.shape):
            dims[8 * i + j] = d
    isf = (ctypes.c_int * max(1, n))(*[int(a.dtype == np.float64) for a in arrs])
    ptrs = (ctypes.c_void_p * max(1, n))(*[a.ctypes.data for a in arrs])
    r = L.gjx_h5_write(file.encode(), group.encode(), mode, n, c_names, ranks, dims, isf, ptrs)
    if r:
        raise GjxError(r, L.gjx_last_error().decode())
