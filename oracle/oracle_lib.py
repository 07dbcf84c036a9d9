"""ctypes access to the oracle's C kernels — TEST INFRASTRUCTURE ONLY."""
import ctypes as C
import os

import numpy as np

import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(_build.build())
        _lib.oracle_tensor_apply.restype = None
        _lib.oracle_max_threads.restype = C.c_int
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def tensor_apply(dim, n, q, cell_map, h, B, G, W, mass, kappa, kappa_pts, order, color_off, x, y, threads=0):
    """y += A x through the reference's tensor schedule (accumulators.jl:1955-2013)."""
    cell_map = np.ascontiguousarray(cell_map, dtype=np.int32)
    h = np.ascontiguousarray(h, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.float64)
    W = np.ascontiguousarray(W, dtype=np.float64)
    order = np.ascontiguousarray(order, dtype=np.int64)
    color_off = np.ascontiguousarray(color_off, dtype=np.int64)
    kp = None if kappa_pts is None else np.ascontiguousarray(kappa_pts, dtype=np.float64)
    lib().oracle_tensor_apply(C.c_int(dim), C.c_int(n), C.c_int(q), C.c_int64(len(h)), _p(cell_map, C.c_int32),
                              _p(h, C.c_double), _p(B, C.c_double), _p(G, C.c_double), _p(W, C.c_double),
                              C.c_double(mass), C.c_double(kappa), _p(kp, C.c_double), C.c_int(len(color_off) - 1),
                              _p(color_off, C.c_int64), _p(order, C.c_int64), _p(x, C.c_double),
                              _p(y, C.c_double), C.c_int(threads))
    return y


def max_threads():
    return int(lib().oracle_max_threads())
