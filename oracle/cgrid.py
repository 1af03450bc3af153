"""ctypes binding of the oracle's FP64 C gridding library (``oracle/cgrid/grid.c``, built by
``oracle/cgrid/Makefile`` into ``oracle/_lib/``) -- TEST INFRASTRUCTURE ONLY.

The same spreading / interpolation arithmetic as :class:`oracle.gridding.GridPlan` (float32 fold,
Kaiser-Bessel weights in double), multithreaded, so the gridding oracle reaches full
configuration sizes. ``available()`` is False when the library has not been built; the numpy
path is then used.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_LIB = Path(__file__).resolve().parent / "_lib" / "libhbgrid.so"
_lib = None


def _load():
    global _lib
    if _lib is None and _LIB.exists():
        lib = C.CDLL(str(_LIB))
        args = [C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_double, C.c_int64, C.c_void_p, C.c_void_p,
                C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        for name in ("hbo_spread", "hbo_interp"):
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = C.c_int
        lib.hbo_set_threads.argtypes = [C.c_int]
        lib.hbo_set_threads.restype = None
        lib.hbo_set_threads(len(os.sched_getaffinity(0)))
        _lib = lib
    return _lib


def available() -> bool:
    return _load() is not None


def _prep(nf, coords):
    nf3 = (1,) * (3 - len(nf)) + tuple(int(v) for v in nf)
    xs = [np.ascontiguousarray(c, dtype=np.float32) for c in coords]
    ptrs = [None] * (3 - len(xs)) + [x.ctypes.data for x in xs]
    return nf3, xs, ptrs


def spread(nf, w: int, beta: float, coords, c) -> np.ndarray:
    """c [T, M] complex -> fine grid [T, *nf] complex128."""
    lib = _load()
    nf3, xs, ptrs = _prep(nf, coords)
    c = np.ascontiguousarray(c, dtype=np.complex128)
    T, M = c.shape
    g = np.zeros((T, *nf), dtype=np.complex128)
    rc = lib.hbo_spread(*nf3, int(w), float(beta), int(M), *ptrs, int(T), c.ctypes.data, g.ctypes.data)
    if rc != 0:
        raise RuntimeError("hbo_spread failed")
    return g


def interp(nf, w: int, beta: float, coords, g) -> np.ndarray:
    """fine grid [T, *nf] -> [T, M] complex128."""
    lib = _load()
    nf3, xs, ptrs = _prep(nf, coords)
    g = np.ascontiguousarray(g, dtype=np.complex128)
    T = g.shape[0]
    M = xs[0].shape[0]
    out = np.empty((T, M), dtype=np.complex128)
    rc = lib.hbo_interp(*nf3, int(w), float(beta), int(M), *ptrs, int(T), g.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise RuntimeError("hbo_interp failed")
    return out
