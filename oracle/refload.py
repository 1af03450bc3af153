"""Drives the reference's own Toeplitz load/store kernels on the CPU (TEST INFRASTRUCTURE ONLY).

``oracle/ref_load/Makefile`` compiles cpp/corelib/lib/fft/kernels/toeplitz_load_{3D,2D}.cu
unchanged (with a host shim) into ``oracle/_ref/libref_toeplitz_load.so``. ``multiplication``
then replays perform_toeplitz_multiplication_cuda_3D / _2D (cpp/corelib/lib/fft/toeplitz.cppm:
232-501): a load launch for batch 0, then per batch the convolution of the scratch and a
store+load launch. The convolution between launches is the straight one
(cpp/corelib/lib/fft/nufft.cppm:448-479 semantics: data in [0,N) of a zeroed 2N scratch, FFT,
times the straight kernel, normalised inverse FFT), because the reference's VkFFT zero-padding
setup leaves that step ambiguous.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parent / "_ref" / "libref_toeplitz_load.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def _load():
    global _lib
    if _lib is None:
        _lib = C.CDLL(str(LIB))
        vp, i = C.c_void_p, C.c_int
        _lib.ref_launch_load_3D.argtypes = [vp, vp, vp, vp, vp] + [i] * 11
        _lib.ref_launch_load_2D.argtypes = [vp, vp, vp, vp, vp] + [i] * 10
        _lib.ref_launch_load_3D.restype = None
        _lib.ref_launch_load_2D.restype = None
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(None)


def multiplication(inp, out, kernel, mult1=None, mult2=None, io_mult=0, in_m1=1, out_m1=2, in_m2=1, out_m2=2,
                   accumulate=0):
    """Reference pipeline on complex64 arrays; returns the new output array."""
    lib = _load()
    inp = np.ascontiguousarray(inp, dtype=np.complex64)
    res = np.ascontiguousarray(np.array(out, dtype=np.complex64, copy=True))
    m1 = None if mult1 is None else np.ascontiguousarray(mult1, dtype=np.complex64)
    m2 = None if mult2 is None else np.ascontiguousarray(mult2, dtype=np.complex64)
    B = inp.shape[0]
    shape = inp.shape[1:]
    d = len(shape)
    scratch = np.zeros(tuple(2 * s for s in shape), dtype=np.complex64)
    K = np.asarray(kernel, dtype=np.complex128)
    flags = [int(io_mult), int(in_m1), int(out_m1), int(in_m2), int(out_m2)]

    def launch(bin_, bout):
        if d == 3:
            NZ, NY, NX = shape
            lib.ref_launch_load_3D(_p(inp), _p(res), _p(scratch), _p(m1), _p(m2), *flags, bin_, bout, NX, NY, NZ,
                                   int(accumulate))
        else:
            NY, NX = shape
            lib.ref_launch_load_2D(_p(inp), _p(res), _p(scratch), _p(m1), _p(m2), *flags, bin_, bout, NX, NY,
                                   int(accumulate))

    data_region = tuple(slice(0, s) for s in shape)
    for b in range(B):
        scratch[...] = 0
        launch(b, -1)  # load batch b into scratch[0:N)
        axes = tuple(range(scratch.ndim))
        conv = np.fft.ifftn(np.fft.fftn(scratch[data_region], s=scratch.shape, axes=axes) * K, axes=axes)
        scratch[...] = conv.astype(np.complex64)
        launch(-1, b)  # store batch b from scratch[N-1 : 2N-1)
    return res
