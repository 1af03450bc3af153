"""Straight Toeplitz kernel / multiply and the SENSE normal operator, restated in numpy (FP64).

- ``toeplitz_kernel``  follows cpp/corelib/lib/fft/nufft.cppm:386-441: type-1 of the sample
  weights onto 2N-1 modes per axis, embedded at [0, 2N-1) of a 2N grid, FFT, times 1/prod(N).
- ``toeplitz_multiply`` follows nufft.cppm:448-479: FFT with zero padding to 2N, times the
  kernel, inverse FFT (normalised), crop [N-1, 2N-1).
- ``toeplitz_multiplication`` applies the reference's multiply flags exactly as
  cpp/corelib/lib/fft/kernels/toeplitz_load_3D.cu:2-79 does around that convolution.
- ``sense_normal`` is NORMAL_T_T1_OP::operator() (cpp/corelib/lib/mri/normal.cppm:65-88):
  sum_c conj(S_c) T(S_c x).
"""
from __future__ import annotations

import numpy as np

from . import gridding, nudft

NONE, MULT, MULT_CONJ = 0, 1, 2


def toeplitz_kernel(coords, shape, weights=None, w: int = 6, sigma: float = 2.0, exact: bool = False):
    """Kernel [2N..] for image shape N. exact=True uses the FP64 NUDFT for the type-1."""
    shape = tuple(int(s) for s in shape)
    M = np.asarray(coords[0]).shape[0]
    nud = np.ones((1, M), dtype=np.complex128) if weights is None else np.asarray(weights, np.complex128).reshape(1, M)
    nm = tuple(2 * s - 1 for s in shape)
    if exact:
        red = nudft.type1(coords, nud, nm, sign=1)[0]
    else:
        red = gridding.nufft1(coords, nud, nm, w=w, sigma=sigma, sign=1)[0]
    import os

    import scipy.fft as sf
    k = np.zeros(tuple(2 * s for s in shape), dtype=np.complex128)
    k[tuple(slice(0, m) for m in nm)] = red
    del red
    k = sf.fftn(k, workers=len(os.sched_getaffinity(0)), overwrite_x=True)
    k /= float(np.prod(shape))
    return k


def toeplitz_multiply(inout, kernel, workers: int | None = None, dtype=np.complex128):
    """inout [B, N..] -> crop(ifftn(fftn(pad 2N) * kernel)) per batch.

    ``workers`` > 1 runs scipy's multithreaded FFT (the timed CPU baseline); ``dtype`` is the
    working precision (complex128 for parity checks)."""
    inout = np.asarray(inout, dtype=dtype)
    shape = inout.shape[1:]
    d = len(shape)
    axes = tuple(range(1, d + 1))
    if workers and workers > 1:
        import scipy.fft as sf
        mid = sf.fftn(inout, s=tuple(2 * s for s in shape), axes=axes, workers=workers)
        mid *= kernel[None].astype(dtype, copy=False)
        mid = sf.ifftn(mid, axes=axes, workers=workers, overwrite_x=True)
    else:
        mid = np.fft.fftn(inout, s=tuple(2 * s for s in shape), axes=axes)
        mid = mid * kernel[None]
        mid = np.fft.ifftn(mid, axes=axes)
    return mid[(slice(None),) + tuple(slice(s - 1, 2 * s - 1) for s in shape)]


def toeplitz_multiply_torch(inout, kernel, dtype=np.complex128, chunk: int = 4):
    """:func:`toeplitz_multiply` evaluated with torch's multithreaded CPU FFT (the same straight
    pad / transform / multiply / inverse / crop sequence, in FP64 by default), ``chunk`` batches at
    a time; for full configuration sizes. Returns a numpy array."""
    import torch
    inout = np.asarray(inout)
    shape = inout.shape[1:]
    d = len(shape)
    tdt = torch.complex128 if dtype == np.complex128 else torch.complex64
    K = torch.from_numpy(np.ascontiguousarray(kernel)).to(tdt)
    out = np.empty(inout.shape, dtype=dtype)
    dims = tuple(range(1, d + 1))
    crop = (slice(None),) + tuple(slice(n - 1, 2 * n - 1) for n in shape)
    for b0 in range(0, inout.shape[0], chunk):
        v = torch.from_numpy(np.ascontiguousarray(inout[b0:b0 + chunk])).to(tdt)
        v = torch.fft.fftn(v, s=tuple(2 * n for n in shape), dim=dims)
        v *= K
        v = torch.fft.ifftn(v, dim=dims)
        out[b0:b0 + chunk] = v[crop].numpy()
    return out


def _m(a, b, t):
    if t == MULT:
        return a * b
    if t == MULT_CONJ:
        return a * np.conj(b)
    return a


def toeplitz_multiplication(inp, out, kernel, mult1=None, mult2=None, io_mult=NONE, in_m1=MULT, out_m1=MULT_CONJ,
                            in_m2=MULT, out_m2=MULT_CONJ, accumulate=0):
    """Flag semantics of toeplitz_multiplication with the straight kernel; returns a new array."""
    inp = np.asarray(inp, dtype=np.complex128)
    t = inp.copy()
    if mult1 is not None:
        t = _m(t, mult1[None], in_m1)
    if mult2 is not None:
        t = _m(t, mult2[None], in_m2)
    v = toeplitz_multiply(t, kernel)
    if mult1 is not None:
        v = _m(v, mult1[None], out_m1)
    if mult2 is not None:
        v = _m(v, mult2[None], out_m2)
    if io_mult != NONE:
        v = _m(v, inp, io_mult)
    if accumulate:
        v = v + np.asarray(out, dtype=np.complex128)
    return v


def sense_normal(x, smaps, kernel, workers: int | None = None, dtype=np.complex128, fast: bool = False):
    """``fast`` evaluates the same convolution by :func:`toeplitz_multiply_torch`."""
    x = np.asarray(x, dtype=dtype)
    s = np.asarray(smaps, dtype=dtype)
    if fast:
        v = toeplitz_multiply_torch(s * x[None], kernel, dtype=dtype)
    else:
        v = toeplitz_multiply(s * x[None], kernel, workers=workers, dtype=dtype)
    return np.sum(np.conj(s) * v, axis=0)


# ---- time-segmented (and noise-weighted) normal operators, cpp/corelib/lib/mri/normal.cppm ----
# Each restates the operator's sequence of toeplitz_multiplication calls (first without, the rest
# with ACCUMULATE) and its TorchScript epilogue.

def normal_idt_t1(kernels, kerneldiags, stacked_diags, x):
    """NORMAL_IDT_T1_OP::operator() (normal.cppm:218-266): flags (io MULT_CONJ, in1 MULT,
    out1 NONE, in2 MULT, out2 MULT_CONJ) with mult1 = x, mult2 = R_l, then the sum over coils."""
    out = np.zeros(np.shape(stacked_diags), dtype=np.complex128)
    for i in range(len(kernels)):
        out = toeplitz_multiplication(stacked_diags, out, kernels[i], x, kerneldiags[i], MULT_CONJ, MULT, NONE, MULT,
                                      MULT_CONJ, 1 if i > 0 else 0)
    return out.sum(axis=0)


def normal_idt_t2(kernels, kerneldiags, x, stacked_diags):
    """NORMAL_IDT_T2_OP::operator() (normal.cppm:322-369): flags (io NONE, in1 MULT,
    out1 MULT_CONJ, in2 MULT, out2 MULT_CONJ) with mult1 = x, mult2 = R_l; no coil sum."""
    out = np.zeros(np.shape(stacked_diags), dtype=np.complex128)
    for i in range(len(kernels)):
        out = toeplitz_multiplication(stacked_diags, out, kernels[i], x, kerneldiags[i], NONE, MULT, MULT_CONJ, MULT,
                                      MULT_CONJ, 1 if i > 0 else 0)
    return out


def normal_idtw_t1(kernels, kerneldiags, stacked_diags, weights, x):
    """NORMAL_IDTW_T1_OP::operator() (normal.cppm:441-491) and its script (:530-534): flags (io NONE,
    in1 MULT, out1 NONE, in2 MULT, out2 MULT_CONJ), then stack_out = W @ stack_out, times
    conj(stacked_diags), summed over coils."""
    out = np.zeros(np.shape(stacked_diags), dtype=np.complex128)
    for i in range(len(kernels)):
        out = toeplitz_multiplication(stacked_diags, out, kernels[i], x, kerneldiags[i], NONE, MULT, NONE, MULT,
                                      MULT_CONJ, 1 if i > 0 else 0)
    C = out.shape[0]
    out = (np.asarray(weights, np.complex128) @ out.reshape(C, -1)).reshape(out.shape)
    return (out * np.conj(np.asarray(stacked_diags, np.complex128))).sum(axis=0)


def normal_idtw_t2(kernels, kerneldiags, x, weights, stacked_diags):
    """NORMAL_IDTW_T2_OP::operator() (normal.cppm:619-668) and its script (:704-708): flags
    (io NONE, in1 MULT, out1 MULT_CONJ, in2 MULT, out2 MULT_CONJ), then stack_out = W @ stack_out."""
    out = normal_idt_t2(kernels, kerneldiags, x, stacked_diags)
    C = out.shape[0]
    return (np.asarray(weights, np.complex128) @ out.reshape(C, -1)).reshape(out.shape)
