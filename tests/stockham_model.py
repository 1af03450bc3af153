"""Pure-Python model of the pass kernel's FFT schedule (csrc/fft.cuh: radix order, Stockham
stage indexing, twiddle-table lookups and the pruned load/store position maps). It lets the CPU
suite check the index arithmetic the CUDA kernel uses against numpy's FFT."""
from __future__ import annotations

import numpy as np


def radices(L: int):
    out, rest = [], L
    for r in (8, 4, 2, 5, 3, 7):
        while rest % r == 0 and rest > 1:
            out.append(r)
            rest //= r
    if rest != 1:
        raise ValueError("not 2,3,5,7-smooth")
    return out


def twiddles(L: int) -> np.ndarray:
    m = np.arange(L)
    return np.exp(-2j * np.pi * m / L).astype(np.complex64)


def _dft(v, inverse):
    R = len(v)
    s = 1 if inverse else -1
    W = np.exp(s * 2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R)
    return W.T @ np.array(v)


def stockham(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    """x: [L, W] columns; returns the unnormalised DFT of each column (sign - or +)."""
    L = x.shape[0]
    tw = twiddles(L)
    a = x.astype(np.complex128)
    p = 1
    for R in radices(L):
        b = np.empty_like(a)
        m = L // R
        twstep = L // (p * R)
        for i in range(m):
            k = i % p
            v = [a[i + r * m] for r in range(R)]
            if p > 1:
                for r in range(1, R):
                    t = tw[r * k * twstep]
                    if inverse:
                        t = np.conj(t)
                    v[r] = v[r] * t
            V = _dft(v, inverse)
            j = (i - k) * R + k
            for r in range(R):
                b[j + r * p] = V[r]
        a = b
        p *= R
    return a


def pruned_pass(x: np.ndarray, L: int, Lin: int, in_shift: int, Lout: int, out_shift: int, inverse: bool):
    """Model of pass_kernel's load -> FFT -> store along axis 0 of x ([Lin, W])."""
    buf = np.zeros((L, x.shape[1]), dtype=np.complex128)
    for pos in range(L):
        l = (pos - in_shift) % L
        if l < Lin:
            buf[pos] = x[l]
    res = stockham(buf, inverse)
    return np.stack([res[(o + out_shift) % L] for o in range(Lout)])
