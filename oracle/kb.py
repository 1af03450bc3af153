"""Kaiser-Bessel spreading kernel and fine-grid sizing (restatement, FP64).

The reference delegates the kernel to cufinufft (cpp/corelib/lib/fft/nufft.cppm:117-165; the
finufft "exponential of semicircle" kernel, source absent). This build uses the Kaiser-Bessel
kernel the hot-path specification names, with Beatty's shape parameter (Beatty, Nishimura,
Pauly, IEEE TMI 24(6) 2005):

    phi(z)    = I0(beta sqrt(1 - (2z/w)^2)) / I0(beta),  |z| < w/2 (fine-grid units)
    beta      = pi sqrt((w/sigma)^2 (sigma - 1/2)^2 - 0.8)
    phihat(x) = w sinh(sqrt(beta^2 - (pi w x)^2)) / sqrt(beta^2 - (pi w x)^2) / I0(beta)

Width from tolerance follows cufinufft's rule for sigma = 2: w = ceil(log10(10/tol)).
"""
from __future__ import annotations

import math

import numpy as np


def width_from_tol(tol: float, sigma: float = 2.0) -> int:
    if sigma >= 2.0:
        w = math.ceil(math.log10(10.0 / tol))
    else:
        w = math.ceil(-math.log(tol) / (math.pi * math.sqrt(1.0 - 1.0 / sigma)))
    return max(2, min(16, w))


def beta(w: int, sigma: float = 2.0) -> float:
    a = w / sigma * (sigma - 0.5)
    v = a * a - 0.8
    return math.pi * math.sqrt(v) if v > 0 else 0.0


def phi(z, w: int, b: float):
    z = np.asarray(z, dtype=np.float64)
    r = 2.0 * z / w
    a = 1.0 - r * r
    out = np.where(a >= 0, np.i0(b * np.sqrt(np.clip(a, 0, None))) / np.i0(b), 0.0)
    return out


def phihat(xi, w: int, b: float):
    xi = np.asarray(xi, dtype=np.float64)
    a = math.pi * w * xi
    d = b * b - a * a
    s = np.sqrt(np.abs(d))
    with np.errstate(invalid="ignore", divide="ignore"):
        v = np.where(d > 1e-12, np.sinh(s) / np.where(s == 0, 1, s),
                     np.where(d < -1e-12, np.sin(s) / np.where(s == 0, 1, s), 1.0))
    return w * v / np.i0(b)


def _smooth235(n: int) -> bool:
    for p in (2, 3, 5):
        while n % p == 0 and n > 1:
            n //= p
    return n == 1


def tiles(dim: int, w: int):
    """Spread tile edge per internal axis (unit leading axes for dim < 3)."""
    if dim == 3:
        e = 8 if w <= 9 else 16
        return (e, e, e)
    if dim == 2:
        return (1, 16, 32)
    return (1, 1, 256)


def fine_size(N: int, sigma: float, w: int, T: int) -> int:
    if N <= 1:
        return 1
    lo = max(math.ceil(sigma * N - 1e-9), 2 * w, T)
    n = lo
    while not (n % T == 0 and _smooth235(n)):
        n += 1
    return n


def fine_grid(nmodes, w: int, sigma: float = 2.0):
    """Fine grid per caller dimension (same rule as the GPU plan)."""
    dim = len(nmodes)
    T = tiles(dim, w)[3 - dim:]
    return tuple(fine_size(int(n), sigma, w, t) for n, t in zip(nmodes, T))
