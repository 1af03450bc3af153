"""FP64 restatement of the gridding NUFFT (same kernel, width, upsampling and fine grid as the
GPU plan) -- the "same algorithm" parity oracle.

The reference hands this to cufinufft (cpp/corelib/lib/fft/nufft.cppm:205-250; finufft
"spread / FFT / deapodise", Barnett, Magland, af Klinteberg, SIAM J. Sci. Comput. 41(5) 2019).
Restated here with the Kaiser-Bessel kernel of ``oracle.kb``:

    type 1:  g[l] = sum_j c_j prod_a phi(l_a - u_ja)        (periodic fine grid, u = x nf / 2pi)
             G[k] = sum_l g[l] exp(+i s 2 pi k.l / nf)
             f[k] = G[k mod nf] / prod_a phihat(k_a / nf_a)
    type 2:  the reverse (pre-deapodise, FFT, interpolate).

Coordinates are folded to the fine grid with float32 arithmetic exactly as the device does, so
both pick the same first cell i0 = ceil(u - w/2) for every point; the kernel is then evaluated in
FP64. Spreading and interpolation run in the multithreaded C restatement (``oracle.cgrid``) when
it is built, else in numpy (``backend`` forces one); the fine-grid FFT runs in scipy, FP64.
"""
from __future__ import annotations

import os

import numpy as np

from . import cgrid, kb


class GridPlan:
    def __init__(self, nmodes, w: int, sigma: float = 2.0, sign: int = 1, backend: str = "auto"):
        self.nmodes = tuple(int(n) for n in nmodes)
        self.dim = len(self.nmodes)
        self.w = int(w)
        self.sigma = float(sigma)
        self.sign = int(sign)
        self.beta = kb.beta(self.w, self.sigma)
        self.nf = kb.fine_grid(self.nmodes, self.w, self.sigma)
        if backend == "auto":
            backend = "c" if cgrid.available() else "numpy"
        self.backend = backend

    # -- coordinates --------------------------------------------------------------------------
    def fold(self, x, nf: int):
        """float32 fold of radians onto [0, nf) (same operation order as the device)."""
        x = np.asarray(x, dtype=np.float32)
        scale = np.float32(nf / (2.0 * np.pi))
        fnf = np.float32(nf)
        u = (x * scale).astype(np.float32)
        q = np.floor((u / fnf).astype(np.float32)).astype(np.float32)
        u = (u - (q * fnf).astype(np.float32)).astype(np.float32)
        u = np.where(u < 0, (u + fnf).astype(np.float32), u).astype(np.float32)
        u = np.where(u >= fnf, (u - fnf).astype(np.float32), u).astype(np.float32)
        return u

    def taps(self, x, nf: int):
        """(cells [M, w] ints, weights [M, w] FP64) for one axis."""
        u = self.fold(x, nf)
        hw = np.float32(0.5 * self.w)
        i0 = np.ceil((u - hw).astype(np.float32)).astype(np.int64)
        d = np.arange(self.w)
        cells = i0[:, None] + d[None, :]
        z = cells.astype(np.float64) - u.astype(np.float64)[:, None]
        wts = kb.phi(z, self.w, self.beta)
        return np.mod(cells, nf), wts

    def deapod(self, axis: int) -> np.ndarray:
        N, nf = self.nmodes[axis], self.nf[axis]
        k = np.arange(N) - N // 2
        return 1.0 / kb.phihat(k / nf, self.w, self.beta)

    # -- spread / interp -------------------------------------------------------------------------
    def _flat_taps(self, coords):
        idx = None
        wt = None
        for a in range(self.dim):
            cells, wts = self.taps(coords[a], self.nf[a])
            if idx is None:
                idx, wt = cells, wts
            else:
                idx = idx[:, :, None] * self.nf[a] + cells[:, None, :]
                wt = wt[:, :, None] * wts[:, None, :]
                idx = idx.reshape(idx.shape[0], -1)
                wt = wt.reshape(wt.shape[0], -1)
        return idx, wt  # [M, w^d]

    def spread(self, coords, c):
        if self.backend == "c":
            return cgrid.spread(self.nf, self.w, self.beta, coords, c)
        c = np.asarray(c, dtype=np.complex128)
        idx, wt = self._flat_taps(coords)
        n = int(np.prod(self.nf))
        out = np.empty((c.shape[0], n), dtype=np.complex128)
        fi = idx.reshape(-1)
        for t in range(c.shape[0]):
            v = (wt * c[t][:, None]).reshape(-1)
            out[t] = np.bincount(fi, weights=v.real, minlength=n) + 1j * np.bincount(fi, weights=v.imag, minlength=n)
        return out.reshape(c.shape[0], *self.nf)

    def interp(self, coords, g):
        if self.backend == "c":
            return cgrid.interp(self.nf, self.w, self.beta, coords, np.asarray(g).reshape(g.shape[0], *self.nf))
        g = np.asarray(g, dtype=np.complex128).reshape(g.shape[0], -1)
        idx, wt = self._flat_taps(coords)
        return np.einsum("tmk,mk->tm", g[:, idx], wt, optimize=True)

    # -- FFT over the fine grid ------------------------------------------------------------------
    def _fft(self, a, sign: int):
        import scipy.fft as sf
        axes = tuple(range(1, self.dim + 1))
        workers = len(os.sched_getaffinity(0))
        if sign < 0:
            return sf.fftn(a, axes=axes, workers=workers)
        n = int(np.prod(self.nf))
        return sf.ifftn(a, axes=axes, workers=workers) * n

    def _mode_index(self, axis: int) -> np.ndarray:
        N, nf = self.nmodes[axis], self.nf[axis]
        return np.mod(np.arange(N) - N // 2, nf)

    def type1(self, coords, c):
        g = self.spread(coords, c)
        G = self._fft(g, self.sign)
        sel = np.ix_(*[self._mode_index(a) for a in range(self.dim)])
        out = G[(slice(None),) + sel]
        for a in range(self.dim):
            shp = [1] * (self.dim + 1)
            shp[a + 1] = -1
            out = out * self.deapod(a).reshape(shp)
        return out

    def type2(self, coords, f):
        f = np.asarray(f, dtype=np.complex128)
        T = f.shape[0]
        fh = f.copy()
        for a in range(self.dim):
            shp = [1] * (self.dim + 1)
            shp[a + 1] = -1
            fh = fh * self.deapod(a).reshape(shp)
        Gh = np.zeros((T, *self.nf), dtype=np.complex128)
        sel = np.ix_(*[self._mode_index(a) for a in range(self.dim)])
        Gh[(slice(None),) + sel] = fh
        g = self._fft(Gh, self.sign)
        return self.interp(coords, g)


def nufft1(coords, c, nmodes, w: int, sigma: float = 2.0, sign: int = 1, backend: str = "auto"):
    return GridPlan(nmodes, w, sigma, sign, backend).type1(coords, c)


def nufft2(coords, f, w: int, sigma: float = 2.0, sign: int = -1, backend: str = "auto"):
    return GridPlan(f.shape[1:], w, sigma, sign, backend).type2(coords, f)
