"""FP64 restatement of the trajectory-design loss and its finite differences -- TEST
INFRASTRUCTURE ONLY.

    L(x, k) = || sum_c conj(S_c) A_k^H (A_k (S_c x) - y_c) ||^2 + lam * slew(k)
    slew(k) = sum over interleaves and axes of (k[t+1] - 2 k[t] + k[t-1])^2

with A_k the type-2 gridding NUFFT (sign -1) of ``oracle.gridding`` at the points k and A_k^H the
type-1 (sign +1) on the same points, the same algorithm the GPU path differentiates. The reference
has no derivatives on this path; its trajectory-design code
(hasty_python/hastycompute/seq_design/gradient_design.py:167-171) produces the coordinates.

Central differences in one coordinate k[a, j] change one sample: A_k S x changes in row j only,
and the type-1 fine grid changes in point j's footprint only. ``coord_fd`` therefore evaluates
L(k +- h e_aj) - L(k) exactly, in FP64, from the base fine grids plus the footprint change
(its transform to the modes by a direct sum over the changed cells), and the difference of the
squared norms as 2 Re<g, d> + ||d||^2 so nothing cancels. The moved coordinate is folded in
FP64 (a float32 fold would quantise a 1e-4 step); the point's other axes, and its base position,
keep the float32 fold the base grid (and the device) used.
"""
from __future__ import annotations

import numpy as np

from . import gridding


class SenseLoss:
    def __init__(self, S, y, coords, w: int, lam: float, interleaves: int, sigma: float = 2.0):
        self.S = np.asarray(S, np.complex128)
        self.shape = self.S.shape[1:]
        self.dim = len(self.shape)
        self.y = np.asarray(y, np.complex128)
        self.k = np.asarray(coords, np.float32)
        self.lam = float(lam)
        self.ninter = int(interleaves)
        self.p2 = gridding.GridPlan(self.shape, w, sigma, sign=-1)
        self.p1 = gridding.GridPlan(self.shape, w, sigma, sign=+1)

    # -- whole loss pieces -----------------------------------------------------------------------
    def _fine2(self, f):
        """type-2 fine grid of images f [C, N..]: FFT(pad(deapodise(f)))"""
        p = self.p2
        fh = np.array(f, dtype=np.complex128)
        for a in range(self.dim):
            shp = [1] * (self.dim + 1)
            shp[a + 1] = -1
            fh = fh * p.deapod(a).reshape(shp)
        G = np.zeros((fh.shape[0], *p.nf), dtype=np.complex128)
        sel = np.ix_(*[p._mode_index(a) for a in range(self.dim)])
        G[(slice(None),) + sel] = fh
        return p._fft(G, -1)

    def _modes1(self, G):
        """type-1 fine grid -> deapodised modes"""
        p = self.p1
        F = p._fft(G, +1)
        sel = np.ix_(*[p._mode_index(a) for a in range(self.dim)])
        out = F[(slice(None),) + sel]
        for a in range(self.dim):
            shp = [1] * (self.dim + 1)
            shp[a + 1] = -1
            out = out * p.deapod(a).reshape(shp)
        return out

    def normal(self, x, coords=None):
        """S^H A^H A S x"""
        k = self.k if coords is None else coords
        G2 = self._fine2(self.S * np.asarray(x, np.complex128)[None])
        r = self.p2.interp(list(k), G2)
        return np.sum(np.conj(self.S) * self._modes1(self.p1.spread(list(k), r)), axis=0)

    def slew(self, k):
        kk = np.asarray(k, np.float64).reshape(self.dim, self.ninter, -1)
        return float(np.sum((kk[:, :, 2:] - 2 * kk[:, :, 1:-1] + kk[:, :, :-2]) ** 2))

    def setup(self, x):
        """Base state at image x and the points k."""
        self.x = np.asarray(x, np.complex128)
        self.G2 = self._fine2(self.S * self.x[None])
        self.r = self.p2.interp(list(self.k), self.G2) - self.y
        self.G1 = self.p1.spread(list(self.k), self.r)
        self.g = np.sum(np.conj(self.S) * self._modes1(self.G1), axis=0)
        self.L = float(np.sum(np.abs(self.g) ** 2)) + self.lam * self.slew(self.k)
        return self.L

    def image_grad(self):
        """torch's gradient of the real loss in x (2 dL/dconj(x)) = 2 S^H A^H A S g."""
        return 2.0 * self.normal(self.g)

    # -- one-point changes -------------------------------------------------------------------------
    def _point_taps(self, plan, kpt, fold64_axis: int | None):
        """cells / weights of one point; the axis ``fold64_axis`` is folded in FP64 (a moved
        coordinate), the others in float32 exactly as the base grid was built."""
        cells, wts = [], []
        for a in range(self.dim):
            nf = plan.nf[a]
            if a == fold64_axis:
                u = np.mod(np.float64(kpt[a]) * nf / (2 * np.pi), nf)
                i0 = int(np.ceil(u - 0.5 * plan.w))
                c = i0 + np.arange(plan.w)
                z = c - u
                wt = gridding.kb.phi(z, plan.w, plan.beta)
                cells.append(np.mod(c, nf))
                wts.append(wt)
            else:
                c, wt = plan.taps(np.array([kpt[a]], np.float32), nf)
                cells.append(c[0])
                wts.append(wt[0])
        return cells, wts

    def _interp_point(self, cells, wts):
        sub = self.G2[(slice(None),) + np.ix_(*cells)]
        w = wts[0]
        for a in range(1, self.dim):
            w = np.multiply.outer(w, wts[a])
        return np.tensordot(sub, w, axes=self.dim)

    def _modes_of_cells(self, cells, vals):
        """deapodised type-1 modes of a fine grid that is `vals` [C, w..] on the cell product"""
        p = self.p1
        out = vals
        for a in range(self.dim):
            N, nf = self.shape[a], p.nf[a]
            kk = np.arange(N) - N // 2
            E = np.exp(2j * np.pi * np.outer(kk, cells[a]) / nf) * p.deapod(a)[:, None]   # [N, w]
            out = np.tensordot(out, E, axes=([1], [1]))      # contracts the next cell axis, appends N
        return out                                            # [C, N..]

    def _delta_g(self, j, a, kpt):
        """change of g when coordinate a of point j moves to kpt[a] (FP64 fold on that axis)."""
        c0, w0 = self._point_taps(self.p1, self.k[:, j], None)
        c1, w1 = self._point_taps(self.p1, kpt, a)
        r1 = self._interp_point(c1, w1) - self.y[:, j]
        def outer(ws):
            w = ws[0]
            for a in range(1, self.dim):
                w = np.multiply.outer(w, ws[a])
            return w
        v1 = r1[(slice(None),) + (None,) * self.dim] * outer(w1)[None]
        v0 = self.r[:, j][(slice(None),) + (None,) * self.dim] * outer(w0)[None]
        dimg = self._modes_of_cells(c1, v1) - self._modes_of_cells(c0, v0)
        return np.sum(np.conj(self.S) * dimg, axis=0)

    def coord_fd(self, a: int, j: int, h: float) -> float:
        """(L(k + h e_aj) - L(k - h e_aj)) / 2h, with the base removed exactly."""
        vals = []
        k64 = self.k.astype(np.float64)
        for sgn in (+1, -1):
            kpt = k64[:, j].copy()
            kpt[a] += sgn * h
            d = self._delta_g(j, a, kpt)
            dL = 2.0 * float(np.sum((np.conj(self.g) * d).real)) + float(np.sum(np.abs(d) ** 2))
            kk = k64.copy()
            kk[a, j] = kpt[a]
            vals.append(dL + self.lam * (self.slew(kk) - self.slew(k64)))
        return (vals[0] - vals[1]) / (2 * h)

    def crosses_cell(self, a: int, j: int, h: float) -> bool:
        """True when moving k[a, j] by +-h changes the point's first fine-grid cell along a (the
        truncated kernel is discontinuous there, so no derivative exists)."""
        nf = self.p1.nf[a]
        c0, _ = self.p1.taps(np.array([self.k[a, j]], np.float32), nf)
        i0s = {int(c0[0, 0])}
        for sgn in (-1, 0, 1):
            u = np.mod(np.float64(self.k[a, j]) * nf / (2 * np.pi) + sgn * h * nf / (2 * np.pi), nf)
            i0s.add(int(np.mod(np.ceil(u - 0.5 * self.p1.w), nf)))
        return len(i0s) > 1
