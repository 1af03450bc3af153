"""Time-segmentation interpolators for off-resonance, as the reference's simulation code fits them
(hasty_python/simul_op.py:11-34, ``tseg_interpolators``), in torch on the device of the rate map.

For a rate map z(r) (complex, per voxel) and sample times t_j, the signal factor exp(-z(r) t_j)
is approximated by sum_l ct_l(r) b_l(t_j) with L segment times tl = linspace(0, T, L):

    weights  h, edges = histogram(Im(2 pi i z), bins)      (flattened map)
    centres  zk = i * 0.5 * (edges[1:] - edges[1])
    Ch[l, k] = exp(tl_l zk_k),  W = diag(sqrt(h))
    P        = pinv(W Ch^T) W                               [L, bins]
    b        = P exp(-zk t^T)                               [L, M]   temporal interpolators
    ct[l]    = exp(-tl_l 2 pi i z)                          [L, N..] spatial factors

exactly the reference's arithmetic (its histogram variable, bin centres and pseudo-inverse), so
the same inputs give the same interpolators. ``b`` and ``ct`` feed ``SenseOffresOp`` (b, c) and the
time-segmented normal operators (``NormalIDTT1Op`` kernel diagonals ct, kernel weights from b).
The pseudo-inverse uses numpy's default cut-off (singular values below 1e-15 of the largest are
dropped) so both follow the same rank decision.
"""
from __future__ import annotations

import math

import torch


def histogram(values: torch.Tensor, bins: int):
    """numpy.histogram(values, bins) for real values: equal-width bins over [min, max] (a zero
    width widened by 0.5 on both sides), the last bin closed. Returns (counts float64, edges)."""
    v = values.reshape(-1).to(torch.float64).contiguous()
    lo, hi = float(v.min()), float(v.max())
    if lo == hi:
        lo, hi = lo - 0.5, hi + 0.5
    edges = torch.linspace(lo, hi, bins + 1, dtype=torch.float64, device=v.device)
    idx = torch.bucketize(v, edges, right=True) - 1
    idx = torch.clamp(idx, 0, bins - 1)  # v == hi lands in the last bin
    counts = torch.bincount(idx, minlength=bins).to(torch.float64)
    return counts, edges


def tseg_interpolators(rate_map: torch.Tensor, t: torch.Tensor, bins: int, lseg: int):
    """(b [lseg, M] complex128, ct [lseg, *rate_map.shape] complex128)."""
    z = rate_map.to(torch.complex128)
    t = t.to(torch.float64).reshape(-1)
    hist_wt, edges = histogram(torch.imag(2j * math.pi * z), bins)
    centers = 0.5 * (edges[1:] - edges[1])
    zk = 1j * centers.to(torch.complex128)
    t = t - t[0]
    T = float(t[-1])
    tl = torch.linspace(0.0, T, lseg, dtype=torch.float64, device=z.device)
    ch = torch.exp(tl[:, None].to(torch.complex128) * zk[None, :])
    w = torch.diag(torch.sqrt(hist_wt)).to(torch.complex128)
    a = w @ ch.transpose(0, 1)
    p = torch.linalg.pinv(a, rtol=1e-15) @ w
    b = p @ torch.exp(-zk[:, None] * t[None, :].to(torch.complex128))
    ct = torch.exp(-tl.reshape((-1,) + (1,) * z.dim()).to(torch.complex128) * (2j * math.pi * z)[None])
    return b, ct
