"""numpy restatement of the reference's time-segmentation interpolators
(hasty_python/simul_op.py:11-34, ``tseg_interpolators``) -- TEST INFRASTRUCTURE ONLY.

Line by line the reference's cupy arithmetic on numpy: the histogram of Im(2 pi i z) over the
flattened map, the bin centres 0.5 * (edges[1:] - edges[1]), Ch = exp(tl zk), P = pinv(W Ch^T) W,
b = P exp(-zk t), ct = exp(-tl 2 pi i z).
"""
from __future__ import annotations

import numpy as np


def tseg_interpolators(rate_map, t, bins: int, lseg: int):
    rate_map = np.asarray(rate_map, dtype=np.complex128)
    t = np.asarray(t, dtype=np.float64)
    hist_wt, bin_edges = np.histogram(np.imag(2j * np.pi * np.concatenate(rate_map)), bins)
    bin_centers = 0.5 * (bin_edges[1:] - bin_edges[1])
    zk = 0 + 1j * bin_centers
    t = t - t[0]
    T = t[-1]
    tl = np.linspace(0, T, lseg)
    ch = np.exp(tl[:, None] * zk[None, ...])
    w = np.diag(np.sqrt(hist_wt))
    p = np.linalg.pinv(w @ np.transpose(ch)) @ w
    b = p @ np.exp(-zk[..., None] * t[None, :])
    ct = np.exp(-tl.reshape((-1,) + (1,) * rate_map.ndim) * (2j * np.pi * rate_map)[None])
    return b, ct
