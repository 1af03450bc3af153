"""Gradient waveform -> k-space -> NUFFT coordinates (hastycucompute_b200.trajectory), the bridge
from the reference's trajectory-design code (hasty_python/hastycompute/seq_design/
gradient_design.py:167-175) into the differentiable NUFFT: the k-space integral and slew rate
against numpy on CPU, and on the GPU the gradient of a trajectory-design loss with respect to the
waveform samples against central differences of the FP64 NUDFT loss."""
import math

import numpy as np
import pytest

from helpers import relerr, to_dev, to_np

GAMMA = 42.577478518e6  # Hz/T
RASTER = 10e-6          # s


def _waveform(B=4, N=200, amp=0.6, seed=0):
    rng = np.random.default_rng(seed)
    t = np.arange(N) / N
    w = np.zeros((B, 3, N))
    for b in range(B):
        ph = 2 * math.pi * b / B + rng.uniform(0, 0.1)
        w[b, 0] = amp * np.sin(2 * math.pi * 3 * t + ph) * t
        w[b, 1] = amp * np.cos(2 * math.pi * 3 * t + ph) * t
        w[b, 2] = 0.1 * amp * np.sin(2 * math.pi * t)
    return w


def _coords_np(w, voxel):
    """FP64 restatement: 1e-3 gamma cumulative trapezoid, then 2 pi k dx, interleaves concatenated."""
    k = 1e-3 * GAMMA * np.cumsum(0.5 * (w[..., 1:] + w[..., :-1]) * RASTER, axis=-1)
    kr = 2 * math.pi * k[:, :2] * np.asarray(voxel)[None, :, None]
    return kr.transpose(1, 0, 2).reshape(2, -1)


def test_kspace_integral_slew_and_coords_match_numpy():
    import torch
    from hastycucompute_b200 import trajectory as tj
    w = _waveform()
    wt = torch.from_numpy(w)
    k = tj.kspace_from_waveform(wt, RASTER, GAMMA).numpy()
    ref = 1e-3 * GAMMA * np.cumsum(0.5 * (w[..., 1:] + w[..., :-1]) * RASTER, axis=-1)
    assert np.allclose(k, ref, rtol=1e-12, atol=1e-12)
    assert np.allclose(tj.slew_rate(wt, RASTER).numpy(), (w[..., 1:] - w[..., :-1]) / (1e3 * RASTER))
    c = tj.waveform_to_coords(wt, RASTER, GAMMA, (0.01, 0.01), axes=(0, 1))
    assert c.dtype == torch.float32 and tuple(c.shape) == (2, 4 * 199)
    assert np.allclose(c.numpy(), _coords_np(w, (0.01, 0.01)), rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
def test_waveform_gradient_through_nufft_matches_finite_differences(cuda):
    import torch
    from hastycucompute_b200 import autograd as ag, synthetic, trajectory as tj
    from oracle import nudft
    N, C, lam = 24, 3, 1e-6
    shape, voxel = (N, N), (0.24 / N, 0.24 / N)
    w0 = _waveform()
    S = synthetic.coil_maps(C, shape)
    x_true = synthetic.image(shape)
    x0 = synthetic.image(shape, seed=5)
    k_true = _coords_np(w0, voxel)
    y = nudft.type2(list(k_true), S * x_true[None], sign=-1)
    pair = ag.NufftPair(shape, C, kernel_width=8)
    Sd, yd, xd = to_dev(S, cuda), to_dev(y.astype(np.complex64), cuda), to_dev(x0, cuda)

    wg = torch.tensor(w0 * 1.05, dtype=torch.float32, device=cuda, requires_grad=True)
    coords = tj.waveform_to_coords(wg, RASTER, GAMMA, voxel, axes=(0, 1))
    r = ag.nufft_forward(Sd * xd[None], coords, pair) - yd
    g = (torch.conj(Sd) * ag.nufft_adjoint(r, coords, pair)).sum(0)
    loss = (g.abs() ** 2).sum() + lam * (tj.slew_rate(wg, RASTER) ** 2).sum()
    loss.backward()
    grad = to_np(wg.grad).astype(np.float64)

    def loss_np(w):
        k = _coords_np(w, voxel)
        Ax = nudft.type2(list(k), S * x0[None], sign=-1)
        gi = (np.conj(S) * nudft.type1(list(k), Ax - y, shape, sign=1)).sum(0)
        sl = (w[..., 1:] - w[..., :-1]) / (1e3 * RASTER)
        return float((np.abs(gi) ** 2).sum() + lam * (sl ** 2).sum())

    base = (w0 * 1.05).astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(9)
    h = 1e-4
    fd, got = [], []
    for _ in range(8):
        b, a, t = int(rng.integers(0, 4)), int(rng.integers(0, 2)), int(rng.integers(1, 150))
        wp, wm = base.copy(), base.copy()
        wp[b, a, t] += h
        wm[b, a, t] -= h
        fd.append((loss_np(wp) - loss_np(wm)) / (2 * h))
        got.append(grad[b, a, t])
    assert relerr(np.array(got), np.array(fd)) <= 1e-3
