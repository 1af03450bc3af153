"""From gradient waveforms to NUFFT coordinates, differentiably.

The reference's trajectory-design code (hasty_python/hastycompute/seq_design/gradient_design.py)
produces gradient waveforms [B, 3, N] (mT/m on the gradient raster) and integrates them to k-space
with ``calculate_kspace_traj`` (:167-171): k = 1e-3 * gamma * cumulative_trapezoid(g, dx = raster
time), in 1/m; its slew rate is the raster difference (:173-175). The NUFFT here takes coordinates
in radians per voxel, coords[i] pairing with image dimension i. ``waveform_to_coords`` chains the
two -- k_rad = 2 pi k dx with dx the voxel size -- in torch, so a loss on the NUFFT output
(``autograd.nufft_forward`` / ``nufft_adjoint``, whose coordinate gradients are the
kernel-derivative kernels) back-propagates to the gradient waveform itself.
"""
from __future__ import annotations

import math
from typing import Sequence

import torch


def kspace_from_waveform(waveform: torch.Tensor, grad_raster_time: float, gamma: float) -> torch.Tensor:
    """k-space trajectory in 1/m from gradient waveforms [B, 3, N] in mT/m (the reference's
    calculate_kspace_traj): 1e-3 * gamma * cumulative trapezoid along the last axis."""
    return (1e-3 * gamma) * torch.cumulative_trapezoid(waveform, dx=grad_raster_time, dim=-1)


def slew_rate(waveform: torch.Tensor, grad_raster_time: float) -> torch.Tensor:
    """Slew rate in T/m/s (the reference's calculate_slew_rate)."""
    return (waveform[..., 1:] - waveform[..., :-1]) / (1e3 * grad_raster_time)


def kspace_to_radians(ktraj: torch.Tensor, voxel_size: Sequence[float]) -> torch.Tensor:
    """[.., dim, M] k in 1/m -> radians per voxel (2 pi k dx per axis), float32."""
    dx = torch.as_tensor([float(v) for v in voxel_size], dtype=ktraj.dtype, device=ktraj.device)
    shape = [1] * ktraj.dim()
    shape[-2] = -1
    return (2.0 * math.pi * ktraj * dx.reshape(shape)).to(torch.float32)


def waveform_to_coords(waveform: torch.Tensor, grad_raster_time: float, gamma: float,
                       voxel_size: Sequence[float], axes: Sequence[int] | None = None) -> torch.Tensor:
    """Gradient waveforms [B, 3, N] -> NUFFT coordinates [dim, B * (N - 1)] (radians per voxel,
    float32, interleaves concatenated), differentiable in the waveform. ``axes`` picks and orders the
    gradient channels that pair with the image dimensions (default: all three, 3-D)."""
    k = kspace_from_waveform(waveform, grad_raster_time, gamma)         # [B, 3, N-1]
    if axes is not None:
        k = k[:, list(axes)]
    kr = kspace_to_radians(k, voxel_size)                               # [B, dim, N-1]
    return kr.permute(1, 0, 2).reshape(kr.shape[1], -1)
