"""Shared helpers for the test suite."""
from __future__ import annotations

import numpy as np


def relerr(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def rand_coords(rng, dim, M, lo=-np.pi, hi=np.pi):
    return [rng.uniform(lo, hi, M).astype(np.float32) for _ in range(dim)]


def crand(rng, *shape):
    return ((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)).astype(np.complex64)


def to_dev(a, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


def to_np(t):
    return t.detach().cpu().numpy()
