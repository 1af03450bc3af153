"""Seeded synthetic inputs with the shapes of the benchmark workloads (no dataset is needed).

Images: complex Gaussian x centred ellipsoid; coil maps: Gaussian magnitude centred on points of a
sphere (radius 40 voxels at 64^3, scaled with N) x a linear phase ramp, root-sum-of-squares 1;
trajectories in radians on [-pi, pi): 3-D golden-means radial, 3-D cones-like spirals with |k|^2
density compensation, golden-angle radial with a per-frame spoke count, 2-D variable-density
spirals. Seeds: image 0, coils 1, noise 2, trajectory 3.
"""
from __future__ import annotations

import math

import numpy as np

PHI1, PHI2 = 0.4656, 0.6823  # 3-D golden means (Chan et al., MRM 2009)


def ellipsoid_mask(shape, axes=(0.42, 0.36, 0.30)):
    grids = np.meshgrid(*[(np.arange(n) - n / 2 + 0.5) / n for n in shape], indexing="ij")
    r2 = sum((g / a) ** 2 for g, a in zip(grids, axes[-len(shape):]))
    return (r2 <= 0.25).astype(np.float64)


def image(shape, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return (x * ellipsoid_mask(shape) / math.sqrt(2)).astype(np.complex64)


def dynamic_images(nframes: int, shape, seed: int = 0) -> np.ndarray:
    """Frames whose ellipsoid intensities vary sinusoidally in time."""
    rng = np.random.default_rng(seed)
    base = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    outer = ellipsoid_mask(shape)
    inner = ellipsoid_mask(shape, axes=(0.2, 0.16, 0.12))
    out = []
    for t in range(nframes):
        a = 1.0 + 0.5 * math.sin(2 * math.pi * t / nframes)
        out.append(base * (outer + (a - 1.0) * inner))
    return (np.stack(out) / math.sqrt(2)).astype(np.complex64)


def coil_maps(ncoils: int, shape, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = len(shape)
    N = max(shape)
    radius = 40.0 * N / 64.0
    grids = np.meshgrid(*[np.arange(n) - n / 2 + 0.5 for n in shape], indexing="ij")
    maps = []
    for c in range(ncoils):
        if d == 3:
            z = 1 - 2 * (c + 0.5) / ncoils
            a = math.pi * (3 - math.sqrt(5)) * c
            center = radius * np.array([z, math.sqrt(1 - z * z) * math.cos(a), math.sqrt(1 - z * z) * math.sin(a)])
        else:
            a = 2 * math.pi * c / ncoils
            center = radius * np.array([math.cos(a), math.sin(a)])
        r2 = sum((g - cc) ** 2 for g, cc in zip(grids, center))
        mag = np.exp(-r2 / (2 * (0.6 * N) ** 2))
        ramp = sum(rng.uniform(-0.5, 0.5) * math.pi * g / n for g, n in zip(grids, shape))
        maps.append(mag * np.exp(1j * (ramp + rng.uniform(0, 2 * math.pi))))
    s = np.stack(maps)
    s /= np.sqrt(np.sum(np.abs(s) ** 2, axis=0, keepdims=True))
    return s.astype(np.complex64)


def _radial_samples(nsamp: int) -> np.ndarray:
    return (np.arange(nsamp) - nsamp / 2) * (2 * math.pi / nsamp)


def golden_means_radial(nspokes: int, nsamp: int, offset: int = 0) -> np.ndarray:
    n = np.arange(offset, offset + nspokes, dtype=np.float64)
    z = np.mod(n * PHI1, 1.0) * 2 - 1
    az = 2 * math.pi * np.mod(n * PHI2, 1.0)
    st = np.sqrt(1 - z * z)
    dirs = np.stack([z, st * np.cos(az), st * np.sin(az)])  # [3, S]; dim 0 pairs with z
    r = _radial_samples(nsamp)
    k = dirs[:, :, None] * r[None, None, :]
    return k.reshape(3, -1).astype(np.float32)


def golden_angle_radial_2d(nspokes: int, nsamp: int) -> np.ndarray:
    ga = math.pi * (3 - math.sqrt(5))
    a = np.arange(nspokes) * ga
    r = _radial_samples(nsamp)
    k = np.stack([np.cos(a)[:, None] * r, np.sin(a)[:, None] * r])
    return k.reshape(2, -1).astype(np.float32)


def cones_spiral(ninter: int, nsamp: int, turns: float = 6.0, seed: int = 3) -> np.ndarray:
    """3-D cones-like spirals: interleave i winds `turns` times around a cone whose axis follows
    a Fibonacci sphere, radius growing linearly to pi."""
    rng = np.random.default_rng(seed)
    i = np.arange(ninter, dtype=np.float64)
    zc = 1 - 2 * (i + 0.5) / ninter
    ac = math.pi * (3 - math.sqrt(5)) * i
    axis = np.stack([zc, np.sqrt(1 - zc * zc) * np.cos(ac), np.sqrt(1 - zc * zc) * np.sin(ac)], axis=1)  # [I,3]
    # orthonormal frame per interleave
    ref = np.where(np.abs(axis[:, 0:1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    e1 = np.cross(axis, ref)
    e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
    e2 = np.cross(axis, e1)
    t = np.arange(nsamp) / nsamp
    r = math.pi * t
    ang = 2 * math.pi * turns * t[None, :] + rng.uniform(0, 2 * math.pi, size=(ninter, 1))
    cone = 0.35  # half-opening of the cone
    k = (r[None, :, None] * (math.cos(cone) * axis[:, None, :]
                             + math.sin(cone) * (np.cos(ang)[:, :, None] * e1[:, None, :]
                                                 + np.sin(ang)[:, :, None] * e2[:, None, :])))
    k = np.clip(k, -math.pi, math.pi * (1 - 1e-6))
    return k.reshape(-1, 3).T.astype(np.float32).copy()


def dcf_k2(coords: np.ndarray) -> np.ndarray:
    """Analytic |k|^2 density compensation, normalised to mean 1."""
    k2 = np.sum(coords.astype(np.float64) ** 2, axis=0)
    return (k2 / k2.mean()).astype(np.float32)


def variable_density_spiral_2d(ninter: int, nsamp: int, alpha: float = 1.5, turns: float = 16.0) -> np.ndarray:
    t = np.arange(nsamp) / nsamp
    r = math.pi * t ** alpha
    base = 2 * math.pi * turns * t
    k = []
    for i in range(ninter):
        a = base + 2 * math.pi * i / ninter
        k.append(np.stack([r * np.cos(a), r * np.sin(a)]))
    k = np.concatenate(k, axis=1)
    return np.clip(k, -math.pi, math.pi * (1 - 1e-6)).astype(np.float32)


def noise(shape, sigma: float, seed: int = 2) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return (sigma * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / math.sqrt(2)).astype(np.complex64)
