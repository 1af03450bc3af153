"""Time-segmentation interpolators (hastycucompute_b200.offres.tseg_interpolators) against the
numpy restatement of the reference's fit (hasty_python/simul_op.py:11-34), on CPU and on the GPU,
and on the GPU feeding the time-segmented normal operator NORMAL_IDT_T1_OP (kernel weights |b_l|^2,
kernel diagonals ct_l) against the oracle's operator with the same inputs."""
import math

import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import offres as ooff


def _rate_map(shape, seed=0):
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*[np.linspace(-1, 1, n) for n in shape], indexing="ij")
    r2 = 5.0 + 45.0 * rng.random(shape)                           # 1/s, varies per voxel
    f = 100.0 * (0.75 - sum(g ** 2 for g in grids) / len(shape))  # Hz, -25 .. 75
    return r2 + 1j * 2 * math.pi * f


@pytest.mark.parametrize("shape,M,lseg", [((12, 12, 12), 800, 6), ((20, 20), 500, 4)])
def test_tseg_interpolators_match_reference_arithmetic_cpu(shape, M, lseg):
    import torch
    from hastycucompute_b200 import offres
    z = _rate_map(shape)
    t = np.linspace(0.0, 5e-3, M)
    bins = z.size // 100
    b_ref, ct_ref = ooff.tseg_interpolators(z, t, bins, lseg)
    b, ct = offres.tseg_interpolators(torch.from_numpy(z), torch.from_numpy(t), bins, lseg)
    assert b.shape == (lseg, M) and tuple(ct.shape) == (lseg, *shape)
    # b passes through the pseudo-inverse of a sampled exponential basis (condition number ~1e8):
    # both sides agree to FP64 rounding times that
    assert relerr(b.numpy(), b_ref) <= 1e-6
    assert relerr(ct.numpy(), ct_ref) <= 1e-12
    counts, edges = offres.histogram(torch.from_numpy(np.imag(2j * np.pi * z)), bins)
    h_ref, e_ref = np.histogram(np.imag(2j * np.pi * z).ravel(), bins)
    assert np.array_equal(counts.numpy(), h_ref) and np.allclose(edges.numpy(), e_ref, rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_tseg_interpolators_on_gpu_feed_the_time_segmented_normal(cuda):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import offres, synthetic
    from oracle import toeplitz as otp
    shape, C, M, lseg, w = (16, 16, 16), 4, 6000, 4, 6
    z = _rate_map(shape, seed=1)
    t = np.linspace(0.0, 4e-3, M)
    bins = z.size // 100
    b_ref, ct_ref = ooff.tseg_interpolators(z, t, bins, lseg)
    b, ct = offres.tseg_interpolators(to_dev(z, cuda), to_dev(t, cuda), bins, lseg)
    assert relerr(to_np(b), b_ref) <= 1e-6
    assert relerr(to_np(ct), ct_ref) <= 1e-12
    rng = np.random.default_rng(2)
    coords = rand_coords(rng, 3, M)
    dc = [to_dev(c, cuda) for c in coords]
    wts = (b.abs() ** 2).to(torch.float32)
    kernels = torch.stack([hb.build_toeplitz_kernel(dc, shape, wts[l].contiguous(), kernel_width=w) for l in range(lseg)])
    diags = ct.to(torch.complex64)
    S = synthetic.coil_maps(C, shape)
    x = crand(rng, *shape)
    op = hb.NormalIDTT1Op(kernels, diags, to_dev(S, cuda))
    got = to_np(op(to_dev(x, cuda)))
    Kn = [to_np(k).astype(np.complex128) for k in kernels]
    ref = otp.normal_idt_t1(Kn, to_np(diags).astype(np.complex128), S, x)
    assert relerr(got, ref) <= 1e-5
