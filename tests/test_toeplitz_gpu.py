"""Toeplitz kernel build, fused multiplication (all reference flag combinations) and the SENSE
normal operator on the GPU through the C ABI, against the oracle. Bar: relative L2 <= 1e-5."""

import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import refload
from oracle import toeplitz as otp

PARITY = 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("shape,M,w", [((12, 10), 3000, 4), ((16, 16), 5000, 6), ((8, 10, 12), 4000, 4),
                                        ((16, 16, 16), 8000, 6)])
def test_toeplitz_kernel(cuda, shape, M, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(M)
    coords = rand_coords(rng, len(shape), M)
    wts = rng.uniform(0.5, 1.5, M).astype(np.float32)
    K = hb.build_toeplitz_kernel([to_dev(c, cuda) for c in coords], shape, to_dev(wts, cuda), kernel_width=w)
    ref = otp.toeplitz_kernel(coords, shape, wts, w=w)
    assert relerr(to_np(K), ref) <= PARITY
    # and the kernel is the NUDFT one up to the NUFFT accuracy
    if np.prod(shape) <= 4096:
        ex = otp.toeplitz_kernel(coords, shape, wts, exact=True)
        assert relerr(to_np(K), ex) <= {4: 2e-3, 6: 3e-5}[w]


FLAGS = [
    (0, 1, 2, 1, 2, 0),  # the reference defaults
    (2, 1, 0, 0, 0, 0),  # NORMAL_T_T1_OP
    (0, 1, 2, 0, 0, 0),  # NORMAL_T_T2_OP
    (0, 1, 2, 1, 2, 1),
    (1, 2, 1, 2, 1, 1),
    (0, 0, 0, 0, 0, 0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(6, 8, 10), (16, 16, 16), (12, 10), (32, 30), (11, 13, 6), (22, 13)])
@pytest.mark.parametrize("flags", FLAGS)
@pytest.mark.parametrize("use_m2", [False, True])
def test_multiplication_flags(cuda, shape, flags, use_m2):
    import torch
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(hash((shape, flags, use_m2)) % 2**32)
    B = 3
    inp = crand(rng, B, *shape)
    out0 = crand(rng, B, *shape)
    m1 = crand(rng, *shape)
    m2 = crand(rng, *shape) if use_m2 else None
    K = crand(rng, *[2 * s for s in shape]).astype(np.complex128)
    io, i1, o1, i2, o2, acc = flags
    ref = otp.toeplitz_multiplication(inp, out0, K, m1, m2, io, i1, o1, i2, o2, acc)
    Kt = hb.transform_toeplitz_kernel(to_dev(K.astype(np.complex64), cuda))
    out = to_dev(out0, cuda)
    hb.toeplitz_multiplication(to_dev(inp, cuda), out, Kt, None, to_dev(m1, cuda),
                               to_dev(m2, cuda) if use_m2 else None, io, i1, o1, i2, o2, acc)
    assert relerr(to_np(out), ref) <= PARITY
    if refload.available():
        r2 = refload.multiplication(inp, out0, K, m1, m2, io, i1, o1, i2, o2, acc)
        assert relerr(to_np(out), r2) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("shape,C", [((16, 16, 16), 8), ((20, 18, 16), 32), ((10, 12, 14), 40), ((64, 64), 12),
                                     ((24, 40), 3)])
def test_sense_normal(cuda, shape, C):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(C)
    x = crand(rng, *shape)
    S = synthetic.coil_maps(C, shape)
    K = crand(rng, *[2 * s for s in shape]).astype(np.complex128)
    op = hb.NormalTT1Op(to_dev(K.astype(np.complex64), cuda), to_dev(S, cuda))
    got = to_np(op(to_dev(x, cuda)))
    ref = otp.sense_normal(x, S, K)
    assert relerr(got, ref) <= PARITY
    # equals the flat multiplication with the NORMAL_T_T1_OP flags followed by the coil sum
    flat = otp.toeplitz_multiplication(S, np.zeros_like(S), K, x, None, 2, 1, 0, 0, 0, 0).sum(0)
    assert relerr(got, flat) <= PARITY


@pytest.mark.gpu
def test_plain_sense_normal_matches_oracle_and_toeplitz(cuda):
    """The plain SENSE normal operator S^H A^H A S (type 2 then type 1, as
    hasty_python/right_precond_test.py:48-73 applies it) against the FP64 gridding oracle, and the
    fused Toeplitz normal operator against the oracle's straight one built from the same points."""
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    from oracle import gridding
    rng = np.random.default_rng(2)
    shape, C, M, w = (16, 16, 16), 8, 12000, 6
    coords = rand_coords(rng, 3, M)
    S = synthetic.coil_maps(C, shape)
    x = crand(rng, *shape)
    dc = [to_dev(c, cuda) for c in coords]
    sense = hb.SenseOp(dc, to_dev(S, cuda), kernel_width=w)
    plain = to_np(sense.normal(to_dev(x, cuda)))
    S128 = S.astype(np.complex128)
    y = gridding.nufft2(coords, S128 * x[None], w=w)
    ref_plain = np.sum(np.conj(S128) * gridding.nufft1(coords, y, shape, w=w), axis=0)
    assert relerr(plain, ref_plain) <= PARITY
    K = hb.build_toeplitz_kernel(dc, shape, kernel_width=w)
    op = hb.NormalTT1Op(K, to_dev(S, cuda))
    got = to_np(op(to_dev(x, cuda)))
    assert relerr(got, otp.sense_normal(x, S, otp.toeplitz_kernel(coords, shape, w=w))) <= PARITY
    # and T = (1/n) A^H A holds up to the NUFFT error of w = 6
    assert relerr(got, plain / np.prod(shape)) <= 1e-4


@pytest.mark.gpu
def test_workspace_argument(cuda):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import toeplitz as tp
    rng = np.random.default_rng(0)
    shape, B = (8, 8, 8), 2
    inp = crand(rng, B, *shape)
    K = crand(rng, 16, 16, 16)
    Kt = hb.transform_toeplitz_kernel(to_dev(K, cuda))
    ws = tp.make_workspace(shape, B, cuda)
    out = torch.zeros((B, *shape), dtype=torch.complex64, device=cuda)
    got = hb.toeplitz_multiply(to_dev(inp, cuda), Kt, ws)
    assert relerr(to_np(got), otp.toeplitz_multiply(inp, K.astype(np.complex128))) <= PARITY
    small = torch.empty(10, dtype=torch.complex64, device=cuda)
    with pytest.raises(hb.HastyError, match="WORKSPACE"):
        hb.toeplitz_multiplication(to_dev(inp, cuda), out, Kt, small)
    with pytest.raises(hb.HastyError, match="INVALID_ARG"):
        hb.toeplitz_multiplication(to_dev(inp, cuda), out, Kt, None, None, None, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,C", [((32, 32, 32), 5), ((64, 64, 64), 2), ((160, 160), 20), ((128, 128), 3),
                                     ((256, 256), 2), ((320, 320), 1), ((32, 64, 160), 3)])
def test_register_fft_lengths_sense_and_flat(cuda, shape, C):
    """2N in {64, 128, 256, 320, 512, 640}: the two-level register FFT kernels."""
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(C + len(shape))
    x = crand(rng, *shape)
    S = synthetic.coil_maps(C, shape)
    K = crand(rng, *[2 * s for s in shape]).astype(np.complex128)
    Kd = to_dev(K.astype(np.complex64), cuda)
    op = hb.NormalTT1Op(Kd, to_dev(S, cuda))
    assert relerr(to_np(op(to_dev(x, cuda))), otp.sense_normal(x, S, K)) <= PARITY
    out0 = crand(rng, C, *shape)
    out = to_dev(out0, cuda)
    hb.toeplitz_multiplication(to_dev(S, cuda), out, op.kernel_t, None, to_dev(x, cuda), None, 2, 1, 0, 0, 0, 1)
    ref = otp.toeplitz_multiplication(S, out0, K, x, None, 2, 1, 0, 0, 0, 1)
    assert relerr(to_np(out), ref) <= PARITY


@pytest.mark.gpu
def test_toeplitz_kernel_register_lengths(cuda):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(3)
    shape, M, w = (32, 32, 32), 20000, 6
    coords = rand_coords(rng, 3, M)
    K = hb.build_toeplitz_kernel([to_dev(c, cuda) for c in coords], shape, kernel_width=w)
    ref = otp.toeplitz_kernel(coords, shape, None, w=w)
    assert relerr(to_np(K), ref) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("shape,C", [((176, 176, 176), 2), ((176, 208, 220), 2), ((208, 220), 4), ((26, 22, 12), 5)])
def test_sense_normal_lengths_with_factors_11_13(cuda, shape, C):
    """2N with a prime factor 11 or 13 (352, 416, 440, 52, 44): the radix-11 / radix-13 Stockham
    stages. The reference convolves any length through VkFFT (cpp/corelib/lib/fft/toeplitz.cppm:449-480)."""
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(sum(shape))
    x = crand(rng, *shape)
    S = synthetic.coil_maps(C, shape)
    K = crand(rng, *[2 * s for s in shape]).astype(np.complex128)
    op = hb.NormalTT1Op(to_dev(K.astype(np.complex64), cuda), to_dev(S, cuda))
    assert relerr(to_np(op(to_dev(x, cuda))), otp.sense_normal(x, S, K, fast=True)) <= PARITY
