"""NORMAL_T_T2_OP, the time-segmented off-resonance SENSE pair and the host-staged adjoint NUFFT
against the oracle."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import gridding, nudft
from oracle import toeplitz as otp


@pytest.mark.gpu
@pytest.mark.parametrize("shape,C", [((16, 16, 16), 4), ((40, 32), 6)])
def test_normal_t2(cuda, shape, C):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(C)
    x = crand(rng, *shape)
    Psi = crand(rng, C, *shape)
    K = crand(rng, *[2 * s for s in shape])
    op = hb.NormalTT2Op(to_dev(K, cuda), to_dev(x, cuda))
    got = to_np(op(to_dev(Psi, cuda)))
    ref = otp.toeplitz_multiplication(Psi, np.zeros_like(Psi), K.astype(np.complex128), x, None, 0, 1, 2, 0, 0, 0)
    assert relerr(got, ref) <= 1e-5


@pytest.mark.gpu
def test_offresonance_sense_pair(cuda):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(5)
    shape, C, L, M = (12, 10, 8), 3, 4, 2500
    coords = rand_coords(rng, 3, M)
    S = synthetic.coil_maps(C, shape)
    b = np.exp(1j * rng.uniform(0, 2 * np.pi, (L, M))).astype(np.complex64) / L
    cmap = np.exp(1j * rng.uniform(0, 2 * np.pi, (L, *shape))).astype(np.complex64)
    x = crand(rng, *shape)
    op = hb.SenseOffresOp([to_dev(c, cuda) for c in coords], to_dev(S, cuda), to_dev(b, cuda), to_dev(cmap, cuda),
                          kernel_width=8)
    y = to_np(op.forward(to_dev(x, cuda)))
    img = (S[:, None] * cmap[None] * x[None, None]).reshape(C * L, *shape)
    ref_y = (nudft.type2(coords, img, sign=-1).reshape(C, L, M) * b[None]).sum(1)
    assert relerr(y, ref_y) <= 1e-5
    yy = crand(rng, C, M)
    xa = to_np(op.adjoint(to_dev(yy, cuda)))
    z = (yy[:, None] * np.conj(b)[None]).reshape(C * L, M)
    im = nudft.type1(coords, z, shape, sign=1).reshape(C, L, *shape)
    ref_x = (np.conj(S) * (im * np.conj(cmap)[None]).sum(1)).sum(0)
    assert relerr(xa, ref_x) <= 1e-5
    # adjointness <A x, y> = <x, A^H y>
    lhs = np.vdot(yy.astype(np.complex128), y)
    rhs = np.vdot(xa.astype(np.complex128), x)
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


@pytest.mark.gpu
def test_backward_cpu_over_cuda(cuda):
    import torch
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(6)
    shape, T, M = (16, 12, 10), 5, 3000
    coords = rand_coords(rng, 3, M)
    data = crand(rng, T, M)
    out = hb.nufft_backward_cpu_over_cuda(shape, torch.from_numpy(data), [to_dev(c, cuda) for c in coords],
                                          kernel_width=7)
    assert not out.is_cuda and tuple(out.shape) == (T, *shape)
    assert relerr(out.numpy(), gridding.nufft1(coords, data, shape, w=7)) <= 1e-5
