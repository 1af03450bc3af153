"""Properties of the oracle itself (CPU): the adjoint identity of the NUDFT and of the gridding
restatement, and the Toeplitz embedding of the normal operator. These hold for any inputs, so
they check the oracle independently of the golden fixtures."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr
from oracle import gridding, nudft
from oracle import toeplitz as otp


def _inner(a, b):
    return np.vdot(np.asarray(a).ravel(), np.asarray(b).ravel())


@pytest.mark.parametrize("shape,M", [((10,), 30), ((6, 8), 50), ((4, 6, 5), 60)])
def test_nudft_pair_is_adjoint(shape, M):
    """<A f, c> = <f, A^H c> with A = type 2 (sign -1) and A^H = type 1 (sign +1)."""
    rng = np.random.default_rng(11)
    coords = rand_coords(rng, len(shape), M)
    f = crand(rng, 2, *shape).astype(np.complex128)
    c = crand(rng, 2, M).astype(np.complex128)
    lhs = _inner(nudft.type2(coords, f, sign=-1), c)
    rhs = _inner(f, nudft.type1(coords, c, shape, sign=1))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("shape,M,w", [((16,), 40, 4), ((8, 10), 80, 6), ((8, 6, 10), 120, 6)])
def test_gridding_pair_is_adjoint(shape, M, w):
    """The gridding restatement's type 2 and type 1 (opposite signs) are exact adjoints: spread is
    the transpose of interpolate, the FFTs are conjugate, the deapodisation is real."""
    rng = np.random.default_rng(12)
    coords = rand_coords(rng, len(shape), M)
    f = crand(rng, 1, *shape).astype(np.complex128)
    c = crand(rng, 1, M).astype(np.complex128)
    lhs = _inner(gridding.nufft2(coords, f, w=w, sign=-1), c)
    rhs = _inner(f, gridding.nufft1(coords, c, shape, w=w, sign=1))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


@pytest.mark.parametrize("shape,M", [((9,), 25), ((6, 8), 60), ((4, 5, 6), 80)])
def test_exact_toeplitz_is_scaled_normal(shape, M):
    """T x = (1/n) A^H diag(w) A x: the straight Toeplitz multiply (fft/nufft.cppm:448-479) with a
    kernel built from the exact type 1 (fft/nufft.cppm:386-441) reproduces the normal operator of
    the NUDFT pair to FP64 rounding, for odd and even edges."""
    rng = np.random.default_rng(13)
    coords = rand_coords(rng, len(shape), M)
    wts = rng.uniform(0.2, 1.5, M)
    x = crand(rng, *shape).astype(np.complex128)
    K = otp.toeplitz_kernel(coords, shape, weights=wts, exact=True)
    got = otp.toeplitz_multiply(x[None], K)[0]
    Ax = nudft.type2(coords, x[None], sign=-1)
    ref = nudft.type1(coords, Ax * wts[None], shape, sign=1)[0] / float(np.prod(shape))
    assert relerr(got, ref) <= 1e-10


def test_sense_normal_is_coil_sum_of_toeplitz():
    """sum_c conj(S_c) T(S_c x) (mri/normal.cppm:65-88) equals the plain SENSE normal operator
    (1/n) sum_c conj(S_c) A^H A (S_c x) when T carries unit weights."""
    rng = np.random.default_rng(14)
    shape, M, C = (6, 6, 4), 70, 3
    coords = rand_coords(rng, 3, M)
    S = crand(rng, C, *shape).astype(np.complex128)
    x = crand(rng, *shape).astype(np.complex128)
    K = otp.toeplitz_kernel(coords, shape, exact=True)
    got = otp.sense_normal(x, S, K)
    Sx = S * x[None]
    ref = (np.conj(S) * nudft.type1(coords, nudft.type2(coords, Sx, sign=-1), shape, sign=1)).sum(0)
    assert relerr(got, ref / float(np.prod(shape))) <= 1e-10
