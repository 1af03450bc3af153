"""CPU checks of the oracle's own pieces that the full-size parity tests rely on: the C gridding
restatement equals the numpy one, the FP64 Toeplitz multiply through torch's CPU FFT equals the
numpy one, and the loss oracle's one-point finite differences equal finite differences of the
whole loss."""
import numpy as np
import pytest

from helpers import relerr
from oracle import cgrid, gridding
from oracle import toeplitz as otp


@pytest.mark.skipif(not cgrid.available(), reason="oracle C gridding library not built")
@pytest.mark.parametrize("shape,w,M,T", [((12,), 4, 300, 2), ((16, 20), 6, 3000, 3), ((16, 16, 16), 4, 4000, 2),
                                         ((10, 12, 14), 7, 2000, 1), ((24, 24, 24), 6, 20000, 3)])
def test_c_gridding_equals_numpy_gridding(shape, w, M, T):
    rng = np.random.default_rng(M)
    coords = [rng.uniform(-np.pi, np.pi, M).astype(np.float32) for _ in shape]
    c = rng.standard_normal((T, M)) + 1j * rng.standard_normal((T, M))
    f = rng.standard_normal((T, *shape)) + 1j * rng.standard_normal((T, *shape))
    assert relerr(gridding.nufft1(coords, c, shape, w, backend="c"), gridding.nufft1(coords, c, shape, w, backend="numpy")) <= 1e-13
    assert relerr(gridding.nufft2(coords, f, w, backend="c"), gridding.nufft2(coords, f, w, backend="numpy")) <= 1e-13


@pytest.mark.parametrize("shape", [(6, 8, 10), (12, 10), (7, 9)])
def test_torch_cpu_toeplitz_equals_numpy(shape):
    rng = np.random.default_rng(sum(shape))
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    S = rng.standard_normal((5, *shape)) + 1j * rng.standard_normal((5, *shape))
    K = rng.standard_normal(tuple(2 * s for s in shape)) + 1j * rng.standard_normal(tuple(2 * s for s in shape))
    assert relerr(otp.sense_normal(x, S, K, fast=True), otp.sense_normal(x, S, K)) <= 1e-13


def test_loss_oracle_one_point_differences_equal_whole_loss_differences():
    from hastycucompute_b200 import synthetic
    from oracle.loss import SenseLoss
    shape, C, ninter, ns, w, lam = (16, 16), 2, 4, 64, 4, 1e-3
    k0 = synthetic.variable_density_spiral_2d(ninter, ns)
    S = synthetic.coil_maps(C, shape).astype(np.complex128)
    x0 = synthetic.image(shape, seed=5).astype(np.complex128)
    y = gridding.nufft2(list(k0), S * synthetic.image(shape)[None], w=w)
    ol = SenseLoss(S, y, k0, w=w, lam=lam, interleaves=ninter)
    L0 = ol.setup(x0)
    # whole-loss evaluation at other points, on a fresh oracle
    def whole(k):
        return SenseLoss(S, y, k, w=w, lam=lam, interleaves=ninter).setup(x0)
    assert abs(whole(k0) - L0) <= 1e-12 * L0
    h = 2e-3
    rng = np.random.default_rng(1)
    checked = 0
    while checked < 6:
        a, j = divmod(int(rng.integers(0, 2 * k0.shape[1])), k0.shape[1])
        if ol.crosses_cell(a, j, h):
            continue
        kp, km = k0.copy(), k0.copy()
        kp[a, j] += np.float32(h)
        km[a, j] -= np.float32(h)
        hh = (float(kp[a, j]) - float(km[a, j])) / 2          # the float32 step actually taken
        ref = (whole(kp) - whole(km)) / (2 * hh)
        got = ol.coord_fd(a, j, hh)
        assert abs(got - ref) <= 1e-4 * abs(ref) + 1e-9 * L0, (a, j, got, ref)
        checked += 1
    # image gradient: torch's convention dL/dRe + i dL/dIm at a few pixels
    g = ol.image_grad()
    for p in rng.choice(np.prod(shape), 4, replace=False):
        i, j = divmod(int(p), shape[1])
        v = []
        for d in (1.0, 1j):
            xp, xm = x0.copy(), x0.copy()
            xp[i, j] += 1e-5 * d
            xm[i, j] -= 1e-5 * d
            v.append((SenseLoss(S, y, k0, w=w, lam=lam, interleaves=ninter).setup(xp)
                      - SenseLoss(S, y, k0, w=w, lam=lam, interleaves=ninter).setup(xm)) / 2e-5)
        assert abs(g[i, j] - (v[0] + 1j * v[1])) <= 1e-5 * abs(g).max()
