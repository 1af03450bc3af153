"""Type-1 spreading with the transforms on the lanes (3-D 8^3 and 2-D 16x32 tiles, widths 4..8,
five or more transforms): parity with the FP64 gridding oracle (relative L2 <= 1e-5) for every
transform chunk (8, 16, 32 lanes and more than 32 transforms), every width, both dimensions,
periodic wrap at the grid edge, dense tiles spread in parts whose partial tiles a second kernel
sums, and bit-identical repeats (the part sums run in a fixed order)."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import gridding

PARITY = 1e-5


def _type1(hb, cuda, coords, c, nmodes, w, maxp=None, kernel="transforms"):
    T = c.shape[0]
    plan = hb.NufftPlan(hb.NufftType.TYPE_1, hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w))
    plan.set_spread_kernel(kernel)
    if maxp is not None:
        plan.set_spread_tuning(maxp, block=(4, 8) if len(nmodes) == 2 else (2, 4, 4))
    plan.setpts([to_dev(x, cuda) for x in coords])
    out = plan(to_dev(c, cuda))
    again = plan(to_dev(c, cuda))
    return to_np(out), to_np(again)


@pytest.mark.gpu
@pytest.mark.parametrize("T", [5, 8, 12, 16, 17, 32, 40])
@pytest.mark.parametrize("w", [4, 6])
def test_lanes_on_transforms_3d_transform_chunks(cuda, T, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(100 * T + w)
    nmodes, M = (20, 24, 16), 7000
    coords = rand_coords(rng, 3, M)
    c = crand(rng, T, M)
    got, again = _type1(hb, cuda, coords, c, nmodes, w)
    assert relerr(got, gridding.nufft1(coords, c, nmodes, w=w)) <= PARITY
    assert np.array_equal(got, again)


@pytest.mark.gpu
@pytest.mark.parametrize("w", [4, 5, 6, 7, 8])
def test_lanes_on_transforms_3d_widths(cuda, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(7 + w)
    nmodes, M, T = (24, 24, 24), 6000, 9
    coords = rand_coords(rng, 3, M)
    c = crand(rng, T, M)
    got, _ = _type1(hb, cuda, coords, c, nmodes, w)
    assert relerr(got, gridding.nufft1(coords, c, nmodes, w=w)) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("nmodes,T,w", [((40, 70), 12, 4), ((32, 48), 32, 6), ((24, 40), 6, 8), ((50, 33), 20, 5)])
def test_lanes_on_transforms_2d(cuda, nmodes, T, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(sum(nmodes) + T)
    M = 5000
    coords = rand_coords(rng, 2, M)
    c = crand(rng, T, M)
    got, _ = _type1(hb, cuda, coords, c, nmodes, w)
    assert relerr(got, gridding.nufft1(coords, c, nmodes, w=w)) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_lanes_on_transforms_periodic_edges(cuda, dim):
    """Points within a kernel half-width of +-pi: footprints wrap onto the first tiles."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(dim)
    nmodes = (16, 20, 24)[-dim:]
    M, T, w = 4000, 16, 6
    coords = [np.where(rng.random(M) < 0.5, rng.uniform(-np.pi, -np.pi + 0.3, M),
                       rng.uniform(np.pi - 0.3, np.pi, M)).astype(np.float32) for _ in range(dim)]
    c = crand(rng, T, M)
    got, _ = _type1(hb, cuda, coords, c, nmodes, w)
    assert relerr(got, gridding.nufft1(coords, c, nmodes, w=w)) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("dim,T,maxp", [(3, 32, None), (3, 32, 64), (3, 12, 32), (2, 12, 64), (3, 8, 128)])
def test_lanes_on_transforms_dense_tiles_in_parts(cuda, dim, T, maxp):
    """Most points in a small ball around k = 0: the centre tiles hold many subproblems, each
    spread by its own CTA into a scratch slot; the partial tiles are summed in part order. The
    cells-on-lanes kernel gives the same transform."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(31 + T + dim)
    nmodes = (32, 32, 32)[-dim:]
    M, w = 30000, 6
    dense = rng.random(M) < 0.7
    coords = [np.where(dense, rng.normal(0.0, 0.15, M), rng.uniform(-np.pi, np.pi, M)).astype(np.float32)
              for _ in range(dim)]
    coords = [np.clip(x, -np.pi, np.pi - 1e-6).astype(np.float32) for x in coords]
    c = crand(rng, T, M)
    got, again = _type1(hb, cuda, coords, c, nmodes, w, maxp=maxp)
    assert relerr(got, gridding.nufft1(coords, c, nmodes, w=w)) <= PARITY
    assert np.array_equal(got, again)
    cells, _ = _type1(hb, cuda, coords, c, nmodes, w, maxp=maxp, kernel="cells")
    assert relerr(cells, got) <= PARITY
