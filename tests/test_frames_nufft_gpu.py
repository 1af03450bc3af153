"""Frame-batched NUFFT (hb_nufft_setpts_frames): several frames, each with its own trajectory and
any number of points (empty frames included), in one plan with one launch per pass. Each frame's
result is checked against the FP64 gridding oracle on that frame alone (relative L2 <= 1e-5) and
against a one-frame plan on the same points; the frame-batched Toeplitz kernel build and the
frame-batched plain SENSE operator against their one-frame counterparts and the oracle."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import gridding
from oracle import toeplitz as otp

PARITY = 1e-5

CASES = [
    # dim, nmodes, points per frame, ntransf, width
    (2, (24, 20), (3000, 0, 1700), 1, 4),
    (2, (32, 32), (2500, 4100), 12, 6),
    (3, (16, 16, 16), (4000, 2500, 0, 3100), 8, 4),
    (3, (16, 12, 20), (5000, 1200), 5, 6),
    (3, (20, 20, 20), (3000, 6000, 2000), 32, 6),
    (3, (12, 14, 10), (2000, 3000), 2, 5),
]


def _frames(rng, dim, counts):
    return [rand_coords(rng, dim, m) for m in counts]


def _plan(hb, ntype, nmodes, T, w):
    return hb.NufftPlan(ntype, hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w))


@pytest.mark.gpu
@pytest.mark.parametrize("dim,nmodes,counts,T,w", CASES)
def test_frames_type1_parity(cuda, dim, nmodes, counts, T, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(101 + sum(counts))
    fr = _frames(rng, dim, counts)
    c = [crand(rng, T, m) for m in counts]
    plan = _plan(hb, hb.NufftType.TYPE_1, nmodes, T, w)
    plan.setpts_frames([[to_dev(x, cuda) for x in f] for f in fr])
    got = to_np(plan(to_dev(np.concatenate(c, axis=1), cuda)))
    assert got.shape == (len(counts), T, *nmodes)
    single = _plan(hb, hb.NufftType.TYPE_1, nmodes, T, w)
    for f, m in enumerate(counts):
        if m == 0:
            assert np.all(got[f] == 0)
            continue
        ref = gridding.nufft1(fr[f], c[f], nmodes, w=w)
        assert relerr(got[f], ref) <= PARITY, f"frame {f}"
        single.setpts([to_dev(x, cuda) for x in fr[f]])
        one = to_np(single(to_dev(c[f], cuda)))
        assert relerr(got[f], one) <= 1e-6, f"frame {f} vs one-frame plan"


@pytest.mark.gpu
@pytest.mark.parametrize("dim,nmodes,counts,T,w", CASES)
def test_frames_type2_parity(cuda, dim, nmodes, counts, T, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(202 + sum(counts))
    fr = _frames(rng, dim, counts)
    modes = crand(rng, len(counts), T, *nmodes)
    plan = _plan(hb, hb.NufftType.TYPE_2, nmodes, T, w)
    plan.setpts_frames([[to_dev(x, cuda) for x in f] for f in fr])
    got = to_np(plan(to_dev(modes, cuda)))
    assert got.shape == (T, sum(counts))
    single = _plan(hb, hb.NufftType.TYPE_2, nmodes, T, w)
    off = np.concatenate([[0], np.cumsum(counts)])
    for f, m in enumerate(counts):
        if m == 0:
            continue
        part = got[:, off[f]: off[f + 1]]
        ref = gridding.nufft2(fr[f], modes[f], w=w)
        assert relerr(part, ref) <= PARITY, f"frame {f}"
        single.setpts([to_dev(x, cuda) for x in fr[f]])
        one = to_np(single(to_dev(modes[f], cuda)))
        assert relerr(part, one) <= 1e-6, f"frame {f} vs one-frame plan"


@pytest.mark.gpu
def test_frames_staged_interpolation_and_spread_kernels(cuda):
    """The staged interpolation kernel and both spreading kernels take frames the same way."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(7)
    nmodes, T, w, counts = (16, 16, 16), 8, 6, (3000, 0, 5000)
    fr = _frames(rng, 3, counts)
    dfr = [[to_dev(x, cuda) for x in f] for f in fr]
    modes = crand(rng, len(counts), T, *nmodes)
    out = {}
    for kind in ("gather", "staged"):
        p = _plan(hb, hb.NufftType.TYPE_2, nmodes, T, w)
        p.set_interp_kernel(kind)
        p.setpts_frames(dfr)
        out[kind] = to_np(p(to_dev(modes, cuda)))
    assert np.array_equal(out["gather"], out["staged"])
    c = crand(rng, T, sum(counts))
    res = {}
    for kind in ("cells", "transforms"):
        p = _plan(hb, hb.NufftType.TYPE_1, nmodes, T, w)
        p.set_spread_kernel(kind)
        p.setpts_frames(dfr)
        res[kind] = to_np(p(to_dev(c, cuda)))
    off = np.concatenate([[0], np.cumsum(counts)])
    for f, m in enumerate(counts):
        if m:
            ref = gridding.nufft1(fr[f], c[:, off[f]: off[f + 1]], nmodes, w=w)
            for kind in res:
                assert relerr(res[kind][f], ref) <= PARITY, (kind, f)


@pytest.mark.gpu
def test_frames_replanned_and_regrown(cuda):
    """A plan re-pointed from one frame to more frames (its grids grow) and back to one frame gives
    the one-frame results."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(9)
    nmodes, T, w = (20, 24), 3, 5
    p = _plan(hb, hb.NufftType.TYPE_1, nmodes, T, w)
    a = rand_coords(rng, 2, 2000)
    ca = crand(rng, T, 2000)
    p.setpts([to_dev(x, cuda) for x in a])
    first = to_np(p(to_dev(ca, cuda)))
    fr = _frames(rng, 2, (1000, 3000, 500))
    c = [crand(rng, T, m) for m in (1000, 3000, 500)]
    p.setpts_frames([[to_dev(x, cuda) for x in f] for f in fr])
    got = to_np(p(to_dev(np.concatenate(c, axis=1), cuda)))
    for f in range(3):
        assert relerr(got[f], gridding.nufft1(fr[f], c[f], nmodes, w=w)) <= PARITY
    p.setpts([to_dev(x, cuda) for x in a])
    again = to_np(p(to_dev(ca, cuda)))
    # three transforms spread with the cells kernel, whose dense tiles add their extra chunks
    # atomically: equal up to the order of those sums
    assert relerr(again, first) <= 1e-6
    assert relerr(again, gridding.nufft1(a, ca, nmodes, w=w)) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("shape,counts", [((12, 10, 14), (2500, 0, 1800)), ((20, 24), (3000, 1200))])
def test_toeplitz_kernels_frames(cuda, shape, counts):
    import torch

    import hastycucompute_b200 as hb
    rng = np.random.default_rng(31 + len(shape))
    dim = len(shape)
    fr = _frames(rng, dim, counts)
    wts = [rng.uniform(0.5, 2.0, m).astype(np.float32) for m in counts]
    dfr = [[to_dev(x, cuda) for x in f] for f in fr]
    K = hb.build_toeplitz_kernels(dfr, shape, weights=[to_dev(v, cuda) for v in wts], kernel_width=6)
    assert tuple(K.shape) == (len(counts), *(2 * s for s in shape))
    for f, m in enumerate(counts):
        if m == 0:
            assert float(K[f].abs().max()) == 0.0
            continue
        one = hb.build_toeplitz_kernel(dfr[f], shape, to_dev(wts[f], cuda), kernel_width=6)
        assert relerr(to_np(K[f]), to_np(one)) <= 1e-6
        ref = otp.toeplitz_kernel(fr[f], shape, wts[f].astype(np.complex128), w=6)
        assert relerr(to_np(K[f]), ref) <= PARITY
    # one group per frame (a small memory bound) gives the same kernels
    K1 = hb.build_toeplitz_kernels(dfr, shape, weights=[to_dev(v, cuda) for v in wts], kernel_width=6, max_bytes=1)
    assert relerr(to_np(K1), to_np(K)) <= 1e-6
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_batched_sense_op_matches_oracle_per_frame(cuda):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(5)
    shape, C, w, counts = (12, 12, 12), 4, 6, (3000, 2200, 4100)
    fr = _frames(rng, 3, counts)
    S = synthetic.coil_maps(C, shape)
    x = crand(rng, len(counts), *shape)
    op = hb.BatchedSenseOp([[to_dev(v, cuda) for v in f] for f in fr], to_dev(S, cuda), kernel_width=w)
    got = to_np(op.normal(to_dev(x, cuda)))
    for f in range(len(counts)):
        y = gridding.nufft2(fr[f], S * x[f][None], w=w)
        ref = (np.conj(S) * gridding.nufft1(fr[f], y, shape, w=w)).sum(0)
        assert relerr(got[f], ref) <= PARITY, f"frame {f}"


@pytest.mark.gpu
def test_frames_coordinate_gradient(cuda):
    """The coordinate gradient of a frame-batched type-2 plan equals each frame's own."""
    import hastycucompute_b200 as hb
    from hastycucompute_b200.autograd import coord_grad
    rng = np.random.default_rng(17)
    nmodes, T, w, counts = (12, 16, 14), 4, 6, (1500, 0, 2600)
    fr = _frames(rng, 3, counts)
    modes = crand(rng, len(counts), T, *nmodes)
    h = crand(rng, T, sum(counts))
    plan = _plan(hb, hb.NufftType.TYPE_2, nmodes, T, w)
    plan.setpts_frames([[to_dev(x, cuda) for x in f] for f in fr])
    got = to_np(coord_grad(plan, to_dev(modes, cuda), to_dev(h, cuda)))
    single = _plan(hb, hb.NufftType.TYPE_2, nmodes, T, w)
    off = np.concatenate([[0], np.cumsum(counts)])
    for f, m in enumerate(counts):
        if m == 0:
            continue
        single.setpts([to_dev(x, cuda) for x in fr[f]])
        one = to_np(coord_grad(single, to_dev(modes[f], cuda), to_dev(np.ascontiguousarray(h[:, off[f]: off[f + 1]]), cuda)))
        assert relerr(got[:, off[f]: off[f + 1]], one) <= 1e-6, f"frame {f}"
