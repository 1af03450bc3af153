"""Frames with their own Toeplitz kernels in one launch per pass (hb_sense_normal_batched) and
frame-batched CG with per-frame scalars, against per-frame applies and the oracle."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import cg as ocg
from oracle import toeplitz as otp

PARITY = 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("shape,F,C", [((16, 16, 16), 3, 4), ((20, 18, 16), 4, 12), ((32, 32, 32), 2, 16),
                                       ((64, 64), 5, 12), ((24, 40), 3, 1)])
def test_batched_normal_matches_per_frame(cuda, shape, F, C):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(F * 10 + C)
    S = synthetic.coil_maps(C, shape)
    Ks = np.stack([crand(rng, *[2 * s for s in shape]) for _ in range(F)])
    x = np.stack([crand(rng, *shape) for _ in range(F)])
    op = hb.BatchedNormalOp(to_dev(Ks, cuda), to_dev(S, cuda))
    got = to_np(op(to_dev(x, cuda)))
    for f in range(F):
        ref = otp.sense_normal(x[f], S, Ks[f].astype(np.complex128))
        assert relerr(got[f], ref) <= PARITY, f
        single = hb.NormalTT1Op(to_dev(Ks[f], cuda), to_dev(S, cuda))
        assert relerr(got[f], to_np(single(to_dev(x[f], cuda)))) <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_batched_cg_matches_per_frame_oracle(cuda, graph):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(4)
    shape, F, C, iters = (12, 12, 12), 3, 4, 8
    S = synthetic.coil_maps(C, shape)
    frames = [rand_coords(rng, 3, int(rng.integers(2000, 5000))) for _ in range(F)]
    Ks = hb.build_toeplitz_kernels([[to_dev(c, cuda) for c in fc] for fc in frames], shape, kernel_width=4)
    op = hb.BatchedNormalOp(Ks, to_dev(S, cuda))
    Kn = to_np(Ks).astype(np.complex128)
    xt = np.stack([synthetic.image(shape, seed=f) for f in range(F)])
    b = np.stack([otp.sense_normal(xt[f], S, Kn[f]) for f in range(F)]).astype(np.complex64)
    solver = hb.BatchedCGSolver(lambda v, o: op.apply(v, o), F, shape, cuda, max_iter=iters, tol=0.0, graph=graph)
    x = to_np(solver.solve(torch.zeros((F, *shape), dtype=torch.complex64, device=cuda), to_dev(b, cuda)))
    rz, it, conv = solver.read()
    for f in range(F):
        ref, hist = ocg.conjugate_gradient(lambda v: otp.sense_normal(v, S, Kn[f]), b[f],
                                           np.zeros(shape, np.complex64), iters, tol=0.0)
        assert relerr(x[f], ref) <= 1e-5, f
        assert it[f] == iters
        assert abs(rz[f] - hist[-1]) <= 1e-3 * hist[-1] + 1e-12


@pytest.mark.gpu
def test_batched_cg_per_frame_early_exit(cuda):
    """Each frame stops on its own residual, like a per-frame loop of the reference CG."""
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(6)
    shape, F, C = (10, 10, 10), 2, 3
    S = synthetic.coil_maps(C, shape)
    frames = [rand_coords(rng, 3, 3000), rand_coords(rng, 3, 4000)]
    Ks = hb.build_toeplitz_kernels([[to_dev(c, cuda) for c in fc] for fc in frames], shape, kernel_width=4)
    Kn = to_np(Ks).astype(np.complex128)
    op = hb.BatchedNormalOp(Ks, to_dev(S, cuda))
    b = np.stack([otp.sense_normal(synthetic.image(shape, seed=f), S, Kn[f]) for f in range(F)]).astype(np.complex64)
    _, h0 = ocg.conjugate_gradient(lambda v: otp.sense_normal(v, S, Kn[0]), b[0], np.zeros(shape, np.complex64), 30, 0.0)
    tol = float(np.sqrt(h0[4])) * 1.0001   # frame 0 breaks after 4 steps
    solver = hb.BatchedCGSolver(lambda v, o: op.apply(v, o), F, shape, cuda, max_iter=12, tol=tol, graph=True)
    x = to_np(solver.solve(torch.zeros((F, *shape), dtype=torch.complex64, device=cuda), to_dev(b, cuda)))
    rz, it, conv = solver.read()
    assert it[0] == 4 and conv[0]
    for f in range(F):
        ref, hist = ocg.conjugate_gradient(lambda v: otp.sense_normal(v, S, Kn[f]), b[f],
                                           np.zeros(shape, np.complex64), 12, tol=tol)
        assert it[f] == len(hist) - 1
        assert relerr(x[f], ref) <= 1e-5
