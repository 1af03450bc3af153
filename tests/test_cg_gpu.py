"""Conjugate gradient on the GPU (device scalars, FP64 dots) against the oracle CG
(cpp/corelib/lib/op/cg.cppm:122-184 restated), plain and CUDA-graph captured."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import cg as ocg
from oracle import toeplitz as otp


def _problem(cuda, shape=(16, 16, 16), C=8, M=10000, w=6, seed=0):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(seed)
    coords = rand_coords(rng, len(shape), M)
    S = synthetic.coil_maps(C, shape)
    x_true = synthetic.image(shape)
    K = hb.build_toeplitz_kernel([to_dev(c, cuda) for c in coords], shape, kernel_width=w)
    op = hb.NormalTT1Op(K, to_dev(S, cuda))
    Kn = to_np(K).astype(np.complex128)
    A_np = lambda v: otp.sense_normal(v, S, Kn)
    b = A_np(x_true).astype(np.complex64)
    return op, A_np, b, shape


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_cg_matches_oracle(cuda, graph):
    import torch
    import hastycucompute_b200 as hb
    op, A_np, b, shape = _problem(cuda)
    iters = 10
    x_ref, hist = ocg.conjugate_gradient(A_np, b, np.zeros(shape, np.complex64), iters, tol=0.0, dtype=np.complex128)
    solver = hb.CGSolver(lambda v, out: op.apply(v, out), shape, cuda, max_iter=iters, tol=0.0, graph=graph)
    x = solver.solve(torch.zeros(shape, dtype=torch.complex64, device=cuda), to_dev(b, cuda))
    assert relerr(to_np(x), x_ref) <= 1e-5
    rz, it, conv = solver.state.read(cuda)
    assert it == iters
    assert abs(rz - hist[-1]) <= 1e-3 * hist[-1] + 1e-12


@pytest.mark.gpu
def test_cg_functional_api(cuda):
    import torch
    import hastycucompute_b200 as hb
    op, A_np, b, shape = _problem(cuda, shape=(12, 14), C=4, M=3000, w=4, seed=1)
    x_ref, _ = ocg.conjugate_gradient(A_np, b, np.zeros(shape, np.complex64), 8, tol=0.0)
    cgl = hb.conjugate_gradient(op, max_iter=8, tol=0.0)
    x = cgl(torch.zeros(shape, dtype=torch.complex64, device=cuda), to_dev(b, cuda))
    assert relerr(to_np(x), x_ref) <= 1e-5


@pytest.mark.gpu
def test_cg_early_exit_matches_reference_break(cuda):
    """Once sqrt(rzold) < tol the remaining steps leave x unchanged (the reference's break)."""
    import torch
    import hastycucompute_b200 as hb
    op, A_np, b, shape = _problem(cuda, shape=(10, 10, 10), C=4, M=6000, w=4, seed=2)
    _, hist = ocg.conjugate_gradient(A_np, b, np.zeros(shape, np.complex64), 30, tol=0.0)
    tol = float(np.sqrt(hist[6])) * 1.0001  # breaks at the top of iteration 7
    x_ref, h2 = ocg.conjugate_gradient(A_np, b, np.zeros(shape, np.complex64), 30, tol=tol)
    assert len(h2) - 1 == 6
    solver = hb.CGSolver(lambda v, out: op.apply(v, out), shape, cuda, max_iter=30, tol=tol, graph=True)
    x = solver.solve(torch.zeros(shape, dtype=torch.complex64, device=cuda), to_dev(b, cuda))
    rz, it, conv = solver.state.read(cuda)
    assert it == 6 and conv
    assert relerr(to_np(x), x_ref) <= 1e-5


@pytest.mark.gpu
def test_vdot_real(cuda):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(5)
    for n in (1, 1000, 1 << 20, 3_000_001):
        a, b = crand(rng, n), crand(rng, n)
        got = hb.vdot_real(to_dev(a, cuda), to_dev(b, cuda)).item()
        ref = float(np.sum(a.real.astype(np.float64) * b.real + a.imag.astype(np.float64) * b.imag))
        assert abs(got - ref) <= 1e-12 * max(1.0, np.sum(np.abs(a) * np.abs(b)))
        # deterministic
        assert hb.vdot_real(to_dev(a, cuda), to_dev(b, cuda)).item() == got
