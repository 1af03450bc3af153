"""Preconditioned / restarted CG (cpp/corelib/lib/op/cg.cppm:16-119) and the power iteration
max_eig (cpp/corelib/lib/op/alg.cppm:15-30) against their FP64 oracle restatements."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import cg as ocg
from oracle import toeplitz as otp


def _dense(seed, n=24):
    rng = np.random.default_rng(seed)
    G = crand(rng, n, n).astype(np.complex128)
    H = G @ G.conj().T + n * np.eye(n)
    return H, crand(rng, n).astype(np.complex128)


def test_oracle_pcg_identity_is_cg():
    H, b = _dense(0)
    A = lambda v: H @ v
    x1 = ocg.conjugate_gradient_precond(A, lambda v: v, b, np.zeros_like(b), 7, 1, tol=0.0)
    x2, _ = ocg.conjugate_gradient(A, b, np.zeros_like(b), 7, tol=0.0)
    assert relerr(x1, x2) <= 1e-12


def test_oracle_pcg_converges_with_restarts():
    H, b = _dense(1)
    d = 1.0 / np.real(np.diag(H))
    x = ocg.conjugate_gradient_precond(lambda v: H @ v, lambda v: d * v, b, np.zeros_like(b), 10, 6, tol=1e-12,
                                       should_restart=lambda x, k: k % 5 == 0)
    assert relerr(H @ x, b) <= 1e-8


def test_oracle_max_eig():
    H, _ = _dense(2)
    m, _ = ocg.max_eig(lambda v: H @ v, np.ones(H.shape[0], np.complex128), 200)
    assert abs(m - np.linalg.eigvalsh(H).max()) <= 1e-6 * m


def _sense_problem(cuda, shape=(12, 12, 12), C=4, M=6000, w=4, seed=3):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(seed)
    coords = rand_coords(rng, len(shape), M)
    S = synthetic.coil_maps(C, shape)
    K = hb.build_toeplitz_kernel([to_dev(c, cuda) for c in coords], shape, kernel_width=w)
    op = hb.NormalTT1Op(K, to_dev(S, cuda))
    Kn = to_np(K).astype(np.complex128)
    A_np = lambda v: otp.sense_normal(v, S, Kn)
    b = A_np(synthetic.image(shape)).astype(np.complex64)
    d = (0.5 + rng.uniform(0, 1, shape)).astype(np.float32)  # positive diagonal preconditioner
    return op, A_np, b, d


@pytest.mark.gpu
def test_pcg_matches_oracle_with_restart(cuda):
    import torch
    import hastycucompute_b200 as hb
    op, A_np, b, d = _sense_problem(cuda)
    dd = to_dev(d, cuda)
    calls = {"n": 0, "after": 0}

    def should_restart(x):
        calls["n"] += 1
        return calls["n"] == 3

    def after(x):
        calls["after"] += 1

    cgl = hb.conjugate_gradient_precond(op, lambda v: v * dd, max_inner_iter=5, max_outer_iter=2, tol=0.0)
    x = cgl(torch.zeros(b.shape, dtype=torch.complex64, device=cuda), to_dev(b, cuda), should_restart, after)
    ref = ocg.conjugate_gradient_precond(A_np, lambda v: d * v, b, np.zeros_like(b), 5, 2, tol=0.0,
                                         should_restart=lambda x, k: k == 3)
    assert relerr(to_np(x), ref) <= 1e-5
    assert calls["after"] == 2
    rz, it, conv = cgl.state.read(cuda)
    assert it == 3 + 5


@pytest.mark.gpu
def test_pcg_no_callbacks_and_break(cuda):
    """Without callbacks nothing is read back; once sqrt(Re<r,z>) < tol the steps are no-ops."""
    import torch
    import hastycucompute_b200 as hb
    op, A_np, b, d = _sense_problem(cuda, shape=(10, 10, 10), seed=4)
    dd = to_dev(d, cuda)
    full = ocg.conjugate_gradient_precond(A_np, lambda v: d * v, b, np.zeros_like(b), 4, 1, tol=0.0)
    cgl = hb.conjugate_gradient_precond(op, lambda v: v * dd, max_inner_iter=4, max_outer_iter=1, tol=0.0)
    x = cgl(torch.zeros(b.shape, dtype=torch.complex64, device=cuda), to_dev(b, cuda))
    assert relerr(to_np(x), full) <= 1e-5
    # a tolerance above the initial residual: no step runs, x stays at x0
    cgl2 = hb.conjugate_gradient_precond(op, lambda v: v * dd, max_inner_iter=4, max_outer_iter=3, tol=1e30)
    x2 = cgl2(torch.zeros(b.shape, dtype=torch.complex64, device=cuda), to_dev(b, cuda))
    assert float(torch.abs(x2).max()) == 0.0
    assert cgl2.state.read(cuda)[1] == 0


@pytest.mark.gpu
def test_max_eig_matches_oracle(cuda):
    import torch
    import hastycucompute_b200 as hb
    op, A_np, b, _ = _sense_problem(cuda, shape=(10, 12, 8), seed=5)
    rng = np.random.default_rng(6)
    x0 = crand(rng, *b.shape)
    m, x = hb.max_eig(op, to_dev(x0, cuda), 12)
    mr, xr = ocg.max_eig(A_np, x0, 12)
    assert abs(m - mr) <= 1e-5 * mr
    assert relerr(to_np(x), xr) <= 1e-4
