"""Time-segmented normal operators NORMAL_IDT_T1/T2_OP and the noise-weighted NORMAL_IDTW_T1/T2_OP
against the FP64 oracle, which restates the reference's toeplitz_multiplication call sequence and
TorchScript epilogues (cpp/corelib/lib/mri/normal.cppm:185-720)."""
import numpy as np
import pytest

from helpers import crand, relerr, to_dev, to_np
from oracle import toeplitz as otp


def _problem(seed, shape, C, L):
    rng = np.random.default_rng(seed)
    x = crand(rng, *shape)
    Psi = crand(rng, C, *shape)
    K = crand(rng, L, *[2 * s for s in shape])
    R = np.exp(1j * rng.uniform(0, 2 * np.pi, (L, *shape))).astype(np.complex64)
    A = crand(rng, C, C)
    W = (A @ A.conj().T + C * np.eye(C)).astype(np.complex64)  # Hermitian positive definite
    return x, Psi, K, R, W


def test_oracle_idtw_identity_weights_is_idt():
    """With W = I the noise-weighted operators reduce to the plain time-segmented ones."""
    x, Psi, K, R, _ = _problem(0, (6, 5, 4), 3, 2)
    I = np.eye(3)
    assert relerr(otp.normal_idtw_t1(K, R, Psi, I, x), otp.normal_idt_t1(K, R, Psi, x)) <= 1e-12
    assert relerr(otp.normal_idtw_t2(K, R, x, I, Psi), otp.normal_idt_t2(K, R, x, Psi)) <= 1e-12


def test_oracle_weight_folding():
    """sum_i conj(Psi_i) sum_j W_ij v_j == sum_j conj(U_j) v_j with U = W^H Psi (the folding the
    fused NORMAL_IDTW_T1 path uses)."""
    rng = np.random.default_rng(1)
    C, n = 5, 40
    Psi, v, W = crand(rng, C, n), crand(rng, C, n), crand(rng, C, C)
    lhs = (np.conj(Psi) * (W @ v)).sum(0)
    U = W.conj().T @ Psi
    rhs = (np.conj(U) * v).sum(0)
    assert relerr(lhs, rhs) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("shape,C,L", [((12, 10, 8), 3, 2), ((20, 16), 4, 3), ((8, 8, 8), 1, 1)])
def test_normal_idt_t1(cuda, shape, C, L):
    import hastycucompute_b200 as hb
    x, Psi, K, R, _ = _problem(C + L, shape, C, L)
    op = hb.NormalIDTT1Op(to_dev(K, cuda), to_dev(R, cuda), to_dev(Psi, cuda))
    got = to_np(op(to_dev(x, cuda)))
    ref = otp.normal_idt_t1(K.astype(np.complex128), R, Psi, x)
    assert relerr(got, ref) <= 1e-5
    # a second apply into the same output buffer gives the same result (the first segment overwrites)
    out = to_dev(np.zeros_like(x), cuda)
    op.apply(to_dev(x, cuda), out)
    op.apply(to_dev(x, cuda), out)
    assert relerr(to_np(out), ref) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("shape,C,L", [((12, 10, 8), 3, 2), ((20, 16), 4, 3)])
def test_normal_idtw_t1(cuda, shape, C, L):
    import hastycucompute_b200 as hb
    x, Psi, K, R, W = _problem(10 + C, shape, C, L)
    op = hb.NormalIDTWT1Op(to_dev(K, cuda), to_dev(R, cuda), to_dev(Psi, cuda), to_dev(W, cuda))
    got = to_np(op(to_dev(x, cuda)))
    ref = otp.normal_idtw_t1(K.astype(np.complex128), R, Psi, W, x)
    assert relerr(got, ref) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("shape,C,L", [((12, 10, 8), 3, 2), ((20, 16), 4, 3)])
def test_normal_idt_t2(cuda, shape, C, L):
    import hastycucompute_b200 as hb
    x, Psi, K, R, W = _problem(20 + C, shape, C, L)
    op = hb.NormalIDTT2Op(to_dev(K, cuda), to_dev(R, cuda), to_dev(x, cuda))
    got = to_np(op(to_dev(Psi, cuda)))
    assert relerr(got, otp.normal_idt_t2(K.astype(np.complex128), R, x, Psi)) <= 1e-5
    opw = hb.NormalIDTWT2Op(to_dev(K, cuda), to_dev(R, cuda), to_dev(x, cuda), to_dev(W, cuda))
    gotw = to_np(opw(to_dev(Psi, cuda)))
    assert relerr(gotw, otp.normal_idtw_t2(K.astype(np.complex128), R, x, W, Psi)) <= 1e-5


@pytest.mark.gpu
def test_sense_normal_ex_reduces_to_sense_normal(cuda):
    """No diagonal, no output maps, no accumulation: the generalised apply is hb_sense_normal."""
    import hastycucompute_b200 as hb
    x, Psi, K, _, _ = _problem(7, (16, 12, 10), 4, 1)
    Kt = hb.transform_toeplitz_kernel(to_dev(K[0], cuda))
    a = hb.sense_normal(to_dev(x, cuda), to_dev(Psi, cuda), Kt)
    b = hb.sense_normal_ex(to_dev(x, cuda), to_dev(Psi, cuda), Kt, to_dev(np.zeros_like(x), cuda))
    assert relerr(to_np(b), to_np(a)) <= 1e-6
    # accumulate adds onto what is there
    c = to_dev(x.copy(), cuda)
    hb.sense_normal_ex(to_dev(x, cuda), to_dev(Psi, cuda), Kt, c, accumulate=True)
    assert relerr(to_np(c), to_np(a) + x) <= 1e-6
