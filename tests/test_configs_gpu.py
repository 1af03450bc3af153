"""Parity at the benchmark configurations' own sizes, each test named for its configuration.

Every result is compared with the FP64 CPU oracle of the same algorithm (``oracle.gridding`` with
its multithreaded C spreading, ``oracle.toeplitz``, ``oracle.cg``, ``oracle.loss``) and must agree
to relative L2 <= 1e-5 (the FP32 parity bar); gradients agree with central differences of the
FP64 oracle loss to <= 1e-3.

- config 0: 64^3, 8 coils, golden-means radial 1024 x 128 (131 k points), KB w=4: Toeplitz kernel,
  plain SENSE A / A^H / A^H A (hasty_python/right_precond_test.py:48-73), every step of the
  10-iteration graph-captured Toeplitz CG and of the 10-iteration plain-operator CG against the
  reference recurrence (cpp/corelib/lib/op/cg.cppm:122-184);
- configs 0 / 2 / 4: 3-D NUFFT type 1 and type 2 at 64^3 and 128^3 modes (fine grids 128^3, 256^3);
- config 1: 160^3, 32 coils, cones 24000 x 256 (6.1 M points), |k|^2 DCF, w=6: Toeplitz kernel,
  type 1 / type 2 (two of the 32 transforms checked) and A^H A (four coils checked);
- config 2: three of the 24 frames (128^3, 16 coils, 300-700 spokes x 128, w=4): per-frame kernel
  and every step of the batched graph-captured 15-iteration CG against the per-frame recurrence;
- config 3: 2-D 256^2, 12 coils, 32 variable-density spirals x 2048, w=4: image gradient and 64
  coordinate gradients of ||A^H(Ax - y)||^2 + lam * slew;
- config 4: 4 volumes of 128^3, 12 coils, 3-D radial 16384 x 128 each, w=4: the batched apply and
  the gradients of 10 unrolled CG iterations in their learnable scalars against central
  differences of the same forward.
"""
import math

import numpy as np
import pytest

from helpers import relerr, to_dev, to_np
from oracle import cg as ocg
from oracle import gridding
from oracle import toeplitz as otp

PARITY = 1e-5


def _stepwise_cg(solver, A_np, iters, b, x0, frames=None):
    """Device CG against the reference recurrence, one iteration at a time: the start (r0 = b - A x0,
    p0 = r0) and then, before every device iteration, one FP64 oracle iteration
    (oracle.cg.cg_iteration, cpp/corelib/lib/op/cg.cppm:139-150) from the device's own x, r, p; the
    device's next x, r, p must equal it. Returns the largest relative L2 error seen.

    Comparing each step rather than the whole run keeps FP32 rounding from being amplified by the
    conditioning of the system: on the un-compensated radial trajectories of configurations 0 and 2
    a CG run in FP32 arithmetic (numpy, FP64 dots) drifts 1e-1 from the FP64 run after 10 iterations,
    the device run 1e-2, while every device step stays at FP32 rounding of the recurrence."""
    solver.start(to_dev(x0, solver.x.device), to_dev(b, solver.x.device))
    nf = 1 if frames is None else frames
    worst = 0.0

    def split(t):
        a = to_np(t).astype(np.complex128)
        return [a] if frames is None else list(a)

    for f, (x, r, p) in enumerate(zip(split(solver.x), split(solver.r), split(solver.p))):
        bf = b if frames is None else b[f]
        xf = x0 if frames is None else x0[f]
        r0 = np.asarray(bf, np.complex128) - A_np(f)(np.asarray(xf, np.complex128))
        worst = max(worst, relerr(r, r0), relerr(p, r0))
    for _ in range(iters):
        before = list(zip(split(solver.x), split(solver.r), split(solver.p)))
        solver.run(1)
        after = list(zip(split(solver.x), split(solver.r), split(solver.p)))
        for f in range(nf):
            xo, ro, po, _ = ocg.cg_iteration(A_np(f), *before[f])
            worst = max(worst, relerr(after[f][0], xo), relerr(after[f][1], ro), relerr(after[f][2], po))
    return worst


def _dev_coords(coords, cuda):
    return [to_dev(np.ascontiguousarray(c), cuda) for c in coords]


def _oracle_sense(coords, S, w):
    """FP64 plain SENSE pair (type 2 sign -1, type 1 sign +1) on the gridding oracle."""
    shape = S.shape[1:]
    fwd = gridding.GridPlan(shape, w, sign=-1)
    adj = gridding.GridPlan(shape, w, sign=+1)
    A = lambda x: fwd.type2(coords, S * np.asarray(x, np.complex128)[None])
    AH = lambda y: np.sum(np.conj(S) * adj.type1(coords, y), axis=0)
    return A, AH


# ---- config 0 ------------------------------------------------------------------------------------

@pytest.mark.gpu
def test_config0_full_size_kernel_sense_and_cg(cuda):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    shape, C, w = (64, 64, 64), 8, 4
    n = int(np.prod(shape))
    coords = synthetic.golden_means_radial(1024, 128)
    dc = _dev_coords(coords, cuda)
    S = synthetic.coil_maps(C, shape)
    x_true = synthetic.image(shape)
    Sd = to_dev(S, cuda)

    # Toeplitz kernel (cpp/corelib/lib/fft/nufft.cppm:386-441)
    K = hb.build_toeplitz_kernel(dc, shape, kernel_width=w)
    assert relerr(to_np(K), otp.toeplitz_kernel(list(coords), shape, w=w)) <= PARITY

    # plain SENSE A, A^H and A^H A against the FP64 gridding oracle
    S128 = S.astype(np.complex128)
    A, AH = _oracle_sense(list(coords), S128, w)
    so = hb.SenseOp(dc, Sd, kernel_width=w)
    y_clean = so.forward(to_dev(x_true, cuda))
    y_ref = A(x_true)
    assert relerr(to_np(y_clean), y_ref) <= PARITY
    y = to_np(y_clean) + synthetic.noise(y_ref.shape, 1e-3, seed=2)
    b_gpu = so.adjoint(to_dev(y, cuda)) / n
    b_ref = AH(y.astype(np.complex128)) / n
    assert relerr(to_np(b_gpu), b_ref) <= PARITY
    nrm = so.normal(to_dev(x_true, cuda))
    assert relerr(to_np(nrm), AH(y_ref)) <= PARITY

    # 10-iteration graph-captured CG on the Toeplitz normal operator: every step against the FP64
    # oracle recurrence on the FP64 straight operator with the same kernel
    b = to_np(b_gpu)
    x0 = np.zeros(shape, np.complex64)
    op = hb.NormalTT1Op(K, Sd)
    Kn = to_np(K).astype(np.complex128)
    A_np = lambda v: otp.sense_normal(v, S128, Kn, fast=True)
    solver = hb.CGSolver(lambda v, out: op.apply(v, out), shape, cuda, max_iter=10, tol=0.0, graph=True)
    assert _stepwise_cg(solver, lambda f: A_np, 10, b, x0) <= PARITY

    # 10-iteration CG on the plain operator (1/n) A^H A, every step against the plain oracle
    sv = hb.CGSolver(lambda v, out: out.copy_(so.normal(v) / n), shape, cuda, max_iter=10, tol=0.0)
    assert _stepwise_cg(sv, lambda f: (lambda v: AH(A(v)) / n), 10, b, x0) <= PARITY


# ---- configs 0 / 2 / 4: 3-D NUFFTs on the register-FFT fine grids ------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("nmodes,spokes,T,w", [
    ((64, 64, 64), 1024, 8, 4),       # config 0 (fine grid 128^3)
    ((64, 64, 64), 1024, 3, 6),
    ((128, 128, 128), 500, 4, 4),     # a config-2 frame (fine grid 256^3)
    ((128, 128, 128), 16384, 2, 4),   # a config-4 volume, 2.1 M points
])
def test_configs_0_2_4_nufft3d_register_lengths(cuda, nmodes, spokes, T, w):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    coords = synthetic.golden_means_radial(spokes, 128)
    dc = _dev_coords(coords, cuda)
    M = coords.shape[1]
    rng = np.random.default_rng(spokes + T)
    c = ((rng.standard_normal((T, M)) + 1j * rng.standard_normal((T, M))) / math.sqrt(2)).astype(np.complex64)
    f = ((rng.standard_normal((T, *nmodes)) + 1j * rng.standard_normal((T, *nmodes))) / math.sqrt(2)).astype(np.complex64)
    opts = hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w)
    p1 = hb.NufftPlan(hb.NufftType.TYPE_1, opts)
    p1.setpts(dc)
    got1 = to_np(p1(to_dev(c, cuda)))
    assert relerr(got1, gridding.nufft1(list(coords), c, nmodes, w=w)) <= PARITY
    p2 = hb.NufftPlan(hb.NufftType.TYPE_2, opts)
    p2.setpts(dc)
    got2 = to_np(p2(to_dev(f, cuda)))
    assert relerr(got2, gridding.nufft2(list(coords), f, w=w)) <= PARITY


# ---- config 1 ------------------------------------------------------------------------------------

@pytest.mark.gpu
def test_config1_full_size_kernel_nufft_and_normal(cuda):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    shape, C, w = (160, 160, 160), 32, 6
    coords = synthetic.cones_spiral(24000, 256)
    dcf = synthetic.dcf_k2(coords)
    dc = _dev_coords(coords, cuda)
    M = coords.shape[1]
    S = synthetic.coil_maps(C, shape)
    x = synthetic.image(shape)

    K = hb.build_toeplitz_kernel(dc, shape, to_dev(dcf, cuda), kernel_width=w)
    K_ref = otp.toeplitz_kernel(list(coords), shape, dcf, w=w)
    assert relerr(to_np(K), K_ref) <= PARITY
    del K_ref

    # all 32 transforms run; the first two are checked against the oracle
    opts = hb.NufftOpts(nmodes=shape, ntransf=C, kernel_width=w)
    p2 = hb.NufftPlan(hb.NufftType.TYPE_2, opts)
    p2.setpts(dc)
    f = to_dev(S, cuda) * to_dev(x, cuda)[None]
    y = p2(f)
    fn = (S[:2] * x[None]).astype(np.complex64)
    assert relerr(to_np(y[:2]), gridding.nufft2(list(coords), fn, w=w)) <= PARITY
    p1 = hb.NufftPlan(hb.NufftType.TYPE_1, opts)
    p1.setpts(dc)
    g = p1(y)
    yn = to_np(y[:2])
    assert relerr(to_np(g[:2]), gridding.nufft1(list(coords), yn, shape, w=w)) <= PARITY
    del p1, p2, f, y, g

    # A^H A on four of the coils (the fused apply treats coils alike, the sum is over those four)
    S4 = to_dev(S[:4], cuda)
    op = hb.NormalTT1Op(K, S4)
    got = to_np(op(to_dev(x, cuda)))
    ref = otp.sense_normal(x, S[:4], to_np(K).astype(np.complex128), fast=True)
    assert relerr(got, ref) <= PARITY
    del op, K
    torch.cuda.empty_cache()


# ---- config 2 ------------------------------------------------------------------------------------

def _config2_frames(nframes=24):
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(3)
    spokes = rng.integers(300, 701, nframes)
    return [synthetic.golden_means_radial(int(ns), 128, offset=int(spokes[:f].sum())) for f, ns in enumerate(spokes)]


@pytest.mark.gpu
def test_config2_batched_graph_cg_three_frames(cuda):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    shape, C, w, iters, F = (128, 128, 128), 16, 4, 15, 3
    n = int(np.prod(shape))
    frames = _config2_frames()[:F]
    xs = synthetic.dynamic_images(24, shape)[:F]
    S = synthetic.coil_maps(C, shape)
    Sd = to_dev(S, cuda)
    dcs = [_dev_coords(fc, cuda) for fc in frames]
    Ks = hb.build_toeplitz_kernels(dcs, shape, kernel_width=w)
    assert relerr(to_np(Ks[0]), otp.toeplitz_kernel(list(frames[0]), shape, w=w)) <= PARITY

    so = hb.SenseOp(dcs[0], Sd, kernel_width=w)
    b = torch.empty((F, *shape), dtype=torch.complex64, device=cuda)
    for f in range(F):
        so.setpts(dcs[f])
        yf = so.forward(to_dev(xs[f], cuda))
        yf = yf + to_dev(synthetic.noise(tuple(yf.shape), 1e-3 * float(yf.abs().max()), seed=2 + f), cuda)
        b[f] = so.adjoint(yf) / n
    op = hb.BatchedNormalOp(Ks, Sd)
    solver = hb.BatchedCGSolver(lambda v, o: op.apply(v, o), F, shape, cuda, max_iter=iters, tol=0.0, graph=True)
    S128 = S.astype(np.complex128)
    Kn = [to_np(Ks[f]).astype(np.complex128) for f in range(F)]
    A_f = lambda f: (lambda v: otp.sense_normal(v, S128, Kn[f], fast=True))
    worst = _stepwise_cg(solver, A_f, iters, to_np(b), np.zeros((F, *shape), np.complex64), frames=F)
    assert worst <= PARITY


# ---- config 3 ------------------------------------------------------------------------------------

@pytest.mark.gpu
def test_config3_full_size_image_and_coordinate_gradients(cuda):
    import torch
    from hastycucompute_b200 import autograd as ag, synthetic
    from oracle.loss import SenseLoss
    shape, C, ninter, ns, w, lam, h = (256, 256), 12, 32, 2048, 4, 1e-3, 1e-4
    k0 = synthetic.variable_density_spiral_2d(ninter, ns)
    M = k0.shape[1]
    S = synthetic.coil_maps(C, shape)
    x_true = synthetic.image(shape)
    x0 = synthetic.image(shape, seed=5)
    Sd = to_dev(S, cuda)
    pair = ag.NufftPair(shape, C, kernel_width=w)
    kk = to_dev(k0, cuda)
    with torch.no_grad():
        y = ag.nufft_forward(Sd * to_dev(x_true, cuda)[None], kk, pair)
    xg = to_dev(x0, cuda).requires_grad_(True)
    kg = kk.clone().requires_grad_(True)
    r = ag.nufft_forward(Sd * xg[None], kg, pair) - y
    gimg = (torch.conj(Sd) * ag.nufft_adjoint(r, kg, pair)).sum(0)
    k3 = kg.reshape(2, ninter, ns)
    slew = ((k3[:, :, 2:] - 2 * k3[:, :, 1:-1] + k3[:, :, :-2]) ** 2).sum()
    loss = (gimg.abs() ** 2).sum() + lam * slew
    loss.backward()

    ol = SenseLoss(S, to_np(y), k0, w=w, lam=lam, interleaves=ninter)
    L = ol.setup(x0)
    assert abs(loss.item() - L) <= 1e-5 * L
    assert relerr(to_np(xg.grad), ol.image_grad()) <= PARITY

    rng = np.random.default_rng(4)
    picks = []
    while len(picks) < 64:
        a, j = divmod(int(rng.integers(0, 2 * M)), M)
        if (a, j) not in picks and not ol.crosses_cell(a, j, h):
            picks.append((a, j))
    fd = np.array([ol.coord_fd(a, j, h) for a, j in picks])
    gk = to_np(kg.grad).astype(np.float64)
    got = np.array([gk[a, j] for a, j in picks])
    assert relerr(got, fd) <= 1e-3


# ---- config 4 ------------------------------------------------------------------------------------

@pytest.mark.gpu
def test_config4_full_size_apply_and_unrolled_scalar_gradients(cuda):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    from hastycucompute_b200.unrolled import UnrolledCG
    F, shape, C, w, K_it = 4, (128, 128, 128), 12, 4, 10
    frames = [synthetic.golden_means_radial(16384, 128, offset=16384 * f) for f in range(F)]
    dcs = [_dev_coords(fc, cuda) for fc in frames]
    Ks = hb.build_toeplitz_kernels(dcs, shape, kernel_width=w)
    del dcs
    S = synthetic.coil_maps(C, shape)
    op = hb.BatchedNormalOp(Ks, to_dev(S, cuda))
    xt = to_dev(synthetic.dynamic_images(F, shape), cuda)
    b = op(xt)
    ref = otp.sense_normal(to_np(xt[0]), S, to_np(Ks[0]).astype(np.complex128), fast=True)
    assert relerr(to_np(b[0]), ref) <= PARITY

    net = UnrolledCG(op, iterations=K_it, step_init=0.9, lam_init=0.01, checkpoint=True).to(cuda)

    def loss_fn():
        return ((net(b) - xt).abs() ** 2).double().sum()

    loss_fn().backward()
    grads = {"steps": net.steps.grad.clone(), "lams": net.lams.grad.clone()}

    def central(param, k, h):
        v0 = float(param[k])
        param[k] = v0 + h
        lp = loss_fn().item()
        param[k] = v0 - h
        lm = loss_fn().item()
        param[k] = v0
        return (lp - lm) / (2 * h)

    # central differences with two Richardson steps, (64 D(h/4) - 20 D(h/2) + D(h)) / 45 (error
    # O(h^6)): the loss bends sharply in the first step, where D(1e-2) alone is 60 % off and one
    # Richardson step still 0.2 %; the weights' gradients are small (0.1 .. 10) and need a wider
    # step to rise above the FP32 rounding of the forward (about 1e-4 in the loss)
    with torch.no_grad():
        for name, param, h in (("steps", net.steps, 4e-3), ("lams", net.lams, 8e-2)):
            fd = [(64 * central(param, k, h / 4) - 20 * central(param, k, h / 2) + central(param, k, h)) / 45
                  for k in range(K_it)]
            assert relerr(to_np(grads[name]), np.array(fd)) <= 1e-3, name
