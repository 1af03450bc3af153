"""Gradients of the NUFFT with respect to data and coordinates (kernel-derivative interpolation),
checked against (1) central finite differences of the FP64 same-algorithm oracle, (2) the exact
derivative of the FP64 NUDFT (within the kernel's accuracy) and (3) autograd end to end."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import gridding, nudft


def _fd_type2(coords, f, W, w, js, h=1e-6):
    """dL/dx_j for L = Re sum conj(W) * nufft2(f)(x) by central differences of the FP64 oracle."""
    plan = gridding.GridPlan(f.shape[1:], w, sign=-1)
    fh = np.asarray(f, np.complex128)
    # oracle fine grid of f (pre-interpolation stage of the type-2 pipeline)
    T = f.shape[0]
    fh2 = fh.copy()
    for a in range(plan.dim):
        shp = [1] * (plan.dim + 1)
        shp[a + 1] = -1
        fh2 = fh2 * plan.deapod(a).reshape(shp)
    Gh = np.zeros((T, *plan.nf), np.complex128)
    Gh[(slice(None),) + np.ix_(*[plan._mode_index(a) for a in range(plan.dim)])] = fh2
    g = plan._fft(Gh, -1)
    out = np.zeros((len(coords), len(js)))
    for n, j in enumerate(js):
        for a in range(len(coords)):
            vals = []
            for sgn in (+1, -1):
                pt = [np.array([np.float64(c[j])]) for c in coords]
                pt[a] = pt[a] + sgn * h
                # fold in float64 for the FD (the float32 fold would quantise h away)
                y = _interp64(plan, pt, g)
                vals.append(np.sum((np.conj(W[:, j:j + 1]) * y).real))
            out[a, n] = (vals[0] - vals[1]) / (2 * h)
    return out


def _interp64(plan, pts, g):
    from oracle import kb
    idx, wt = None, None
    for a in range(plan.dim):
        nf = plan.nf[a]
        u = np.mod(np.asarray(pts[a], np.float64) * nf / (2 * np.pi), nf)
        i0 = np.ceil(u - 0.5 * plan.w).astype(np.int64)
        cells = i0[:, None] + np.arange(plan.w)[None, :]
        wts = kb.phi(cells - u[:, None], plan.w, plan.beta)
        cells = np.mod(cells, nf)
        if idx is None:
            idx, wt = cells, wts
        else:
            idx = (idx[:, :, None] * nf + cells[:, None, :]).reshape(idx.shape[0], -1)
            wt = (wt[:, :, None] * wts[:, None, :]).reshape(wt.shape[0], -1)
    gf = g.reshape(g.shape[0], -1)
    return np.einsum("tmk,mk->tm", gf[:, idx], wt)


@pytest.mark.gpu
@pytest.mark.parametrize("nmodes,w,T", [((12, 14, 10), 6, 3), ((32, 24), 4, 5), ((40,), 6, 2), ((16, 16, 16), 8, 12)])
def test_type2_coordinate_gradient(cuda, nmodes, w, T):
    import torch
    from hastycucompute_b200 import autograd as ag
    rng = np.random.default_rng(len(nmodes) * 10 + w)
    dim, M = len(nmodes), 1500
    coords = rand_coords(rng, dim, M)
    f = crand(rng, T, *nmodes)
    W = crand(rng, T, M)
    pair = ag.NufftPair(nmodes, T, kernel_width=w)
    pair.setpts(to_dev(np.stack(coords), cuda))
    got = to_np(ag.coord_grad(pair.fwd, to_dev(f, cuda), to_dev(np.conj(W), cuda)))
    js = rng.choice(M, 24, replace=False)
    fd = _fd_type2(coords, f, W, w, js)
    assert relerr(got[:, js], fd) <= 2e-4
    # the exact NUDFT derivative: dc_j/dx_ja = sum_k f_k (-i k_a) e^{-i k x_j}
    ex = np.zeros((dim, len(js)))
    for a in range(dim):
        k = (np.arange(nmodes[a]) - nmodes[a] // 2).reshape([-1 if i == a else 1 for i in range(dim)])
        dy = nudft.type2_at(coords, f * (-1j * k)[None], js, sign=-1)
        ex[a] = np.sum((np.conj(W[:, js]) * dy).real, axis=0)
    # the kernel's accuracy for derivatives (about N times its accuracy for values)
    assert relerr(got[:, js], ex) <= {4: 2e-2, 6: 5e-4, 8: 5e-5}[w]


@pytest.mark.gpu
@pytest.mark.parametrize("nmodes,w,T", [((12, 14, 10), 6, 3), ((32, 24), 6, 2)])
def test_type1_coordinate_gradient(cuda, nmodes, w, T):
    """f = A^H c (type 1, sign +1): dL/dx_j for L = Re sum conj(Wf) f against the exact NUDFT
    derivative  df_k/dx_ja = c_j (i k_a) e^{i k x_j}."""
    import torch
    from hastycucompute_b200 import autograd as ag
    rng = np.random.default_rng(7 + w)
    dim, M = len(nmodes), 1200
    coords = rand_coords(rng, dim, M)
    c = crand(rng, T, M)
    Wf = crand(rng, T, *nmodes)
    pair = ag.NufftPair(nmodes, T, kernel_width=w)
    xc = to_dev(np.stack(coords), cuda).requires_grad_(True)
    cd = to_dev(c, cuda)
    fo = ag.nufft_adjoint(cd, xc, pair)
    L = (torch.conj(to_dev(Wf, cuda)) * fo).real.sum()
    L.backward()
    got = to_np(xc.grad)
    # exact: dL/dx_ja = Re sum_c sum_k conj(Wf_k) c_j (i k_a) e^{i k x_j} = Re sum_c c_j * conj(A_ja Wf)
    # where (A_a Wf)_j = sum_k Wf_k (-i k_a) e^{-i k x_j}
    ex = np.zeros((dim, M))
    for a in range(dim):
        k = (np.arange(nmodes[a]) - nmodes[a] // 2).reshape([-1 if i == a else 1 for i in range(dim)])
        t = nudft.type2(coords, Wf * (-1j * k)[None], sign=-1)   # [T, M]
        ex[a] = np.sum((c * np.conj(t)).real, axis=0)
    assert relerr(got, ex) <= 5e-4


@pytest.mark.gpu
def test_data_gradients_are_adjoints(cuda):
    import torch
    from hastycucompute_b200 import autograd as ag
    rng = np.random.default_rng(3)
    nmodes, T, M = (16, 12, 10), 2, 3000
    coords = np.stack(rand_coords(rng, 3, M))
    pair = ag.NufftPair(nmodes, T, kernel_width=6)
    f = to_dev(crand(rng, T, *nmodes), cuda).requires_grad_(True)
    W = to_dev(crand(rng, T, M), cuda)
    y = ag.nufft_forward(f, to_dev(coords, cuda), pair)
    (torch.conj(W) * y).real.sum().backward()
    ref = nudft.type1(list(coords), to_np(W), nmodes, sign=1)   # A^H W
    assert relerr(to_np(f.grad), ref) <= 5e-5


@pytest.mark.gpu
def test_trajectory_design_loss_matches_finite_differences(cuda):
    """Config-3 style: L = ||A^H(A x - y)||^2 + lam * slew(k) in 2-D with coils; gradients in x
    and in 64 random coordinates against central differences (h = 1e-4) of the FP64 NUDFT loss."""
    import torch
    from hastycucompute_b200 import autograd as ag, synthetic
    rng = np.random.default_rng(11)
    N, C, ninter, ns = 24, 3, 4, 96
    shape = (N, N)
    k0 = synthetic.variable_density_spiral_2d(ninter, ns)          # [2, M]
    M = k0.shape[1]
    S = synthetic.coil_maps(C, shape)
    x_true = synthetic.image(shape)
    y = nudft.type2(list(k0), S * x_true[None], sign=-1).astype(np.complex64)
    x0 = synthetic.image(shape, seed=5)
    lam = 1e-3
    pair = ag.NufftPair(shape, C, kernel_width=8)

    def loss_torch(x, k):
        Ax = ag.nufft_forward(torch.as_tensor(S, device=cuda) * x[None], k, pair)
        r = Ax - torch.as_tensor(y, device=cuda)
        g = (torch.conj(torch.as_tensor(S, device=cuda)) * ag.nufft_adjoint(r, k, pair)).sum(0)
        kk = k.reshape(2, ninter, ns)
        slew = ((kk[:, :, 2:] - 2 * kk[:, :, 1:-1] + kk[:, :, :-2]) ** 2).sum()
        return (g.abs() ** 2).sum() + lam * slew

    def loss_np(x, k):
        Ax = nudft.type2(list(k), S * x[None], sign=-1)
        g = (np.conj(S) * nudft.type1(list(k), Ax - y, shape, sign=1)).sum(0)
        kk = k.reshape(2, ninter, ns)
        slew = ((kk[:, :, 2:] - 2 * kk[:, :, 1:-1] + kk[:, :, :-2]) ** 2).sum()
        return float((np.abs(g) ** 2).sum() + lam * slew)

    xt = to_dev(x0, cuda).requires_grad_(True)
    kt = to_dev(k0, cuda).requires_grad_(True)
    loss_torch(xt, kt).backward()
    gk = to_np(kt.grad).astype(np.float64)
    gx = to_np(xt.grad)
    h = 1e-4
    picks = rng.choice(2 * M, 64, replace=False)
    fd = []
    k64 = k0.astype(np.float64)
    for p in picks:
        a, j = divmod(int(p), M)
        kp, km = k64.copy(), k64.copy()
        kp[a, j] += h
        km[a, j] -= h
        fd.append((loss_np(x0, kp) - loss_np(x0, km)) / (2 * h))
    got = np.array([gk[divmod(int(p), M)] for p in picks])
    assert relerr(got, np.array(fd)) <= 1e-3
    # image gradient (Wirtinger: dL/dRe + i dL/dIm) at 16 random pixels
    fdx = []
    pix = rng.choice(N * N, 16, replace=False)
    for p in pix:
        i, j = divmod(int(p), N)
        v = []
        for d in (1.0, 1j):
            xp, xm = x0.astype(np.complex128), x0.astype(np.complex128)
            xp[i, j] += h * d
            xm[i, j] -= h * d
            v.append((loss_np(xp, k64) - loss_np(xm, k64)) / (2 * h))
        fdx.append(v[0] + 1j * v[1])
    gotx = np.array([gx[divmod(int(p), N)] for p in pix])
    assert relerr(gotx, np.array(fdx)) <= 1e-3
