"""Unrolled differentiable Toeplitz SENSE-CG with learnable steps and regularisation: gradients
in the scalars against central differences, recomputation equal to plain backprop, and lower
peak memory with checkpointing."""
import numpy as np
import pytest

from helpers import rand_coords, relerr, to_dev


def _setup(cuda, F=2, shape=(16, 16, 16), C=3):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    rng = np.random.default_rng(0)
    S = to_dev(synthetic.coil_maps(C, shape), cuda)
    frames = [[to_dev(c, cuda) for c in rand_coords(rng, 3, 6000 + 500 * f)] for f in range(F)]
    Ks = hb.build_toeplitz_kernels(frames, shape, kernel_width=4)
    op = hb.BatchedNormalOp(Ks, S)
    xt = to_dev(np.stack([synthetic.image(shape, seed=f) for f in range(F)]), cuda)
    b = op(xt)
    return op, b, xt


@pytest.mark.gpu
def test_unrolled_cg_scalar_gradients_match_finite_differences(cuda):
    import torch
    from hastycucompute_b200.unrolled import UnrolledCG
    op, b, xt = _setup(cuda)
    K = 5
    net = UnrolledCG(op, iterations=K, step_init=0.9, lam_init=0.01, checkpoint=True).to(cuda)

    def loss_fn():
        x = net(b)
        return ((x - xt).abs() ** 2).sum().double()

    loss = loss_fn()
    loss.backward()
    gs, gl = net.steps.grad.clone(), net.lams.grad.clone()
    h = 1e-3
    for param, grad in ((net.steps, gs), (net.lams, gl)):
        fd = []
        for k in range(K):
            with torch.no_grad():
                param[k] += h
                lp = loss_fn().item()
                param[k] -= 2 * h
                lm = loss_fn().item()
                param[k] += h
            fd.append((lp - lm) / (2 * h))
        fd = np.array(fd)
        assert relerr(grad.cpu().numpy(), fd) <= 1e-3


@pytest.mark.gpu
def test_recomputation_equals_plain_backprop_and_saves_memory(cuda):
    import torch
    from hastycucompute_b200.unrolled import UnrolledCG
    op, b, xt = _setup(cuda, F=2, shape=(32, 32, 32), C=4)
    grads, peaks = [], []
    for ck in (False, True):
        net = UnrolledCG(op, iterations=8, step_init=1.0, lam_init=0.0, checkpoint=ck).to(cuda)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        base = torch.cuda.memory_allocated()
        loss = ((net(b) - xt).abs() ** 2).sum()
        loss.backward()
        torch.cuda.synchronize()
        peaks.append(torch.cuda.max_memory_allocated() - base)
        grads.append(torch.cat([net.steps.grad, net.lams.grad]).cpu().numpy())
    assert relerr(grads[1], grads[0]) <= 1e-5
    assert peaks[1] < peaks[0]
