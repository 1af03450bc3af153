"""hb.HostPipeline: host-to-host applies with overlapped copies give the same results as applying
each item on its own."""
import numpy as np
import pytest

from helpers import crand, relerr, to_dev, to_np


@pytest.mark.gpu
def test_host_pipeline_matches_serial(cuda):
    import torch
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(11)
    shape, C, items = (16, 12, 10), 3, 5
    S = crand(rng, C, *shape)
    K = crand(rng, *[2 * s for s in shape])
    op = hb.NormalTT1Op(to_dev(K, cuda), to_dev(S, cuda))
    xs = [crand(rng, *shape) for _ in range(items)]
    host_in = [torch.from_numpy(x).pin_memory() for x in xs]
    host_out = [torch.empty_like(h).pin_memory() for h in host_in]
    pipe = hb.HostPipeline(lambda a, b: op.apply(a, b), shape, cuda)
    pipe.run(host_in, host_out)
    torch.cuda.synchronize()
    for x, h in zip(xs, host_out):
        ref = to_np(op(to_dev(x, cuda)))
        assert relerr(h.numpy(), ref) <= 1e-6
    # a second run reuses the device buffers
    pipe.run(host_in[::-1], host_out)
    torch.cuda.synchronize()
    for x, h in zip(xs[::-1], host_out):
        assert relerr(h.numpy(), to_np(op(to_dev(x, cuda)))) <= 1e-6
