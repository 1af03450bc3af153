"""Frames and coils across ranks on CPU (gloo, world size 2, launched the way torchrun launches
ranks). The distribution code is the library's (hastycucompute_b200.frames); the per-frame solve
and the per-shard apply are CPU stand-ins with the operator interface (the oracle's Toeplitz SENSE
normal operator and CG), since the fused CUDA operators need a GPU. Checked: the frames split
over two ranks and gathered equal the single-rank reconstruction exactly, and the coil-sharded
apply with its all-reduce equals the apply over all coils."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from hastycucompute_b200.frames import coil_partition, frame_partition  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


SHAPE, C, W = (12, 10), 4, 4
SPOKES = [30, 55, 41, 70, 36]  # ragged frames: samples per frame differ


def _frame_problem(f):
    from hastycucompute_b200 import synthetic
    from oracle import toeplitz as otp
    k = synthetic.golden_angle_radial_2d(SPOKES[f], 24)
    k = np.roll(k, f, axis=1)
    S = synthetic.coil_maps(C, SHAPE)
    x = synthetic.image(SHAPE, seed=10 + f)
    K = otp.toeplitz_kernel(list(k), SHAPE, w=W)
    return S, K, otp.sense_normal(x, S, K)


def _solve(ids):
    """CPU stand-in of the per-rank batched recon: oracle CG (5 iterations) per frame."""
    import torch
    from oracle import cg as ocg, toeplitz as otp
    out = []
    for f in ids:
        S, K, b = _frame_problem(f)
        x, _ = ocg.conjugate_gradient(lambda v: otp.sense_normal(v, S, K), b, np.zeros(SHAPE, np.complex128), 5, tol=0.0)
        out.append(torch.from_numpy(x))
    return torch.stack(out) if out else torch.zeros((0, *SHAPE), dtype=torch.complex128)


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch
    import torch.distributed as dist
    from hastycucompute_b200.frames import CoilShardedNormal, coil_partition, distributed_frames
    from oracle import toeplitz as otp
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    weights = [s * 24 for s in SPOKES]
    full = distributed_frames(len(SPOKES), world, rank, _solve, weights=weights)
    torch.save(full, Path(out_dir, f"frames{rank}.pt"))
    # coil sharding of frame 0: partial apply over this rank's coils, all-reduce of the image
    S, K, _ = _frame_problem(0)
    sl = coil_partition(C, world, rank)
    x = torch.from_numpy(np.asarray(_frame_problem(1)[2]))
    op = CoilShardedNormal(lambda v, out: out.copy_(torch.from_numpy(otp.sense_normal(v.numpy(), S[sl], K))), world)
    torch.save(op(x), Path(out_dir, f"coils{rank}.pt"))
    dist.destroy_process_group()


def test_frame_partition_covers_each_frame_once_and_balances_samples():
    for nframes, world in [(24, 1), (24, 2), (24, 8), (5, 2), (3, 4), (7, 7), (0, 3)]:
        w = list(np.random.default_rng(nframes + world).integers(300, 701, nframes) * 128) if nframes else None
        parts = [frame_partition(nframes, world, r, w) for r in range(world)]
        flat = [f for p in parts for f in p]
        assert flat == list(range(nframes))
        if nframes >= world:
            assert all(len(p) >= 1 for p in parts)
        if nframes >= 4 * world and w is not None:
            loads = [sum(w[f] for f in p) for p in parts]
            assert max(loads) <= sum(w) / world + max(w)
    assert [coil_partition(10, 3, r) for r in range(3)] == [slice(0, 4), slice(4, 7), slice(7, 10)]


@pytest.mark.timeout(300)
def test_two_gloo_ranks_split_frames_and_shard_coils(tmp_path):
    import torch
    import torch.multiprocessing as mp
    from oracle import toeplitz as otp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    single = _solve(list(range(len(SPOKES))))
    for r in range(world):
        got = torch.load(tmp_path / f"frames{r}.pt")
        assert torch.equal(got, single)
    S, K, _ = _frame_problem(0)
    ref = otp.sense_normal(_frame_problem(1)[2], S, K)
    for r in range(world):
        got = torch.load(tmp_path / f"coils{r}.pt").numpy()
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
