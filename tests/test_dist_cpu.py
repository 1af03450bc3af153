"""The multi-rank path of bench.py on CPU: two gloo ranks, launched the way torchrun launches them
(RANK / WORLD_SIZE / LOCAL_RANK / MASTER_* in the environment). Frames are independent replicas,
so the only cross-rank steps are the barrier and the max-over-ranks of the timed region."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup(False)
    assert (w, r, local) == (world, rank, rank)
    # each rank times a different amount of work; every rank must report the slowest
    v = bench.max_over_ranks(10.0 * (rank + 1), w, "cpu")
    bench.barrier(w)
    Path(out_dir, f"rank{rank}.txt").write_text(repr(v))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_max_and_meet_at_the_barrier(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        assert float((tmp_path / f"rank{r}.txt").read_text()) == 20.0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.pop("WORLD_SIZE", None)
    w, r, _ = bench.dist_setup(False)
    assert (w, r) == (1, 0)
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    bench.barrier(1)
