"""Frames and coils across ranks (one process per GPU, torch.distributed).

The reference spreads its per-frame / per-coil work over a thread pool of devices and gathers the
results on the CPU (cpp/corelib/lib/threading/threading.cppm:142-352,
cpp/corelib/lib/mri/adjoint.cppm:145-156). Here:

- frames (and batch volumes) are independent systems: ``frame_partition`` gives every rank a
  contiguous run of frames balanced by their sample counts, each rank reconstructs its frames with
  the batched operator and CG on its own GPU, and ``gather_frames`` assembles the [F, N..] result
  on every rank with one all-gather at the end -- no collective on the data path;
- within one frame, coils can be sharded: ``coil_partition`` splits the coils and
  ``CoilShardedNormal`` sums the ranks' partial SENSE normal applies with one all-reduce of the
  image per apply (the only exchange the operator has: the sum over coils).
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import torch


def frame_partition(nframes: int, world: int, rank: int, weights: Optional[Sequence[float]] = None) -> list:
    """Contiguous frames of `rank`: cut points at the quantiles of the cumulative weight (sample
    counts), so every rank gets about the same work; each rank gets at least one frame while there
    are as many frames as ranks. The same on every rank (no communication)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    if nframes <= 0:
        return []
    w = [1.0] * nframes if weights is None else [float(v) for v in weights]
    if len(w) != nframes:
        raise ValueError("one weight per frame")
    total = sum(w)
    cuts = [0]
    acc = 0.0
    f = 0
    for r in range(1, world):
        target = total * r / world
        while f < nframes and acc + 0.5 * w[f] < target:
            acc += w[f]
            f += 1
        # leave at least one frame for each remaining rank when there are enough frames
        lo = cuts[-1] + (1 if nframes >= world else 0)
        hi = nframes - (world - r if nframes >= world else 0)
        cuts.append(min(max(f, lo), hi))
    cuts.append(nframes)
    return list(range(cuts[rank], cuts[rank + 1]))


def gather_frames(local: torch.Tensor, nframes: int, world: int, weights: Optional[Sequence[float]] = None,
                  group=None) -> torch.Tensor:
    """All ranks' frames [len(frames of rank), N..] -> the full [nframes, N..] on every rank (one
    all-gather of equal-sized, zero-padded blocks)."""
    if world == 1:
        return local
    import torch.distributed as dist
    parts = [frame_partition(nframes, world, r, weights) for r in range(world)]
    cap = max(len(p) for p in parts)
    tail = tuple(local.shape[1:])
    buf = torch.zeros((cap, *tail), dtype=local.dtype, device=local.device)
    buf[: local.shape[0]] = local
    bufs = [torch.empty_like(buf) for _ in range(world)]
    real = (lambda t: torch.view_as_real(t)) if local.is_complex() else (lambda t: t)
    dist.all_gather([real(b) for b in bufs], real(buf), group=group)
    out = torch.empty((nframes, *tail), dtype=local.dtype, device=local.device)
    for r, ids in enumerate(parts):
        if ids:
            out[ids[0]: ids[-1] + 1] = bufs[r][: len(ids)]
    return out


def distributed_frames(nframes: int, world: int, rank: int, solve: Callable[[list], torch.Tensor],
                       weights: Optional[Sequence[float]] = None, gather: bool = True, group=None):
    """Runs ``solve(frame_ids)`` (returns [len(frame_ids), N..]) on this rank's frames and, with
    ``gather``, returns the full result on every rank."""
    ids = frame_partition(nframes, world, rank, weights)
    local = solve(ids)
    return gather_frames(local, nframes, world, weights, group) if gather else local


def coil_partition(ncoils: int, world: int, rank: int) -> slice:
    """Contiguous coils of `rank` (sizes differ by at most one)."""
    base, rem = divmod(ncoils, world)
    lo = rank * base + min(rank, rem)
    return slice(lo, lo + base + (1 if rank < rem else 0))


class CoilShardedNormal:
    """sum over all coils of conj(S_c) T(S_c x) when every rank holds a shard of the coils:
    ``local_apply(x, out)`` writes this rank's partial sum (the fused SENSE normal apply over its
    coils), then one all-reduce (sum) of the image completes it on every rank."""

    def __init__(self, local_apply: Callable[[torch.Tensor, torch.Tensor], torch.Tensor], world: int, group=None):
        self.local_apply = local_apply
        self.world = int(world)
        self.group = group

    def apply(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        if out is None:
            out = torch.empty_like(x)
        self.local_apply(x, out)
        if self.world > 1:
            import torch.distributed as dist
            if out.is_complex():
                dist.all_reduce(torch.view_as_real(out), group=self.group)
            else:
                dist.all_reduce(out, group=self.group)
        return out

    __call__ = apply
