"""Gridding autotuner: picks the spreading kernel, its cell block and the points per spread
subproblem for a given problem by timing type-1 plans on the device, and the interpolation lane
groups by timing type-2 plans, and caches the choices as JSON.

Spreading search space (all exact, all give the same result up to float rounding):
- the kernel: transforms on the lanes (each thread owns 4 rows x 8 cells of one transform; dense
  tiles are spread in parts whose partial tiles a second kernel sums) or cells on the lanes (each
  thread owns one cell; dense tiles as extra subproblems);
- for cells on the lanes, the 32-cell block each warp owns inside a spread tile: 3-D tiles are
  8x8x8, so any (bz, by, bx) with bz*by*bx = 32 and each edge dividing 8; 2-D tiles are 16x32;
- points per subproblem (when a tile is dense enough to split): 256 .. 8192.

Interpolation search space: the transforms a lane group gathers per point (32, 16, 8 or 4 lanes;
all give bit-identical results).

Cache key: dimensionality, modes, transforms, kernel width, number of points and a coarse
density signature of the trajectory (quartiles of |k|), so the same trajectory family reuses the
choice. Cache file: $HASTY_B200_TUNE_CACHE or ~/.cache/hastycucompute_b200/spread_tuning.json.
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Optional, Sequence

import torch

from .nufft import NufftOpts, NufftPlan, NufftType

BLOCKS_3D = [(2, 4, 4), (4, 4, 2), (2, 2, 8), (4, 2, 4), (1, 4, 8), (8, 2, 2), (2, 8, 2)]
BLOCKS_2D = [(1, 4, 8), (1, 8, 4), (1, 2, 16), (1, 16, 2), (1, 1, 32)]
MAXP = [1024, 2048, 4096, 8192]
MAXP_TRANSFORMS = [256, 512, 1024, 2048, 4096]


def cache_path() -> Path:
    p = os.environ.get("HASTY_B200_TUNE_CACHE")
    if p:
        return Path(p)
    return Path.home() / ".cache" / "hastycucompute_b200" / "spread_tuning.json"


def _key(nmodes, ntransf, width, coords) -> str:
    r = torch.sqrt(sum(c.float() ** 2 for c in coords))
    q = torch.quantile(r[:: max(1, r.numel() // 100000)], torch.tensor([0.25, 0.5, 0.75], device=r.device))
    sig = ",".join(f"{v:.2f}" for v in q.tolist())
    M = coords[0].shape[0]
    return f"d{len(nmodes)}|n{'x'.join(map(str, nmodes))}|t{ntransf}|w{width}|m{M // 1000}k|q{sig}"


def _load() -> dict:
    p = cache_path()
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


def _store(d: dict) -> None:
    p = cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    p.write_text(json.dumps(d, indent=1, sort_keys=True))


def tune_spread(nmodes: Sequence[int], ntransf: int, coords: Sequence[torch.Tensor], kernel_width: int,
                reps: int = 3, use_cache: bool = True, candidates: Optional[list] = None) -> dict:
    """Times type-1 executes over the search space; returns {"kernel", "block", "max_candidates",
    "ms", "timings"} for the fastest and stores it in the cache. ``candidates`` entries are
    (kernel, block, max_candidates)."""
    nmodes = tuple(int(n) for n in nmodes)
    key = _key(nmodes, ntransf, kernel_width, coords)
    cache = _load() if use_cache else {}
    if key in cache:
        return dict(cache[key], cached=True)
    dev = coords[0].device
    blocks = BLOCKS_3D if len(nmodes) == 3 else BLOCKS_2D
    if candidates is None:
        candidates = [("transforms", blocks[0], m) for m in MAXP_TRANSFORMS]
        candidates += [("cells", b, m) for b in blocks for m in MAXP]
    M = coords[0].shape[0]
    data = torch.randn((ntransf, M), dtype=torch.complex64, device=dev)
    out = torch.empty((ntransf, *nmodes), dtype=torch.complex64, device=dev)
    timings = []
    for kernel, block, maxp in candidates:
        plan = NufftPlan(NufftType.TYPE_1, NufftOpts(nmodes=nmodes, ntransf=ntransf, kernel_width=kernel_width))
        try:
            plan.set_spread_kernel(kernel)
            plan.set_spread_tuning(maxp, block)
        except Exception:
            plan.free()
            continue
        plan.setpts(list(coords))
        plan.execute(data, out)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            plan.execute(data, out)
        e1.record()
        torch.cuda.synchronize(dev)
        timings.append((e0.elapsed_time(e1) / reps, kernel, list(block), int(maxp)))
        plan.free()
    timings.sort(key=lambda r: r[0])
    best = {"kernel": timings[0][1], "block": timings[0][2], "max_candidates": timings[0][3],
            "ms": round(timings[0][0], 4), "timings": [[round(t, 4), k, b, m] for t, k, b, m in timings]}
    if use_cache:
        cache = _load()
        cache[key] = best
        _store(cache)
    return dict(best, cached=False)


INTERP_GROUPS = [32, 16, 8, 4]


def tune_interp(nmodes: Sequence[int], ntransf: int, coords: Sequence[torch.Tensor], kernel_width: int,
                reps: int = 3, use_cache: bool = True) -> dict:
    """Times type-2 executes over the interpolation lane-group sizes; returns {"interp_group",
    "ms", "timings"} for the fastest and stores it in the cache."""
    nmodes = tuple(int(n) for n in nmodes)
    key = "interp|" + _key(nmodes, ntransf, kernel_width, coords)
    cache = _load() if use_cache else {}
    if key in cache:
        return dict(cache[key], cached=True)
    dev = coords[0].device
    M = coords[0].shape[0]
    img = torch.randn((ntransf, *nmodes), dtype=torch.complex64, device=dev)
    out = torch.empty((ntransf, M), dtype=torch.complex64, device=dev)
    timings = []
    for grp in INTERP_GROUPS:
        plan = NufftPlan(NufftType.TYPE_2, NufftOpts(nmodes=nmodes, ntransf=ntransf, kernel_width=kernel_width))
        try:
            plan.set_interp_tuning(grp)
        except Exception:
            plan.free()
            continue
        plan.setpts(list(coords))
        plan.execute(img, out)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            plan.execute(img, out)
        e1.record()
        torch.cuda.synchronize(dev)
        timings.append((e0.elapsed_time(e1) / reps, grp))
        plan.free()
    timings.sort(key=lambda r: r[0])
    best = {"interp_group": int(timings[0][1]), "ms": round(timings[0][0], 4),
            "timings": [[round(t, 4), g] for t, g in timings]}
    if use_cache:
        cache = _load()
        cache[key] = best
        _store(cache)
    return dict(best, cached=False)


def apply(plan: NufftPlan, choice: dict) -> None:
    """Applies a tuner choice (from tune_spread, tune_interp or both merged) to a plan, before its
    setpts."""
    if "max_candidates" in choice:
        plan.set_spread_kernel(choice.get("kernel", "auto"))
        plan.set_spread_tuning(int(choice["max_candidates"]), tuple(choice["block"]))
    if "interp_group" in choice:
        plan.set_interp_tuning(int(choice["interp_group"]))
