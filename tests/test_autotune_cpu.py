"""Host side of the spreading autotuner (no GPU): the search space honours the tuning contract of
hb_nufft_set_spread_tuning, the cache key separates problems, and a cached choice is returned
without timing anything."""
import json

import numpy as np
import torch

from hastycucompute_b200 import autotune
from helpers import rand_coords


def _coords(M, dim=3, seed=0):
    return [torch.from_numpy(c) for c in rand_coords(np.random.default_rng(seed), dim, M)]


def test_search_space_tiles_the_spread_tile():
    """32 cells per warp block; edges are powers of two dividing the tile (8x8x8 in 3-D, 16x32 in
    2-D with a unit z edge)."""
    for bz, by, bx in autotune.BLOCKS_3D:
        assert bz * by * bx == 32 and all(8 % e == 0 for e in (bz, by, bx))
    for bz, by, bx in autotune.BLOCKS_2D:
        assert bz == 1 and by * bx == 32 and 16 % by == 0 and 32 % bx == 0
    assert all(32 <= m <= 65536 and m & (m - 1) == 0 for m in autotune.MAXP)


def test_cache_key_is_stable_and_separates_problems():
    c = _coords(20000)
    k = autotune._key((32, 32, 32), 8, 6, c)
    assert k == autotune._key((32, 32, 32), 8, 6, [t.clone() for t in c])
    others = {
        autotune._key((32, 32, 24), 8, 6, c),
        autotune._key((32, 32, 32), 4, 6, c),
        autotune._key((32, 32, 32), 8, 4, c),
        autotune._key((32, 32, 32), 8, 6, _coords(40000)),
        autotune._key((32, 32, 32), 8, 6, [t * 0.5 for t in c]),  # denser centre
    }
    assert k not in others and len(others) == 5


def test_cached_choice_is_returned_without_timing(tmp_path, monkeypatch):
    monkeypatch.setenv("HASTY_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    c = _coords(5000)
    key = autotune._key((16, 16, 16), 2, 6, c)
    choice = {"block": [4, 4, 2], "max_candidates": 2048, "ms": 0.5, "timings": []}
    autotune._store({key: choice})

    def no_plans(*a, **k):
        raise AssertionError("a cached choice must not build plans")

    monkeypatch.setattr(autotune, "NufftPlan", no_plans)
    got = autotune.tune_spread((16, 16, 16), 2, c, 6)
    assert got["cached"] is True and got["block"] == [4, 4, 2] and got["max_candidates"] == 2048
    assert json.loads((tmp_path / "tune.json").read_text()) == {key: choice}


def test_unreadable_cache_counts_as_empty(tmp_path, monkeypatch):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    monkeypatch.setenv("HASTY_B200_TUNE_CACHE", str(p))
    assert autotune._load() == {}
    monkeypatch.setenv("HASTY_B200_TUNE_CACHE", str(tmp_path / "missing.json"))
    assert autotune._load() == {}


def test_interp_choice_is_cached_apart_from_spreading(tmp_path, monkeypatch):
    """The interpolation tuner keys its choices apart from the spreading tuner's, returns a cached
    choice without building plans, and apply() sets only what a choice holds."""
    monkeypatch.setenv("HASTY_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    c = _coords(5000)
    key = autotune._key((16, 16, 16), 12, 4, c)
    autotune._store({"interp|" + key: {"interp_group": 4, "ms": 0.1, "timings": []},
                     key: {"kernel": "cells", "block": [2, 4, 4], "max_candidates": 1024, "ms": 0.2, "timings": []}})

    def no_plans(*a, **k):
        raise AssertionError("a cached choice must not build plans")

    monkeypatch.setattr(autotune, "NufftPlan", no_plans)
    got = autotune.tune_interp((16, 16, 16), 12, c, 4)
    assert got["cached"] is True and got["interp_group"] == 4
    spread = autotune.tune_spread((16, 16, 16), 12, c, 4)
    assert spread["cached"] is True and spread["kernel"] == "cells"

    calls = []

    class FakePlan:
        def set_spread_kernel(self, k):
            calls.append(("kernel", k))

        def set_spread_tuning(self, m, b):
            calls.append(("tuning", m, b))

        def set_interp_tuning(self, g):
            calls.append(("interp", g))

    autotune.apply(FakePlan(), got)
    assert calls == [("interp", 4)]
    calls.clear()
    autotune.apply(FakePlan(), dict(spread, **got))
    assert calls == [("kernel", "cells"), ("tuning", 1024, (2, 4, 4)), ("interp", 4)]


def test_cache_key_separates_trajectory_families():
    """Radial spokes, cones spirals and uniform random points with the same point count and
    problem get different keys (a choice tuned on one family is not reused for another), while a
    re-drawn trajectory of the same family reuses it."""
    from hastycucompute_b200 import synthetic
    radial = [torch.from_numpy(np.ascontiguousarray(c)) for c in synthetic.golden_means_radial(256, 128)]
    cones = [torch.from_numpy(np.ascontiguousarray(c)) for c in synthetic.cones_spiral(128, 256)]
    uniform = _coords(32768)
    keys = {autotune._key((32, 32, 32), 8, 6, c) for c in (radial, cones, uniform)}
    assert len(keys) == 3
    radial2 = [torch.from_numpy(np.ascontiguousarray(c)) for c in synthetic.golden_means_radial(256, 128, offset=256)]
    assert autotune._key((32, 32, 32), 8, 6, radial2) == autotune._key((32, 32, 32), 8, 6, radial)
