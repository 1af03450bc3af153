"""Spreading autotuner: every candidate gives the default's result; the choice is cached."""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import gridding


@pytest.mark.gpu
@pytest.mark.parametrize("nmodes,w", [((20, 20, 20), 6), ((48, 40), 4)])
def test_every_tuning_gives_the_same_transform(cuda, nmodes, w):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import autotune
    rng = np.random.default_rng(2)
    M, T = 20000, 5
    coords = rand_coords(rng, len(nmodes), M)
    coords[0][: M // 2] *= 0.05   # a dense core so subproblems split
    c = crand(rng, T, M)
    ref = gridding.nufft1(coords, c, nmodes, w=w)
    blocks = autotune.BLOCKS_3D if len(nmodes) == 3 else autotune.BLOCKS_2D
    for block in blocks:
        for maxp in (64, 4096):
            p = hb.NufftPlan(hb.NufftType.TYPE_1, hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w))
            p.set_spread_tuning(maxp, block)
            p.setpts([to_dev(x, cuda) for x in coords])
            assert relerr(to_np(p(to_dev(c, cuda))), ref) <= 1e-5, (block, maxp)


@pytest.mark.gpu
def test_tuner_picks_and_caches(cuda, tmp_path, monkeypatch):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import autotune
    monkeypatch.setenv("HASTY_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(3)
    coords = [to_dev(x, cuda) for x in rand_coords(rng, 3, 30000)]
    cand = [((2, 4, 4), 1024), ((4, 4, 2), 2048), ((1, 4, 8), 512)]
    first = autotune.tune_spread((24, 24, 24), 8, coords, 6, candidates=cand)
    assert not first["cached"] and (tuple(first["block"]), first["max_candidates"]) in cand
    assert len(first["timings"]) == 3
    again = autotune.tune_spread((24, 24, 24), 8, coords, 6, candidates=cand)
    assert again["cached"] and again["block"] == first["block"]
    p = hb.NufftPlan(hb.NufftType.TYPE_1, hb.NufftOpts(nmodes=(24, 24, 24), ntransf=8, kernel_width=6))
    autotune.apply(p, first)
    p.setpts(coords)
    with pytest.raises(RuntimeError):
        p.set_spread_tuning(1024, (2, 4, 4))


def test_tuning_arguments_are_checked_on_the_host():
    from hastycucompute_b200 import _lib
    import ctypes as C
    lib = _lib.load()
    h = C.c_void_p()
    # makeplan allocates device memory, so only the pure argument checks run here
    assert lib.hb_nufft_set_spread_tuning(None, 1024, 2, 4, 4) == 1
