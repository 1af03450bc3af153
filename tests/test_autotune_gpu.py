"""Spreading autotuner: every candidate (both kernels, every cell block, small and large
subproblems) gives the oracle's result; the choice is cached; a plan that cannot put the
transforms on the lanes refuses that kernel."""
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
    for kernel, bl in (("cells", blocks), ("transforms", blocks[:1])):
        for block in bl:
            for maxp in (64, 4096):
                p = hb.NufftPlan(hb.NufftType.TYPE_1, hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w))
                p.set_spread_kernel(kernel)
                p.set_spread_tuning(maxp, block)
                p.setpts([to_dev(x, cuda) for x in coords])
                assert relerr(to_np(p(to_dev(c, cuda))), ref) <= 1e-5, (kernel, block, maxp)


@pytest.mark.gpu
def test_tuner_picks_and_caches(cuda, tmp_path, monkeypatch):
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import autotune
    monkeypatch.setenv("HASTY_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(3)
    coords = [to_dev(x, cuda) for x in rand_coords(rng, 3, 30000)]
    cand = [("cells", (2, 4, 4), 1024), ("cells", (4, 4, 2), 2048), ("transforms", (2, 4, 4), 512)]
    first = autotune.tune_spread((24, 24, 24), 8, coords, 6, candidates=cand)
    assert not first["cached"] and (first["kernel"], tuple(first["block"]), first["max_candidates"]) in cand
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


@pytest.mark.gpu
def test_transforms_on_lanes_is_refused_where_the_plan_does_not_allow_it(cuda):
    import hastycucompute_b200 as hb
    p = hb.NufftPlan(hb.NufftType.TYPE_1, hb.NufftOpts(nmodes=(16, 16, 16), ntransf=2, kernel_width=6))
    with pytest.raises(hb.HastyError, match="INVALID_ARG"):
        p.set_spread_kernel("transforms")
    p.set_spread_kernel("cells")


@pytest.mark.gpu
def test_interp_tuner_picks_caches_and_applies(cuda, tmp_path, monkeypatch):
    """Type-2 lane-group tuning: every size is timed, the choice is cached, and a plan given it
    interpolates the oracle's samples."""
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import autotune
    monkeypatch.setenv("HASTY_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    rng = np.random.default_rng(4)
    nmodes, T, w, M = (40, 48), 12, 4, 20000
    coords = rand_coords(rng, 2, M)
    dcoords = [to_dev(x, cuda) for x in coords]
    first = autotune.tune_interp(nmodes, T, dcoords, w)
    assert not first["cached"] and first["interp_group"] in autotune.INTERP_GROUPS
    assert sorted(g for _, g in first["timings"]) == sorted(autotune.INTERP_GROUPS)
    again = autotune.tune_interp(nmodes, T, dcoords, w)
    assert again["cached"] and again["interp_group"] == first["interp_group"]
    f = crand(rng, T, *nmodes)
    p = hb.NufftPlan(hb.NufftType.TYPE_2, hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w))
    autotune.apply(p, first)
    p.setpts(dcoords)
    assert relerr(to_np(p(to_dev(f, cuda))), gridding.nufft2(coords, f, w=w)) <= 1e-5
