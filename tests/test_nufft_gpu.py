"""NUFFT type 1 / type 2 on the GPU through the C ABI, against the oracle.

Parity bar: relative L2 error <= 1e-5 against the same-algorithm FP64 restatement
(oracle.gridding); against the FP64 NUDFT the error is the kernel's own accuracy (stated per case).
"""
import numpy as np
import pytest

from helpers import crand, rand_coords, relerr, to_dev, to_np
from oracle import gridding, kb, nudft

PARITY = 1e-5
# NUDFT error of the Kaiser-Bessel kernel at sigma = 2 by width (measured on the oracle)
NUDFT_TOL = {4: 2e-3, 5: 2e-4, 6: 3e-5, 7: 5e-6, 8: 3e-6}

CASES = [
    # dim, nmodes, M, ntransf, width
    (1, (37,), 500, 2, 4),
    (2, (24, 20), 3000, 1, 4),
    (2, (32, 32), 4000, 3, 6),
    (2, (17, 30), 2500, 12, 5),
    (3, (12, 14, 10), 4000, 1, 4),
    (3, (16, 16, 16), 6000, 8, 4),
    (3, (16, 12, 20), 5000, 5, 6),
    (3, (20, 20, 20), 8000, 32, 6),
    (3, (10, 10, 10), 3000, 40, 7),
    (3, (24, 24, 24), 6000, 2, 10),
]


def _plan(hb, ntype, nmodes, ntransf, w, sign=None):
    opts = hb.NufftOpts(nmodes=nmodes, ntransf=ntransf, kernel_width=w, sign=sign)
    return hb.NufftPlan(ntype, opts)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,nmodes,M,T,w", CASES)
def test_type1_parity(cuda, dim, nmodes, M, T, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(11 + M)
    coords = rand_coords(rng, dim, M)
    c = crand(rng, T, M)
    plan = _plan(hb, hb.NufftType.TYPE_1, nmodes, T, w)
    plan.setpts([to_dev(x, cuda) for x in coords])
    got = to_np(plan(to_dev(c, cuda)))
    ref = gridding.nufft1(coords, c, nmodes, w=w)
    e = relerr(got, ref)
    assert e <= PARITY, f"type1 parity {e:.2e}"
    if np.prod(nmodes) * M <= 4096 * 8000:
        ex = nudft.type1(coords, c, nmodes, sign=1)
        assert relerr(got, ex) <= NUDFT_TOL.get(w, 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,nmodes,M,T,w", CASES)
def test_type2_parity(cuda, dim, nmodes, M, T, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(21 + M)
    coords = rand_coords(rng, dim, M)
    f = crand(rng, T, *nmodes)
    plan = _plan(hb, hb.NufftType.TYPE_2, nmodes, T, w)
    plan.setpts([to_dev(x, cuda) for x in coords])
    got = to_np(plan(to_dev(f, cuda)))
    ref = gridding.nufft2(coords, f, w=w)
    e = relerr(got, ref)
    assert e <= PARITY, f"type2 parity {e:.2e}"
    if np.prod(nmodes) * M <= 4096 * 8000:
        ex = nudft.type2(coords, f, sign=-1)
        assert relerr(got, ex) <= NUDFT_TOL.get(w, 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("sign", [1, -1])
def test_signs(cuda, sign):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(5)
    nm, M = (12, 10, 8), 2000
    coords = rand_coords(rng, 3, M)
    c = crand(rng, 2, M)
    p1 = _plan(hb, hb.NufftType.TYPE_1, nm, 2, 6, sign=sign)
    p1.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(p1(to_dev(c, cuda))), nudft.type1(coords, c, nm, sign=sign)) <= NUDFT_TOL[6]
    f = crand(rng, 2, *nm)
    p2 = _plan(hb, hb.NufftType.TYPE_2, nm, 2, 6, sign=sign)
    p2.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(p2(to_dev(f, cuda))), nudft.type2(coords, f, sign=sign)) <= NUDFT_TOL[6]


@pytest.mark.gpu
def test_adjointness(cuda):
    """<A f, c> == <f, A^H c> for the type-2 / type-1 pair on the same points."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(8)
    nm, M, T = (16, 16, 16), 7000, 3
    coords = rand_coords(rng, 3, M)
    f, c = crand(rng, T, *nm), crand(rng, T, M)
    p1 = _plan(hb, hb.NufftType.TYPE_1, nm, T, 6)
    p2 = _plan(hb, hb.NufftType.TYPE_2, nm, T, 6)
    for p in (p1, p2):
        p.setpts([to_dev(x, cuda) for x in coords])
    Af = to_np(p2(to_dev(f, cuda))).astype(np.complex128)
    Ahc = to_np(p1(to_dev(c, cuda))).astype(np.complex128)
    lhs = np.vdot(c, Af)
    rhs = np.vdot(Ahc, f)
    assert abs(lhs - rhs) / (np.linalg.norm(Af) * np.linalg.norm(c)) <= 1e-6


@pytest.mark.gpu
def test_coordinates_outside_pi(cuda):
    """Coordinates are periodic: x and x + 2 pi m give the same transform."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(9)
    nm, M = (16, 16), 3000
    coords = rand_coords(rng, 2, M)
    shifted = [(x + 2 * np.pi * rng.integers(-3, 4, M)).astype(np.float32) for x in coords]
    c = crand(rng, 1, M)
    p = _plan(hb, hb.NufftType.TYPE_1, nm, 1, 6)
    p.setpts([to_dev(x, cuda) for x in shifted])
    got = to_np(p(to_dev(c, cuda)))
    ref = gridding.nufft1(shifted, c, nm, w=6)
    assert relerr(got, ref) <= PARITY
    assert relerr(got, nudft.type1(coords, c, nm)) <= 1e-4


@pytest.mark.gpu
def test_dense_center_and_edges(cuda):
    """Heavy tiles (many points in one bin, split into subproblems) and points on the grid edge."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(10)
    nm = (20, 20, 20)
    M1 = 30000
    center = [rng.normal(0, 0.05, M1).astype(np.float32) for _ in range(3)]
    edge = [np.full(500, -np.pi, np.float32), np.full(500, np.float32(np.pi) * np.float32(0.9999999)),
            rng.uniform(-np.pi, np.pi, 500).astype(np.float32)]
    coords = [np.concatenate([a, b]) for a, b in zip(center, edge)]
    M = coords[0].shape[0]
    c = crand(rng, 4, M)
    p = _plan(hb, hb.NufftType.TYPE_1, nm, 4, 6)
    p.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(p(to_dev(c, cuda))), gridding.nufft1(coords, c, nm, w=6)) <= PARITY
    f = crand(rng, 4, *nm)
    q = _plan(hb, hb.NufftType.TYPE_2, nm, 4, 6)
    q.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(q(to_dev(f, cuda))), gridding.nufft2(coords, f, w=6)) <= PARITY


@pytest.mark.gpu
def test_empty_points(cuda):
    import torch
    import hastycucompute_b200 as hb
    nm = (8, 8, 8)
    p = _plan(hb, hb.NufftType.TYPE_1, nm, 2, 4)
    z = torch.zeros(0, dtype=torch.float32, device=cuda)
    p.setpts([z, z, z])
    out = p(torch.zeros((2, 0), dtype=torch.complex64, device=cuda))
    assert torch.count_nonzero(out).item() == 0
    q = _plan(hb, hb.NufftType.TYPE_2, nm, 2, 4)
    q.setpts([z, z, z])
    assert q(torch.ones((2, *nm), dtype=torch.complex64, device=cuda)).shape == (2, 0)


@pytest.mark.gpu
def test_nonfinite_coordinate_is_an_error(cuda):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(3)
    coords = rand_coords(rng, 2, 100)
    coords[1][17] = np.nan
    p = _plan(hb, hb.NufftType.TYPE_1, (8, 8), 1, 4)
    with pytest.raises(hb.HastyError, match="HB_ERR_RANGE"):
        p.setpts([to_dev(x, cuda) for x in coords])
    with pytest.raises(RuntimeError):
        p(to_dev(crand(rng, 1, 100), cuda))


@pytest.mark.gpu
def test_plan_reuse_and_resetpts(cuda):
    """setpts twice on one plan (growing and shrinking M) gives fresh results."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(4)
    nm = (12, 12, 12)
    p = _plan(hb, hb.NufftType.TYPE_2, nm, 3, 5)
    f = crand(rng, 3, *nm)
    for M in (1000, 5000, 300):
        coords = rand_coords(rng, 3, M)
        p.setpts([to_dev(x, cuda) for x in coords])
        assert relerr(to_np(p(to_dev(f, cuda))), gridding.nufft2(coords, f, w=5)) <= PARITY


@pytest.mark.gpu
def test_type1_resetpts_reuses_scratch(cuda):
    """Type-1 plans keep their sort scratch between setpts calls: re-pointing with more, fewer and
    again more points (different densities) gives fresh, correct results each time."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(14)
    nm = (14, 12, 16)
    p = _plan(hb, hb.NufftType.TYPE_1, nm, 3, 5)
    for M, spread in ((2000, np.pi), (9000, 0.3), (400, np.pi), (12000, 1.0)):
        coords = [rng.uniform(-spread, spread, M).astype(np.float32) for _ in range(3)]
        c = crand(rng, 3, M)
        p.setpts([to_dev(x, cuda) for x in coords])
        assert relerr(to_np(p(to_dev(c, cuda))), gridding.nufft1(coords, c, nm, w=5)) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("nmodes", [(48, 40, 44), (96, 80)])
def test_type1_mostly_empty_grid(cuda, nmodes):
    """A few points in a large grid: almost every spread tile has no candidate and is zeroed by the
    empty-tile path; the result matches the oracle everywhere."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(15)
    M = 60
    coords = rand_coords(rng, len(nmodes), M)
    c = crand(rng, 2, M)
    p = _plan(hb, hb.NufftType.TYPE_1, nmodes, 2, 4)
    p.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(p(to_dev(c, cuda))), gridding.nufft1(coords, c, nmodes, w=4)) <= PARITY


@pytest.mark.gpu
def test_plan_info_matches_oracle_grid(cuda):
    import hastycucompute_b200 as hb
    for nm, w in [((64, 64, 64), 4), ((160, 160, 160), 6), ((256, 256), 4), ((319, 319, 319), 6)]:
        p = _plan(hb, hb.NufftType.TYPE_1, nm, 1, w)
        info = p.info()
        assert info.fine == kb.fine_grid(nm, w)
        assert info.width == w
        assert abs(info.beta - kb.beta(w)) < 1e-9
        p.free()


# Fine grids of 64..640 points run the two-level register FFT kernels; other sizes the generic
# shared-memory kernel. These cases cover every register length.
@pytest.mark.gpu
@pytest.mark.parametrize("nmodes,w", [((32, 32), 4), ((64, 60), 4), ((128, 128), 4), ((160, 150), 6),
                                      ((256, 250), 4), ((320, 300), 4), ((24, 160), 6)])
def test_register_fft_lengths(cuda, nmodes, w):
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(sum(nmodes))
    M, T = 4000, 3
    coords = rand_coords(rng, 2, M)
    c = crand(rng, T, M)
    f = crand(rng, T, *nmodes)
    p1 = _plan(hb, hb.NufftType.TYPE_1, nmodes, T, w)
    p1.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(p1(to_dev(c, cuda))), gridding.nufft1(coords, c, nmodes, w=w)) <= PARITY
    p2 = _plan(hb, hb.NufftType.TYPE_2, nmodes, T, w)
    p2.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(p2(to_dev(f, cuda))), gridding.nufft2(coords, f, w=w)) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("dim,nmodes,M,T,w", [(3, (24, 20, 16), 6000, 8, 6), (2, (40, 36), 4000, 12, 8),
                                               (3, (32, 32, 32), 8000, 32, 7)])
def test_upsampfac_1_25(cuda, dim, nmodes, M, T, w):
    """nufft_upsamp_cuda UPSAMP_1_25 (cpp/corelib/lib/fft/nufft.cppm:59-63, 148-152): the fine grid
    is 1.25 N (rounded up to the tile / FFT rule) and the Kaiser-Bessel shape follows sigma; both
    types against the gridding oracle at the same sigma."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(M + T)
    coords = rand_coords(rng, dim, M)
    c = crand(rng, T, M)
    f = crand(rng, T, *nmodes)
    opts = hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w, upsamp=hb.NufftUpsamp.UPSAMP_1_25)
    p1 = hb.NufftPlan(hb.NufftType.TYPE_1, opts)
    p1.setpts([to_dev(x, cuda) for x in coords])
    assert p1.info().fine == kb.fine_grid(nmodes, w, 1.25)
    assert relerr(to_np(p1(to_dev(c, cuda))), gridding.nufft1(coords, c, nmodes, w=w, sigma=1.25)) <= PARITY
    p2 = hb.NufftPlan(hb.NufftType.TYPE_2, opts)
    p2.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(p2(to_dev(f, cuda))), gridding.nufft2(coords, f, w=w, sigma=1.25)) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("nmodes,T,w", [((20, 24, 16), 32, 6), ((24, 20, 16), 16, 4), ((40, 36), 12, 4)])
@pytest.mark.parametrize("per_group", [0, 32, 16, 8, 4])
def test_interp_lane_groups_agree(cuda, nmodes, T, w, per_group):
    """hb_nufft_set_interp_tuning: every lane-group size gathers the same sums (vs the oracle)."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(T + w + per_group)
    M = 5000
    coords = rand_coords(rng, len(nmodes), M)
    f = crand(rng, T, *nmodes)
    p = hb.NufftPlan(hb.NufftType.TYPE_2, hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w))
    p.set_interp_tuning(per_group)
    p.setpts([to_dev(x, cuda) for x in coords])
    assert relerr(to_np(p(to_dev(f, cuda))), gridding.nufft2(coords, f, w=w)) <= PARITY


@pytest.mark.gpu
@pytest.mark.parametrize("nmodes,T,w", [((20, 24, 16), 8, 6), ((24, 24, 24), 32, 6), ((16, 20, 18), 12, 4),
                                        ((18, 16, 20), 5, 5), ((20, 20, 20), 16, 7), ((4, 6, 5), 9, 4)])
def test_staged_interp_matches_gather_and_oracle(cuda, nmodes, T, w):
    """Type 2 from staged tile regions: bit-identical to the gathering kernel (same sums, same
    order) and within parity of the FP64 oracle, with points clustered at k = 0 (dense tiles in
    parts) and at the periodic edge (regions that wrap), odd transform counts and grids with a
    single tile along an axis."""
    import hastycucompute_b200 as hb
    rng = np.random.default_rng(sum(nmodes) + T + w)
    M = 9000
    kind = rng.random(M)
    coords = []
    for _ in range(3):
        x = np.where(kind < 0.4, rng.normal(0.0, 0.05, M),
                     np.where(kind < 0.6, rng.uniform(np.pi - 0.2, np.pi, M), rng.uniform(-np.pi, np.pi, M)))
        coords.append(np.clip(x, -np.pi, np.pi - 1e-6).astype(np.float32))
    f = crand(rng, T, *nmodes)
    outs = {}
    for kernel, after in (("gather", False), ("staged", False), ("staged", True)):
        p = hb.NufftPlan(hb.NufftType.TYPE_2, hb.NufftOpts(nmodes=nmodes, ntransf=T, kernel_width=w))
        if not after:
            p.set_interp_kernel(kernel)
        p.setpts([to_dev(x, cuda) for x in coords])
        if after:  # chosen once the points are set: the job list is built then
            p.set_interp_kernel(kernel)
        outs[(kernel, after)] = to_np(p(to_dev(f, cuda)))
    assert np.array_equal(outs[("staged", False)], outs[("gather", False)])
    assert np.array_equal(outs[("staged", True)], outs[("gather", False)])
    outs["staged"] = outs[("staged", False)]
    assert relerr(outs["staged"], gridding.nufft2(coords, f, w=w)) <= 1e-5


@pytest.mark.gpu
def test_staged_interp_is_refused_where_the_plan_does_not_allow_it(cuda):
    import hastycucompute_b200 as hb
    for nmodes, w, typ in (((32, 32), 4, hb.NufftType.TYPE_2), ((16, 16, 16), 8, hb.NufftType.TYPE_2),
                           ((16, 16, 16), 6, hb.NufftType.TYPE_1)):
        p = hb.NufftPlan(typ, hb.NufftOpts(nmodes=nmodes, ntransf=4, kernel_width=w))
        with pytest.raises(hb.HastyError, match="INVALID_ARG"):
            p.set_interp_kernel("staged")
        p.set_interp_kernel("gather")
