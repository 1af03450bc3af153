"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py): they pin the oracle
(CPU) and the GPU path (gpu marker) to the FP64 NUDFT and to the reference's own Toeplitz
load/store kernels."""
from pathlib import Path

import numpy as np
import pytest

from helpers import relerr, to_dev, to_np
from oracle import gridding, nudft, refload
from oracle import toeplitz as otp

G = Path(__file__).resolve().parent / "golden"
NUDFT_TOL = {4: 2e-3, 6: 3e-5, 8: 3e-6}


def load(name):
    return dict(np.load(G / name))


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_nudft_fixture_reproduces(dim):
    d = load(f"nudft_{dim}d.npz")
    nm = tuple(int(v) for v in d["nmodes"])
    assert relerr(nudft.type1(list(d["coords"]), d["c"], nm, sign=1), d["type1"]) < 1e-12
    assert relerr(nudft.type2(list(d["coords"]), d["f"], sign=-1), d["type2"]) < 1e-12


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("w", [4, 6, 8])
def test_gridding_oracle_against_nudft_fixture(dim, w):
    d = load(f"nudft_{dim}d.npz")
    nm = tuple(int(v) for v in d["nmodes"])
    assert relerr(gridding.nufft1(list(d["coords"]), d["c"], nm, w=w), d["type1"]) < NUDFT_TOL[w]
    assert relerr(gridding.nufft2(list(d["coords"]), d["f"], w=w), d["type2"]) < NUDFT_TOL[w]


@pytest.mark.parametrize("dim", [2, 3])
def test_toeplitz_oracle_against_reference_kernel_fixture(dim):
    d = load(f"ref_toeplitz_{dim}d.npz")
    for fl, ref in zip(d["flags"], d["outputs"]):
        io, i1, o1, i2, o2, acc = (int(v) for v in fl)
        got = otp.toeplitz_multiplication(d["input"], d["out0"], d["kernel"].astype(np.complex128), d["mult1"],
                                          d["mult2"], io, i1, o1, i2, o2, acc)
        assert relerr(got, ref) < 1e-6, fl


@pytest.mark.skipif(not refload.available(), reason="reference kernels not built (oracle/_ref)")
@pytest.mark.parametrize("dim", [2, 3])
def test_reference_kernel_build_reproduces_fixture(dim):
    d = load(f"ref_toeplitz_{dim}d.npz")
    for fl, ref in zip(d["flags"], d["outputs"]):
        got = refload.multiplication(d["input"], d["out0"], d["kernel"].astype(np.complex128), d["mult1"], d["mult2"],
                                     *(int(v) for v in fl))
        assert relerr(got, ref) < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_gpu_nufft_against_nudft_fixture(cuda, dim):
    import hastycucompute_b200 as hb
    d = load(f"nudft_{dim}d.npz")
    nm = tuple(int(v) for v in d["nmodes"])
    coords = [to_dev(c, cuda) for c in d["coords"]]
    for w in (4, 6, 8):
        p1 = hb.NufftPlan(hb.NufftType.TYPE_1, hb.NufftOpts(nmodes=nm, ntransf=2, kernel_width=w))
        p1.setpts(coords)
        assert relerr(to_np(p1(to_dev(d["c"], cuda))), d["type1"]) < NUDFT_TOL[w]
        p2 = hb.NufftPlan(hb.NufftType.TYPE_2, hb.NufftOpts(nmodes=nm, ntransf=2, kernel_width=w))
        p2.setpts(coords)
        assert relerr(to_np(p2(to_dev(d["f"], cuda))), d["type2"]) < NUDFT_TOL[w]


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_gpu_toeplitz_against_reference_kernel_fixture(cuda, dim):
    import hastycucompute_b200 as hb
    d = load(f"ref_toeplitz_{dim}d.npz")
    Kt = hb.transform_toeplitz_kernel(to_dev(d["kernel"], cuda))
    for fl, ref in zip(d["flags"], d["outputs"]):
        out = to_dev(d["out0"], cuda)
        hb.toeplitz_multiplication(to_dev(d["input"], cuda), out, Kt, None, to_dev(d["mult1"], cuda),
                                   to_dev(d["mult2"], cuda), *(int(v) for v in fl))
        assert relerr(to_np(out), ref) < 1e-5, fl
