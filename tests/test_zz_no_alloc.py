"""The allocation-free SENSE normal entry point, hb_sense_normal_noalloc.

It serves callers that cannot allocate device memory (a runtime embedded in another framework
that owns every allocation, a driver layer that only hands out fixed buffers): its workspace and
twiddle tables are fixed device arrays inside the library. This file checks it through the C ABI
against the allocating entry point hb_sense_normal and against the FP64 oracle of the SENSE
normal operator (NORMAL_T_T1_OP, cpp/corelib/lib/mri/normal.cppm:65-88), on two calls in a row
(the arrays keep the previous call's contents); that a second call changes neither the device's
free memory nor torch's allocator; and that a problem larger than its fixed workspace is refused
before anything runs. The file name sorts last so a run that stops at the first failure has run
every other test first.
"""

import numpy as np
import pytest

from helpers import crand, relerr, to_dev, to_np

TOL = 1e-5  # the suite's parity bar


def _call(name, shape, C_, x, S, Kt, out, ws=None):
    from hastycucompute_b200 import _lib
    from hastycucompute_b200._torch import ptr, stream_ptr
    shp = _lib.i64_array(shape)
    if name == "hb_sense_normal":
        nb = ws.numel() * ws.element_size()
        _lib.call(name, len(shape), shp, C_, ptr(x), ptr(S), ptr(Kt), ptr(out), ptr(ws), nb, stream_ptr(x.device))
    else:
        _lib.call(name, len(shape), shp, C_, ptr(x), ptr(S), ptr(Kt), ptr(out), stream_ptr(x.device))


@pytest.mark.gpu
@pytest.mark.parametrize("shape,C_", [((16, 20, 24), 4), ((64, 80), 8), ((32, 32, 32), 3)])
def test_noalloc_matches_allocating_entry_and_oracle_twice(cuda, shape, C_):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic, toeplitz as tp
    from oracle import toeplitz as otp
    rng = np.random.default_rng(C_)
    Sn = synthetic.coil_maps(C_, shape)
    S = to_dev(Sn, cuda)
    Kn = crand(rng, *[2 * s for s in shape])
    Kt = hb.transform_toeplitz_kernel(to_dev(Kn, cuda))
    ws = tp.make_workspace(shape, C_, cuda)
    for call in range(2):
        xn = crand(rng, *shape)
        x = to_dev(xn, cuda)
        ref = torch.empty_like(x)
        got = torch.full_like(x, float("nan"))
        _call("hb_sense_normal", shape, C_, x, S, Kt, ref, ws)
        _call("hb_sense_normal_noalloc", shape, C_, x, S, Kt, got)
        torch.cuda.synchronize()
        assert relerr(to_np(got), to_np(ref)) <= TOL, f"call {call}"
        oracle = otp.sense_normal(xn, Sn, Kn.astype(np.complex128))
        assert relerr(to_np(got), oracle) <= TOL, f"call {call} vs oracle"


@pytest.mark.gpu
def test_noalloc_second_call_allocates_nothing(cuda):
    import torch
    import hastycucompute_b200 as hb
    from hastycucompute_b200 import synthetic
    shape, C_ = (24, 24, 24), 4
    rng = np.random.default_rng(11)
    S = to_dev(synthetic.coil_maps(C_, shape), cuda)
    Kt = hb.transform_toeplitz_kernel(to_dev(crand(rng, *[2 * s for s in shape]), cuda))
    x = to_dev(crand(rng, *shape), cuda)
    outs = [torch.empty_like(x) for _ in range(2)]
    _call("hb_sense_normal_noalloc", shape, C_, x, S, Kt, outs[0])  # loads the module and its arrays
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(cuda)[0]
    alloc0, reserved0 = torch.cuda.memory_allocated(cuda), torch.cuda.memory_reserved(cuda)
    _call("hb_sense_normal_noalloc", shape, C_, x, S, Kt, outs[1])
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(cuda)[0] == free0
    assert (torch.cuda.memory_allocated(cuda), torch.cuda.memory_reserved(cuda)) == (alloc0, reserved0)
    assert relerr(to_np(outs[1]), to_np(outs[0])) == 0.0


@pytest.mark.gpu
def test_noalloc_refuses_problems_beyond_its_workspace(cuda):
    import torch
    import hastycucompute_b200 as hb
    shape, C_ = (64, 64, 64), 32  # needs 6 * 64^3 * 32 * 8 B = 384 MiB > 32 MiB
    x = torch.zeros(shape, dtype=torch.complex64, device=cuda)
    S = torch.zeros((C_, *shape), dtype=torch.complex64, device=cuda)
    Kt = torch.zeros(tuple(2 * s for s in shape), dtype=torch.complex64, device=cuda)
    out = torch.zeros_like(x)
    with pytest.raises(hb.HastyError, match="HB_ERR_WORKSPACE"):
        _call("hb_sense_normal_noalloc", shape, C_, x, S, Kt, out)
