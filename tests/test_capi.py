"""The C ABI library loads, exports every function include/hasty_b200.h declares, and validates
arguments on the host (no GPU needed: none of these calls reaches a kernel)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "hasty_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    from hastycucompute_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 17
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), "binding table and header disagree"


def test_version_and_state_size():
    from hastycucompute_b200 import _lib
    lib = _lib.load()
    assert lib.hb_version() >= 10000
    assert lib.hb_cg_state_bytes() >= 64


def test_makeplan_rejects_bad_arguments():
    from hastycucompute_b200 import _lib
    lib = _lib.load()
    h = C.c_void_p()
    nm = _lib.i64_array([16, 16])
    assert lib.hb_nufft_makeplan(3, 2, nm, 0, 1, 1e-5, 0, 2.0, 3, C.byref(h)) == 1
    assert b"type" in lib.hb_last_error()
    assert lib.hb_nufft_makeplan(1, 4, nm, 0, 1, 1e-5, 0, 2.0, 3, C.byref(h)) == 1
    assert lib.hb_nufft_makeplan(1, 2, nm, 0, 0, 1e-5, 0, 2.0, 3, C.byref(h)) == 1
    assert lib.hb_nufft_makeplan(1, 2, nm, 2, 1, 1e-5, 0, 2.0, 3, C.byref(h)) == 1
    assert lib.hb_nufft_makeplan(1, 2, nm, 0, 1, 1e-5, 17, 2.0, 3, C.byref(h)) == 1
    assert lib.hb_nufft_makeplan(1, 2, nm, 0, 1, 1e-5, 0, 2.0, 7, C.byref(h)) == 1
    assert lib.hb_nufft_makeplan(1, 2, nm, 0, 1, 0.0, 0, 2.0, 3, C.byref(h)) == 1
    assert lib.hb_nufft_destroy(None) == 0


def test_toeplitz_workspace_size_is_host_arithmetic():
    from hastycucompute_b200 import _lib
    lib = _lib.load()
    n = C.c_size_t()
    assert lib.hb_toeplitz_workspace_size(3, _lib.i64_array([160, 160, 160]), 32, C.byref(n)) == 0
    N, B = 160, 32
    assert n.value == 8 * (N * N * 2 * N * B + N * 2 * N * 2 * N * B)
    assert lib.hb_toeplitz_workspace_size(2, _lib.i64_array([256, 256]), 12, C.byref(n)) == 0
    assert n.value == 8 * 256 * 512 * 12
    assert lib.hb_toeplitz_workspace_size(3, _lib.i64_array([11, 8, 8]), 1, C.byref(n)) == 1  # 22 not 2,3,5,7-smooth
    assert lib.hb_toeplitz_workspace_size(1, _lib.i64_array([8]), 1, C.byref(n)) == 1


def test_multiplication_rejects_bad_flags_before_touching_the_device():
    from hastycucompute_b200 import _lib
    lib = _lib.load()
    shp = _lib.i64_array([8, 8, 8])
    dummy = C.c_void_p(16)
    for bad in range(6):
        flags = [0, 0, 0, 0, 0, 0]
        flags[bad] = 3 if bad < 5 else 2
        st = lib.hb_toeplitz_multiplication(3, shp, 1, dummy, dummy, dummy, dummy, 1 << 30, None, None, *flags, None)
        assert st == 1, (bad, lib.hb_last_error())
        assert b"Invalid" in lib.hb_last_error()
