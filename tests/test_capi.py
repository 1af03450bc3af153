"""The C ABI library loads, exports every function include/hasty_b200.h declares, and validates
arguments on the host (no GPU needed: none of these calls reaches a kernel)."""
import ctypes as C
import re
from pathlib import Path


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


_SCALARS = {"int": C.c_int, "int64_t": C.c_int64, "float": C.c_float, "double": C.c_double,
             "size_t": C.c_size_t, "hb_nufft_plan": C.c_void_p}
_POINTEES = {"int": C.c_int, "int64_t": C.c_int64, "float": C.c_float, "double": C.c_double,
             "size_t": C.c_size_t, "hb_nufft_plan": C.c_void_p}


def declarations():
    """{name: (return type, [parameter types])} from the header, const and names stripped."""
    text = (ROOT / "include" / "hasty_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for ret, name, params in re.findall(r"([A-Za-z_][\w \*]*?)\s*\b(hb_\w+)\s*\(([^)]*)\)\s*;", text):
        types = []
        for p in params.split(","):
            p = " ".join(p.replace("const", " ").split())
            if p in ("", "void"):
                continue
            types.append(re.sub(r"\s*\b\w+$", "", p).replace(" ", "") if not p.endswith("*") else p.replace(" ", ""))
        out[name] = (" ".join(ret.replace("const", " ").split()).replace(" *", "*"), types)
    return out


def _matches(ctype, ctext):
    """ctypes type against a C type: scalars exactly; pointers as c_void_p / c_char_p or a
    POINTER to the same pointee."""
    if ctext.endswith("*"):
        base = ctext[:-1]
        if ctype in (C.c_void_p,):
            return True
        if ctype is C.c_char_p:
            return base == "char"
        return getattr(ctype, "_type_", None) is _POINTEES.get(base)
    return ctype is _SCALARS.get(ctext)


def test_binding_signatures_match_header():
    """Every ctypes signature has the header's arity, pointer-ness and scalar types (a drifted
    argument list would pass garbage through the ABI without any error)."""
    from hastycucompute_b200 import _lib
    decl = declarations()
    assert set(decl) == set(_lib.SIGNATURES)
    for name, (ret, params) in decl.items():
        res, args = _lib.SIGNATURES[name]
        assert len(args) == len(params), (name, len(args), params)
        for i, (a, p) in enumerate(zip(args, params)):
            assert _matches(a, p), (name, i, a, p)
        assert _matches(res, ret) or (ret == "char*" and res is C.c_char_p), (name, res, ret)


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
    assert lib.hb_toeplitz_workspace_size(3, _lib.i64_array([11, 8, 8]), 1, C.byref(n)) == 0  # 22 = 2 * 11
    assert lib.hb_toeplitz_workspace_size(3, _lib.i64_array([17, 8, 8]), 1, C.byref(n)) == 1  # 34 = 2 * 17
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


def test_frame_entry_points_reject_bad_arguments_before_touching_the_device():
    """hb_nufft_setpts_frames and hb_toeplitz_kernels_frames check their host arguments first."""
    from hastycucompute_b200 import _lib
    lib = _lib.load()
    npts = _lib.i64_array([100, 0, 50])
    dummy = C.c_void_p(16)
    assert lib.hb_nufft_setpts_frames(None, 3, npts, dummy, dummy, dummy, None) == 1
    assert b"plan" in lib.hb_last_error()
    kshape = _lib.i64_array([16, 16, 16])
    assert lib.hb_toeplitz_kernels_frames(4, kshape, 3, npts, dummy, dummy, dummy, dummy, dummy, 6, None) == 1
    assert lib.hb_toeplitz_kernels_frames(3, kshape, 0, npts, dummy, dummy, dummy, dummy, dummy, 6, None) == 1
    assert lib.hb_toeplitz_kernels_frames(3, kshape, 3, None, dummy, dummy, dummy, dummy, dummy, 6, None) == 1
    assert lib.hb_toeplitz_kernels_frames(3, _lib.i64_array([16, 15, 16]), 3, npts, dummy, dummy, dummy, dummy, dummy,
                                          6, None) == 2
