"""ctypes binding of libhasty_b200.so (the C ABI in include/hasty_b200.h).

The shared library is built in-tree (``python -m hastycucompute_b200.build``). Loading it is
lazy; every call raises :class:`HastyError` with the library's message on a non-zero status.
There is no fallback: without the library, every operator raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libhasty_b200.so"
_lib = None

HB_OK = 0
STATUS_NAMES = {
    1: "HB_ERR_INVALID_ARG",
    2: "HB_ERR_SHAPE",
    3: "HB_ERR_CUDA",
    4: "HB_ERR_ALLOC",
    5: "HB_ERR_STATE",
    6: "HB_ERR_RANGE",
    7: "HB_ERR_WORKSPACE",
}

# Every function the header declares, with (restype, argtypes).
_vp, _i, _i64, _f, _d, _sz = C.c_void_p, C.c_int, C.c_int64, C.c_float, C.c_double, C.c_size_t
_pi64 = C.POINTER(C.c_int64)
SIGNATURES = {
    "hb_last_error": (C.c_char_p, []),
    "hb_version": (_i, []),
    "hb_nufft_makeplan": (_i, [_i, _i, _pi64, _i, _i, _f, _i, _d, _i, C.POINTER(_vp)]),
    "hb_nufft_setpts": (_i, [_vp, _i64, _vp, _vp, _vp, _vp]),
    "hb_nufft_setpts_frames": (_i, [_vp, _i, _pi64, _vp, _vp, _vp, _vp]),
    "hb_nufft_execute": (_i, [_vp, _vp, _vp, _vp]),
    "hb_nufft_destroy": (_i, [_vp]),
    "hb_nufft_coord_grad": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "hb_nufft_set_spread_tuning": (_i, [_vp, _i, _i, _i, _i]),
    "hb_nufft_set_spread_kernel": (_i, [_vp, _i, _i]),
    "hb_nufft_set_interp_tuning": (_i, [_vp, _i]),
    "hb_nufft_set_interp_kernel": (_i, [_vp, _i]),
    "hb_nufft_get_info": (_i, [_vp, _pi64, C.POINTER(_i), C.POINTER(_d), C.POINTER(_sz)]),
    "hb_toeplitz_kernel": (_i, [_i, _pi64, _i64, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "hb_toeplitz_kernels_frames": (_i, [_i, _pi64, _i, _pi64, _vp, _vp, _vp, _vp, _vp, _i, _vp]),
    "hb_transform_toeplitz_kernel": (_i, [_i, _pi64, _vp, _vp, _vp]),
    "hb_toeplitz_workspace_size": (_i, [_i, _pi64, _i64, C.POINTER(_sz)]),
    "hb_toeplitz_multiplication": (_i, [_i, _pi64, _i64, _vp, _vp, _vp, _vp, _sz, _vp, _vp,
                                        _i, _i, _i, _i, _i, _i, _vp]),
    "hb_sense_normal": (_i, [_i, _pi64, _i64, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "hb_sense_normal_noalloc": (_i, [_i, _pi64, _i64, _vp, _vp, _vp, _vp, _vp]),
    "hb_sense_normal_ex": (_i, [_i, _pi64, _i64, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp, _sz, _vp]),
    "hb_sense_normal_batched": (_i, [_i, _pi64, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "hb_transform_toeplitz_kernels": (_i, [_i, _pi64, _i64, _vp, _vp, _vp]),
    "hb_cgb_state_bytes": (_sz, [_i64]),
    "hb_cgb_init": (_i, [_i64, _i64, _vp, _vp, _vp, _vp, _vp, _d, _vp]),
    "hb_cgb_step": (_i, [_i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hb_cgb_read_state": (_i, [_vp, _i64, C.POINTER(_d), _pi64, C.POINTER(_i), _vp]),
    "hb_cg_state_bytes": (_sz, []),
    "hb_cg_init": (_i, [_i64, _vp, _vp, _vp, _vp, _vp, _d, _vp]),
    "hb_cg_step": (_i, [_i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hb_cg_read_state": (_i, [_vp, C.POINTER(_d), _pi64, C.POINTER(_i), _vp]),
    "hb_pcg_residual": (_i, [_i64, _vp, _vp, _vp, _vp]),
    "hb_pcg_start": (_i, [_i64, _vp, _vp, _vp, _vp, _d, _vp]),
    "hb_pcg_step1": (_i, [_i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "hb_pcg_step2": (_i, [_i64, _vp, _vp, _vp, _vp, _i, _vp]),
    "hb_vdot_real": (_i, [_i64, _vp, _vp, _vp, _vp]),
    "hb_timing_enable": (_i, [_i]),
    "hb_timing_read": (_i, [C.c_char_p, _sz, C.POINTER(_f), _i, C.POINTER(_i), C.POINTER(_i)]),
}


class HastyError(RuntimeError):
    """A libhasty_b200 call returned a non-zero status."""

    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed ({STATUS_NAMES.get(status, status)}): {msg}")
        self.status = status


def lib_path() -> Path:
    return Path(os.environ.get("HASTY_B200_LIB", _LIB_PATH))


def load(path: str | os.PathLike | None = None):
    """Loads (once) and returns the ctypes library with all signatures declared."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else lib_path()
    if not p.exists():
        raise HastyError("load", -1, f"{p} not found; run `python -m hastycucompute_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    lib = load()
    st = getattr(lib, name)(*args)
    if st != HB_OK:
        msg = lib.hb_last_error()
        raise HastyError(name, st, msg.decode() if msg else "")


def i64_array(vals) -> C.Array:
    vals = [int(v) for v in vals]
    return (C.c_int64 * max(1, len(vals)))(*vals)


def timing_enable(on: bool = True) -> None:
    call("hb_timing_enable", 1 if on else 0)


def timing_read(cap: int = 64) -> tuple[dict, int]:
    """Per-kernel summed milliseconds since the last read, and the number of launches."""
    buf = C.create_string_buffer(4096)
    ms = (C.c_float * cap)()
    nn = C.c_int()
    nl = C.c_int()
    call("hb_timing_read", buf, 4096, ms, cap, C.byref(nn), C.byref(nl))
    names = buf.value.decode().split("\n") if nn.value else []
    return {n: float(ms[i]) for i, n in enumerate(names[:cap])}, int(nl.value)
