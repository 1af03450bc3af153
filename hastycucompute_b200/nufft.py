"""NUFFT plans: the B200 replacement of ``hasty::fft::nufft_plan`` (cpp/corelib/lib/fft/nufft.cppm).

Mirrors the reference's make / setpts / execute / free life cycle and its option struct
(``nufft_opts``, nufft.cppm:78-95): modes in image order, coordinates in radians with
``coords[i]`` pairing with image dimension ``i``, centred (CMCL) mode order, type-1 sign +1 and
type-2 sign -1 by default. Data are complex64 CUDA tensors; the transform runs on torch's current
stream and allocates nothing per call.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass
from typing import Sequence

import torch

from . import _lib
from ._torch import check_tensor, ptr, stream_ptr


class NufftType(enum.IntEnum):
    """nufft_type, nufft.cppm:42-48."""
    TYPE_1 = 1
    TYPE_2 = 2
    FORWARD = 2
    BACKWARD = 1


class NufftSign(enum.IntEnum):
    """nufft_sign, nufft.cppm:50-55."""
    POS = 1
    NEG = -1
    DEFAULT_TYPE_1 = 1
    DEFAULT_TYPE_2 = -1


class NufftUpsamp(enum.Enum):
    """nufft_upsamp_cuda, nufft.cppm:59-63 (DEFAULT is 2.0 here, as in cufinufft)."""
    UPSAMP_2_0 = 2.0
    UPSAMP_1_25 = 1.25
    DEFAULT = 0.0


class NufftMethod(enum.IntEnum):
    """nufft_method_cuda, nufft.cppm:65-70. All select the same bin-sorted tile kernels."""
    GM_NO_SORT = 0
    GM_SORT = 1
    SM = 2
    DEFAULT = 3


@dataclass
class NufftOpts:
    """nufft_opts<cuda_t, f32_t, DIM> (nufft.cppm:78-95) plus an explicit kernel width.

    ``kernel_width`` > 0 overrides the width derived from ``tol`` (w = ceil(log10(10/tol))).
    """
    nmodes: Sequence[int]
    ntransf: int = 1
    tol: float = 1e-5
    sign: NufftSign | int | None = None
    upsamp: NufftUpsamp = NufftUpsamp.DEFAULT
    method: NufftMethod = NufftMethod.DEFAULT
    kernel_width: int = 0
    device_idx: int | None = None

    def get_sign(self, ntype: NufftType) -> int:
        if self.sign is None:
            return 1 if ntype == NufftType.TYPE_1 else -1
        return int(self.sign)


@dataclass
class PlanInfo:
    fine: tuple
    width: int
    beta: float
    device_bytes: int


class NufftPlan:
    """nufft_plan<cuda_t, f32_t, DIM, NT> (nufft.cppm:103-310)."""

    def __init__(self, ntype: NufftType, opts: NufftOpts):
        self._h = C.c_void_p()
        self.type = NufftType(ntype)
        self.opts = opts
        self.dim = len(opts.nmodes)
        if not 1 <= self.dim <= 3:
            raise ValueError("nmodes must have 1..3 entries")
        self.nmodes = tuple(int(n) for n in opts.nmodes)
        self.ntransf = int(opts.ntransf)
        self.device = torch.device("cuda", opts.device_idx if opts.device_idx is not None else torch.cuda.current_device())
        self.M = None
        self.nframes = None  # set by setpts_frames: execute then takes / gives frame-stacked modes
        self.frame_points = None
        self._coords = None
        with torch.cuda.device(self.device):
            _lib.call("hb_nufft_makeplan", int(self.type), self.dim, _lib.i64_array(self.nmodes),
                      opts.get_sign(self.type), self.ntransf, float(opts.tol), int(opts.kernel_width),
                      float(opts.upsamp.value), int(opts.method), C.byref(self._h))

    # -- reference API --------------------------------------------------------------------------
    @classmethod
    def make(cls, ntype: NufftType, opts: NufftOpts) -> "NufftPlan":
        """nufft_plan::make (nufft.cppm:107-172)."""
        return cls(ntype, opts)

    def setpts(self, coords: Sequence[torch.Tensor]) -> None:
        """nufft_plan::setpts (nufft.cppm:175-203). coords[i] (float32, [M]) pairs with dim i."""
        if len(coords) != self.dim:
            raise ValueError(f"expected {self.dim} coordinate arrays")
        M = coords[0].shape[0]
        for i, c in enumerate(coords):
            check_tensor(c, f"coords[{i}]", torch.float32, (M,), self.device)
        if self.dim >= 2 and coords[0].shape[0] != coords[1].shape[0]:
            raise ValueError("x and y coords have different lengths")
        cp = [ptr(c) for c in coords] + [C.c_void_p(None)] * (3 - self.dim)
        with torch.cuda.device(self.device):
            _lib.call("hb_nufft_setpts", self._h, int(M), cp[0], cp[1], cp[2], stream_ptr(self.device))
        self.M = int(M)
        self.nframes = None
        self.frame_points = None
        self._coords = tuple(coords)

    def setpts_frames(self, frame_coords: Sequence[Sequence[torch.Tensor]]) -> None:
        """Points of several frames (each its own trajectory, any number of points, zero allowed)
        in one plan: one bin sort now and one launch per pass at every execute, in place of one
        plan execute per frame (the per-frame loops of hasty_python/simul_op.py:39-91 and
        right_precond_test.py:48-73). After it, execute takes / gives

            type 1: input [ntransf, M] -> output [nframes, ntransf, *nmodes]
            type 2: input [nframes, ntransf, *nmodes] -> output [ntransf, M]

        with M the total point count and the frames' points back to back along M."""
        F = len(frame_coords)
        if F < 1:
            raise ValueError("need at least one frame")
        counts = []
        for f, coords in enumerate(frame_coords):
            if len(coords) != self.dim:
                raise ValueError(f"frame {f}: expected {self.dim} coordinate arrays")
            m = coords[0].shape[0]
            for i, c in enumerate(coords):
                check_tensor(c, f"frame {f} coords[{i}]", torch.float32, (m,), self.device)
            counts.append(int(m))
        cat = [torch.cat([fc[i] for fc in frame_coords]).contiguous() for i in range(self.dim)]
        cp = [ptr(c) for c in cat] + [C.c_void_p(None)] * (3 - self.dim)
        with torch.cuda.device(self.device):
            _lib.call("hb_nufft_setpts_frames", self._h, F, _lib.i64_array(counts), cp[0], cp[1], cp[2],
                      stream_ptr(self.device))
        self.M = int(sum(counts))
        self.nframes = F
        self.frame_points = tuple(counts)
        self._coords = tuple(cat)

    def _mode_shape(self) -> tuple:
        base = (self.ntransf, *self.nmodes)
        return base if self.nframes is None else (self.nframes, *base)

    def execute(self, input: torch.Tensor, output: torch.Tensor) -> torch.Tensor:
        """nufft_plan::execute (nufft.cppm:205-250).

        type 1: input [ntransf, M] -> output [ntransf, *nmodes];
        type 2: input [ntransf, *nmodes] -> output [ntransf, M].
        """
        if self.M is None:
            raise RuntimeError("execute called before setpts")
        if self.type == NufftType.TYPE_1:
            check_tensor(input, "input", torch.complex64, (self.ntransf, self.M), self.device)
            check_tensor(output, "output", torch.complex64, self._mode_shape(), self.device)
        else:
            check_tensor(input, "input", torch.complex64, self._mode_shape(), self.device)
            check_tensor(output, "output", torch.complex64, (self.ntransf, self.M), self.device)
        with torch.cuda.device(self.device):
            _lib.call("hb_nufft_execute", self._h, ptr(input), ptr(output), stream_ptr(self.device))
        return output

    def free(self) -> None:
        """nufft_plan::free (nufft.cppm:279-297)."""
        if self._h:
            _lib.call("hb_nufft_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # -- extras ----------------------------------------------------------------------------------
    def set_spread_tuning(self, max_candidates: int = 4096, block=(2, 4, 4)) -> None:
        """Spreading knobs (before setpts): points per subproblem and the warp's cell block
        (image order; 2-D plans take (1, by, bx)). Without a call, setpts picks the subproblem
        size from the number of points."""
        if self.M is not None:
            raise RuntimeError("set the spread tuning before setpts")
        b = tuple(int(v) for v in block)
        if len(b) == 2:
            b = (1,) + b
        _lib.call("hb_nufft_set_spread_tuning", self._h, int(max_candidates), *b)

    def set_spread_kernel(self, kind: str = "auto", transforms_per_cta: int = 0) -> None:
        """Spreading kernel (before setpts): "auto", "cells" (one cell per lane) or "transforms"
        (transforms on the lanes), and for the latter the transforms one CTA spreads (8, 16, 32;
        0 = automatic). All compute the same sums."""
        if self.M is not None:
            raise RuntimeError("set the spreading kernel before setpts")
        code = {"auto": 0, "cells": 1, "transforms": 2}[kind]
        _lib.call("hb_nufft_set_spread_kernel", self._h, code, int(transforms_per_cta))

    def set_interp_tuning(self, transforms_per_group: int = 0) -> None:
        """Interpolation (type 2): transforms per lane group (points per warp = 32 / that; 0 =
        automatic). All choices compute the same sums."""
        _lib.call("hb_nufft_set_interp_tuning", self._h, int(transforms_per_group))

    def set_interp_kernel(self, kind: str = "auto") -> None:
        """Interpolation (type 2): "gather" (each point's cells from global memory), "staged" (per
        8^3 tile and 8 transforms, the reachable region copied to shared memory first; 3-D, widths
        4..7) or "auto". Both give bit-identical samples."""
        kinds = {"auto": 0, "gather": 1, "staged": 2}
        if kind not in kinds:
            raise ValueError(f"interpolation kernel must be one of {sorted(kinds)}")
        _lib.call("hb_nufft_set_interp_kernel", self._h, kinds[kind])

    def info(self) -> PlanInfo:
        fine = (C.c_int64 * 3)()
        w = C.c_int()
        beta = C.c_double()
        nb = C.c_size_t()
        _lib.call("hb_nufft_get_info", self._h, fine, C.byref(w), C.byref(beta), C.byref(nb))
        return PlanInfo(tuple(fine[: self.dim]), w.value, beta.value, nb.value)

    def __call__(self, input: torch.Tensor) -> torch.Tensor:
        if self.type == NufftType.TYPE_1:
            out = torch.empty(self._mode_shape(), dtype=torch.complex64, device=self.device)
        else:
            out = torch.empty((self.ntransf, self.M), dtype=torch.complex64, device=self.device)
        return self.execute(input, out)


def nufft_type1(coords: Sequence[torch.Tensor], data: torch.Tensor, nmodes: Sequence[int], **kw) -> torch.Tensor:
    """One-shot adjoint NUFFT: data [ntransf, M] -> [ntransf, *nmodes]."""
    opts = NufftOpts(nmodes=tuple(nmodes), ntransf=data.shape[0], **kw)
    plan = NufftPlan(NufftType.TYPE_1, opts)
    plan.setpts(coords)
    out = plan(data)
    return out


def nufft_type2(coords: Sequence[torch.Tensor], image: torch.Tensor, **kw) -> torch.Tensor:
    """One-shot forward NUFFT: image [ntransf, *nmodes] -> [ntransf, M]."""
    opts = NufftOpts(nmodes=tuple(image.shape[1:]), ntransf=image.shape[0], **kw)
    plan = NufftPlan(NufftType.TYPE_2, opts)
    plan.setpts(coords)
    return plan(image)


def nufft_backward_cpu_over_cuda(dimshape: Sequence[int], input: torch.Tensor, coords: Sequence[torch.Tensor],
                                 kernel_width: int = 0, tol: float = 1e-6) -> torch.Tensor:
    """nufft_backward_cpu_over_cuda (cpp/corelib/lib/fft/nufft.cppm:316-382): adjoint NUFFT of host
    data [T, M] at device coordinates, returned on the host as [T, *dimshape]. The reference moves
    and transforms one row at a time with a device synchronisation around each; here all T rows go
    in one pinned copy and one batched execute. tol 1e-6 is the reference's float default."""
    if input.is_cuda:
        raise ValueError("input must be a host tensor")
    dev = coords[0].device
    T = input.shape[0]
    host = input.to(torch.complex64).contiguous().pin_memory()
    d = host.to(dev, non_blocking=True)
    plan = NufftPlan(NufftType.TYPE_1, NufftOpts(nmodes=tuple(dimshape), ntransf=T, tol=tol, kernel_width=kernel_width))
    plan.setpts(list(coords))
    out = plan(d)
    res = torch.empty(out.shape, dtype=torch.complex64).pin_memory()
    res.copy_(out, non_blocking=True)
    torch.cuda.current_stream(dev).synchronize()
    plan.free()
    return res.to(input.dtype) if input.dtype != torch.complex64 and input.is_complex() else res
