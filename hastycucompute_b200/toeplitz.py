"""Toeplitz-embedded normal operator: the B200 replacement of ``hasty::fft::toeplitz_kernel`` /
``transform_toeplitz_kernel`` / ``toeplitz_multiplication`` and of ``NORMAL_T_T1_OP``.

Reference: cpp/corelib/lib/fft/nufft.cppm:386-479 (kernel, straight multiply),
cpp/corelib/lib/fft/toeplitz.cppm:47-56 (enums), :510-712 (transform, multiplication),
:722-857 (torch-op shaped entry) and cpp/corelib/lib/mri/normal.cppm:43-93 (SENSE A^H A).

Operator (2N zero padding, centred crop, as the reference's straight path defines it):
    T(t) = crop_{[N-1, 2N-1)}( IFFT( FFT(pad_{2N}(t)) * K ) ),
    K    = FFT( embed_{[0, 2N-1)}( type1(w; 2N-1 modes) ) ) / prod(N),
so T = (1/prod(N)) A^H diag(w) A with A the type-2 NUFFT on the same points.
"""
from __future__ import annotations

import ctypes as C
import enum
from typing import Optional, Sequence

import torch

from . import _lib
from ._torch import check_tensor, ptr, stream_ptr


class ToeplitzMultType(enum.IntEnum):
    """toeplitz.cppm:47-51."""
    NONE = 0
    MULT = 1
    MULT_CONJ = 2


class ToeplitzAccumulateType(enum.IntEnum):
    """toeplitz.cppm:53-56."""
    NONE = 0
    ACCUMULATE = 1


def toeplitz_kernel(coords: Sequence[torch.Tensor], kernel: torch.Tensor, nudata: torch.Tensor,
                    kernel_width: int = 0) -> torch.Tensor:
    """toeplitz_kernel (nufft.cppm:386-441): fills ``kernel`` ([2N..], complex64) in place.

    ``nudata`` is [1, M] (or [M]) complex64 weights (ones, or a density compensation).
    ``kernel_width`` <= 0 derives the width from tol 1e-5 (w = 6 at upsampling 2).
    """
    dim = kernel.dim()
    if dim not in (2, 3):
        raise ValueError("kernel must be 2-D or 3-D")
    check_tensor(kernel, "kernel", torch.complex64)
    M = coords[0].shape[0]
    if len(coords) != dim:
        raise ValueError(f"expected {dim} coordinate arrays")
    for i, c in enumerate(coords):
        check_tensor(c, f"coords[{i}]", torch.float32, (M,), kernel.device)
    nd = nudata.reshape(-1)
    if nd.shape[0] != M:
        raise ValueError("shape<1>() of nudata didn't match length of coord vectors")
    check_tensor(nd, "nudata", torch.complex64, (M,), kernel.device)
    cp = [ptr(c) for c in coords] + [C.c_void_p(None)] * (3 - dim)
    with torch.cuda.device(kernel.device):
        _lib.call("hb_toeplitz_kernel", dim, _lib.i64_array(kernel.shape), int(M), cp[0], cp[1], cp[2],
                  ptr(nd), ptr(kernel), int(kernel_width), stream_ptr(kernel.device))
    return kernel


def toeplitz_kernels_frames(frame_coords: Sequence[Sequence[torch.Tensor]], kernels: torch.Tensor,
                            frame_nudata: Optional[Sequence[torch.Tensor]] = None, kernel_width: int = 0) -> torch.Tensor:
    """toeplitz_kernel for F frames in one call: fills ``kernels`` ([F, 2N..], complex64). Frame f
    has its own points ``frame_coords[f]`` (any count, zero allowed) and weights
    ``frame_nudata[f]`` ([M_f] or [1, M_f]; ones when None). One frame-batched type-1 NUFFT and
    one launch per FFT pass serve all frames, in place of one plan per frame."""
    F = kernels.shape[0]
    dim = kernels.dim() - 1
    if dim not in (2, 3):
        raise ValueError("kernels must be [F, 2N..] with 2-D or 3-D frames")
    if len(frame_coords) != F:
        raise ValueError("one coordinate set per frame")
    check_tensor(kernels, "kernels", torch.complex64, None, kernels.device)
    dev = kernels.device
    counts, nds = [], []
    for f, coords in enumerate(frame_coords):
        if len(coords) != dim:
            raise ValueError(f"frame {f}: expected {dim} coordinate arrays")
        m = coords[0].shape[0]
        for i, c in enumerate(coords):
            check_tensor(c, f"frame {f} coords[{i}]", torch.float32, (m,), dev)
        if frame_nudata is None:
            nds.append(torch.ones(m, dtype=torch.complex64, device=dev))
        else:
            nd = frame_nudata[f].reshape(-1).to(torch.complex64)
            if nd.shape[0] != m:
                raise ValueError(f"frame {f}: nudata length differs from the coordinates")
            nds.append(nd)
        counts.append(int(m))
    cat = [torch.cat([fc[i] for fc in frame_coords]).contiguous() for i in range(dim)]
    nd = torch.cat(nds).contiguous()
    cp = [ptr(c) for c in cat] + [C.c_void_p(None)] * (3 - dim)
    with torch.cuda.device(dev):
        _lib.call("hb_toeplitz_kernels_frames", dim, _lib.i64_array(kernels.shape[1:]), F, _lib.i64_array(counts),
                  cp[0], cp[1], cp[2], ptr(nd), ptr(kernels), int(kernel_width), stream_ptr(dev))
    return kernels


def transform_toeplitz_kernel(kernel: torch.Tensor) -> torch.Tensor:
    """transform_toeplitz_kernel (toeplitz.cppm:510-609): returns the kernel in the layout the
    fused multiplication reads (a new tensor, same element count)."""
    check_tensor(kernel, "kernel", torch.complex64)
    out = torch.empty_like(kernel)
    with torch.cuda.device(kernel.device):
        _lib.call("hb_transform_toeplitz_kernel", kernel.dim(), _lib.i64_array(kernel.shape), ptr(kernel),
                  ptr(out), stream_ptr(kernel.device))
    return out


def workspace_bytes(shape: Sequence[int], nbatch: int) -> int:
    n = C.c_size_t()
    _lib.call("hb_toeplitz_workspace_size", len(shape), _lib.i64_array(shape), int(nbatch), C.byref(n))
    return int(n.value)


def make_workspace(shape: Sequence[int], nbatch: int, device) -> torch.Tensor:
    nb = workspace_bytes(shape, nbatch)
    return torch.empty((nb + 7) // 8, dtype=torch.complex64, device=device)


def toeplitz_multiplication(input: torch.Tensor, output: torch.Tensor, kernel: torch.Tensor,
                            scratch: Optional[torch.Tensor] = None, mult1: Optional[torch.Tensor] = None,
                            mult2: Optional[torch.Tensor] = None,
                            input_output_mult_type: int = ToeplitzMultType.NONE,
                            input_mult1_type: int = ToeplitzMultType.MULT,
                            output_mult1_type: int = ToeplitzMultType.MULT_CONJ,
                            input_mult2_type: int = ToeplitzMultType.MULT,
                            output_mult2_type: int = ToeplitzMultType.MULT_CONJ,
                            accumulate_type: int = ToeplitzAccumulateType.NONE) -> torch.Tensor:
    """toeplitz_multiplication / ops_toeplitz_multiplication (toeplitz.cppm:611-857).

    input/output: [B, N..] complex64; kernel: transformed kernel [2N..]; mult1/mult2: [N..] or
    None; scratch: a workspace tensor from :func:`make_workspace` or None (then allocated
    stream-ordered per call). Enum defaults follow perform_toeplitz_multiplication_cuda_3D.
    """
    dim = input.dim() - 1
    if dim not in (2, 3):
        raise ValueError("input and output must be 3D or 4D (with batch)")
    check_tensor(input, "input", torch.complex64)
    check_tensor(output, "output", torch.complex64, input.shape, input.device)
    img = tuple(input.shape[1:])
    check_tensor(kernel, "kernel", torch.complex64, tuple(2 * s for s in img), input.device)
    for name, m in (("mult1", mult1), ("mult2", mult2)):
        if m is not None:
            check_tensor(m, name, torch.complex64, img, input.device)
    sb = 0
    if scratch is not None:
        check_tensor(scratch, "scratch", scratch.dtype, device=input.device)
        sb = scratch.numel() * scratch.element_size()
    with torch.cuda.device(input.device):
        _lib.call("hb_toeplitz_multiplication", dim, _lib.i64_array(img), int(input.shape[0]), ptr(input),
                  ptr(output), ptr(kernel), ptr(scratch), sb, ptr(mult1), ptr(mult2), int(input_output_mult_type),
                  int(input_mult1_type), int(output_mult1_type), int(input_mult2_type), int(output_mult2_type),
                  int(accumulate_type), stream_ptr(input.device))
    return output


def toeplitz_multiply(inout: torch.Tensor, kernel_t: torch.Tensor, scratch: Optional[torch.Tensor] = None) -> torch.Tensor:
    """toeplitz_multiply (nufft.cppm:448-479): inout[b] <- T(inout[b]) for every batch b, with the
    transformed kernel. Returns a new tensor (the reference rebinds its argument)."""
    out = torch.empty_like(inout)
    return toeplitz_multiplication(inout, out, kernel_t, scratch, None, None, ToeplitzMultType.NONE,
                                   ToeplitzMultType.NONE, ToeplitzMultType.NONE, ToeplitzMultType.NONE,
                                   ToeplitzMultType.NONE, ToeplitzAccumulateType.NONE)


def sense_normal(x: torch.Tensor, smaps: torch.Tensor, kernel_t: torch.Tensor, out: Optional[torch.Tensor] = None,
                 scratch: Optional[torch.Tensor] = None) -> torch.Tensor:
    """sum_c conj(S_c) T(S_c x) in one fused apply (NORMAL_T_T1_OP::operator(), normal.cppm:65-88)."""
    dim = x.dim()
    check_tensor(x, "x", torch.complex64)
    check_tensor(smaps, "smaps", torch.complex64, (smaps.shape[0], *x.shape), x.device)
    check_tensor(kernel_t, "kernel", torch.complex64, tuple(2 * s for s in x.shape), x.device)
    if out is None:
        out = torch.empty_like(x)
    check_tensor(out, "out", torch.complex64, x.shape, x.device)
    sb = 0
    if scratch is not None:
        sb = scratch.numel() * scratch.element_size()
    with torch.cuda.device(x.device):
        _lib.call("hb_sense_normal", dim, _lib.i64_array(x.shape), int(smaps.shape[0]), ptr(x), ptr(smaps),
                  ptr(kernel_t), ptr(out), ptr(scratch), sb, stream_ptr(x.device))
    return out


def sense_normal_ex(x: torch.Tensor, smaps: torch.Tensor, kernel_t: torch.Tensor, out: torch.Tensor,
                    smaps_out: Optional[torch.Tensor] = None, diag: Optional[torch.Tensor] = None,
                    accumulate: bool = False, scratch: Optional[torch.Tensor] = None) -> torch.Tensor:
    """out (+)= conj(R) sum_c conj(U_c) T(R S_c x): one time segment of NORMAL_IDT_T1_OP /
    NORMAL_IDTW_T1_OP (cpp/corelib/lib/mri/normal.cppm:218-266, 441-535) as one fused apply.
    U = smaps_out (default smaps), R = diag (default 1)."""
    dim = x.dim()
    check_tensor(x, "x", torch.complex64)
    check_tensor(smaps, "smaps", torch.complex64, (smaps.shape[0], *x.shape), x.device)
    if smaps_out is not None:
        check_tensor(smaps_out, "smaps_out", torch.complex64, tuple(smaps.shape), x.device)
    if diag is not None:
        check_tensor(diag, "diag", torch.complex64, tuple(x.shape), x.device)
    check_tensor(kernel_t, "kernel", torch.complex64, tuple(2 * s for s in x.shape), x.device)
    check_tensor(out, "out", torch.complex64, x.shape, x.device)
    sb = 0 if scratch is None else scratch.numel() * scratch.element_size()
    with torch.cuda.device(x.device):
        _lib.call("hb_sense_normal_ex", dim, _lib.i64_array(x.shape), int(smaps.shape[0]), ptr(x), ptr(smaps),
                  ptr(smaps_out), ptr(diag), 1 if accumulate else 0, ptr(kernel_t), ptr(out), ptr(scratch), sb,
                  stream_ptr(x.device))
    return out
