"""SENSE operators around the NUFFT and the Toeplitz normal operator.

``NormalTT1Op`` is ``NORMAL_T_T1_OP`` (cpp/corelib/lib/mri/normal.cppm:43-93): built from a
Toeplitz kernel and the stacked coil maps, it maps an image x to sum_c conj(S_c) T(S_c x). Here
the coil expand, the padded convolution, the coil reduce and the sum run as one fused apply with
a workspace held by the operator (no per-call allocation, graph capturable).

``SenseOp`` is the plain (non-Toeplitz) SENSE pair the Python experiments use
(hasty_python/right_precond_test.py:48-73, with the reference's 1/sqrt(prod N) scaling optional):
forward y_c = NUFFT2(S_c x), adjoint x = sum_c conj(S_c) NUFFT1(y_c).
"""
from __future__ import annotations

from typing import Optional, Sequence

import torch

from .nufft import NufftOpts, NufftPlan, NufftType
from .toeplitz import make_workspace, sense_normal, toeplitz_kernel, transform_toeplitz_kernel


class NormalTT1Op:
    """B x = sum_c conj(S_c) T (S_c x); operator API of op/op.cppm:14-102 (square, same type)."""

    class_name = "NORMAL_T_T1_OP"

    def __init__(self, kernel: torch.Tensor, stacked_diags: torch.Tensor, transformed: bool = False):
        self.dim = kernel.dim()
        self.kernel_t = kernel if transformed else transform_toeplitz_kernel(kernel)
        self.smaps = stacked_diags.contiguous()
        self.shape = tuple(self.smaps.shape[1:])
        if tuple(2 * s for s in self.shape) != tuple(kernel.shape):
            raise ValueError("kernel must have shape 2N for image shape N")
        self.ncoils = self.smaps.shape[0]
        self.device = self.smaps.device
        self.workspace = make_workspace(self.shape, self.ncoils, self.device)

    # operator API (device_type_t / input_tensor_type_t / ranks)
    device_type_t = "cuda"
    input_tensor_type_t = torch.complex64
    output_tensor_type_t = torch.complex64

    @property
    def input_rank_t(self) -> int:
        return self.dim

    @property
    def output_rank_t(self) -> int:
        return self.dim

    def apply(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        return sense_normal(x, self.smaps, self.kernel_t, out, self.workspace)

    __call__ = apply


def build_toeplitz_kernel(coords: Sequence[torch.Tensor], shape: Sequence[int], weights: Optional[torch.Tensor] = None,
                          kernel_width: int = 0) -> torch.Tensor:
    """Kernel [2N..] for image shape N and per-sample weights (ones by default)."""
    dev = coords[0].device
    M = coords[0].shape[0]
    if weights is None:
        nud = torch.ones((1, M), dtype=torch.complex64, device=dev)
    else:
        nud = weights.reshape(1, M).to(torch.complex64).contiguous()
    kernel = torch.zeros(tuple(2 * s for s in shape), dtype=torch.complex64, device=dev)
    return toeplitz_kernel(coords, kernel, nud, kernel_width=kernel_width)


class SenseOp:
    """Plain SENSE A (forward) / A^H (adjoint) with batched coils on one NUFFT plan pair."""

    def __init__(self, coords: Sequence[torch.Tensor], smaps: torch.Tensor, kernel_width: int = 0, tol: float = 1e-5,
                 scale: float = 1.0):
        self.smaps = smaps.contiguous()
        self.shape = tuple(smaps.shape[1:])
        self.ncoils = smaps.shape[0]
        self.scale = float(scale)
        opts = NufftOpts(nmodes=self.shape, ntransf=self.ncoils, tol=tol, kernel_width=kernel_width)
        self.fwd = NufftPlan(NufftType.TYPE_2, opts)
        self.adj = NufftPlan(NufftType.TYPE_1, opts)
        self.fwd.setpts(coords)
        self.adj.setpts(coords)
        self.M = coords[0].shape[0]

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        y = self.fwd(self.smaps * x.unsqueeze(0))
        return y * self.scale if self.scale != 1.0 else y

    def adjoint(self, y: torch.Tensor) -> torch.Tensor:
        img = self.adj(y.contiguous())
        out = (self.smaps.conj() * img).sum(0)
        return out * self.scale if self.scale != 1.0 else out

    def normal(self, x: torch.Tensor) -> torch.Tensor:
        return self.adjoint(self.forward(x))
