"""Differentiable NUFFT and Toeplitz operators (torch.autograd), with gradients with respect to
both the data and the k-space coordinates.

- image / data gradients are the adjoint transforms: for c = A f (type 2, sign s),
  dL/df = A^H dL/dc (a type 1 of sign -s); for f = B c (type 1, sign s), dL/dc = B^H dL/df
  (a type 2 of sign -s);
- coordinate gradients come from hb_nufft_coord_grad, the kernel-derivative interpolation: the
  exact derivative of the implemented gridding operator with respect to the points;
- the Toeplitz SENSE normal operator is self-adjoint, so its backward is one more apply.

The reference has no derivatives on this path; its trajectory-design code
(hasty_python/hastycompute/seq_design/gradient_design.py:167-171) produces the coordinates these
operators differentiate through.
"""
from __future__ import annotations

from typing import Sequence

import torch

from . import _lib
from ._torch import check_tensor, ptr, stream_ptr
from .nufft import NufftOpts, NufftPlan, NufftType


def coord_grad(plan2: NufftPlan, modes: torch.Tensor, h: torch.Tensor) -> torch.Tensor:
    """hb_nufft_coord_grad: [dim, M] float32 gradient for the points of type-2 `plan2` (a plan set
    with ``setpts_frames`` takes frame-stacked modes [F, ntransf, N..] and gives every frame's
    points' gradients back to back along M)."""
    modes = modes.contiguous()
    h = h.contiguous()
    check_tensor(modes, "modes", torch.complex64, plan2._mode_shape(), plan2.device)
    check_tensor(h, "h", torch.complex64, (plan2.ntransf, plan2.M), plan2.device)
    grad = torch.empty((plan2.dim, plan2.M), dtype=torch.float32, device=plan2.device)
    _lib.call("hb_nufft_coord_grad", plan2._h, ptr(modes), ptr(h), ptr(grad), stream_ptr(plan2.device))
    return grad


class NufftPair:
    """Type-2 plan of sign s and type-1 plan of sign -s on one set of points (an operator A and
    its adjoint), re-pointed by ``setpts`` whenever the coordinates change."""

    def __init__(self, nmodes: Sequence[int], ntransf: int, kernel_width: int = 6, sign: int = -1,
                 device=None):
        self.nmodes = tuple(int(n) for n in nmodes)
        self.ntransf = int(ntransf)
        self.sign = int(sign)
        kw = dict(nmodes=self.nmodes, ntransf=self.ntransf, kernel_width=kernel_width,
                  device_idx=None if device is None else torch.device(device).index)
        self.fwd = NufftPlan(NufftType.TYPE_2, NufftOpts(sign=self.sign, **kw))     # A
        self.adj = NufftPlan(NufftType.TYPE_1, NufftOpts(sign=-self.sign, **kw))    # A^H
        self._key = None

    def setpts(self, coords: torch.Tensor) -> None:
        key = (coords.data_ptr(), coords._version, tuple(coords.shape))
        if key == self._key:
            return
        cs = [coords[i].detach().contiguous() for i in range(coords.shape[0])]
        self.fwd.setpts(cs)
        self.adj.setpts(cs)
        self._key = key


class _Type2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, coords, pair):
        pair.setpts(coords)
        ctx.pair = pair
        ctx.save_for_backward(f, coords)
        return pair.fwd(f.contiguous())

    @staticmethod
    def backward(ctx, gy):
        f, coords = ctx.saved_tensors
        pair = ctx.pair
        pair.setpts(coords)
        gy = gy.contiguous()
        gf = pair.adj(gy) if ctx.needs_input_grad[0] else None
        gx = coord_grad(pair.fwd, f.contiguous(), gy.conj().resolve_conj()) if ctx.needs_input_grad[1] else None
        return gf, gx, None


class _Type1(torch.autograd.Function):
    @staticmethod
    def forward(ctx, c, coords, pair):
        # f = A^H c with A the pair's type 2: a type 1 of sign -s
        pair.setpts(coords)
        ctx.pair = pair
        ctx.save_for_backward(c, coords)
        return pair.adj(c.contiguous())

    @staticmethod
    def backward(ctx, gf):
        c, coords = ctx.saved_tensors
        pair = ctx.pair
        pair.setpts(coords)
        gf = gf.contiguous()
        gc = pair.fwd(gf) if ctx.needs_input_grad[0] else None
        gx = coord_grad(pair.fwd, gf, c.conj().resolve_conj().contiguous()) if ctx.needs_input_grad[1] else None
        return gc, gx, None


def nufft_forward(f: torch.Tensor, coords: torch.Tensor, pair: NufftPair) -> torch.Tensor:
    """c = A f: [T, N..] -> [T, M] (type 2, sign of the pair), differentiable in f and coords."""
    return _Type2.apply(f, coords, pair)


def nufft_adjoint(c: torch.Tensor, coords: torch.Tensor, pair: NufftPair) -> torch.Tensor:
    """f = A^H c: [T, M] -> [T, N..] (type 1, opposite sign), differentiable in c and coords."""
    return _Type1.apply(c, coords, pair)


class _Normal(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, op):
        ctx.op = op
        return op.apply(x.contiguous())

    @staticmethod
    def backward(ctx, g):
        return ctx.op.apply(g.contiguous()), None


def normal_apply(op, x: torch.Tensor) -> torch.Tensor:
    """B x for a NormalTT1Op, differentiable in x (B is Hermitian, so dL/dx = B dL/dB x)."""
    return _Normal.apply(x, op)
