"""Unrolled, differentiable Toeplitz SENSE-CG with per-iteration recomputation.

Each iteration k solves toward (B + lam_k I) x = b with the CG recurrence of
cpp/corelib/lib/op/cg.cppm:139-150 and a learnable step s_k that scales alpha:

    Ap = B p + lam_k p;  alpha = rzold / Re<p, Ap>
    x += s_k alpha p;    r -= s_k alpha Ap;  rznew = Re<r, r>;  p = r + (rznew / rzold) p

B is a (batched) Toeplitz SENSE normal operator, Hermitian, so its backward is one more apply.
With ``checkpoint=True`` every iteration runs under torch.utils.checkpoint: the forward keeps
only each iteration's inputs (x, r, p, rzold) and the backward recomputes the iteration, so
activation memory stays O(1) iterations instead of O(K).
"""
from __future__ import annotations

from typing import Optional

import torch
from torch.utils.checkpoint import checkpoint

from .autograd import normal_apply


def _rdot(a: torch.Tensor, b: torch.Tensor, frames: bool) -> torch.Tensor:
    """Re<a,b> in float64, per frame when `frames` (leading dim) else total."""
    v = (a.real.double() * b.real.double() + a.imag.double() * b.imag.double())
    if frames:
        return v.reshape(v.shape[0], -1).sum(1)
    return v.sum()


class UnrolledCG(torch.nn.Module):
    """K unrolled CG iterations with learnable float32 steps and regularisation weights.

    ``op`` is a NormalTT1Op (one volume) or BatchedNormalOp (volumes along dim 0)."""

    def __init__(self, op, iterations: int = 10, step_init: float = 1.0, lam_init: float = 0.0,
                 checkpoint: bool = True):
        super().__init__()
        self.op = op
        self.iterations = int(iterations)
        self.frames = hasattr(op, "nframes")
        self.steps = torch.nn.Parameter(torch.full((self.iterations,), float(step_init), dtype=torch.float32))
        self.lams = torch.nn.Parameter(torch.full((self.iterations,), float(lam_init), dtype=torch.float32))
        self.use_checkpoint = bool(checkpoint)

    def _bshape(self, v: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
        return v.reshape((-1,) + (1,) * (x.dim() - 1)) if self.frames else v

    def _iteration(self, x, r, p, rzold, step, lam):
        Ap = normal_apply(self.op, p) + lam.to(p.dtype) * p
        alpha = rzold / _rdot(p, Ap, self.frames)
        a = (step.double() * alpha).float()
        a = self._bshape(a, x).to(x.dtype)
        x = x + a * p
        r = r - a * Ap
        rznew = _rdot(r, r, self.frames)
        beta = self._bshape((rznew / rzold).float(), x).to(x.dtype)
        p = r + beta * p
        return x, r, p, rznew

    def forward(self, b: torch.Tensor, x0: Optional[torch.Tensor] = None) -> torch.Tensor:
        x = torch.zeros_like(b) if x0 is None else x0
        r = b - (normal_apply(self.op, x) + self.lams[0].to(b.dtype) * x)
        p = r
        rzold = _rdot(r, r, self.frames)
        for k in range(self.iterations):
            if self.use_checkpoint and torch.is_grad_enabled():
                x, r, p, rzold = checkpoint(self._iteration, x, r, p, rzold, self.steps[k], self.lams[k],
                                            use_reentrant=False)
            else:
                x, r, p, rzold = self._iteration(x, r, p, rzold, self.steps[k], self.lams[k])
        return x
