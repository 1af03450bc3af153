"""Small algorithms on square operators (cpp/corelib/lib/op/alg.cppm)."""
from __future__ import annotations

from typing import Callable, Tuple

import torch

from .cg import vdot_real


def max_eig(A: Callable[[torch.Tensor], torch.Tensor], x0: torch.Tensor, max_iter: int = 10) -> Tuple[float, torch.Tensor]:
    """max_eig (cpp/corelib/lib/op/alg.cppm:15-30): power iteration y = A x, maxeig = ||y||,
    x = y / maxeig, max_iter times. Returns (maxeig, x). The norm is accumulated in FP64 on the
    device; the value is read back once at the end."""
    x = x0
    nrm = None
    for _ in range(int(max_iter)):
        y = A(x)
        nrm = torch.sqrt(vdot_real(y, y))
        x = y / nrm.to(torch.float32)
    return (float(nrm.item()) if nrm is not None else 0.0), x
