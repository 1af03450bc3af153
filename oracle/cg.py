"""Conjugate gradient following cpp/corelib/lib/op/cg.cppm:122-184 (TorchScript step :139-150).

    r = b - A x; p = r; rzold = Re<r,r>; resid = sqrt(rzold)
    for it < max_iter:
        if resid < tol: break
        Ap = A p; alpha = rzold / Re<p,Ap>
        x += alpha p; r -= alpha Ap
        rznew = Re<r,r>; p = r + (rznew / rzold) p; rzold = rznew; resid = sqrt(rzold)

``dtype`` selects the vector precision (complex64 mirrors the device, complex128 is the FP64
reference); inner products are always accumulated in FP64.
"""
from __future__ import annotations

import numpy as np


def _rdot(a, b) -> float:
    return float(np.sum(a.real.astype(np.float64) * b.real + a.imag.astype(np.float64) * b.imag))


def conjugate_gradient(A, b, x0, max_iter: int, tol: float = 1e-6, dtype=np.complex128):
    x = np.array(x0, dtype=dtype)
    b = np.asarray(b, dtype=dtype)
    r = (b - A(x)).astype(dtype)
    p = r.copy()
    rzold = _rdot(r, r)
    resid = np.sqrt(rzold)
    hist = [rzold]
    for _ in range(max_iter):
        if resid < tol:
            break
        Ap = np.asarray(A(p), dtype=dtype)
        alpha = rzold / _rdot(p, Ap)
        if dtype == np.complex64:
            alpha = np.float32(alpha)
        x = (x + alpha * p).astype(dtype)
        r = (r - alpha * Ap).astype(dtype)
        rznew = _rdot(r, r)
        beta = rznew / rzold
        if dtype == np.complex64:
            beta = np.float32(beta)
        p = (r + beta * p).astype(dtype)
        rzold = rznew
        resid = np.sqrt(rzold)
        hist.append(rzold)
    return x, hist
