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


def cg_iteration(A, x, r, p, rzold=None):
    """One iteration of the recurrence above (cpp/corelib/lib/op/cg.cppm:139-150) from the state
    (x, r, p) in FP64: returns (x', r', p', rznew)."""
    x = np.asarray(x, dtype=np.complex128)
    r = np.asarray(r, dtype=np.complex128)
    p = np.asarray(p, dtype=np.complex128)
    if rzold is None:
        rzold = _rdot(r, r)
    Ap = np.asarray(A(p), dtype=np.complex128)
    alpha = rzold / _rdot(p, Ap)
    x = x + alpha * p
    r = r - alpha * Ap
    rznew = _rdot(r, r)
    p = r + (rznew / rzold) * p
    return x, r, p, rznew


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


def conjugate_gradient_precond(A, P, b, x0, max_inner_iter: int, max_outer_iter: int, tol: float = 1e-6,
                               should_restart=None, dtype=np.complex128):
    """Preconditioned / restarted CG following cpp/corelib/lib/op/cg.cppm:16-119 (steps :35-56,
    loop :66-111). ``should_restart(x, k)`` gets the iterate and the number of steps taken."""
    x = np.array(x0, dtype=dtype)
    b = np.asarray(b, dtype=dtype)
    r = (b - A(x)).astype(dtype)
    z = np.asarray(P(r), dtype=dtype)
    p = z.copy()
    rzold = _rdot(r, z)
    resid = np.sqrt(rzold)
    k = 0
    for _outer in range(max_outer_iter):
        for _inner in range(max_inner_iter):
            if resid < tol:
                break
            Ap = np.asarray(A(p), dtype=dtype)
            alpha = rzold / _rdot(p, Ap)
            x = (x + alpha * p).astype(dtype)
            r = (r - alpha * Ap).astype(dtype)
            z = np.asarray(P(r), dtype=dtype)
            k += 1
            restart = bool(should_restart(x, k)) if should_restart is not None else False
            rznew = _rdot(r, z)
            p = z.copy() if restart else (z + (rznew / rzold) * p).astype(dtype)
            rzold = rznew
            resid = np.sqrt(rzold)
            if restart:
                break
    return x


def max_eig(A, x0, max_iter: int = 10):
    """Power iteration of cpp/corelib/lib/op/alg.cppm:15-30."""
    x = np.asarray(x0, dtype=np.complex128)
    m = 0.0
    for _ in range(max_iter):
        y = np.asarray(A(x), dtype=np.complex128)
        m = float(np.linalg.norm(y.ravel()))
        x = y / m
    return m, x
