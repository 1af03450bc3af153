"""Conjugate gradient: the B200 replacement of ``hasty::conjugate_gradient``
(cpp/corelib/lib/op/cg.cppm:122-184).

The reference fuses the step arithmetic into a TorchScript string and reads ``rzold.item()`` on
the host every iteration. Here the scalars never leave the device: ``hb_cg_step`` computes
Re<p,Ap>, alpha, the x / r updates, Re<r,r>, beta and the direction update in three kernels with
FP64 fixed-order dots, and performs the reference's ``if resid < tol: break`` on the device
(later steps leave x, r, p unchanged). A whole iteration, operator apply included, can therefore
be captured in one CUDA graph and replayed ``max_iter`` times.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional

import torch

from . import _lib
from ._torch import check_tensor, ptr, stream_ptr


class CGState:
    """Device-side CG scalars (rzold, alpha, beta, the break flag, an iteration count)."""

    def __init__(self, device):
        nbytes = _lib.load().hb_cg_state_bytes()
        self.buf = torch.zeros(nbytes, dtype=torch.uint8, device=device)

    def read(self, device=None):
        rz = C.c_double()
        it = C.c_int64()
        conv = C.c_int()
        _lib.call("hb_cg_read_state", ptr(self.buf), C.byref(rz), C.byref(it), C.byref(conv), stream_ptr(device))
        return rz.value, it.value, bool(conv.value)


def cg_init(b: torch.Tensor, Ax: torch.Tensor, r: torch.Tensor, p: torch.Tensor, state: CGState, tol: float) -> None:
    _lib.call("hb_cg_init", b.numel(), ptr(b), ptr(Ax), ptr(r), ptr(p), ptr(state.buf), float(tol), stream_ptr(b.device))


def cg_step(x: torch.Tensor, r: torch.Tensor, p: torch.Tensor, Ap: torch.Tensor, state: CGState) -> None:
    _lib.call("hb_cg_step", x.numel(), ptr(x), ptr(r), ptr(p), ptr(Ap), ptr(state.buf), stream_ptr(x.device))


def vdot_real(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """Re<a, b> accumulated in FP64 (a 0-dim float64 CUDA tensor)."""
    out = torch.empty((), dtype=torch.float64, device=a.device)
    _lib.call("hb_vdot_real", a.numel(), ptr(a), ptr(b), ptr(out), stream_ptr(a.device))
    return out


class CGSolver:
    """Fixed-shape CG driver for an operator ``A(x, out)`` that writes A x into ``out``.

    ``solve(x, b)`` runs ``max_iter`` iterations (fewer take effect once sqrt(rzold) < tol). With
    ``graph=True`` one iteration is captured in a CUDA graph on first use and replayed.
    """

    def __init__(self, A: Callable[[torch.Tensor, torch.Tensor], torch.Tensor], shape, device, max_iter: int = 10,
                 tol: float = 1e-6, graph: bool = False):
        self.A = A
        self.max_iter = int(max_iter)
        self.tol = float(tol)
        self.device = torch.device(device)
        z = lambda: torch.zeros(shape, dtype=torch.complex64, device=self.device)
        self.x, self.r, self.p, self.Ap, self.b = z(), z(), z(), z(), z()
        self.state = CGState(self.device)
        self.use_graph = graph
        self.graph: Optional[torch.cuda.CUDAGraph] = None

    def _iteration(self):
        self.A(self.p, self.Ap)
        cg_step(self.x, self.r, self.p, self.Ap, self.state)

    def _capture(self):
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            # warm-up outside capture (creates FFT tables, loads kernels) on a scratch copy
            saved = [t.clone() for t in (self.x, self.r, self.p, self.Ap)] + [self.state.buf.clone()]
            self._iteration()
            for t, v in zip((self.x, self.r, self.p, self.Ap, self.state.buf), saved):
                t.copy_(v)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._iteration()
        self.graph = g

    def start(self, x0: torch.Tensor, b: torch.Tensor) -> None:
        self.x.copy_(x0)
        self.b.copy_(b)
        self.A(self.x, self.Ap)
        cg_init(self.b, self.Ap, self.r, self.p, self.state, self.tol)

    def run(self, iters: Optional[int] = None) -> torch.Tensor:
        n = self.max_iter if iters is None else int(iters)
        if self.use_graph and self.graph is None:
            self._capture()
        for _ in range(n):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._iteration()
        return self.x

    def solve(self, x0: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        self.start(x0, b)
        return self.run()


def conjugate_gradient(A: Callable[[torch.Tensor], torch.Tensor], max_iter: int = 0, tol: float = 1e-6):
    """conjugate_gradient(A, max_iter, tol) (cg.cppm:122-184): returns ``cgl(x, b) -> x``.

    ``A`` maps an image to an image (e.g. :class:`NormalTT1Op`). ``x`` is updated in place and
    returned, like the reference's lambda.
    """

    def cgl(x: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        check_tensor(x, "x", torch.complex64)
        check_tensor(b, "b", torch.complex64, x.shape, x.device)
        r = torch.empty_like(x)
        p = torch.empty_like(x)
        state = CGState(x.device)
        cg_init(b, A(x), r, p, state, tol)
        for _ in range(max_iter):
            Ap = A(p)
            cg_step(x, r, p, Ap, state)
        return x

    return cgl


class BatchedCGSolver:
    """CG on F independent systems at once (vectors [F, N..], per-frame device scalars and early
    exit): one batched operator apply plus three fused kernels per iteration, optionally captured
    in one CUDA graph and replayed."""

    def __init__(self, A: Callable[[torch.Tensor, torch.Tensor], torch.Tensor], nframes: int, shape, device,
                 max_iter: int = 10, tol: float = 1e-6, graph: bool = False):
        self.A = A
        self.nframes = int(nframes)
        self.shape = (self.nframes, *tuple(shape))
        self.n = int(torch.tensor(shape).prod().item())
        self.max_iter = int(max_iter)
        self.tol = float(tol)
        self.device = torch.device(device)
        z = lambda: torch.zeros(self.shape, dtype=torch.complex64, device=self.device)
        self.x, self.r, self.p, self.Ap, self.b = z(), z(), z(), z(), z()
        nbytes = _lib.load().hb_cgb_state_bytes(self.nframes)
        self.state = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
        self.use_graph = graph
        self.graph: Optional[torch.cuda.CUDAGraph] = None

    def _iteration(self):
        self.A(self.p, self.Ap)
        _lib.call("hb_cgb_step", self.n, self.nframes, ptr(self.x), ptr(self.r), ptr(self.p), ptr(self.Ap),
                  ptr(self.state), stream_ptr(self.device))

    def _capture(self):
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            saved = [t.clone() for t in (self.x, self.r, self.p, self.Ap, self.state)]
            self._iteration()
            for t, v in zip((self.x, self.r, self.p, self.Ap, self.state), saved):
                t.copy_(v)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._iteration()
        self.graph = g

    def start(self, x0: torch.Tensor, b: torch.Tensor) -> None:
        self.x.copy_(x0)
        self.b.copy_(b)
        self.A(self.x, self.Ap)
        _lib.call("hb_cgb_init", self.n, self.nframes, ptr(self.b), ptr(self.Ap), ptr(self.r), ptr(self.p),
                  ptr(self.state), self.tol, stream_ptr(self.device))

    def run(self, iters: Optional[int] = None) -> torch.Tensor:
        n = self.max_iter if iters is None else int(iters)
        if self.use_graph and self.graph is None:
            self._capture()
        for _ in range(n):
            if self.graph is not None:
                self.graph.replay()
            else:
                self._iteration()
        return self.x

    def solve(self, x0: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        self.start(x0, b)
        return self.run()

    def read(self):
        rz = (C.c_double * self.nframes)()
        it = (C.c_int64 * self.nframes)()
        cv = (C.c_int * self.nframes)()
        _lib.call("hb_cgb_read_state", ptr(self.state), self.nframes, rz, it, cv, stream_ptr(self.device))
        return list(rz), list(it), [bool(v) for v in cv]


def conjugate_gradient_precond(A: Callable[[torch.Tensor], torch.Tensor], P: Callable[[torch.Tensor], torch.Tensor],
                               max_inner_iter: int, max_outer_iter: int, tol: float = 1e-6):
    """conjugate_gradient(A, P, max_inner_iter, max_outer_iter, tol) (cpp/corelib/lib/op/cg.cppm:
    16-119): preconditioned CG with restarts. Returns ``cgl(x, b, should_restart_callback=None,
    after_restart_callback=None) -> x`` like the reference's lambda.

    The scalars stay on the device (hb_pcg_*); the reference's ``if resid < tol: break`` is the
    device break flag, so without callbacks no iteration reads anything back. A
    ``should_restart_callback(x) -> bool`` is a host decision per iteration, so with one the
    driver reads the break flag first (one synchronisation per iteration), as the reference
    evaluates ``resid`` before it. ``after_restart_callback(x)`` runs after every outer loop."""

    def cgl(x: torch.Tensor, b: torch.Tensor, should_restart_callback=None, after_restart_callback=None) -> torch.Tensor:
        check_tensor(x, "x", torch.complex64)
        check_tensor(b, "b", torch.complex64, x.shape, x.device)
        dev = x.device
        n = x.numel()
        r = torch.empty_like(x)
        p = torch.empty_like(x)
        state = CGState(dev)
        _lib.call("hb_pcg_residual", n, ptr(b), ptr(A(x)), ptr(r), stream_ptr(dev))
        z = P(r)
        _lib.call("hb_pcg_start", n, ptr(r), ptr(z), ptr(p), ptr(state.buf), float(tol), stream_ptr(dev))
        for _outer in range(int(max_outer_iter)):
            for _inner in range(int(max_inner_iter)):
                if should_restart_callback is not None and state.read(dev)[2]:
                    break
                Ap = A(p)
                _lib.call("hb_pcg_step1", n, ptr(x), ptr(r), ptr(p), ptr(Ap), ptr(state.buf), stream_ptr(dev))
                z = P(r)
                restart = bool(should_restart_callback(x)) if should_restart_callback is not None else False
                _lib.call("hb_pcg_step2", n, ptr(r), ptr(z), ptr(p), ptr(state.buf), 1 if restart else 0,
                          stream_ptr(dev))
                if restart:
                    break
            if after_restart_callback is not None:
                after_restart_callback(x)
        cgl.state = state
        return x

    return cgl
