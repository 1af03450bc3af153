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
from .toeplitz import make_workspace, sense_normal, sense_normal_ex, toeplitz_kernel, transform_toeplitz_kernel


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
                 scale: float = 1.0, spread_tuning: Optional[dict] = None):
        self.smaps = smaps.contiguous()
        self.shape = tuple(smaps.shape[1:])
        self.ncoils = smaps.shape[0]
        self.scale = float(scale)
        opts = NufftOpts(nmodes=self.shape, ntransf=self.ncoils, tol=tol, kernel_width=kernel_width)
        self.fwd = NufftPlan(NufftType.TYPE_2, opts)
        self.adj = NufftPlan(NufftType.TYPE_1, opts)
        if spread_tuning is not None:  # an autotune.tune_spread choice for the adjoint's spreading
            from .autotune import apply
            apply(self.adj, spread_tuning)
        self.setpts(coords)

    def setpts(self, coords: Sequence[torch.Tensor]) -> None:
        """Re-points both plans (a new frame's trajectory); the plans keep their buffers."""
        self.fwd.setpts(list(coords))
        self.adj.setpts(list(coords))
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


class BatchedSenseOp:
    """Plain SENSE A / A^H over frames with their own (ragged) trajectories and shared coil maps,
    one frame-batched NUFFT plan pair: every pass of the type 2 and type 1 covers all frames' points
    in one launch (the per-frame plan loop of hasty_python/right_precond_test.py:48-73 and
    simul_op.py:39-91 replaced). Images are [F, N..]; non-uniform data [C, M] with the frames'
    points back to back along M."""

    def __init__(self, frame_coords, smaps: torch.Tensor, kernel_width: int = 0, tol: float = 1e-5,
                 scale: float = 1.0, spread_tuning: Optional[dict] = None):
        self.smaps = smaps.contiguous()
        self.shape = tuple(smaps.shape[1:])
        self.ncoils = smaps.shape[0]
        self.scale = float(scale)
        opts = NufftOpts(nmodes=self.shape, ntransf=self.ncoils, tol=tol, kernel_width=kernel_width)
        self.fwd = NufftPlan(NufftType.TYPE_2, opts)
        self.adj = NufftPlan(NufftType.TYPE_1, opts)
        if spread_tuning is not None:
            from .autotune import apply
            apply(self.adj, spread_tuning)
        self.setpts(frame_coords)

    def setpts(self, frame_coords) -> None:
        self.fwd.setpts_frames(frame_coords)
        self.adj.setpts_frames(frame_coords)
        self.nframes = len(frame_coords)
        self.frame_points = self.fwd.frame_points
        self.M = self.fwd.M

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        y = self.fwd((self.smaps.unsqueeze(0) * x.unsqueeze(1)).contiguous())
        return y * self.scale if self.scale != 1.0 else y

    def adjoint(self, y: torch.Tensor) -> torch.Tensor:
        img = self.adj(y.contiguous())
        out = (self.smaps.conj().unsqueeze(0) * img).sum(1)
        return out * self.scale if self.scale != 1.0 else out

    def normal(self, x: torch.Tensor) -> torch.Tensor:
        return self.adjoint(self.forward(x))


class BatchedNormalOp:
    """Frames with their own Toeplitz kernels and shared coil maps in one apply:
    out[f] = sum_c conj(S_c) T_f(S_c x[f]) for x [F, N..]. Every pass runs all F x C columns in
    one launch (hb_sense_normal_batched); the reference loops NORMAL_T_T1_OP over frames."""

    def __init__(self, kernels: torch.Tensor, stacked_diags: torch.Tensor):
        from . import _lib
        from ._torch import check_tensor, ptr, stream_ptr
        self.nframes = kernels.shape[0]
        self.dim = kernels.dim() - 1
        self.smaps = stacked_diags.contiguous()
        self.shape = tuple(self.smaps.shape[1:])
        self.ncoils = self.smaps.shape[0]
        self.device = self.smaps.device
        if tuple(kernels.shape[1:]) != tuple(2 * s for s in self.shape):
            raise ValueError("kernels must be [F, 2N..] for image shape N")
        check_tensor(kernels, "kernels", torch.complex64, device=self.device)
        self.kernels_t = torch.empty_like(kernels)
        _lib.call("hb_transform_toeplitz_kernels", self.dim, _lib.i64_array(kernels.shape[1:]), self.nframes,
                  ptr(kernels), ptr(self.kernels_t), stream_ptr(self.device))
        self.workspace = make_workspace(self.shape, self.nframes * self.ncoils, self.device)

    def apply(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        from . import _lib
        from ._torch import check_tensor, ptr, stream_ptr
        check_tensor(x, "x", torch.complex64, (self.nframes, *self.shape), self.device)
        if out is None:
            out = torch.empty_like(x)
        ws = self.workspace
        _lib.call("hb_sense_normal_batched", self.dim, _lib.i64_array(self.shape), self.nframes, self.ncoils, ptr(x),
                  ptr(self.smaps), ptr(self.kernels_t), ptr(out), ptr(ws), ws.numel() * ws.element_size(),
                  stream_ptr(self.device))
        return out

    __call__ = apply


def build_toeplitz_kernels(frame_coords, shape, weights=None, kernel_width: int = 0,
                           max_bytes: int = 16 << 30) -> torch.Tensor:
    """Straight kernels [F, 2N..] for frames with their own (ragged) trajectories: frame-batched
    builds (one type-1 NUFFT launch per pass over a group of frames), in groups whose temporary
    grids stay under about ``max_bytes``."""
    from .toeplitz import toeplitz_kernels_frames
    F = len(frame_coords)
    dev = frame_coords[0][0].device
    kshape = tuple(2 * int(s) for s in shape)
    per_frame = 8 * 2 * (2 ** len(shape)) * int(torch.tensor(kshape).prod().item())  # fine grid + pass buffers
    group = max(1, min(F, int(max_bytes) // max(per_frame, 1)))
    out = torch.empty((F, *kshape), dtype=torch.complex64, device=dev)
    for f0 in range(0, F, group):
        f1 = min(F, f0 + group)
        w = None if weights is None else [weights[f] for f in range(f0, f1)]
        toeplitz_kernels_frames([frame_coords[f] for f in range(f0, f1)], out[f0:f1], w, kernel_width=kernel_width)
    return out


class NormalTT2Op:
    """NORMAL_T_T2_OP (cpp/corelib/lib/mri/normal.cppm:111-160): the normal operator in the coil
    maps, (B Psi)_i = conj(x) T (x Psi_i), i.e. the fused multiplication with the reference's flags
    (input mult1 = x MULT, output mult1 = x MULT_CONJ)."""

    class_name = "NORMAL_T_T2_OP"

    def __init__(self, kernel: torch.Tensor, x: torch.Tensor, transformed: bool = False):
        from .toeplitz import transform_toeplitz_kernel
        self.kernel_t = kernel if transformed else transform_toeplitz_kernel(kernel)
        self.x = x.contiguous()
        self.shape = tuple(self.x.shape)
        self._ws = {}

    def apply(self, stacked_diags: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        from .toeplitz import ToeplitzAccumulateType as A, ToeplitzMultType as T, toeplitz_multiplication
        B = stacked_diags.shape[0]
        if B not in self._ws:
            self._ws[B] = make_workspace(self.shape, B, self.x.device)
        if out is None:
            out = torch.empty_like(stacked_diags)
        return toeplitz_multiplication(stacked_diags.contiguous(), out, self.kernel_t, self._ws[B], self.x, None,
                                       T.NONE, T.MULT, T.MULT_CONJ, T.NONE, T.NONE, A.NONE)

    __call__ = apply


class SenseOffresOp:
    """Time-segmented off-resonance SENSE pair, sense_forward_offresonance /
    sense_adjoint_offresonance (cpp/corelib/lib/mri/forward.cppm:35-165, adjoint.cppm:32-171):

        forward:  y_c = sum_l b_l * NUFFT2(c_l * S_c * x)
        adjoint:  x   = sum_c conj(S_c) sum_l conj(c_l) * NUFFT1(conj(b_l) * y_c)

    with b [L, M] per-sample temporal interpolators and c [L, N..] spatial phase maps (L = 1, b = c
    = 1 is plain SENSE). All C x L transforms run as one batched NUFFT instead of the reference's
    per-coil host tasks (and without its double conj(S) in the adjoint, adjoint.cppm:116-117)."""

    def __init__(self, coords: Sequence[torch.Tensor], smaps: torch.Tensor, b: torch.Tensor, c: torch.Tensor,
                 kernel_width: int = 0, tol: float = 1e-5):
        self.smaps = smaps.contiguous()
        self.C = smaps.shape[0]
        self.shape = tuple(smaps.shape[1:])
        self.b = b.to(torch.complex64).contiguous()
        self.c = c.to(torch.complex64).contiguous()
        self.L = self.b.shape[0]
        opts = NufftOpts(nmodes=self.shape, ntransf=self.C * self.L, tol=tol, kernel_width=kernel_width)
        self.fwd = NufftPlan(NufftType.TYPE_2, opts)
        self.adj = NufftPlan(NufftType.TYPE_1, opts)
        self.fwd.setpts(list(coords))
        self.adj.setpts(list(coords))
        self.M = coords[0].shape[0]

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        img = (self.smaps[:, None] * self.c[None] * x[None, None]).reshape(self.C * self.L, *self.shape)
        y = self.fwd(img.contiguous()).reshape(self.C, self.L, self.M)
        return (y * self.b[None]).sum(1)

    def adjoint(self, y: torch.Tensor) -> torch.Tensor:
        z = (y[:, None] * self.b.conj()[None]).reshape(self.C * self.L, self.M)
        img = self.adj(z.contiguous()).reshape(self.C, self.L, *self.shape)
        return (self.smaps.conj() * (img * self.c.conj()[None]).sum(1)).sum(0)

    def normal(self, x: torch.Tensor) -> torch.Tensor:
        return self.adjoint(self.forward(x))


def _transform_all(kernels: torch.Tensor, transformed: bool) -> torch.Tensor:
    if transformed:
        return kernels.contiguous()
    return torch.stack([transform_toeplitz_kernel(k.contiguous()) for k in kernels])


class NormalIDTT1Op:
    """NORMAL_IDT_T1_OP (cpp/corelib/lib/mri/normal.cppm:185-270): time-segmented SENSE normal
    operator B x = sum_l R_l^H [sum_s Psi_s^H F^H T_l F Psi_s] R_l x, from L (kernel T_l,
    diagonal R_l) pairs and the stacked coil maps Psi. Each segment is one fused apply (coil
    expand, padded convolution, coil reduce, conj(R_l), accumulate into the output); the
    reference's [C, N..] per-coil intermediate and its separate sum over coils do not exist here."""

    class_name = "NORMAL_IDT_T1_OP"

    def __init__(self, kernels: torch.Tensor, kerneldiags: torch.Tensor, stacked_diags: torch.Tensor,
                 transformed: bool = False):
        if kernels.shape[0] != kerneldiags.shape[0]:
            raise RuntimeError("Number of kernels and kernel diagonals must match.")
        self.kernels_t = _transform_all(kernels, transformed)
        self.kerneldiags = kerneldiags.contiguous()
        self.smaps = stacked_diags.contiguous()
        self.smaps_out: Optional[torch.Tensor] = None
        self.shape = tuple(self.smaps.shape[1:])
        self.dim = len(self.shape)
        if tuple(self.kerneldiags.shape[1:]) != self.shape:
            raise ValueError("kernel diagonals must have the image shape")
        self.workspace = make_workspace(self.shape, self.smaps.shape[0], self.smaps.device)

    def apply(self, x: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        if out is None:
            out = torch.empty_like(x)
        for l in range(self.kernels_t.shape[0]):
            sense_normal_ex(x, self.smaps, self.kernels_t[l], out, self.smaps_out, self.kerneldiags[l],
                            accumulate=l > 0, scratch=self.workspace)
        return out

    __call__ = apply


class NormalIDTWT1Op(NormalIDTT1Op):
    """NORMAL_IDTW_T1_OP (cpp/corelib/lib/mri/normal.cppm:405-580): B = sum_{i,j} W_ij Psi_i^H
    [sum_l R_l^H F^H T_l F R_l] Psi_j with W the inverse noise covariance. The reference forms the
    per-coil results, mixes them with torch.mm(W, .) and reduces with conj(Psi). Since
    sum_i conj(Psi_i) sum_j W_ij v_j = sum_j conj(U_j) v_j with U = W^H Psi, the mixing is folded
    once into output coil maps U and every segment stays one fused apply."""

    class_name = "NORMAL_IDTW_T1_OP"

    def __init__(self, kernels: torch.Tensor, kerneldiags: torch.Tensor, stacked_diags: torch.Tensor,
                 weights: torch.Tensor, transformed: bool = False):
        super().__init__(kernels, kerneldiags, stacked_diags, transformed)
        C = self.smaps.shape[0]
        if tuple(weights.shape) != (C, C):
            raise ValueError("weights must be [C, C]")
        self.weights = weights.contiguous()
        self.smaps_out = torch.mm(self.weights.conj().t().contiguous(), self.smaps.reshape(C, -1)).reshape(self.smaps.shape)


class NormalIDTT2Op:
    """NORMAL_IDT_T2_OP (cpp/corelib/lib/mri/normal.cppm:292-372): the time-segmented operator in
    the coil maps, (B Psi)_i = X^H [sum_l R_l^H F^H T_l F R_l] X Psi_i: for each segment one
    batched multiplication with the reference's flags (input x and R_l, output conj(x) and
    conj(R_l)), accumulated over segments."""

    class_name = "NORMAL_IDT_T2_OP"

    def __init__(self, kernels: torch.Tensor, kerneldiags: torch.Tensor, x: torch.Tensor, transformed: bool = False):
        if kernels.shape[0] != kerneldiags.shape[0]:
            raise RuntimeError("Number of kernels and kernel diagonals must match.")
        self.kernels_t = _transform_all(kernels, transformed)
        self.kerneldiags = kerneldiags.contiguous()
        self.x = x.contiguous()
        self.shape = tuple(self.x.shape)
        self._ws = {}

    def _segments(self, stacked_diags: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        from .toeplitz import ToeplitzAccumulateType as A, ToeplitzMultType as T, toeplitz_multiplication
        B = stacked_diags.shape[0]
        if B not in self._ws:
            self._ws[B] = make_workspace(self.shape, B, self.x.device)
        sd = stacked_diags.contiguous()
        for l in range(self.kernels_t.shape[0]):
            toeplitz_multiplication(sd, out, self.kernels_t[l], self._ws[B], self.x, self.kerneldiags[l], T.NONE,
                                    T.MULT, T.MULT_CONJ, T.MULT, T.MULT_CONJ, A.ACCUMULATE if l > 0 else A.NONE)
        return out

    def apply(self, stacked_diags: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        if out is None:
            out = torch.empty_like(stacked_diags)
        return self._segments(stacked_diags, out)

    __call__ = apply


class NormalIDTWT2Op(NormalIDTT2Op):
    """NORMAL_IDTW_T2_OP (cpp/corelib/lib/mri/normal.cppm:586-720): NORMAL_IDT_T2_OP followed by
    the coil mixing stack_out = W @ stack_out (one complex GEMM over [C, prod N])."""

    class_name = "NORMAL_IDTW_T2_OP"

    def __init__(self, kernels: torch.Tensor, kerneldiags: torch.Tensor, x: torch.Tensor, weights: torch.Tensor,
                 transformed: bool = False):
        super().__init__(kernels, kerneldiags, x, transformed)
        self.weights = weights.contiguous()

    def apply(self, stacked_diags: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        C = stacked_diags.shape[0]
        tmp = self._segments(stacked_diags, torch.empty_like(stacked_diags))
        mixed = torch.mm(self.weights, tmp.reshape(C, -1)).reshape(stacked_diags.shape)
        if out is None:
            return mixed
        out.copy_(mixed)
        return out

    __call__ = apply
