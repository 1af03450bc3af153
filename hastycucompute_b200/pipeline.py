"""Host-to-host application of an operator with the PCIe copies hidden behind the applies.

A serving loop hands images in host memory and wants results in host memory. Applied one item
at a time, every apply waits for its input copy and the next item waits for the result copy.
``HostPipeline`` keeps two device input/output buffer pairs and three streams: item i+1's
host-to-device copy and item i-1's device-to-host copy (one copy engine each) run while item i is
applied on the caller's stream, so a run of K items costs about max(apply, copy) per item instead
of apply + copies. Every item is still copied in and out; host buffers must be pinned for the
copies to be asynchronous.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import torch


class HostPipeline:
    """``run(host_in, host_out)`` applies ``op(x_dev, out_dev)`` to each ``host_in[i]`` into
    ``host_out[i]``. ``op`` has the operator signature ``apply(x, out)``. Shapes and dtypes of the
    inputs / outputs are fixed at construction."""

    def __init__(self, op: Callable[[torch.Tensor, torch.Tensor], torch.Tensor], in_shape, device,
                 out_shape=None, dtype=torch.complex64):
        self.op = op
        self.device = torch.device(device)
        out_shape = in_shape if out_shape is None else out_shape
        self.xin = [torch.empty(in_shape, dtype=dtype, device=self.device) for _ in range(2)]
        self.xout = [torch.empty(out_shape, dtype=dtype, device=self.device) for _ in range(2)]
        self.h2d = torch.cuda.Stream(self.device)
        self.d2h = torch.cuda.Stream(self.device)

    def run(self, host_in: Sequence[torch.Tensor], host_out: Sequence[torch.Tensor],
            compute: Optional[torch.cuda.Stream] = None) -> None:
        if len(host_in) != len(host_out):
            raise ValueError("host_in and host_out must have the same length")
        comp = compute if compute is not None else torch.cuda.current_stream(self.device)
        start = torch.cuda.Event()
        start.record(comp)
        self.h2d.wait_event(start)
        self.d2h.wait_event(start)
        in_ready = [torch.cuda.Event(), torch.cuda.Event()]
        applied = [torch.cuda.Event(), torch.cuda.Event()]
        copied_out = [torch.cuda.Event(), torch.cuda.Event()]
        used = [False, False]
        for i, (hi, ho) in enumerate(zip(host_in, host_out)):
            b = i & 1
            with torch.cuda.stream(self.h2d):
                if used[b]:
                    self.h2d.wait_event(applied[b])  # the apply of item i-2 has read xin[b]
                self.xin[b].copy_(hi, non_blocking=True)
                in_ready[b].record(self.h2d)
            with torch.cuda.stream(comp):
                comp.wait_event(in_ready[b])
                if used[b]:
                    comp.wait_event(copied_out[b])  # item i-2's result has left xout[b]
                self.op(self.xin[b], self.xout[b])
                applied[b].record(comp)
            with torch.cuda.stream(self.d2h):
                self.d2h.wait_event(applied[b])
                ho.copy_(self.xout[b], non_blocking=True)
                copied_out[b].record(self.d2h)
            used[b] = True
        # the caller's stream sees every result copy before anything it enqueues next
        for b in range(2):
            if used[b]:
                comp.wait_event(copied_out[b])
