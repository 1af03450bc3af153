"""Torch tensor plumbing for the C ABI: device pointers, the current stream, checks."""
from __future__ import annotations

import ctypes as C

import torch


def stream_ptr(device: torch.device | None = None) -> C.c_void_p:
    """cudaStream_t of torch's current stream on `device` (so calls are graph-capturable)."""
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(t: torch.Tensor | None) -> C.c_void_p:
    return C.c_void_p(t.data_ptr() if t is not None else None)


def check_tensor(t: torch.Tensor, name: str, dtype: torch.dtype, shape=None, device=None) -> None:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} was not a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name} dtype must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
    if device is not None and t.device != device:
        raise ValueError(f"{name} must be on {device}, got {t.device}")
