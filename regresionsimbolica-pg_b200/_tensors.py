"""Tensor plumbing for the ctypes boundary: pointer extraction, reference-style checks, stream
and workspace handling.  PyTorch is used only for device memory and streams."""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as N


def check_cuda(t: torch.Tensor, name: str) -> None:
    """CHECK_CUDA / CHECK_CONTIGUOUS of the reference (rpn_kernels.cu:10-12)."""
    if not t.is_cuda:
        raise RuntimeError("%s must be a CUDA tensor" % name)
    if not t.is_contiguous():
        raise RuntimeError("%s must be contiguous" % name)


def ptr(t) -> C.c_void_p:
    if t is None:
        return C.c_void_p(0)
    return C.c_void_p(t.data_ptr())


def dtype_code(dt: torch.dtype) -> int:
    if dt == torch.float32:
        return N.WS_F32
    if dt == torch.float64:
        return N.WS_F64
    raise RuntimeError("expected float32 or float64, got %s" % dt)


_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def stream_of(t: torch.Tensor) -> C.c_void_p:
    """The current torch stream on the tensor's device (launches never use the legacy
    default stream unless it is current).  Read as a raw handle when torch offers it (a
    fraction of a microsecond; building a Stream object costs a few, which shows on
    microsecond kernels)."""
    if _raw_stream is not None and t.is_cuda:
        return C.c_void_p(_raw_stream(t.device.index if t.device.index is not None
                                      else torch.cuda.current_device()))
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    """Scratch from torch's caching allocator (stream-ordered, 512-byte aligned)."""
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
