"""Device plumbing: one library context per CUDA device, tensor conversion, stream handles.

PyTorch holds the device memory and the stream; the arithmetic is done by libnebula_b200.so.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

_contexts: dict[int, int] = {}


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("the CUDA SPH path needs a CUDA device (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def ctx(device: torch.device | None = None) -> int:
    dev = require_cuda() if device is None else device
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    c = _contexts.get(idx)
    if c is None:
        torch.cuda.init()
        c = _lib.lib().nb_create(idx)
        if not c:
            raise _lib.NebulaCudaError(f"nb_create failed on cuda:{idx}")
        _contexts[idx] = c
    return c


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def dev_f64(a, shape=None) -> torch.Tensor:
    """A contiguous float64 CUDA tensor (copied from NumPy or another device when needed)."""
    d = require_cuda()
    if isinstance(a, torch.Tensor):
        t = a.to(device=d, dtype=torch.float64)
    else:
        t = torch.as_tensor(np.asarray(a, dtype=np.float64), device=d)
    if shape is not None:
        t = t.expand(shape)
    return t.contiguous()


def dev_i64(a) -> torch.Tensor:
    d = require_cuda()
    if isinstance(a, torch.Tensor):
        return a.to(device=d, dtype=torch.int64).contiguous()
    return torch.as_tensor(np.asarray(a, dtype=np.int64), device=d).contiguous()


def ptr(t: torch.Tensor | None):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def to_numpy(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)
