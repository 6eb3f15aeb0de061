"""Device-memory plumbing for the Python layer (torch tensors as buffers).

The native library takes raw device pointers and a CUDA stream; torch only
provides the allocations and the current stream. Everything fails loudly
when no CUDA device is present: there is no host fallback.
"""

from __future__ import annotations

import numpy as np


def torch():
    import torch as _t

    return _t


def require_cuda(device: int) -> None:
    t = torch()
    if not t.cuda.is_available():
        raise RuntimeError("loki_b200: a CUDA device is required (no CPU fallback)")
    if device < 0 or device >= t.cuda.device_count():
        raise RuntimeError(f"loki_b200: invalid device_id {device}")


def stream_ptr(device: int) -> int:
    return torch().cuda.current_stream(device).cuda_stream


def to_device_f32(x, device: int):
    """A contiguous float32 CUDA tensor on `device` (copies host arrays)."""
    t = torch()
    if isinstance(x, t.Tensor):
        if x.device.type == "cuda" and x.device.index == device and x.dtype == t.float32 and x.is_contiguous():
            return x
        return x.to(device=f"cuda:{device}", dtype=t.float32).contiguous()
    arr = np.ascontiguousarray(x, dtype=np.float32)
    return t.from_numpy(arr).to(device=f"cuda:{device}")


def empty_f32(n: int, device: int):
    t = torch()
    return t.empty(int(n), dtype=t.float32, device=f"cuda:{device}")


def ptr(tensor) -> int:
    return tensor.data_ptr()


def is_device_tensor(x) -> bool:
    try:
        t = torch()
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, t.Tensor) and x.device.type == "cuda"
