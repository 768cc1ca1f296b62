"""Array plumbing between the reference-style API and device memory.

The reference's operators take and return float64 memoryviews on the host.
janus_b200 accepts the same numpy arrays (copied to the GPU, the result
copied back into the caller's array or a new one) and also CUDA torch
tensors, which are used in place with no host round trip.  PyTorch is only
the device-memory and stream plumbing here; all arithmetic runs in the
native library.
"""
from __future__ import annotations

import numpy as np
import torch

FLOAT_DTYPES = {
    "float64": torch.float64, "f64": torch.float64, np.float64: torch.float64,
    torch.float64: torch.float64,
    "float32": torch.float32, "f32": torch.float32, np.float32: torch.float32,
    torch.float32: torch.float32,
}


def torch_dtype(dtype) -> torch.dtype:
    if dtype is None:
        return torch.float64
    if isinstance(dtype, np.dtype):
        dtype = dtype.type
    try:
        return FLOAT_DTYPES[dtype]
    except (KeyError, TypeError):
        raise ValueError(f"unsupported dtype {dtype!r} (float64 or float32)")


def jb_dtype(dtype: torch.dtype) -> int:
    return 0 if dtype == torch.float64 else 1


def is_tensor(a) -> bool:
    return isinstance(a, torch.Tensor)


def shape_of(a):
    if a is None:
        return None
    return tuple(int(s) for s in a.shape)


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def device():
    if not torch.cuda.is_available():
        raise RuntimeError("janus_b200 needs a CUDA device (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def to_device(a, dtype: torch.dtype) -> torch.Tensor:
    """Contiguous CUDA tensor of `dtype` holding a's values."""
    if is_tensor(a):
        t = a
        if t.device.type != "cuda":
            t = t.to(device())
        if t.dtype != dtype:
            t = t.to(dtype)
        return t.contiguous()
    arr = np.ascontiguousarray(np.asarray(a), dtype=np.float64 if dtype == torch.float64
                               else np.float32)
    return torch.from_numpy(arr).to(device(), non_blocking=False)


def as_numpy_float64(a) -> np.ndarray:
    return np.asarray(a, dtype=np.float64)


class Output:
    """Destination of an operator: the caller's array/tensor, or a new one.

    ``target`` is the device tensor the kernel writes to; ``finish()``
    returns what the reference's API returns (for a host output, a view
    whose ``.base`` is the caller's array).
    """

    def __init__(self, out, shape, dtype, like):
        self.user = out
        self.host = not is_tensor(like) if out is None else not is_tensor(out)
        if out is None:
            self.target = torch.empty(shape, dtype=dtype, device=device())
        elif is_tensor(out):
            if (out.device.type == "cuda" and out.dtype == dtype and out.is_contiguous()):
                self.target = out
            else:
                self.target = torch.empty(shape, dtype=dtype, device=device())
        else:
            self.target = torch.empty(shape, dtype=dtype, device=device())

    def finish(self):
        t = self.target
        if self.user is None:
            if self.host:
                return t.cpu().numpy().astype(np.float64, copy=False)
            return t
        if is_tensor(self.user):
            if t is not self.user:
                self.user.copy_(t)
            return self.user
        self.user[...] = t.cpu().numpy()
        return self.user[...]
