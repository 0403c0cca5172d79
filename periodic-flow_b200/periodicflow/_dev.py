"""Device-array plumbing for the operator API: torch CUDA tensors in, raw
pointers out.  NumPy inputs are copied to the device and results copied back
into them (the reference's operators mutate their output arguments)."""
from __future__ import annotations

import numpy as np

from . import _native as N


def torch():
    import torch as _t
    if not _t.cuda.is_available():
        raise RuntimeError("periodicflow CUDA backend: no CUDA device is visible")
    return _t


class Arg:
    """One operator argument on the device, with write-back for NumPy inputs."""

    def __init__(self, a, real_dtype, complex_):
        t = torch()
        self.src = a
        self.numpy = isinstance(a, np.ndarray)
        if self.numpy:
            dt = (np.complex128 if real_dtype == t.float64 else np.complex64) if complex_ else (
                np.float64 if real_dtype == t.float64 else np.float32)
            self.t = t.from_numpy(np.ascontiguousarray(a, dtype=dt)).cuda()
        else:
            want = (t.complex128 if real_dtype == t.float64 else t.complex64) if complex_ else real_dtype
            if a.dtype != want or not a.is_cuda or not a.is_contiguous():
                raise TypeError(f"expected a contiguous CUDA tensor of {want}, got {a.dtype}")
            self.t = a

    @property
    def ptr(self):
        return self.t.data_ptr()

    def write_back(self):
        if self.numpy:
            self.src[...] = self.t.cpu().numpy()


def precision_of(a) -> int:
    """PF_FP64 for float64/complex128 data, PF_FP32 for float32/complex64."""
    if isinstance(a, np.ndarray):
        return N.PF_FP64 if a.dtype in (np.float64, np.complex128) else N.PF_FP32
    t = torch()
    return N.PF_FP64 if a.dtype in (t.float64, t.complex128) else N.PF_FP32


def real_dtype(prec: int):
    t = torch()
    return t.float64 if prec == N.PF_FP64 else t.float32


def stream_ptr():
    return torch().cuda.current_stream().cuda_stream
