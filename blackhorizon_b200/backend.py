"""Array backend dispatch with the ``b200`` backend added.

Mirrors blackhorizon/backend.py:24-59 (``gpu_available``, ``get_xp``,
``xp_of``, ``to_numpy``) and adds ``'b200'``: arrays are PyTorch CUDA tensors
and every physics call goes through libbh_b200.so.  ``get_xp('b200')`` returns
a small array namespace (``asarray``, ``full``, ``zeros``, ``empty``, dtypes)
so callers written against ``xp`` keep working.
"""

from __future__ import annotations

from typing import Any

import numpy

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None

Array = Any


def b200_available() -> bool:
    """True when a CUDA device is visible and libbh_b200.so loads."""
    if torch is None or not torch.cuda.is_available():
        return False
    from . import _lib

    try:
        _lib.load()
    except (OSError, RuntimeError):
        return False
    return True


def gpu_available() -> bool:
    """The reference's 'gpu' (CuPy) backend is not part of this package; the
    b200 backend replaces it."""
    return b200_available()


class _B200Namespace:
    """The ``xp`` of the b200 backend: NumPy-style constructors that return
    float64/int CUDA tensors on the current device."""

    float64 = torch.float64 if torch is not None else None
    float32 = torch.float32 if torch is not None else None
    int32 = torch.int32 if torch is not None else None
    int64 = torch.int64 if torch is not None else None

    @staticmethod
    def _device():
        return torch.device("cuda", torch.cuda.current_device())

    def asarray(self, a, dtype=None):
        if isinstance(a, numpy.ndarray) and dtype is None:
            dtype = {numpy.dtype("float64"): torch.float64,
                     numpy.dtype("float32"): torch.float32,
                     numpy.dtype("int32"): torch.int32,
                     numpy.dtype("int64"): torch.int64}.get(a.dtype, None)
        return torch.as_tensor(a, dtype=dtype, device=self._device())

    def full(self, shape, value, dtype=None):
        return torch.full(shape if isinstance(shape, tuple) else (shape,), value,
                          dtype=dtype or torch.float64, device=self._device())

    def zeros(self, shape, dtype=None):
        return torch.zeros(shape, dtype=dtype or torch.float64, device=self._device())

    def empty(self, shape, dtype=None):
        return torch.empty(shape, dtype=dtype or torch.float64, device=self._device())


_B200 = _B200Namespace()


def get_xp(backend: str):
    """Return the array module for 'cpu' (numpy) or 'b200'.

    Errors follow blackhorizon/backend.py:34-45: RuntimeError when the device
    is unavailable, ValueError for an unknown name."""
    if backend == "cpu":
        return numpy
    if backend in ("b200", "gpu"):
        if not b200_available():
            raise RuntimeError(
                "b200 backend requested but no CUDA device is visible or "
                "libbh_b200.so is not built (python -m blackhorizon_b200.build)"
            )
        return _B200
    raise ValueError(f"Unknown backend {backend!r}, expected 'cpu' or 'b200'.")


def is_device_array(array: Array) -> bool:
    return torch is not None and isinstance(array, torch.Tensor)


def xp_of(array: Array):
    """The array module owning `array` (blackhorizon/backend.py:48-52)."""
    if is_device_array(array):
        return _B200
    return numpy


def to_numpy(array: Array) -> numpy.ndarray:
    """Copy an array to host memory as a NumPy ndarray."""
    if is_device_array(array):
        return array.detach().cpu().numpy()
    return numpy.asarray(array)


# --------------------------------------------------------------- helpers
def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def to_device_f64(a, name: str = "array"):
    """(tensor, host_dtype): a contiguous float64 CUDA tensor for `a` and the
    NumPy dtype to return results in when `a` came from the host (else None)."""
    if is_device_array(a):
        if not a.is_cuda:
            t = a.to(device=_B200._device(), dtype=torch.float64)
            return t.contiguous(), None
        if a.dtype != torch.float64:
            return a.to(torch.float64).contiguous(), None
        return a.contiguous(), None
    arr = numpy.asarray(a)
    if arr.dtype.kind not in "fiu":
        raise TypeError(f"{name} must be a numeric array")
    t = torch.as_tensor(numpy.ascontiguousarray(arr, dtype=numpy.float64),
                        device=_B200._device())
    return t, arr.dtype


def out_like(t, host_dtype, src=None):
    """Return device tensor `t` as the caller's array type: NumPy with the
    input's float dtype when the input was NumPy; a device tensor with the
    input's float dtype otherwise."""
    if host_dtype is not None:
        out = t.cpu().numpy()
        if host_dtype.kind == "f" and out.dtype.kind == "f" and host_dtype != out.dtype:
            out = out.astype(host_dtype)
        return out
    if src is not None and is_device_array(src) and src.dtype.is_floating_point \
            and t.dtype.is_floating_point and src.dtype != t.dtype:
        return t.to(src.dtype)
    return t


def ptr(t) -> int:
    return 0 if t is None else t.data_ptr()
