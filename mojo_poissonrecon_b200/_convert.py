"""Host-side conversion guards, with the reference's rules and messages.

Reference: python/mojo_poissonrecon/_lib.py:93-145 (f64, i64, addr).  `f64`
and `i64` accept anything array-like (NumPy arrays, lists, CPU or CUDA torch
tensors) and return a C-contiguous NumPy array or, for a torch tensor, a
contiguous torch tensor on the same device.  `addr` is the device-side
counterpart of the reference's buffer guard: it returns the address of a
contiguous CUDA float64/int64 tensor.
"""

from __future__ import annotations

import numpy as np
import torch

_LIMIT = 1 << 53


def _check_numpy_real(source: np.ndarray, target: str) -> None:
    if np.issubdtype(source.dtype, np.complexfloating):
        raise TypeError(f"complex values cannot be converted to {target}")


def f64(values, *, copy: bool = False):
    """Float64 conversion that refuses silent narrowing (_lib.py:93-110)."""
    if isinstance(values, torch.Tensor):
        if values.is_complex():
            raise TypeError("complex values cannot be converted to Float64")
        if values.dtype == torch.bool or not values.is_floating_point():
            if values.dtype != torch.bool and values.numel():
                if bool((values > _LIMIT).any()) or bool((values < -_LIMIT).any()):
                    raise ValueError("integer value cannot be represented exactly as Float64")
        out = values.to(torch.float64)
        out = out.contiguous()
        return out.clone() if copy and out is values else out
    source = np.asarray(values)
    _check_numpy_real(source, "Float64")
    if not (np.issubdtype(source.dtype, np.number) or np.issubdtype(source.dtype, np.bool_)):
        raise TypeError("values must be real numbers")
    if np.issubdtype(source.dtype, np.floating) and source.dtype.itemsize > 8:
        raise TypeError("extended-precision floats cannot be narrowed to Float64")
    if np.issubdtype(source.dtype, np.integer):
        if source.size and (np.any(source > _LIMIT) or np.any(source < -_LIMIT)):
            raise ValueError("integer value cannot be represented exactly as Float64")
    if copy:
        return np.array(values, dtype=np.float64, order="C", copy=True)
    return np.ascontiguousarray(values, dtype=np.float64)


def i64(values, *, copy: bool = False):
    """Int64 conversion that refuses fractions and overflow (_lib.py:113-132)."""
    if isinstance(values, torch.Tensor):
        if values.is_complex():
            raise TypeError("complex values cannot be converted to Int64")
        if values.is_floating_point() and values.numel():
            if not bool(torch.isfinite(values).all()) or bool((values != torch.trunc(values)).any()):
                raise ValueError("Int64 values must be finite integers")
        return values.to(torch.int64).contiguous()
    source = np.asarray(values)
    _check_numpy_real(source, "Int64")
    if np.issubdtype(source.dtype, np.floating):
        if source.size and (not np.isfinite(source).all() or np.any(source != np.trunc(source))):
            raise ValueError("Int64 values must be finite integers")
    elif not (np.issubdtype(source.dtype, np.integer) or np.issubdtype(source.dtype, np.bool_)):
        raise TypeError("values cannot be converted safely to Int64")
    info = np.iinfo(np.int64)
    if source.size and (np.any(source < info.min) or np.any(source > info.max)):
        raise OverflowError("value is outside the Int64 range")
    if copy:
        return np.array(values, dtype=np.int64, order="C", copy=True)
    return np.ascontiguousarray(values, dtype=np.int64)


def addr(values) -> int:
    """Address of a device buffer for the C ABI (_lib.py:135-145 on the GPU)."""
    if not isinstance(values, torch.Tensor):
        raise TypeError("FFI buffers must be CUDA torch tensors")
    if values.dtype not in (torch.float64, torch.int64):
        raise TypeError("FFI buffers must have native Float64 or Int64 dtype")
    if not values.is_cuda:
        raise TypeError("FFI buffers must live on a CUDA device")
    if not values.is_contiguous():
        raise ValueError("FFI buffers must be aligned and C-contiguous")
    address = int(values.data_ptr())
    if address == 0:
        raise ValueError("FFI buffers must have a non-null address")
    return address
