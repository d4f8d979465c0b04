"""Functional entry points over the C ABI on torch CUDA tensors.

Each function takes float32, C-contiguous CUDA tensors (ITK layout, shape
z, y, x), enqueues the kernels on the current torch stream (or ``stream``) and
returns without synchronising.  Errors raise ``RtkbError``.
"""
from __future__ import annotations

import ctypes as C

from ._capi import check, load
from .image import shape_of


def _torch():
    import torch

    return torch


def _ptr(t):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("expected a CUDA tensor (there is no CPU path)")
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise TypeError("expected a contiguous float32 tensor")
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    torch = _torch()
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def _check_shape(t, desc, what):
    if tuple(t.shape) != shape_of(desc):
        raise ValueError(f"{what}: shape {tuple(t.shape)} does not match description {shape_of(desc)}")


def _backproject(fn, geometry, vol_desc, proj_desc, proj, vol_in, out, stream):
    torch = _torch()
    _check_shape(proj, proj_desc, "projections")
    _check_shape(vol_in, vol_desc, "volume")
    if out is None:
        out = torch.empty_like(vol_in)
    _check_shape(out, vol_desc, "output")
    check(fn(geometry.handle, C.byref(vol_desc), C.byref(proj_desc), _ptr(proj), _ptr(vol_in), _ptr(out),
             _stream(stream)))
    return out


def fdk_backproject(geometry, vol_desc, proj_desc, proj, vol_in, out=None, stream=None):
    """rtk::FDKBackProjectionImageFilter: out = vol_in + FDK backprojection."""
    return _backproject(load().rtkb_fdk_backproject, geometry, vol_desc, proj_desc, proj, vol_in, out, stream)


def voxel_backproject(geometry, vol_desc, proj_desc, proj, vol_in, out=None, stream=None):
    """rtk::BackProjectionImageFilter (voxel-based): out = vol_in + backprojection."""
    return _backproject(load().rtkb_voxel_backproject, geometry, vol_desc, proj_desc, proj, vol_in, out, stream)


def device_status(stream=None) -> int:
    """Synchronises the stream and returns (and clears) the kernels' status word."""
    st = C.c_int(0)
    check(load().rtkb_device_status(_stream(stream), C.byref(st)))
    return st.value
