"""Combined deskew / rotate after deconvolution (drop-in for the reference's MATLAB function).

``deskewRotateFrame3D(vol, angle, dz, xyPixelSize, reverse=..., Crop=..., bbox=..., objectiveScan=...,
xStepThresh=..., resampleFactor=..., gpuProcess=..., save16bit=..., interpMethod=...)`` mirrors
microscopeDataProcessing/deskew_rotate/deskewRotateFrame3D.m:1-260 on its default path (linear
interpolation, no resampling), which RLdecon.m:487-491 takes for deconvolved frames; the work runs
on the GPU through libpkdecon.so.  ``deskew_rotate_device`` takes and returns device buffers, so a
volume deconvolved with ``decon.decon_device`` is deskewed without leaving the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, i64x3, lib, ptr

_DT = {np.dtype(np.uint16): 0, np.dtype(np.float32): 1}


def _bbox(bbox):
    if bbox is None or len(bbox) == 0:
        return None
    if len(bbox) != 6:
        raise ValueError("bbox must have 6 elements [y1 x1 z1 y2 x2 z2]")
    return (C.c_int64 * 6)(*[int(v) for v in bbox])


def deskewRotateFrame3D(vol, angle, dz, xyPixelSize, reverse=False, Crop=True, bbox=None, objectiveScan=False,
                        xStepThresh=2.0, resampleFactor=None, gpuProcess=False, save16bit=False,
                        interpMethod="linear", ctx=None):
    """volout = deskewRotateFrame3D(vol, angle, dz, xyPixelSize, ...) (uint16 or single input)."""
    if resampleFactor is not None and len(resampleFactor) and np.any(np.asarray(resampleFactor) != 1):
        raise NotImplementedError("resampleFactor: the reference's imwarp path is not built")
    if str(interpMethod).lower() != "linear":
        raise NotImplementedError("interpMethod 'cubic': the reference's imwarp path is not built")
    ctx = ctx or _lib.default_context()
    a = np.asarray(vol)
    if a.dtype not in _DT:
        a = a.astype(np.float32)
    while a.ndim < 3:
        a = a[..., None]
    a = np.asfortranarray(a)
    od = (C.c_int64 * 3)()
    bb = _bbox(bbox)
    args = (ctx.handle, ptr(a), _DT[a.dtype], i64x3(a.shape), float(angle), float(dz), float(xyPixelSize),
            int(bool(reverse)), int(bool(objectiveScan)), float(xStepThresh), bb, int(bool(save16bit)))
    check(lib.pk_deskew_rotate(*args, None, od))
    u16 = bool(save16bit) and a.dtype == np.uint16
    out = np.empty(tuple(int(v) for v in od), np.uint16 if u16 else np.float32, order="F")
    check(lib.pk_deskew_rotate(*args, ptr(out), od))
    return out


def deskew_rotate_device(d_in, in_dtype, dims, angle, dz, xyPixelSize, d_out=None, reverse=False, bbox=None,
                         objectiveScan=False, xStepThresh=2.0, save16bit=False, ctx=None, stream=None):
    """Device-buffer variant (``d_in`` / ``d_out``: torch CUDA tensors or device pointers).  With
    ``d_out=None`` only the output size is returned."""
    ctx = ctx or _lib.default_context()
    od = (C.c_int64 * 3)()
    t = _DT[np.dtype(str(in_dtype).replace("torch.", ""))]
    check(lib.pk_deskew_rotate_device(ctx.handle, ptr(d_in), t, i64x3(dims), float(angle), float(dz),
                                      float(xyPixelSize), int(bool(reverse)), int(bool(objectiveScan)),
                                      float(xStepThresh), _bbox(bbox), int(bool(save16bit)), ptr(d_out), od,
                                      ptr(stream)))
    return tuple(int(v) for v in od)
