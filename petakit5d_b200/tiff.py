"""TIFF volumes (drop-ins for the reference's io/readtiff.m, io/writetiff.m and getImageSizeMex).

The reference reads and writes every volume of the deconvolution pipeline with its parallel
libtiff MEX files (io/cpp-tiff/src/parallelreadtiff.cpp, parallelwritetiff.cpp).  These functions
call libpkdecon.so's own reader / writer (no libtiff): a MATLAB-ordered [ny nx nz] array is stored as
nz pages of ny rows by nx columns; ``writetiff`` writes BigTIFF with LZW (the reference default) or
no compression; ``readtiff`` decodes strips on all host cores and can place the volume in pinned
(page-locked) memory, so the following host-buffer deconvolution call uploads it at full PCIe rate.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

from ._lib import check, i64x3, lib, ptr

_W = {np.dtype(np.uint8): (8, 0), np.dtype(np.uint16): (16, 0), np.dtype(np.float32): (32, 1),
      np.dtype(np.float64): (64, 1), np.dtype(np.uint32): (32, 0)}


def _dtype(bits, is_float):
    for d, (b, f) in _W.items():
        if b == bits and f == int(bool(is_float)):
            return d
    raise TypeError(f"unsupported TIFF sample type: {bits} bits, float={bool(is_float)}")


def getImageSize(filepath):
    """[ny, nx, nz] of a TIFF file (getImageSizeMex)."""
    d = (C.c_int64 * 3)()
    check(lib.pk_tiff_info(os.fsencode(str(filepath)), d, None, None))
    return tuple(int(v) for v in d)


def pinned_empty(shape, dtype):
    """A Fortran-ordered numpy array in page-locked host memory (freed with the array)."""
    dtype = np.dtype(dtype)
    n = int(np.prod(shape)) * dtype.itemsize
    p = C.c_void_p()
    check(lib.pk_host_alloc(n, C.byref(p)))
    buf = (C.c_char * max(n, 1)).from_address(p.value)
    weakref.finalize(buf, lib.pk_host_free, C.c_void_p(p.value))
    return np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape, order="F")


def readtiff(filepath, range=None, pinned=False, threads=0):
    """data = readtiff(filepath[, range=[z1 z2]]) (io/readtiff.m -> parallelReadTiff).

    A single page comes back 2D, as in MATLAB.  ``pinned=True`` reads into page-locked memory."""
    path = os.fsencode(str(filepath))
    d = (C.c_int64 * 3)()
    bits = C.c_int32()
    isf = C.c_int32()
    check(lib.pk_tiff_info(path, d, C.byref(bits), C.byref(isf)))
    dt = _dtype(bits.value, isf.value)
    ny, nx, nz = (int(v) for v in d)
    rng = None
    if range is not None and len(range):
        if len(range) != 2:
            raise ValueError("Input range is not 2")
        rng = (C.c_int64 * 2)(int(range[0]), int(range[1]))
        nz = int(range[1]) - int(range[0]) + 1
    shape = (ny, nx, max(nz, 0))
    out = pinned_empty(shape, dt) if pinned else np.empty(shape, dt, order="F")
    check(lib.pk_tiff_read(path, rng, ptr(out), out.nbytes, int(threads)))
    return out[:, :, 0] if out.shape[2] == 1 else out


def writetiff(img, filepath, Compression="lzw", threads=0):
    """writetiff(img, filepath, Compression='lzw') (io/writetiff.m -> parallelWriteTiff)."""
    a = np.asarray(img)
    if a.dtype == np.bool_:
        a = a.astype(np.uint8)
    if a.dtype not in _W:
        raise TypeError(f"writetiff: unsupported data type {a.dtype}")
    comp = str(Compression).lower()
    if comp not in ("lzw", "none"):
        raise ValueError("Compression must be 'lzw' or 'none'")
    while a.ndim < 3:
        a = a[..., None]
    a = np.asfortranarray(a)
    bits, isf = _W[a.dtype]
    d = os.path.dirname(os.path.abspath(str(filepath)))
    os.makedirs(d, exist_ok=True)
    check(lib.pk_tiff_write(os.fsencode(str(filepath)), ptr(a), i64x3(a.shape), bits, isf, int(comp == "lzw"),
                            int(threads)))
