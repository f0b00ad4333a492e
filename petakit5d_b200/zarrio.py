"""Zarr v2 volumes (drop-ins for the reference's io/readzarr.m and io/writezarr.m).

The reference reads and writes Zarr through its cpp-zarr MEX files (io/cpp-zarr/src/
parallelreadzarr.cpp, parallelwritezarr.cpp).  These functions call libpkdecon.so's own reader /
writer: a MATLAB-ordered [ny nx nz] array is the Zarr array of that shape, chunks are decoded and
encoded on all host cores, and a region read (``inputBbox``) touches only the chunks that meet it.
Compressors: none, zlib, gzip and blosc (the reference's default: cname lz4, clevel 5, byte shuffle;
lz4, zstd or zlib inside).  ``compressor="blosc"`` writes blosc-lz4; "blosc-zstd" and "blosc-zlib"
choose the codec inside.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil

import numpy as np

from ._lib import check, i64x3, lib, ptr
from .tiff import pinned_empty

_W = {np.dtype(np.uint8): (8, 0), np.dtype(np.uint16): (16, 0), np.dtype(np.uint32): (32, 0),
      np.dtype(np.float32): (32, 1), np.dtype(np.float64): (64, 1)}
_COMP = {"none": 0, None: 0, "zlib": 1, "gzip": 2, "blosc": 3, "blosc-lz4": 3, "blosc-zstd": 4, "blosc-zlib": 5}
_BLOSC = {3: "lz4", 4: "zstd", 5: "zlib"}


def _dtype(bits, is_float):
    for d, (b, f) in _W.items():
        if b == bits and f == int(bool(is_float)):
            return d
    raise TypeError(f"unsupported Zarr dtype: {bits} bits, float={bool(is_float)}")


def getZarrInfo(filepath):
    """(shape, chunks, dtype) of a Zarr array."""
    d, c = (C.c_int64 * 3)(), (C.c_int64 * 3)()
    bits, isf = C.c_int32(), C.c_int32()
    check(lib.pk_zarr_info(os.fsencode(str(filepath)), d, c, C.byref(bits), C.byref(isf)))
    return tuple(int(v) for v in d), tuple(int(v) for v in c), _dtype(bits.value, isf.value)


def readzarr(filepath, inputBbox=None, pinned=False, threads=0):
    """data = readzarr(filepath, 'inputBbox', [y1 x1 z1 y2 x2 z2]) (io/readzarr.m)."""
    shape, _, dt = getZarrInfo(filepath)
    bb = None
    if inputBbox is not None and len(inputBbox):
        if len(inputBbox) != 6:
            raise ValueError("inputBbox must have 6 elements")
        bb = (C.c_int64 * 6)(*[int(v) for v in inputBbox])
        shape = tuple(int(inputBbox[k + 3]) - int(inputBbox[k]) + 1 for k in range(3))
    out = pinned_empty(shape, dt) if pinned else np.empty(shape, dt, order="F")
    check(lib.pk_zarr_read(os.fsencode(str(filepath)), bb, ptr(out), out.nbytes, int(threads)))
    return out


def writezarr(data, filepath, blockSize=(500, 500, 500), compressor="zlib", overwrite=False, threads=0,
              dimSeparator="."):
    """writezarr(data, filepath, 'blockSize', [...], 'dimSeparator', ...) (io/writezarr.m): order F;
    chunk keys joined by '.' (the default) or '/' (nested folders)."""
    if dimSeparator not in (".", "/"):
        raise ValueError("dimSeparator must be '.' or '/'")
    a = np.asarray(data)
    if a.dtype == np.bool_:
        a = a.astype(np.uint8)
    if a.dtype not in _W:
        raise TypeError(f"writezarr: unsupported data type {a.dtype}")
    while a.ndim < 3:                       # expand2dDim (the reference default)
        a = a[..., None]
    a = np.asfortranarray(a)
    bs = list(blockSize) + [1] * (3 - len(blockSize))
    if np.ndim(data) == 2:
        bs[2] = 1
    if overwrite and os.path.isdir(str(filepath)):
        shutil.rmtree(str(filepath))
    os.makedirs(os.path.dirname(os.path.abspath(str(filepath))), exist_ok=True)
    bits, isf = _W[a.dtype]
    comp = _COMP[compressor if compressor is None else str(compressor).lower()]
    if dimSeparator == "/":                 # the metadata, then the whole array as one region write
        import json
        os.makedirs(str(filepath), exist_ok=True)
        if comp >= 3:
            cmeta = {"blocksize": 0, "clevel": 5, "cname": _BLOSC[comp], "id": "blosc", "shuffle": 1}
        else:
            cmeta = None if comp == 0 else {"id": "zlib" if comp == 1 else "gzip", "level": 1}
        meta = {"chunks": [int(min(b, n)) for b, n in zip(bs, a.shape)],
                "compressor": cmeta,
                "dimension_separator": "/", "dtype": f"<{'f' if isf else 'u'}{bits // 8}", "fill_value": 0,
                "filters": None, "order": "F", "shape": [int(n) for n in a.shape], "zarr_format": 2}
        with open(os.path.join(str(filepath), ".zarray"), "w") as f:
            json.dump(meta, f, indent=4)
        writezarr_region(a, filepath, [1, 1, 1, *a.shape], threads=threads)
        return
    check(lib.pk_zarr_write(os.fsencode(str(filepath)), ptr(a), i64x3(a.shape), bits, isf, i64x3(bs), comp,
                            int(threads)))


def writezarr_region(data, filepath, bbox, threads=0):
    """writezarr(data, filepath, 'bbox', [y1 x1 z1 y2 x2 z2]) into an existing array: the region must
    cover whole chunks (it may end at the array's edge)."""
    a = np.asfortranarray(np.asarray(data))
    shape, _, dt = getZarrInfo(filepath)
    if a.dtype != dt:
        raise TypeError(f"writezarr: the array holds {dt}, not {a.dtype}")
    while a.ndim < 3:
        a = a[..., None]
    want = tuple(int(bbox[k + 3]) - int(bbox[k]) + 1 for k in range(3))
    if a.shape != want:
        raise ValueError(f"data of shape {a.shape} does not fill the region {want}")
    bb = (C.c_int64 * 6)(*[int(v) for v in bbox])
    check(lib.pk_zarr_write_region(os.fsencode(str(filepath)), ptr(a), bb, int(threads)))
