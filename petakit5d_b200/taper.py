"""Edge taper of the raw volume before deconvolution (RLdecon.m:351-357).

``edgetaper_slices(vol, PSF)`` runs MATLAB's ``edgetaper(vol(:,:,iz), PSF)`` on every z slice on the
GPU through libpkdecon.so (pk_edgetaper); ``edgetaper(I, PSF)`` is the one-image form and
``fspecial_gaussian(hsize, sigma)`` builds the kernel that RLdecon passes,
``fspecial('gaussian', nTapering + 30, nTapering)`` (host parameter setup, float64).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, i64x3, lib, ptr

_DT = {np.dtype(np.uint16): 0, np.dtype(np.float32): 1}


def fspecial_gaussian(hsize, sigma):
    """fspecial('gaussian', hsize, sigma): exp(-(x^2 + y^2) / (2 sigma^2)) on an hsize x hsize grid
    centred at (hsize - 1) / 2, values below eps * max dropped, normalised to sum 1 (float64)."""
    r = np.arange(int(hsize), dtype=np.float64) - (int(hsize) - 1) / 2.0
    h = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / (2.0 * float(sigma) ** 2))
    h[h < np.finfo(np.float64).eps * h.max()] = 0.0
    return h / h.sum()


def edgetaper_slices(vol, psf, out=None, ctx=None):
    """edgetaper(vol(:,:,iz), psf) for every z slice of a uint16 / single [ny, nx, nz] volume; the
    result keeps the volume's class.  ``out`` (Fortran order, same class and shape) may be ``vol``."""
    ctx = ctx or _lib.default_context()
    a = np.asarray(vol)
    if a.dtype not in _DT:
        a = a.astype(np.float32)
    two_d = a.ndim == 2
    if a.ndim not in (2, 3):
        raise ValueError("edgetaper: volume must be 2-D or 3-D")
    a = np.asfortranarray(a if not two_d else a[:, :, None])
    h = np.asfortranarray(np.asarray(psf, np.float64))
    if h.ndim != 2:
        raise ValueError("edgetaper: PSF must be 2-D")
    if out is None:
        out = np.empty(a.shape, a.dtype, order="F")
    elif (not out.flags.f_contiguous or out.dtype != a.dtype
          or out.reshape(out.shape + (1,) * (3 - out.ndim)).shape != a.shape):
        raise ValueError("out must be a Fortran-ordered array of the volume's class and shape")
    check(lib.pk_edgetaper(ctx.handle, ptr(a), _DT[a.dtype], i64x3(a.shape), ptr(h), (C.c_int64 * 2)(*h.shape),
                           ptr(out)))
    return out[:, :, 0] if two_d and out.ndim == 3 else out


def edgetaper(img, psf, ctx=None):
    """edgetaper(I, PSF) for one 2-D uint16 / single image."""
    return edgetaper_slices(img, psf, ctx=ctx)
