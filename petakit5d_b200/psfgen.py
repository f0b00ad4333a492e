"""PSF preparation before deconvolution (drop-ins for the reference's MATLAB code).

* ``psf_gen_new(psf, dz_psf, dz_data, medFactor=1.5, PSFGenMethod='masked')`` mirrors
  microscopeDataProcessing/decon/psf_gen_new.m:1-140 (background subtraction, peak-component mask,
  centring, axial resampling) and runs on the GPU through libpkdecon.so.
* ``rldecon_psf_crop(psf, data_size, RLMethod)`` mirrors the PSF crops RLdecon.m:249-265 applies
  after it: the non-OMW methods crop to the PSF's nonzero bounding box (one voxel of margin, centre
  kept), and a PSF larger than the data is cropped around its centre (host index arithmetic).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, i64x3, lib, ptr

_METHODS = {"masked": 0, "median": 1}


def psf_gen_new(psf, dz_psf, dz_data, medFactor=1.5, PSFGenMethod="masked", ctx=None):
    """psf = psf_gen_new(psf, dz_psf, dz_data, medFactor, PSFGenMethod).

    Returns a float32 array (MATLAB returns double after the axial resampling)."""
    ctx = ctx or _lib.default_context()
    m = str(PSFGenMethod).lower()
    if m not in _METHODS:
        raise ValueError(f"PSFGenMethod must be 'masked' or 'median', not {PSFGenMethod!r}")
    a = np.asarray(psf, dtype=np.float32)
    two_d = a.ndim == 2
    while a.ndim < 3:
        a = a[..., None]
    a = np.asfortranarray(a)
    od = (C.c_int64 * 3)()
    ny, nx, nz = a.shape
    buf = np.empty(ny * nx * (2 * nz + 8), np.float32)       # the output bound stated in pkdecon.h
    check(lib.pk_psf_gen(ctx.handle, ptr(a), i64x3(a.shape), float(dz_psf), float(dz_data), float(medFactor),
                         _METHODS[m], ptr(buf), buf.size, od))
    shape = tuple(int(v) for v in od)
    out = buf[:int(np.prod(shape))].reshape(shape, order="F")
    return out[:, :, 0] if two_d and shape[2] == 1 else out


def rldecon_psf_crop(psf, data_size, RLMethod="omw"):
    """The PSF crops of RLdecon.m:249-265 (after psf_gen_new)."""
    psf = np.asarray(psf)
    while psf.ndim < 3:
        psf = psf[..., None]
    psz = np.array(psf.shape)
    if str(RLMethod).lower() != "omw":
        lo = np.zeros(3, int)
        for d in range(3):
            nzi = np.flatnonzero(psf.sum(axis=tuple(a for a in range(3) if a != d)))
            if nzi.size == 0:
                raise ValueError("RLdecon: the PSF is all zero")
            lo[d] = min(nzi[0], psz[d] - 1 - nzi[-1]) - 1
        lo = np.maximum(0, lo)
        psf = psf[lo[0]:psz[0] - lo[0], lo[1]:psz[1] - lo[1], lo[2]:psz[2] - lo[2]]
        psz = np.array(psf.shape)
    im = np.array(tuple(data_size) + (1,) * (3 - len(data_size)))
    if np.any(psz > im):
        s = np.maximum(0, (psz - im) // 2)
        t = s + np.minimum(psz, im)
        psf = psf[s[0]:t[0], s[1]:t[1], s[2]:t[2]]
    return psf
