"""Backprojector generators (drop-ins for the reference's MATLAB functions).

* ``omw_backprojector_generation(psf, alpha, skewed, ...)`` mirrors
  microscopeDataProcessing/decon/omw_backprojector_generation.m:1-166 and returns
  ``(b_omw, OTF_bp_omw, abs_OTF_c, OTF_mask)``.
* ``BackProjector(PSF_fp, bp_type, alpha, beta, n, resFlag, iRes)`` mirrors
  third_parties/WBDeconvolution/BackProjector.m:1-233 (all five bp_types) and returns
  ``(PSF_bp, OTF_bp)``.

Both run on the GPU through libpkdecon.so (float64 transforms at PSF size).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, i64x3, lib, ptr


def _psf3(psf):
    a = np.asarray(psf, dtype=np.float32)
    while a.ndim < 3:
        a = a[..., None]
    return np.asfortranarray(a)


def omw_backprojector_generation(psf, alpha, skewed, OTFCumThresh=0.9, OTFAreaThresh=100, hannWinBounds=(0.8, 1.0),
                                 minIntThrsh=1e-3, ctx=None):
    """[b_omw, OTF_bp_omw, abs_OTF_c, OTF_mask] = omw_backprojector_generation(psf, alpha, skewed, ...).

    ``skewed``: True/False, or None for the reference's auto-detection (``skewed = []``).
    """
    ctx = ctx or _lib.default_context()
    p = _psf3(psf)
    if p.size == 0:
        raise ValueError("A valid nonzero PSF needs to be provided!")
    sk = -1 if skewed is None or (hasattr(skewed, "__len__") and len(skewed) == 0) else (1 if skewed else 0)
    lo, hi = [float(v) for v in hannWinBounds]
    b = np.empty(p.shape, np.float32, order="F")
    omw = np.empty(p.shape, np.complex64, order="F")
    absc = np.empty(p.shape, np.float32, order="F")
    mask = np.empty(p.shape, np.uint8, order="F")
    check(lib.pk_omw_backprojector(ctx.handle, ptr(p), i64x3(p.shape), float(alpha), sk, float(OTFCumThresh),
                                   float(OTFAreaThresh), lo, hi, float(minIntThrsh), ptr(b), ptr(omw), ptr(absc),
                                   ptr(mask)))
    return b, omw, absc, mask.astype(bool) if mask.max(initial=0) <= 1 else mask


BP_TYPES = {"traditional": 0, "gaussian": 1, "butterworth": 2, "wiener": 3, "wiener-butterworth": 4}


def BackProjector(PSF_fp, bp_type="traditional", alpha=0.001, beta=1, n=10, resFlag=1, iRes=(0, 0, 0),
                  verboseFlag=0, ctx=None):
    """[PSF_bp, OTF_bp] = BackProjector(PSF_fp, bp_type, alpha, beta, n, resFlag, iRes, verboseFlag).

    bp_type: 'traditional', 'gaussian', 'butterworth', 'wiener' or 'wiener-butterworth'
    (BackProjector.m:163-231); anything else raises ValueError as the reference errors.
    """
    if bp_type not in BP_TYPES:
        raise ValueError("bp_type does not match any back-projector type")
    ctx = ctx or _lib.default_context()
    p = _psf3(PSF_fp)
    out = np.empty(p.shape, np.float64, order="F")
    otf = np.empty(p.shape, np.complex128, order="F")
    ires = (C.c_double * 3)(*[float(v) for v in (list(iRes) + [0, 0, 0])[:3]])
    check(lib.pk_backprojector(ctx.handle, ptr(p), i64x3(p.shape), BP_TYPES[bp_type], float(alpha), float(beta), int(n),
                               int(resFlag), ires, ptr(out), ptr(otf)))
    return out, otf
