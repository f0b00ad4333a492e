"""Drop-in host API for the deconvolution hot path, mirroring the reference MATLAB functions.

``decon_lucy_function`` and ``decon_lucy_omw_function`` take the same positional arguments and
name/value parameters as microscopeDataProcessing/decon/decon_lucy_function.m:1-36 and
decon_lucy_omw_function.m:1-30 and return the same outputs.  Arrays are indexed like MATLAB
(``I[y, x, z]``, ``size(I) == I.shape``); they are passed to libpkdecon.so in column-major order.
Parameter names are matched case-insensitively, as the reference's inputParser does.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import PK_F32, PK_F64, PK_U16, DeconParams, check, i64x3, lib, ptr

_DEFAULTS = {"background": None, "usegpu": True, "save16bit": True, "dampfactor": 1.0, "scalefactor": 1.0,
             "deconoffset": 0.0, "edgeerosion": 0, "bbox": None, "debug": False, "debug_folder": "./debug/",
             "savestep": 1}


def _parse(kw):
    opts = dict(_DEFAULTS)
    ctx = kw.pop("ctx", None)
    for k, v in kw.items():
        key = k.lower()
        if key not in opts:
            raise TypeError(f"'{k}' is not a recognized parameter")
        opts[key] = v
    if not opts["usegpu"]:
        raise ValueError("useGPU=false: this implementation runs on the GPU only (no CPU path)")
    return opts, ctx


def _params(opts):
    p = DeconParams()
    lib.pk_params_default(p)
    bg = opts["background"]
    p.background = 0.0 if bg is None or (hasattr(bg, "__len__") and len(bg) == 0) else float(bg)
    p.damp_factor = float(opts["dampfactor"])
    p.scale_factor = float(opts["scalefactor"])
    p.decon_offset = float(opts["deconoffset"])
    p.edge_erosion = int(opts["edgeerosion"])
    p.save16bit = 1 if opts["save16bit"] else 0
    bb = opts["bbox"]
    if bb is not None and len(bb) > 0:
        if len(bb) != 6:
            raise ValueError("bbox must have 6 elements [y1 x1 z1 y2 x2 z2]")
        p.has_bbox = 1
        for i in range(6):
            p.bbox[i] = int(bb[i])
    return p


def _volume(I):
    a = np.asarray(I)
    if a.ndim > 3:
        raise ValueError("only 2D/3D volumes are supported")
    while a.ndim < 3:
        a = a[..., None]
    if a.dtype == np.uint16:
        t = PK_U16
    elif a.dtype == np.float32:
        t = PK_F32
    elif a.dtype == np.float64:
        t = PK_F64
    else:
        a = a.astype(np.float32)
        t = PK_F32
    return np.asfortranarray(a), t


def _psf(P):
    a = np.asarray(P, dtype=np.float32)
    while a.ndim < 3:
        a = a[..., None]
    return np.asfortranarray(a)


def _out(dims, p):
    od = i64x3([0, 0, 0])
    check(lib.pk_output_dims(i64x3(dims), p, od))
    shape = tuple(int(v) for v in od)
    return np.empty(shape, dtype=np.uint16 if p.save16bit else np.float32, order="F")


def _debug_run(method, vol, t, pf, pb, numit, p, opts, ctx, out):
    """debug = true: err_mat from the library, uint16(J) of every saveStep-th iteration written to
    debug_folder/Iter_%04d.tif (decon_lucy_omw_function.m:113-141, decon_lucy_function.m:144-171)."""
    import os
    from .tiff import writetiff
    estep = int(opts["savestep"])
    numit = int(numit)
    nsnap = numit // estep if estep >= 1 else 0
    snaps = np.empty((max(nsnap, 1),) + vol.shape[::-1], np.uint16)      # C order of [nz nx ny] per volume
    err = np.zeros((max(numit, 1), 4), np.float64)
    rows = _lib.C.c_int32(0)
    check(lib.pk_decon_debug(ctx.handle, int(method), ptr(vol), t, i64x3(vol.shape), ptr(pf), i64x3(pf.shape),
                             ptr(pb) if pb is not None else None, i64x3(pb.shape if pb is not None else pf.shape),
                             numit, p, estep, ptr(out), ptr(err), _lib.C.byref(rows),
                             ptr(snaps) if nsnap > 0 else None))
    n = int(rows.value)
    err_mat = err.reshape(-1, order="C").view()[: 4 * n].reshape(4, n).T.copy()   # column-major n x 4
    folder = opts["debug_folder"]
    os.makedirs(folder, exist_ok=True)
    for s in range(nsnap):
        writetiff(snaps[s].T, os.path.join(folder, f"Iter_{(s + 1) * estep:04d}.tif"))
    return err_mat


def decon_lucy_function(I, PSF, NUMIT, **kw):
    """[J_2, err_mat, k] = decon_lucy_function(I, PSF, NUMIT, ...) (Biggs-accelerated RL)."""
    opts, ctx = _parse(kw)
    ctx = ctx or _lib.default_context()
    vol, t = _volume(I)
    psf = _psf(PSF)
    p = _params(opts)
    out = _out(vol.shape, p)
    if opts["debug"]:
        err_mat = _debug_run(0, vol, t, psf, None, NUMIT, p, opts, ctx, out)
        return _squeeze_like(out, I), err_mat, int(NUMIT)
    k = _lib.C.c_int32(0)
    check(lib.pk_decon_lucy(ctx.handle, ptr(vol), t, i64x3(vol.shape), ptr(psf), i64x3(psf.shape), int(NUMIT), p,
                            ptr(out), _lib.C.byref(k)))
    return _squeeze_like(out, I), np.zeros((int(NUMIT), 4)), int(k.value)


def decon_lucy_omw_function(I, PSF_f, PSF_b, NUMIT, **kw):
    """[J, err_mat] = decon_lucy_omw_function(I, PSF_f, PSF_b, NUMIT, ...) (OMW / WB backprojector RL)."""
    opts, ctx = _parse(kw)
    ctx = ctx or _lib.default_context()
    vol, t = _volume(I)
    pf = _psf(PSF_f)
    pb = _psf(PSF_b)
    p = _params(opts)
    out = _out(vol.shape, p)
    if opts["debug"]:
        err_mat = _debug_run(1, vol, t, pf, pb, NUMIT, p, opts, ctx, out)
        return _squeeze_like(out, I), err_mat
    check(lib.pk_decon_lucy_omw(ctx.handle, ptr(vol), t, i64x3(vol.shape), ptr(pf), i64x3(pf.shape), ptr(pb),
                                i64x3(pb.shape), int(NUMIT), p, ptr(out)))
    return _squeeze_like(out, I), np.zeros((int(NUMIT), 4))


_INFLIGHT = {}


def decon_submit(method, I, PSF_f, PSF_b, NUMIT, out, ctx=None, **kw):
    """Queue one host-buffer deconvolution ('omw' or 'rl') and return its ticket at once.

    ``out`` receives the result (the shape and dtype ``decon_lucy_*_function`` would return, in
    Fortran order); ``I`` and ``out`` should be page-locked (``tiff.pinned_empty``, torch
    ``pin_memory``) for the copies to overlap other calls' compute.  Collect with ``decon_wait``."""
    opts, _ = _parse(kw)
    ctx = ctx or _lib.default_context()
    vol, t = _volume(I)
    pf = _psf(PSF_f)
    pb = _psf(PSF_b) if method == "omw" else None
    p = _params(opts)
    od = i64x3([0, 0, 0])
    check(lib.pk_output_dims(i64x3(vol.shape), p, od))
    dt = np.dtype(np.uint16 if p.save16bit else np.float32)
    if out.dtype != dt or out.size < int(np.prod([int(v) for v in od])):
        raise ValueError(f"out must hold {tuple(int(v) for v in od)} {dt}")
    tk = _lib.C.c_int64()
    check(lib.pk_decon_submit(ctx.handle, 1 if method == "omw" else 0, ptr(vol), t, i64x3(vol.shape), ptr(pf),
                              i64x3(pf.shape), ptr(pb), i64x3(pb.shape if pb is not None else pf.shape), int(NUMIT),
                              p, ptr(out), _lib.C.byref(tk)))
    _INFLIGHT[(ctx.handle, tk.value)] = (vol, out)       # keep the buffers alive until the wait
    return tk.value


def decon_wait(ticket, timeout_ms=-1, ctx=None):
    """Wait for a ``decon_submit`` ticket (raises PkError PK_ERR_TIMEOUT when ``timeout_ms`` passes)."""
    ctx = ctx or _lib.default_context()
    check(lib.pk_decon_wait(ctx.handle, int(ticket), int(timeout_ms)))
    _INFLIGHT.pop((ctx.handle, int(ticket)), None)


def _squeeze_like(out, I):
    nd = np.asarray(I).ndim
    if nd < 3 and out.shape[2] == 1:
        out = out[..., 0]
        if nd < 2 and out.shape[1] == 1:
            out = out[:, 0]
    return out


def decon_device(method, d_in, in_dtype, dims, psf_f, psf_b=None, numit=2, ctx=None, stream=None, **kw):
    """Device-pointer call (``d_in``/``d_out`` are device pointers or torch CUDA tensors).

    method: 'omw' or 'rl'.  Returns the DeconParams used and writes into ``kw['out']``.
    """
    opts, _ = _parse({k: v for k, v in kw.items() if k != "out"})
    ctx = ctx or _lib.default_context()
    out = kw["out"]
    p = _params(opts)
    t = {"uint16": PK_U16, "float32": PK_F32, "float64": PK_F64}[str(in_dtype).replace("torch.", "")]
    pf = _psf(psf_f)
    s = ptr(stream) if stream is not None else None
    if method == "omw":
        pb = _psf(psf_b)
        check(lib.pk_decon_lucy_omw_device(ctx.handle, ptr(d_in), t, i64x3(dims), ptr(pf), i64x3(pf.shape),
                                           ptr(pb), i64x3(pb.shape), int(numit), p, ptr(out), s))
    else:
        check(lib.pk_decon_lucy_device(ctx.handle, ptr(d_in), t, i64x3(dims), ptr(pf), i64x3(pf.shape), int(numit),
                                       p, ptr(out), s))
    return p


def psf2otf_half(psf, dims, ctx=None):
    """decon_psf2otf(PSF./sum(PSF(:)), dims) as the half spectrum ``[floor(ny/2)+1, nx, nz]`` complex64."""
    ctx = ctx or _lib.default_context()
    pf = _psf(psf)
    d = [int(v) for v in dims] + [1] * (3 - len(dims))
    out = np.empty((d[0] // 2 + 1, d[1], d[2]), dtype=np.complex64, order="F")
    check(lib.pk_psf2otf(ctx.handle, ptr(pf), i64x3(pf.shape), i64x3(d), ptr(out)))
    return out


def fft3_r2c(d_in, dims, d_spec, ctx=None, stream=None):
    ctx = ctx or _lib.default_context()
    check(lib.pk_fft3_r2c_device(ctx.handle, ptr(d_in), i64x3(dims), ptr(d_spec), ptr(stream) if stream else None))


def fft3_c2r(d_spec, dims, d_out, ctx=None, stream=None):
    ctx = ctx or _lib.default_context()
    check(lib.pk_fft3_c2r_device(ctx.handle, ptr(d_spec), i64x3(dims), ptr(d_out), ptr(stream) if stream else None))


def decon_mask_edge_erosion(mask, EdgeErosion, ctx=None):
    """mask = decon_mask_edge_erosion(mask, EdgeErosion) (decon/decon_mask_edge_erosion.m:1-30) on the
    GPU: ``mask > 0`` eroded at the volume's edges (full mask: EdgeErosion voxels off each face;
    otherwise faces cleared, then strel('disk', EdgeErosion - 1) per plane and a line of
    2 * EdgeErosion - 1 in z).  ``mask`` may be logical, uint8, uint16 or single; returns logical."""
    ctx = ctx or _lib.default_context()
    a = np.asarray(mask)
    shape = a.shape
    if a.dtype not in (np.uint16, np.float32):
        a = (a > 0).astype(np.uint16)
    while a.ndim < 3:
        a = a[..., None]
    a = np.asfortranarray(a)
    out = np.empty(a.shape, np.uint8, order="F")
    check(lib.pk_mask_edge_erosion(ctx.handle, ptr(a), _lib.PK_U16 if a.dtype == np.uint16 else _lib.PK_F32,
                                   i64x3(a.shape), int(EdgeErosion), ptr(out)))
    return out.astype(bool).reshape(shape, order="F")
