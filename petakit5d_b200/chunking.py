"""Chunked deconvolution: the callers of the hot path for volumes split into overlapping chunks.

* ``find_good_factor_number``  -- utils/findGoodFactorNumber.m:1-26
* ``zarr_chunk_coordinates``   -- microscopeDataProcessing/stitch/XR_zarrChunkCoordinatesExtraction.m:1-83
* ``border_size``              -- ``round((size(psf)+10)/2)`` (RLdecon_large_in_memory.m:177)
* ``batch_decon``              -- many chunks in shared launches (pk_batch_decon)
* ``decon_large_in_memory``    -- RLdecon_large_in_memory.m:177-260: chunk grid with borders, decon of
                                  every chunk cropped to its region (deconBbox), paste back
* ``edge_erosion_mask``        -- the runner's bwdist edge erosion (RLdecon_large_in_memory.m:146-168)
* ``RLdecon_large_in_memory``  -- the whole runner for TIFF files (RLdecon_large_in_memory.m:1-300)
* ``RLdecon_large_in_place``   -- the Zarr runner, region by region (RLdecon_large_in_place.m:1-277)
"""
from __future__ import annotations

import ctypes as C
import math
import os
import shutil

import numpy as np

from . import _lib
from ._lib import PK_F32, PK_F64, PK_U16, Chunk, check, i64x3, lib, ptr
from .decon import _params, _parse, _psf


def find_good_factor_number(n, direction=1, allow_odd_seven=False):
    return int(lib.pk_find_good_factor_number(int(n), int(direction), 1 if allow_odd_seven else 0))


def border_size(psf_size):
    return [int(np.floor((s + 10) / 2.0 + 0.5)) for s in psf_size]


def zarr_chunk_coordinates(vol_size, batch_size=(1024, 1024, 1024), block_size=(256, 256, 256), bbox=None,
                           same_batch_size=True, border=50):
    """(batchBBoxes, regionBBoxes, localBBoxes) as n x 6 int64 arrays, 1-based inclusive."""
    border = list(np.broadcast_to(np.asarray(border, dtype=np.int64), (3,)))
    block = list(np.broadcast_to(np.asarray(block_size, dtype=np.int64), (3,)))
    bb = None
    if bbox is not None and len(bbox) == 6:
        bb = (C.c_int64 * 6)(*[int(v) for v in bbox])
    n = lib.pk_chunk_coordinates(i64x3(vol_size), i64x3(batch_size), i64x3(block), bb, 1 if same_batch_size else 0,
                                 i64x3(border), None, None, None)
    if n < 0:
        raise ValueError("invalid chunk grid arguments")
    out = [np.zeros((n, 6), np.int64) for _ in range(3)]
    lib.pk_chunk_coordinates(i64x3(vol_size), i64x3(batch_size), i64x3(block), bb, 1 if same_batch_size else 0,
                             i64x3(border), ptr(out[0]), ptr(out[1]), ptr(out[2]))
    return tuple(out)


_TYPES = {np.dtype(np.uint16): PK_U16, np.dtype(np.float32): PK_F32, np.dtype(np.float64): PK_F64}


def batch_decon(chunks, psfs, psf_ids, numit=2, method="omw", psfs_b=None, bboxes=None, pad_good=False, ctx=None,
                outputs=None, **kw):
    """Deconvolve ``chunks`` (list of [y, x, z] arrays of one dtype) in shared launches.

    ``psfs[psf_ids[i]]`` (and ``psfs_b[...]`` for OMW) is chunk i's PSF pair; ``bboxes[i]`` its 1-based
    inclusive output crop (deconBbox) or None.  Returns the list of outputs (uint16 when save16bit).
    For the host->device copies to overlap the compute, pass chunks in pinned memory.
    """
    opts, _ = _parse(dict(kw))
    ctx = ctx or _lib.default_context()
    m = {"omw": 1, "rl": 0}[method]
    if m == 1 and psfs_b is None:
        raise ValueError("OMW needs backprojectors (psfs_b)")
    vols = [np.asfortranarray(c) for c in chunks]
    dt = {v.dtype for v in vols}
    if len(dt) != 1 or next(iter(dt)) not in _TYPES:
        raise ValueError("all chunks must share one dtype among uint16/float32/float64")
    t = _TYPES[next(iter(dt))]
    pf = [_psf(p) for p in psfs]
    shapes = {p.shape for p in pf}
    pb = [_psf(p) for p in psfs_b] if psfs_b is not None else None
    if pb is not None:
        for a, b in zip(pf, pb):
            if a.shape != b.shape:
                raise ValueError("PSF_f and PSF_b of one id must have the same size")
    del shapes
    p = _params(opts)
    n = len(vols)
    arr = (Chunk * n)()
    outs = []
    for i, v in enumerate(vols):
        q = _params(opts)
        bb = None if bboxes is None else bboxes[i]
        if bb is not None and len(bb) == 6:
            q.has_bbox = 1
            for k in range(6):
                q.bbox[k] = int(bb[k])
        od = i64x3([0, 0, 0])
        check(lib.pk_output_dims(i64x3(v.shape), q, od))
        o = outputs[i] if outputs is not None else np.empty(tuple(od), np.uint16 if p.save16bit else np.float32, order="F")
        outs.append(o)
        arr[i].in_ = v.ctypes.data
        arr[i].dims = i64x3(v.shape)
        arr[i].psf_id = int(psf_ids[i])
        arr[i].has_bbox = q.has_bbox
        for k in range(6):
            arr[i].bbox[k] = q.bbox[k]
        arr[i].out = o.ctypes.data
    npsf = len(pf)
    fptrs = (C.c_void_p * npsf)(*[a.ctypes.data for a in pf])
    bptrs = (C.c_void_p * npsf)(*[a.ctypes.data for a in pb]) if pb is not None else None
    dims = np.array([list(a.shape) for a in pf], dtype=np.int64).ravel()
    check(lib.pk_batch_decon(ctx.handle, m, n, arr, t, npsf, fptrs, bptrs, dims.ctypes.data, int(numit), p,
                             1 if pad_good else 0, 0))
    return outs


def decon_large_in_memory(volume, psf, numit=2, method="omw", psf_b=None, batch_size=(512, 512, 512), ctx=None,
                          pad_good=False, **kw):
    """RLdecon_large_in_memory.m:177-260 on one GPU: chunk grid with BorderSize = round((size(psf)+10)/2)
    (sameBatchSize false), every chunk deconvolved and cropped to its region, pasted into the output."""
    vol = np.asfortranarray(volume)
    border = border_size(np.asarray(psf).shape[:3])
    bb, rb, _ = zarr_chunk_coordinates(vol.shape, batch_size=batch_size, block_size=batch_size, same_batch_size=False,
                                       border=border)
    chunks, boxes = [], []
    for b, r in zip(bb, rb):
        chunks.append(np.asfortranarray(vol[b[0] - 1:b[3], b[1] - 1:b[4], b[2] - 1:b[5]]))
        st = r[:3] - b[:3] + 1
        en = r[3:] - b[:3] + 1
        boxes.append([*st, *en])
    outs = batch_decon(chunks, [psf], [0] * len(chunks), numit, method, [psf_b] if psf_b is not None else None,
                       boxes, pad_good, ctx, **kw)
    save16 = kw.get("save16bit", kw.get("Save16bit", True))
    out = np.empty(vol.shape, np.uint16 if save16 else np.float32, order="F")
    for r, o in zip(rb, outs):
        out[r[0] - 1:r[3], r[1] - 1:r[4], r[2] - 1:r[5]] = o
    return out


def edge_erosion_mask(im, erosion, out=None, ctx=None):
    """RLdecon_large_in_memory.m:146-168, 267-270 on the GPU: the mask ``bwdist(~(im > 0, faces
    cleared)) > erosion - 1``; ``out`` (uint16 / single, Fortran order) is multiplied by it in place."""
    ctx = ctx or _lib.default_context()
    a = np.asfortranarray(im)
    if a.dtype not in (np.uint16, np.float32):
        a = np.asfortranarray(a.astype(np.float32))
    mask = np.empty(a.shape, np.uint8, order="F")
    t = _lib.PK_U16 if a.dtype == np.uint16 else _lib.PK_F32
    ot = 0
    if out is not None:
        if not out.flags.f_contiguous or out.shape != a.shape or out.dtype not in (np.uint16, np.float32):
            raise ValueError("out must be a Fortran-ordered uint16/single array of the volume's shape")
        ot = _lib.PK_U16 if out.dtype == np.uint16 else _lib.PK_F32
    check(lib.pk_edge_erosion_edt(ctx.handle, ptr(a), t, i64x3(a.shape), int(erosion), ptr(out), ot, ptr(mask)))
    return mask.astype(bool)


def _runner_options(name, defaults, kw):
    low = {k.lower(): k for k in defaults}
    o = dict(defaults)
    for k, v in kw.items():
        if k.lower() not in low:
            raise TypeError(f"{name}: unknown parameter {k!r}")
        o[low[k.lower()]] = v
    if o["maskFullpaths"] and len(o["maskFullpaths"]) and o["maskFullpaths"][0] and len(o["maskFullpaths"]) != 3:
        raise ValueError("maskFullpaths: three 2-D Zarr masks (xy, xz, yz) are needed")
    if str(o["RLMethod"]) not in ("simplified", "omw"):
        raise NotImplementedError(f"RLMethod '{o['RLMethod']}' is not built")
    return o


_MASK_AXES = ((0, 1), (1, 2), (0, 2))          # finds = [1, 2; 2, 3; 1, 3]: xy, xz, yz


def _round_half_away(v):
    return math.floor(v + 0.5) if v >= 0 else math.ceil(v - 0.5)


def region_masked_out(mask_paths, region):
    """True when a region need not be deconvolved (RLdecon_large_in_memory.m:201-216,
    RLdecon_for_zarr_block.m:111-128): one of the three 2-D Zarr masks (xy, xz, yz maximum-projection
    masks, in that order) is all zero over the region's window ``[start(a) 1 end(a) 1]``."""
    from . import zarrio as Z
    if not mask_paths or not len(mask_paths) or not mask_paths[0]:
        return False
    r = [int(v) for v in region]
    for f, (a, b) in enumerate(_MASK_AXES):
        win = Z.readzarr(mask_paths[f], inputBbox=[r[a], r[b], 1, r[a + 3], r[b + 3], 1])
        if not np.any(win):
            return True
    return False


def _runner_psfs(psfFullpath, decon_path, dz, o, ctx):
    """The PSF that sets the chunk borders (RLdecon_large_in_memory.m:93-123,
    RLdecon_large_in_place.m:112-141; written to <deconPath>/psfgen/) and the PSF each chunk's RLdecon
    call prepares from the same file (RLdecon.m:241-265: its own dz ratio, sind(|SkewAngle|))."""
    from . import psfgen as P
    from . import tiff as T
    pp = T.readtiff(psfFullpath).astype(np.float32)
    skew = float(o["SkewAngle"])
    method = str(o["RLMethod"])
    if not o["psfGen"]:
        return pp, pp
    ratio = math.sin(math.radians(skew)) if o["Deskew"] else 1.0
    g = P.psf_gen_new(pp, o["dzPSF"], dz * ratio, 1.5, "masked", ctx=ctx)
    psf = P.rldecon_psf_crop(g, g.shape, "simplified")          # bounding box +-1 only
    os.makedirs(os.path.join(decon_path, "psfgen"), exist_ok=True)
    gen_fn = os.path.join(decon_path, "psfgen", os.path.splitext(os.path.basename(psfFullpath))[0] + ".tif")
    if not os.path.exists(gen_fn):
        T.writetiff(psf, gen_fn)
    cpsf = P.psf_gen_new(pp, o["dzPSF"], dz * math.sin(math.radians(abs(skew))), 1.5, "masked", ctx=ctx)
    if method != "omw":
        cpsf = P.rldecon_psf_crop(cpsf, cpsf.shape, "simplified")
    return psf, cpsf


def _decon_chunks(chunks, boxes, cpsf, o, ctx, bg, edge_erosion=0):
    """Every chunk deconvolved as RLdecon would (PSF cropped to the chunk when larger, :260-265; OMW
    backprojector of that PSF), cropped to its region; one batched call."""
    from . import backprojector as B
    from . import psfgen as P
    method = str(o["RLMethod"])
    psfs, psfs_b, ids, key = [], [], [], {}
    for c in chunks:
        cp = P.rldecon_psf_crop(cpsf, c.shape, "omw")
        k = cp.shape
        if k not in key:
            key[k] = len(psfs)
            p32 = np.asarray(cp, np.float32)
            psfs.append(p32 / np.float32(p32.sum(dtype=np.float32)))
            if method == "omw":
                bp = B.omw_backprojector_generation(cp, float(o["wienerAlpha"]), o["skewed"],
                                                    OTFCumThresh=float(o["OTFCumThresh"]),
                                                    hannWinBounds=o["hannWinBounds"], ctx=ctx)[0]
                psfs_b.append(P.rldecon_psf_crop(bp, c.shape, "omw"))
        ids.append(key[k])
    scale = 1.0 if o["scaleFactor"] is None or np.size(o["scaleFactor"]) == 0 else float(o["scaleFactor"])
    return batch_decon(chunks, psfs, ids, int(o["DeconIter"]), "omw" if method == "omw" else "rl",
                       psfs_b if method == "omw" else None, boxes, False, ctx, Background=bg,
                       save16bit=bool(o["save16bit"]), dampFactor=o["dampFactor"], scaleFactor=scale,
                       deconOffset=o["deconOffset"], EdgeErosion=int(edge_erosion))


def RLdecon_large_in_memory(frameFullpath, psfFullpath, deconFullpath, xyPixelSize, dz, **kw):
    """RLdecon_large_in_memory(frameFullpath, psfFullpath, deconFullpath, xyPixelSize, dz, ...)
    (decon/RLdecon_large_in_memory.m:1-300) for TIFF files: the PSF prepared with psf_gen_new and
    saved under ``<deconPath>/psfgen/``, the volume read whole, cut into ``batchSize`` chunks with
    ``round((size(psf) + 10) / 2)`` borders, every chunk deconvolved as RLdecon would (one batched
    call), the regions pasted back, the edge-erosion mask applied, and the result and its z MIP
    written.  The input may be TIFF or Zarr (:129-135); ``saveZarr`` writes the result as Zarr
    (:288-293); regions that ``maskFullpaths`` masks out are left zero without deconvolution
    (:201-216)."""
    from . import tiff as T
    from . import zarrio as Z
    o = _runner_options("RLdecon_large_in_memory", dict(
        save16bit=True, Rotate=False, Deskew=False, SkewAngle=-32.45, flipZstack=False, Background=None,
        dzPSF=0.1, DeconIter=15, EdgeErosion=8, ErodeMaskfile="", SaveMaskfile=False, dampFactor=1.0,
        scaleFactor=None, deconOffset=0.0, maskFullpaths=(), saveZarr=False, RLMethod="simplified",
        wienerAlpha=0.005, OTFCumThresh=0.9, hannWinBounds=(0.8, 1.0), skewed=None, fixIter=True,
        errThresh=None, batchSize=(1024, 1024, 1024), Overlap=200, CPUMaxMem=500, parseCluster=True, uuid="",
        debug=False, psfGen=True, useGPU=True, ctx=None, EdgeSoften=5, zEdgeSoften=2, Crop=None, zFlip=False,
        GenMaxZproj=(0, 0, 1)), kw)
    # Deskew sets the dz ratio of the border PSF (:102-106); each chunk's RLdecon call would also
    # deskew / rotate it (:240-247), but only its first output, the deconvolved chunk, is kept
    if o["Deskew"] and not o["Rotate"]:
        raise NotImplementedError("Deskew without Rotate: each chunk's RLdecon call would run deskewFrame3D "
                                  "with 'interpMethod', which its inputParser does not accept (the reference "
                                  "errors as written)")
    ctx = o["ctx"]
    bg = 99.0 if o["Background"] is None or np.size(o["Background"]) == 0 else float(o["Background"])   # :81-83
    erosion = int(o["EdgeErosion"])
    if o["ErodeMaskfile"] and os.path.exists(o["ErodeMaskfile"]):
        erosion = 0
    decon_path = os.path.dirname(deconFullpath)
    fsname = os.path.splitext(os.path.basename(frameFullpath))[0]
    psf, cpsf = _runner_psfs(psfFullpath, decon_path, dz, o, ctx)
    if str(frameFullpath).rstrip("/").endswith(".zarr"):
        im = Z.readzarr(frameFullpath, pinned=True)
    else:
        im = T.readtiff(frameFullpath, pinned=True)
    if im.ndim == 2:
        im = im[:, :, None]
    if o["flipZstack"]:
        im = np.asfortranarray(im[:, :, ::-1])
    border = border_size(np.asarray(psf).shape[:3] + (1,) * (3 - np.asarray(psf).ndim))
    bs = tuple(int(v) for v in o["batchSize"])
    bb, rb, _ = zarr_chunk_coordinates(im.shape, batch_size=bs, block_size=bs, same_batch_size=False, border=border)
    keep = [not region_masked_out(o["maskFullpaths"], r) for r in rb]
    bb, rb = bb[keep], rb[keep]
    chunks, boxes = [], []
    for b, r in zip(bb, rb):
        chunks.append(np.asfortranarray(im[b[0] - 1:b[3], b[1] - 1:b[4], b[2] - 1:b[5]]))
        boxes.append([*(r[:3] - b[:3] + 1), *(r[3:] - b[:3] + 1)])
    outs = _decon_chunks(chunks, boxes, cpsf, o, ctx, bg) if chunks else []
    out = np.zeros(im.shape, np.uint16 if o["save16bit"] else np.float32, order="F")
    for r, ob in zip(rb, outs):
        out[r[0] - 1:r[3], r[1] - 1:r[4], r[2] - 1:r[5]] = ob
    if erosion > 0:                                                                     # :146-168, 267-270
        mp = os.path.join(decon_path, "Masks", f"{fsname}_eroded.tif")
        if o["SaveMaskfile"] and os.path.exists(mp):       # the common mask saved for this name (:149-157)
            out *= (T.readtiff(mp) > 0).reshape(out.shape, order="F")
        else:
            mask = edge_erosion_mask(im, erosion, out=out, ctx=ctx)
            if o["SaveMaskfile"]:                                                       # :160-164
                os.makedirs(os.path.dirname(mp), exist_ok=True)
                tmp = os.path.join(os.path.dirname(mp), f"{fsname}_eroded_{o['uuid'] or os.getpid()}.tif")
                T.writetiff(mask.astype(np.uint8), tmp)
                os.replace(tmp, mp)
    if o["ErodeMaskfile"] and os.path.exists(o["ErodeMaskfile"]):
        out *= (T.readtiff(o["ErodeMaskfile"]) > 0).reshape(out.shape, order="F").astype(out.dtype)
    os.makedirs(decon_path or ".", exist_ok=True)
    if o["saveZarr"]:
        tmp = f"{os.path.splitext(deconFullpath)[0]}_{o['uuid'] or os.getpid()}.zarr"
        Z.writezarr(out, tmp, overwrite=True)
        if os.path.isdir(deconFullpath):
            shutil.rmtree(deconFullpath)
        os.replace(tmp, deconFullpath)
    else:
        T.writetiff(out, deconFullpath)
    mip_dir = os.path.join(decon_path, "MIPs")
    os.makedirs(mip_dir, exist_ok=True)
    T.writetiff(out.max(axis=2), os.path.join(mip_dir, f"{fsname}_MIP_z.tif"))
    return out


def RLdecon_large_in_place(frameFullpath, psfFullpath, deconPath, xyPixelSize, dz, **kw):
    """RLdecon_large_in_place(frameFullpath, xyPixelSize, dz, deconPath, PSF, ...)
    (decon/RLdecon_large_in_place.m:1-277 with RLdecon_for_zarr_block.m:101-171) for Zarr input: the
    output ``<deconPath>/<name>.zarr`` is skipped when it exists, else built in a temporary array and
    renamed; batches of the same size (``sameBatchSize``) with ``round((size(psf) + 10) / 2)`` borders
    are read from the input region by region, deconvolved as RLdecon would (EdgeErosion per batch, as
    RLdecon applies it) ``groupSize`` batches per batched call, and their regions written into the
    output chunk by chunk; regions that ``maskFullpaths`` masks out are written as zeros without
    deconvolution.  Batches run in tasks of ``taskSize`` (:192-197) whose completion is flagged under
    ``<deconPath>/zarr_flag/<name>_<uuid>/`` (:164-167, :217-221), so a second call with the same
    ``uuid`` resumes at the first unfinished task; at the end the temporary array is renamed, the
    flags removed (:272-280) and the y/x/z MIPs written (XR_MIP_zarr, :283-289).  The job
    distribution over a cluster is replaced by one process per GPU.  Returns the output path."""
    from . import zarrio as Z
    o = _runner_options("RLdecon_large_in_place", dict(
        save16bit=True, Rotate=False, Deskew=False, SkewAngle=-32.45, flipZstack=False, Background=None,
        dzPSF=0.1, DeconIter=15, EdgeErosion=0, dampFactor=1.0, scaleFactor=None, deconOffset=0.0,
        maskFullpaths=(), RLMethod="simplified", wienerAlpha=0.005, OTFCumThresh=0.9, hannWinBounds=(0.8, 1.0),
        skewed=None, fixIter=True, errThresh=None, batchSize=(1024, 1024, 1024), blockSize=(256, 256, 256),
        largeFile=False, largeMethod="inplace", parseCluster=False, parseParfor=False, jobLogDir="",
        cpusPerTask=8, uuid="", maxTrialNum=3, unitWaitTime=1, debug=False, psfGen=True, useGPU=True,
        GPUJob=False, ctx=None, groupSize=8), kw)
    # flipZstack is passed on to RLdecon_for_zarr_block, which parses it and never uses it (:27, :54);
    # Deskew only sets the dz ratio of the border PSF (:122-126): the blocks run without it (:137-138)
    ctx = o["ctx"]
    bg = 0.0 if o["Background"] is None or np.size(o["Background"]) == 0 else float(o["Background"])
    fsname = os.path.splitext(os.path.basename(str(frameFullpath).rstrip("/")))[0]
    out_path = os.path.join(deconPath, f"{fsname}.zarr")
    if os.path.isdir(out_path):                                                   # :102-105
        return out_path
    os.makedirs(deconPath, exist_ok=True)
    uid = str(o["uuid"] or os.getpid())
    tmp_path = f"{out_path}_{uid}"
    psf, cpsf = _runner_psfs(psfFullpath, deconPath, dz, o, ctx)
    im_size, _, in_dt = Z.getZarrInfo(frameFullpath)
    border = border_size(np.asarray(psf).shape[:3] + (1,) * (3 - np.asarray(psf).ndim))
    bb, rb, _ = zarr_chunk_coordinates(im_size, batch_size=tuple(int(v) for v in o["batchSize"]),
                                       block_size=tuple(int(v) for v in o["blockSize"]), same_batch_size=True,
                                       border=border)
    order = np.lexsort(tuple(np.asarray(bb)[:, ::-1].T) + (np.prod(bb[:, 3:] - bb[:, :3] + 1, axis=1),))
    bb, rb = bb[order], rb[order]                                                 # sortrows by size, then box
    out_dt = np.uint16 if o["save16bit"] else np.float32
    bs = tuple(int(min(a, b)) for a, b in zip(o["blockSize"], im_size))
    if not os.path.isdir(tmp_path):
        _create_empty_zarr(tmp_path, im_size, bs, out_dt)
    # tasks of taskSize batches (:192-197), each flagged when its regions are written (:217-221), so that
    # a second call with the same uuid resumes at the first unflagged task
    n = len(bb)
    task = 20
    if (o["parseCluster"] or o["GPUJob"] or str(o["RLMethod"]) == "omw") and n > 200:
        task = max(100, int(_round_half_away(n / 5000)))
    flag_dir = os.path.join(deconPath, "zarr_flag", f"{fsname}_{uid}")
    os.makedirs(flag_dir, exist_ok=True)
    g = max(1, int(o["groupSize"]))
    for t0 in range(0, n, task):
        t1 = min(n, t0 + task)
        flag = os.path.join(flag_dir, f"blocks_{t0 + 1}_{t1}.mat")
        if os.path.exists(flag):
            continue
        for s0 in range(t0, t1, g):
            s1 = min(t1, s0 + g)
            chunks, boxes, regions = [], [], []
            for b, r in zip(bb[s0:s1], rb[s0:s1]):
                if region_masked_out(o["maskFullpaths"], r):              # RLdecon_for_zarr_block.m:111-128
                    Z.writezarr_region(np.zeros(tuple(r[3:] - r[:3] + 1), out_dt, order="F"), tmp_path, list(r))
                    continue
                chunks.append(Z.readzarr(frameFullpath, inputBbox=list(b), pinned=True))
                boxes.append([*(r[:3] - b[:3] + 1), *(r[3:] - b[:3] + 1)])
                regions.append(r)
            outs = _decon_chunks(chunks, boxes, cpsf, o, ctx, bg, o["EdgeErosion"]) if chunks else []
            for r, ob in zip(regions, outs):
                Z.writezarr_region(ob, tmp_path, list(r))
        open(flag, "wb").close()
    if os.path.isdir(out_path):                                                   # :272-280
        shutil.rmtree(out_path)
    os.replace(tmp_path, out_path)
    shutil.rmtree(flag_dir, ignore_errors=True)
    zarr_mips(out_path, os.path.join(deconPath, "MIPs"), bs[2])                   # XR_MIP_zarr, axis [1 1 1]
    return out_path


def zarr_mips(path, mip_dir, slab_z=256):
    """XR_MIP_zarr(path, 'axis', [1 1 1]) (io/XR_MIP_zarr.m:56-67): the y, x and z maximum projections
    of a Zarr array written as ``<mip_dir>/<name>_MIP_{y,x,z}.tif`` (each skipped when it exists),
    reading the array in z-slabs of ``slab_z`` planes."""
    from . import tiff as T
    from . import zarrio as Z
    fsname = os.path.splitext(os.path.basename(str(path).rstrip("/")))[0]
    names = [os.path.join(mip_dir, f"{fsname}_MIP_{a}.tif") for a in "yxz"]
    if all(os.path.exists(f) for f in names):
        return names
    (ny, nx, nz), _, dt = Z.getZarrInfo(path)
    my = np.empty((nx, nz), dt, order="F")
    mx = np.empty((ny, nz), dt, order="F")
    mz = None
    for z0 in range(0, nz, max(1, int(slab_z))):
        z1 = min(nz, z0 + max(1, int(slab_z)))
        v = Z.readzarr(path, inputBbox=[1, 1, z0 + 1, ny, nx, z1])
        my[:, z0:z1] = v.max(axis=0)
        mx[:, z0:z1] = v.max(axis=1)
        mz = v.max(axis=2) if mz is None else np.maximum(mz, v.max(axis=2))
    os.makedirs(mip_dir, exist_ok=True)
    for f, m in zip(names, (my, mx, mz)):
        if not os.path.exists(f):
            T.writetiff(np.asfortranarray(m), f)
    return names


def _create_empty_zarr(path, shape, chunks, dtype):
    """An order-F, zlib, fill-value-0 array with no chunk files yet (createzarr's role); "/" chunk keys
    when it has more than 10000 chunks, else "." (RLdecon_large_in_place.m:186-191)."""
    import json
    if os.path.isdir(path):
        shutil.rmtree(path)
    os.makedirs(path)
    meta = {"chunks": [int(c) for c in chunks], "compressor": {"id": "zlib", "level": 1},
            "dimension_separator": "/" if np.prod(-(-np.asarray(shape) // np.asarray(chunks))) > 10000 else ".",
            "dtype": np.dtype(dtype).newbyteorder("<").str, "fill_value": 0,
            "filters": None, "order": "F", "shape": [int(v) for v in shape], "zarr_format": 2}
    with open(os.path.join(path, ".zarray"), "w") as f:
        json.dump(meta, f)


def shard(n_items, rank, world):
    """Indices of ``n_items`` independent chunks / requests owned by ``rank`` of ``world`` replicas
    (round robin).  The path has no exchange step, so replicas need no data-path collective."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return list(range(rank, int(n_items), world))
