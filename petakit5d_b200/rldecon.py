"""Per-file deconvolution driver: drop-in for microscopeDataProcessing/decon/RLdecon.m.

``RLdecon(inputFn, outputFn, PSFfn, xyPixelSize, dz, dzPSF, **options)`` follows RLdecon.m:1-571 for
TIFF files: the PSF is prepared with psf_gen_new and cached under ``<deconPath>/psfgen/`` (:207-281),
the OMW backprojector is generated or loaded from its cache file (:283-333), the volume is read
(:335-344), edge-tapered slice by slice when ``nTapering > 0`` (:351-357), deconvolved with
``decon_lucy_omw_function`` / ``decon_lucy_function`` and masked by an existing Zarr erosion mask
(``ErodeMaskfile``, :409-413) when one is given (:366-412), optionally deskewed and rotated
in one step (``deskewRotateFrame3D``, :487-491), and the results and their maximum projections are
written (:494-571).  Every compute step runs on the GPU through libpkdecon.so (the erosion-mask
multiply of the returned host result is one host pass, as in the reference); the files are read and
written by its TIFF / Zarr readers and writer.

Zarr input (``.zarr`` inputFn) and output (``saveZarr``, chunked by ``blockSize``) go through the
Zarr reader / writer; maximum projections stay TIFF, as in the reference.

Not built (each raises NotImplementedError): the 'original' (MATLAB's deconvlucy) and 'cudagen' methods, the separate deskew and rotate steps
(``DSRCombined=false``, deskew without rotation, objective-scan rotation: RLdecon.m:448-449,
:485-486 and :499-500 pass 'interpMethod' to deskewFrame3D / rotateFrame3D, whose inputParsers
accept only 'Interp' (pointDetection/src/deskewFrame3D.m:28-37, pointDetection/src/rotateFrame3D.m:26-35),
so those reference branches stop with MATLAB's unmatched-parameter error as written) and
resampling / cubic interpolation in the deskew.
"""
from __future__ import annotations

import math
import os
import shutil
import uuid as _uuid

import numpy as np

from . import backprojector as B
from . import decon as D
from . import deskew as G
from . import psfgen as P
from . import taper as TP
from . import tiff as T
from . import zarrio as Z

_NO_IMWARP = ("%s is not built: RLdecon.m passes it 'interpMethod', which its inputParser does not "
              "accept (only 'Interp'), so the reference branch errors as written")

_DEFAULTS = dict(rawdata=None, nTapering=0, save16bit=True, objectiveScan=False, Deskew=False, Rotate=False,
                 DSRCombined=True, Reverse=False, SkewAngle=32.45, flipZstack=False, interpMethod="linear",
                 Crop=False, xStepThresh=2.0, Background=None, Resample=None, DeconIter=15, RLMethod="omw",
                 wienerAlpha=0.005, OTFCumThresh=0.9, hannWinBounds=(0.8, 1.0), skewed=None, fixIter=True,
                 errThresh=None, saveZarr=False, blockSize=(256, 256, 256), dampFactor=1.0, scaleFactor=None,
                 deconOffset=0.0, EdgeErosion=0, ErodeMaskfile="", deconBbox=None, debug=False, saveStep=5,
                 useGPU=True, save3Dstack=(True, True, True), mipAxis=(0, 0, 1), psfGen=True, uuid="", ctx=None)


def _opts(kw):
    low = {k.lower(): k for k in _DEFAULTS}
    o = dict(_DEFAULTS)
    for k, v in kw.items():
        if k.lower() not in low:
            raise TypeError(f"RLdecon: unknown parameter {k!r}")
        o[low[k.lower()]] = v
    return o


def _move_into_place(write, final):
    """Write to a temporary name beside the target, then rename (the reference's tmp + movefile)."""
    root, ext = os.path.splitext(final)
    tmp = f"{root}_{_uuid.uuid4().hex[:8]}{ext or '.tif'}"
    write(tmp)
    if os.path.isdir(final):                         # movefile replaces an existing Zarr folder
        shutil.rmtree(final)
    os.replace(tmp, final)


def _read(fn, pinned=False):
    """readtiff / readzarr by extension (RLdecon.m:337-343, :423-428)."""
    if str(fn).endswith(".zarr"):
        return Z.readzarr(fn, pinned=pinned)
    return T.readtiff(fn, pinned=pinned)


def _size(fn):
    return Z.getZarrInfo(fn)[0] if str(fn).endswith(".zarr") else T.getImageSize(fn)


def _writer(o):
    """writezarr with the run's blockSize when saveZarr is set (:455-461, :514-517, :560-562), else writetiff."""
    if o["saveZarr"]:
        bs = tuple(int(v) for v in o["blockSize"])
        return lambda a, f: Z.writezarr(a, f, blockSize=bs)
    return lambda a, f: T.writetiff(a, f)


def _u16(a):
    a = np.asarray(a)
    if a.dtype == np.uint16:
        return a
    return np.clip(np.where(a >= 0, np.floor(a.astype(np.float64) + 0.5), 0), 0, 65535).astype(np.uint16)


def save_mip_frame(im, mip_fullname, axis=(0, 0, 1)):
    """saveMIP_frame (tools/MIP/saveMIP_frame.m): uint16 maximum projections along the flagged axes,
    written as ``<prefix>_MIP_{y,x,z}.tif``; skipped when the file already exists."""
    if os.path.exists(mip_fullname) or not any(axis):
        return
    os.makedirs(os.path.dirname(mip_fullname), exist_ok=True)
    im = _u16(im)
    prefix = mip_fullname[:-10]
    for d, lab in enumerate("yxz"):
        if axis[d]:
            mip = im.max(axis=d) if im.ndim > d else im
            _move_into_place(lambda f, m=mip: T.writetiff(m, f), f"{prefix}_MIP_{lab}.tif")


def _crop_to(a, im_size):
    """Crop an array larger than the data around its centre (RLdecon.m:260-265, :326-332)."""
    sz = np.array(a.shape[:3] + (1,) * (3 - a.ndim))
    im = np.array(tuple(im_size) + (1,) * (3 - len(im_size)))
    if np.any(sz > im):
        s = np.maximum(0, (sz - im) // 2)
        t = s + np.minimum(sz, im)
        a = a.reshape(tuple(sz))[s[0]:t[0], s[1]:t[1], s[2]:t[2]]
    return a


def RLdecon(inputFn, outputFn, PSFfn, xyPixelSize, dz, dzPSF, **kw):
    """[deconvolved, ds, dsr] = RLdecon(inputFn, outputFn, PSFfn, xyPixelSize, dz, dzPSF, ...)."""
    o = _opts(kw)
    ctx = o["ctx"]
    method = str(o["RLMethod"])
    if method in ("original", "cudagen"):
        raise NotImplementedError(f"RLMethod '{method}' is not built (the reference calls "
                                  f"{'deconvlucy' if method == 'original' else 'the undefined decon_lucy_cuda_function'})")
    if method not in ("omw", "simplified"):
        raise ValueError(f"unknown RLMethod {method!r}")
    # an existing erosion mask replaces the decon functions' own edge erosion (:364, :382-385, :409-413)
    use_exist_mask = o["EdgeErosion"] > 0 and bool(o["ErodeMaskfile"]) and os.path.exists(o["ErodeMaskfile"])
    skew = abs(float(o["SkewAngle"]))
    objective = bool(o["objectiveScan"])
    deskew, rotate, combined = bool(o["Deskew"]), bool(o["Rotate"]), bool(o["DSRCombined"])
    dz_ratio = math.sin(math.radians(skew)) if not objective else 1.0
    save16 = bool(o["save16bit"])
    s3 = o["save3Dstack"]
    save3d = [bool(s3)] * 3 if np.ndim(s3) == 0 or len(s3) == 1 else [bool(v) for v in s3]
    if inputFn:
        data_path, fsname = os.path.split(os.path.splitext(inputFn)[0])
    else:
        data_path, fsname = "", os.path.splitext(os.path.basename(outputFn))[0] if outputFn else "frame"
    if outputFn:
        decon_path, out_fsn = os.path.split(os.path.splitext(outputFn)[0])
    else:
        decon_path, out_fsn = os.path.join(data_path, "matlab_decon"), fsname
    if objective:
        deskew = False
        if rotate:
            raise NotImplementedError(_NO_IMWARP % "rotateFrame3D")
    if not deskew and rotate:
        deskew, combined = True, True
    if deskew and not combined:
        raise NotImplementedError(_NO_IMWARP % "deskewFrame3D")
    if deskew and not rotate:
        raise NotImplementedError(_NO_IMWARP % "deskewFrame3D")
    ext = ".zarr" if o["saveZarr"] else ".tif"                    # :126-130
    write = _writer(o)
    dsr_fn = os.path.join(decon_path, "DSR", f"{out_fsn}{ext}") if rotate else None
    if not rotate:
        save3d[2] = False
    save3d[1] = False
    exists = [bool(save3d[0] and outputFn and os.path.exists(outputFn)), True,
              bool(not rotate or (save3d[2] and os.path.exists(dsr_fn)))]

    rawdata = o["rawdata"]
    im_size = _size(inputFn) if rawdata is None else tuple(np.shape(rawdata)) + (1,) * (3 - np.ndim(rawdata))

    # ---- PSF (RLdecon.m:207-281) and backprojector (:283-333)
    psf = psf_b = None
    if isinstance(PSFfn, str) and PSFfn:
        psf_fsn, ext = os.path.splitext(os.path.basename(PSFfn))
        if ext not in (".tif", ".tiff"):
            raise NotImplementedError("only .tif PSF files are supported")
        psfgen_path = os.path.join(decon_path, "psfgen")
        psf_gen = bool(o["psfGen"])
        if psf_gen or inputFn or method == "omw":
            os.makedirs(psfgen_path, exist_ok=True)
        gen_fn = os.path.join(psfgen_path, f"{psf_fsn}_{method}.tif")
        if psf_gen and os.path.exists(gen_fn):
            psf = T.readtiff(gen_fn).astype(np.float32)
            psf_gen = False
        else:
            psf = T.readtiff(PSFfn).astype(np.float32)
        if psf_gen:
            psf = P.psf_gen_new(psf, dzPSF, dz * dz_ratio, 1.5, "masked", ctx=ctx)
            if method != "omw":
                psf = P.rldecon_psf_crop(psf, psf.shape, "simplified")
        psf = _crop_to(psf, im_size)
        if inputFn and not os.path.exists(gen_fn):
            _move_into_place(lambda f: T.writetiff(np.asarray(psf, np.float32), f), gen_fn)
        if method == "omw":
            a, t = float(o["wienerAlpha"]), float(o["OTFCumThresh"])
            bp_fn = os.path.join(psfgen_path, f"{psf_fsn}_back_projector_alpha_{a:0.6f}_otf_cum_thresh_{t:0.6f}.tif")
            if os.path.exists(bp_fn):
                psf_b = T.readtiff(bp_fn)
            else:
                psf_b, _, abs_c, mask = B.omw_backprojector_generation(psf, a, o["skewed"], OTFCumThresh=t,
                                                                       hannWinBounds=o["hannWinBounds"], ctx=ctx)
                _move_into_place(lambda f: T.writetiff(psf_b, f), bp_fn)
                _move_into_place(lambda f: T.writetiff(abs_c, f), os.path.join(psfgen_path, f"{psf_fsn}_OTF.tif"))
                _move_into_place(lambda f: T.writetiff(np.asarray(mask, np.uint8), f),
                                 os.path.join(psfgen_path, f"{psf_fsn}_OTF_mask_otf_cum_thresh_{t:0.6f}.tif"))
            psf_b = _crop_to(np.asarray(psf_b, np.float32), im_size)
    elif PSFfn is not None and not isinstance(PSFfn, str):
        raise TypeError("PSFfn must be a .tif file name")

    # ---- deconvolution (:335-412)
    deconvolved = None
    n_iter = int(o["DeconIter"])
    if not exists[0]:
        if rawdata is None:
            rawdata = _read(inputFn, pinned=True)
        if o["flipZstack"]:
            rawdata = np.asfortranarray(np.asarray(rawdata)[:, :, ::-1])
        if o["nTapering"] > 0:                   # soften the x-y borders (:351-357)
            nt = o["nTapering"]
            rawdata = TP.edgetaper_slices(rawdata, TP.fspecial_gaussian(int(nt) + 30, float(nt)), ctx=ctx)
        if n_iter > 0 and np.any(rawdata):
            scale = 1.0 if o["scaleFactor"] is None or np.size(o["scaleFactor"]) == 0 else float(o["scaleFactor"])
            p32 = np.asarray(psf, np.float32)
            p32 = p32 / np.float32(p32.sum(dtype=np.float32))
            debug_folder = "/tmp/"
            save_step = int(o["saveStep"])
            if o["debug"]:
                debug_folder = os.path.join(decon_path, f"{fsname}_debug")
                os.makedirs(debug_folder, exist_ok=True)
                save_step = min(save_step, n_iter)
            common = dict(Background=o["Background"], useGPU=True, save16bit=save16, dampFactor=o["dampFactor"],
                          scaleFactor=scale, deconOffset=o["deconOffset"], bbox=o["deconBbox"],
                          EdgeErosion=0 if use_exist_mask else o["EdgeErosion"], debug=o["debug"], debug_folder=debug_folder,
                          saveStep=save_step, ctx=ctx)
            if method == "omw":
                deconvolved = D.decon_lucy_omw_function(rawdata, p32, psf_b, n_iter, **common)[0]
            else:
                deconvolved = D.decon_lucy_function(rawdata, p32, n_iter, **common)[0]
            if use_exist_mask:
                mask = Z.readzarr(o["ErodeMaskfile"])
                if mask.shape != deconvolved.shape:
                    raise ValueError(f"ErodeMaskfile: mask size {mask.shape} differs from the result's "
                                     f"{deconvolved.shape}")
                deconvolved *= mask > 0
        else:
            deconvolved = np.asarray(rawdata)
            bb = o["deconBbox"]
            if bb is not None and len(bb):
                deconvolved = deconvolved[bb[0] - 1:bb[3], bb[1] - 1:bb[4], bb[2] - 1:bb[5]]
    elif deskew or rotate:
        deconvolved = _read(outputFn)
    rawdata = None

    # ---- deskew / rotate in one step (:487-491) and its output (:499-520)
    dsr = None
    if rotate and not exists[2]:
        vol = deconvolved if deconvolved.dtype in (np.uint16, np.float32) else deconvolved.astype(np.float32)
        dsr = G.deskewRotateFrame3D(vol, skew, dz, xyPixelSize, reverse=bool(o["Reverse"]), Crop=True,
                                    objectiveScan=objective, resampleFactor=o["Resample"],
                                    interpMethod=o["interpMethod"], xStepThresh=float(o["xStepThresh"]),
                                    save16bit=save16, ctx=ctx)
        dsr = _u16(dsr) if save16 else dsr.astype(np.float32)
        dsr_path = os.path.dirname(dsr_fn)
        save_mip_frame(dsr, os.path.join(dsr_path, "MIPs", f"{fsname}_MIP_z.tif"), o["mipAxis"])
        if save3d[2]:
            os.makedirs(dsr_path, exist_ok=True)
            _move_into_place(lambda f: write(dsr, f), dsr_fn)

    # ---- the deconvolved volume (:528-571)
    if not outputFn or not any(save3d) or exists[0]:
        return deconvolved, None, dsr
    if save16:
        deconvolved = _u16(deconvolved)
    if len(o["mipAxis"]) == 3 and any(o["mipAxis"]):
        save_mip_frame(deconvolved, os.path.join(decon_path, "MIPs", f"{fsname}_MIP_z.tif"), o["mipAxis"])
    if save3d[0]:
        os.makedirs(decon_path, exist_ok=True)
        _move_into_place(lambda f: write(deconvolved, f), outputFn)
    return deconvolved, None, dsr


_FRAME3D_DEFAULTS = dict(
    PSFfile="", Overwrite=False, save16bit=True, Rotate=False, Deskew=False, SkewAngle=-32.45, flipZstack=False,
    Reverse=True, Background=None, EdgeSoften=5, zEdgeSoften=2, dzPSF=0.1, DeconIter=15, EdgeErosion=8,
    ErodeMaskfile="", SaveMaskfile=False, RLMethod="simplified", wienerAlpha=0.005, OTFCumThresh=0.9,
    hannWinBounds=(0.8, 1.0), skewed=None, fixIter=False, errThresh=None, CPUMaxMem=500,
    batchSize=(1024, 1024, 1024), blockSize=(256, 256, 256), largeFile=False, largeMethod="inmemory",
    saveZarr=False, save3Dstack=(True, True, True), mipAxis=(0, 0, 1), dampFactor=1.0, scaleFactor=None,
    deconOffset=0.0, maskFullpaths=(), parseCluster=True, parseParfor=False, masterCompute=True, masterCPU=False,
    GPUJob=False, jobLogDir="../job_logs", cpusPerTask=4, uuid="", maxTrialNum=3, unitWaitTime=2, debug=False,
    saveStep=5, psfGen=True, mccMode=False, configFile="", GPUConfigFile="", ctx=None)


def XR_RLdeconFrame3D(frameFullpaths, xyPixelSize, dz, deconPath="", **kw):
    """XR_RLdeconFrame3D(frameFullpaths, xyPixelSize, dz, deconPath, ...)
    (decon/XR_RLdeconFrame3D.m:1-316): for each frame, skip a missing input or an existing result
    (unless ``Overwrite``); frames whose ``prod(size) * 4 B * 10`` exceeds ``CPUMaxMem`` GB (and every
    frame after one, as the reference keeps ``largeFile`` set) go to the large-file runner of
    ``largeMethod`` ('inplace' or 'inmemory', after which the call returns, as in the reference);
    the others to RLdecon, with the eroded mask of the raw data saved as
    ``<deconPath>/Masks/<name>_eroded.zarr`` and used as ``ErodeMaskfile`` when ``SaveMaskfile``
    (:205-231).  The Slurm / parfor job options are accepted; the work runs in this process."""
    import warnings
    from . import chunking as K
    from . import decon as D
    low = {k.lower(): k for k in _FRAME3D_DEFAULTS}
    o = dict(_FRAME3D_DEFAULTS)
    for k, v in kw.items():
        if k.lower() not in low:
            raise TypeError(f"XR_RLdeconFrame3D: unknown parameter {k!r}")
        o[low[k.lower()]] = v
    if isinstance(frameFullpaths, str):
        frameFullpaths = [frameFullpaths]
    uid = o["uuid"] or _uuid.uuid4().hex[:8]
    s3 = o["save3Dstack"]
    save3d = [bool(s3)] * 3 if np.ndim(s3) == 0 or len(s3) == 1 else [bool(v) for v in s3]
    save3d[1] = save3d[1] and bool(o["Deskew"])
    save3d[2] = save3d[2] and bool(o["Rotate"])
    large = bool(o["largeFile"])
    if not large and not any(save3d) and not any(np.asarray(o["mipAxis"]) > 0):
        raise ValueError("Either the 3D stack or the MIP for at least one axis needs to be saved!")
    ext_out = ".zarr" if o["saveZarr"] else ".tif"
    for frame in frameFullpaths:
        if not os.path.exists(frame):
            warnings.warn(f"{frame} does not exist! Skip it!")
            continue
        pathstr, name = os.path.split(str(frame).rstrip("/"))
        fsname = os.path.splitext(name)[0]
        dpath = deconPath or os.path.join(pathstr, "matlab_decon")
        os.makedirs(dpath, exist_ok=True)
        im_size = _size(frame)
        if np.prod(im_size) * 4 / 2 ** 30 * 10 > float(o["CPUMaxMem"]):
            large = True
        decon_fn = os.path.join(dpath, fsname + ext_out)
        dsr_fn = os.path.join(dpath, "DSR", fsname + ext_out)
        if os.path.exists(decon_fn) and not o["Overwrite"]:
            continue
        common = dict(save16bit=o["save16bit"], Deskew=o["Deskew"], SkewAngle=o["SkewAngle"],
                      Background=o["Background"], dzPSF=o["dzPSF"], DeconIter=o["DeconIter"], RLMethod=o["RLMethod"],
                      skewed=o["skewed"], wienerAlpha=o["wienerAlpha"], OTFCumThresh=o["OTFCumThresh"],
                      hannWinBounds=o["hannWinBounds"], fixIter=o["fixIter"], dampFactor=o["dampFactor"],
                      scaleFactor=o["scaleFactor"], deconOffset=o["deconOffset"], debug=o["debug"],
                      psfGen=o["psfGen"], ctx=o["ctx"])
        if not large:
            erode_fn = o["ErodeMaskfile"]
            if o["EdgeErosion"] > 0 and o["SaveMaskfile"]:                        # :205-231
                raw = _read(frame)
                if o["flipZstack"]:
                    raw = np.asfortranarray(np.asarray(raw)[:, :, ::-1])
                m = D.decon_mask_edge_erosion(raw, o["EdgeErosion"], ctx=o["ctx"])
                raw = None
                erode_fn = os.path.join(dpath, "Masks", f"{fsname}_eroded.zarr")
                tmp = os.path.join(dpath, "Masks", f"{fsname}_eroded_{uid}.zarr")
                Z.writezarr(m.astype(np.uint8), tmp, blockSize=tuple(int(v) for v in o["blockSize"]), overwrite=True)
                if os.path.isdir(erode_fn):
                    shutil.rmtree(erode_fn)
                os.replace(tmp, erode_fn)
            RLdecon(frame, decon_fn, o["PSFfile"], xyPixelSize, dz, o["dzPSF"], Rotate=o["Rotate"], DSRCombined=True,
                    Reverse=o["Reverse"], saveZarr=o["saveZarr"], blockSize=o["blockSize"], flipZstack=o["flipZstack"],
                    EdgeErosion=o["EdgeErosion"], ErodeMaskfile=erode_fn, errThresh=o["errThresh"],
                    saveStep=o["saveStep"], useGPU=o["GPUJob"], save3Dstack=save3d, mipAxis=o["mipAxis"],
                    **{k: v for k, v in common.items() if k != "dzPSF"})
            if (save3d[0] and os.path.exists(decon_fn)) or (save3d[2] and os.path.exists(dsr_fn)):
                continue
        method = str(o["largeMethod"]).lower()
        if method == "inplace":
            K.RLdecon_large_in_place(frame, o["PSFfile"], dpath, xyPixelSize, dz, flipZstack=o["flipZstack"],
                                     batchSize=o["batchSize"], blockSize=o["blockSize"], EdgeErosion=o["EdgeErosion"],
                                     maskFullpaths=o["maskFullpaths"], parseCluster=o["parseCluster"],
                                     parseParfor=o["parseParfor"], cpusPerTask=o["cpusPerTask"], GPUJob=o["GPUJob"],
                                     uuid=uid, **common)
            return
        if method == "inmemory":
            K.RLdecon_large_in_memory(frame, o["PSFfile"], decon_fn, xyPixelSize, dz, flipZstack=o["flipZstack"],
                                      EdgeErosion=o["EdgeErosion"], batchSize=o["batchSize"], saveZarr=o["saveZarr"],
                                      maskFullpaths=o["maskFullpaths"], useGPU=o["GPUJob"], uuid=uid, **common)
            return
