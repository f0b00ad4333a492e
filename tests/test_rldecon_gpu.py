"""RLdecon drop-in (per-file driver): files in, files out, every step on the GPU, and the same
numbers as calling the steps one by one."""
import os

import numpy as np
import pytest

from petakit5d_b200 import backprojector as B
from petakit5d_b200 import decon as D
from petakit5d_b200 import deskew as G
from petakit5d_b200 import psfgen as P
from petakit5d_b200 import synth
from petakit5d_b200 import tiff as T
from petakit5d_b200 import zarrio as Z
from petakit5d_b200.rldecon import RLdecon

pytestmark = pytest.mark.gpu


def _files(tmp_path):
    psf_true = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((96, 80, 48), 60, psf_true, seed=5)
    bead = synth.measured_psf((32, 32, 41), sigma_xy=1.3, sigma_z=3.0, seed=6)
    raw = str(tmp_path / "data" / "frame_CamA.tif")
    pfn = str(tmp_path / "psf" / "psf_CamA.tif")
    T.writetiff(vol, raw)
    T.writetiff(bead, pfn)
    return vol, bead, raw, pfn


def test_rldecon_omw_with_deskew_rotate(tmp_path):
    vol, bead, raw, pfn = _files(tmp_path)
    out = str(tmp_path / "data" / "matlab_decon" / "frame_CamA.tif")
    J, ds, dsr = RLdecon(raw, out, pfn, 0.108, 0.3, 0.1, Background=100, DeconIter=2, RLMethod="omw",
                         wienerAlpha=0.005, OTFCumThresh=0.6, Deskew=True, Rotate=True, Reverse=True)
    dpath = os.path.dirname(out)
    assert os.path.exists(out) and os.path.exists(os.path.join(dpath, "DSR", "frame_CamA.tif"))
    assert os.path.exists(os.path.join(dpath, "MIPs", "frame_CamA_MIP_z.tif"))
    assert os.path.exists(os.path.join(dpath, "DSR", "MIPs", "frame_CamA_MIP_z.tif"))
    gen = os.path.join(dpath, "psfgen", "psf_CamA_omw.tif")
    bpf = os.path.join(dpath, "psfgen", "psf_CamA_back_projector_alpha_0.005000_otf_cum_thresh_0.600000.tif")
    assert os.path.exists(gen) and os.path.exists(bpf)
    # the same steps one by one
    psf = P.rldecon_psf_crop(P.psf_gen_new(bead, 0.1, 0.3 * np.sin(np.radians(32.45))), vol.shape, "omw")
    np.testing.assert_array_equal(T.readtiff(gen), psf)
    bp = B.omw_backprojector_generation(psf, 0.005, None, OTFCumThresh=0.6)[0]
    np.testing.assert_array_equal(T.readtiff(bpf), bp)
    p32 = psf / np.float32(psf.sum(dtype=np.float32))
    ref, _ = D.decon_lucy_omw_function(vol, p32, bp, 2, Background=100)
    np.testing.assert_array_equal(J, ref)
    np.testing.assert_array_equal(T.readtiff(out), ref)
    ref_dsr = G.deskewRotateFrame3D(ref, 32.45, 0.3, 0.108, reverse=True, save16bit=True)
    np.testing.assert_array_equal(dsr, ref_dsr)
    np.testing.assert_array_equal(T.readtiff(os.path.join(dpath, "DSR", "frame_CamA.tif")), ref_dsr)
    np.testing.assert_array_equal(T.readtiff(os.path.join(dpath, "MIPs", "frame_CamA_MIP_z.tif")), ref.max(axis=2))
    # a second call finds the outputs and the cached PSF files and does not redo the work
    mtime = os.path.getmtime(out)
    J2, _, _ = RLdecon(raw, out, pfn, 0.108, 0.3, 0.1, Background=100, DeconIter=2, OTFCumThresh=0.6)
    assert os.path.getmtime(out) == mtime and J2 is None


def test_rldecon_simplified_crops_the_psf_and_the_output(tmp_path):
    vol, bead, raw, pfn = _files(tmp_path)
    out = str(tmp_path / "o" / "frame_CamA.tif")
    bbox = [5, 7, 3, 90, 70, 38]
    J, _, _ = RLdecon(raw, out, pfn, 0.108, 0.3, 0.1, Background=100, DeconIter=3, RLMethod="simplified",
                      deconBbox=bbox, save16bit=False, mipAxis=[1, 1, 1])
    psf = P.psf_gen_new(bead, 0.1, 0.3 * np.sin(np.radians(32.45)))
    psf = P.rldecon_psf_crop(psf, vol.shape, "simplified")
    p32 = psf / np.float32(psf.sum(dtype=np.float32))
    ref = D.decon_lucy_function(vol, p32, 3, Background=100, bbox=bbox, save16bit=False)[0]
    assert J.shape == (86, 64, 36)
    np.testing.assert_array_equal(J, ref)
    for ax in "yxz":
        assert os.path.exists(os.path.join(os.path.dirname(out), "MIPs", f"frame_CamA_MIP_{ax}.tif"))


def test_rldecon_existing_erosion_mask(tmp_path):
    vol, bead, raw, pfn = _files(tmp_path)
    mask = np.ones(vol.shape, np.uint8)
    mask[:10] = 0
    mask[:, -7:] = 0
    mfn = str(tmp_path / "mask.zarr")
    Z.writezarr(mask, mfn, blockSize=(64, 64, 32))
    kw = dict(Background=100, DeconIter=3, RLMethod="simplified", EdgeErosion=6, save16bit=False)
    J, _, _ = RLdecon(raw, str(tmp_path / "a" / "frame_CamA.tif"), pfn, 0.108, 0.3, 0.1, ErodeMaskfile=mfn, **kw)
    psf = P.rldecon_psf_crop(P.psf_gen_new(bead, 0.1, 0.3 * np.sin(np.radians(32.45))), vol.shape, "simplified")
    p32 = psf / np.float32(psf.sum(dtype=np.float32))
    ref = D.decon_lucy_function(vol, p32, 3, Background=100, save16bit=False, EdgeErosion=0)[0]
    np.testing.assert_array_equal(J, ref * (mask > 0))               # RLdecon.m:382-385, 409-413
    # a mask file that does not exist: the decon function erodes the edges itself (:364)
    J2, _, _ = RLdecon(raw, str(tmp_path / "b" / "frame_CamA.tif"), pfn, 0.108, 0.3, 0.1,
                       ErodeMaskfile=str(tmp_path / "absent.zarr"), **kw)
    ref2 = D.decon_lucy_function(vol, p32, 3, Background=100, save16bit=False, EdgeErosion=6)[0]
    np.testing.assert_array_equal(J2, ref2)


def test_rldecon_zarr_input_and_output(tmp_path):
    vol, bead, raw, pfn = _files(tmp_path)
    zin = str(tmp_path / "data" / "frame_CamA.zarr")
    Z.writezarr(vol, zin, blockSize=(64, 64, 32))
    kw = dict(Background=100, DeconIter=2, RLMethod="omw", wienerAlpha=0.005, OTFCumThresh=0.6, Deskew=True,
              Rotate=True, Reverse=True)
    Jt, _, dt = RLdecon(raw, str(tmp_path / "t" / "frame_CamA.tif"), pfn, 0.108, 0.3, 0.1, **kw)
    out = str(tmp_path / "z" / "frame_CamA.zarr")
    Jz, _, dz = RLdecon(zin, out, pfn, 0.108, 0.3, 0.1, saveZarr=True, blockSize=[64, 64, 64], **kw)
    np.testing.assert_array_equal(Jz, Jt)
    np.testing.assert_array_equal(dz, dt)
    np.testing.assert_array_equal(Z.readzarr(out), Jt)
    dsr_fn = str(tmp_path / "z" / "DSR" / "frame_CamA.zarr")
    np.testing.assert_array_equal(Z.readzarr(dsr_fn), dt)
    assert os.path.exists(str(tmp_path / "z" / "DSR" / "MIPs" / "frame_CamA_MIP_z.tif"))
    # the deconvolved Zarr exists and the rotated one does not: it is read back and rotated (:420-428)
    import shutil
    shutil.rmtree(dsr_fn)
    J3, _, d3 = RLdecon(zin, out, pfn, 0.108, 0.3, 0.1, saveZarr=True, blockSize=[64, 64, 64], **kw)
    np.testing.assert_array_equal(J3, Jt)
    np.testing.assert_array_equal(d3, dt)
    np.testing.assert_array_equal(Z.readzarr(dsr_fn), dt)


def test_frame3d_saves_the_eroded_mask_and_uses_it(tmp_path):
    """XR_RLdeconFrame3D.m:205-231: the eroded mask of the raw data saved as Masks/<name>_eroded.zarr and
    used as ErodeMaskfile gives the result of RLdecon's own erosion."""
    from oracle.decon import mask_edge_erosion
    from petakit5d_b200.rldecon import XR_RLdeconFrame3D
    vol, bead, raw, pfn = _files(tmp_path)
    dpath = str(tmp_path / "out")
    kw = dict(Background=100, DeconIter=2, RLMethod="simplified", EdgeErosion=4, save16bit=False)
    XR_RLdeconFrame3D([raw], 0.108, 0.3, dpath, PSFfile=pfn, SaveMaskfile=True, **kw)
    m = Z.readzarr(os.path.join(dpath, "Masks", "frame_CamA_eroded.zarr"))
    np.testing.assert_array_equal(m.astype(bool), mask_edge_erosion(vol > 0, 4))
    J = T.readtiff(os.path.join(dpath, "frame_CamA.tif"))
    ref, _, _ = RLdecon(raw, str(tmp_path / "ref" / "frame_CamA.tif"), pfn, 0.108, 0.3, 0.1, **kw)
    np.testing.assert_array_equal(J, ref)
