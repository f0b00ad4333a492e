"""The large-file runner (RLdecon_large_in_memory) for TIFF files and its bwdist edge erosion."""
import os

import numpy as np
import pytest

from oracle import chunking as OC
from petakit5d_b200 import chunking as K
from petakit5d_b200 import decon as D
from petakit5d_b200 import psfgen as P
from petakit5d_b200 import synth
from petakit5d_b200 import tiff as T

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("E", [1, 3, 8])
@pytest.mark.parametrize("dtype", [np.uint16, np.float32])
def test_edge_erosion_mask_matches_exact_edt(E, dtype):
    rng = np.random.default_rng(E)
    im = (rng.random((37, 45, 23)) > 0.03).astype(dtype) * rng.integers(1, 500, (37, 45, 23)).astype(dtype)
    im[5:12, 20:30, 8:15] = 0                      # a hole well inside
    out = (rng.random(im.shape) * 1000).astype(np.float32, order="F")
    ref_out = out.copy(order="F")
    m = K.edge_erosion_mask(im, E, out=out)
    ref = OC.edt_erosion_mask(im, E)
    np.testing.assert_array_equal(m, ref)
    np.testing.assert_array_equal(out, ref_out * ref)


@pytest.mark.parametrize("method", ["simplified", "omw"])
def test_large_runner_tiff_matches_chunked_composition(tmp_path, method):
    psf_true = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((150, 130, 64), 150, psf_true, seed=11)
    bead = synth.measured_psf((32, 32, 41), sigma_xy=1.3, sigma_z=3.0, seed=12)
    fin, pfn = str(tmp_path / "raw.tif"), str(tmp_path / "psf.tif")
    T.writetiff(vol, fin)
    T.writetiff(bead, pfn)
    fout = str(tmp_path / "decon" / "raw.tif")
    out = K.RLdecon_large_in_memory(fin, pfn, fout, 0.108, 0.3, RLMethod=method, DeconIter=3,
                                    batchSize=(64, 64, 64), EdgeErosion=4, OTFCumThresh=0.6)
    assert os.path.exists(fout) and os.path.exists(os.path.join(tmp_path, "decon", "MIPs", "raw_MIP_z.tif"))
    np.testing.assert_array_equal(T.readtiff(fout), out)
    # the same, composed: chunk grid, per-chunk decon with the region crop, paste, erosion
    cpsf = P.psf_gen_new(bead, 0.1, 0.3 * np.sin(np.radians(32.45)))
    if method != "omw":
        cpsf = P.rldecon_psf_crop(cpsf, cpsf.shape, "simplified")
    g = P.psf_gen_new(bead, 0.1, 0.3)
    border = K.border_size(P.rldecon_psf_crop(g, g.shape, "simplified").shape)
    bb, rb, _ = K.zarr_chunk_coordinates(vol.shape, batch_size=(64, 64, 64), block_size=(64, 64, 64),
                                         same_batch_size=False, border=border)
    ref = np.zeros(vol.shape, np.uint16, order="F")
    from petakit5d_b200 import backprojector as B
    for b, r in zip(bb, rb):
        c = np.asfortranarray(vol[b[0] - 1:b[3], b[1] - 1:b[4], b[2] - 1:b[5]])
        cp = P.rldecon_psf_crop(cpsf, c.shape, "omw")
        p32 = cp / np.float32(cp.sum(dtype=np.float32))
        box = [*(r[:3] - b[:3] + 1), *(r[3:] - b[:3] + 1)]
        if method == "omw":
            bp = P.rldecon_psf_crop(B.omw_backprojector_generation(cp, 0.005, None, OTFCumThresh=0.6)[0], c.shape, "omw")
            j, _ = D.decon_lucy_omw_function(c, p32, bp, 3, Background=99, bbox=box)
        else:
            j = D.decon_lucy_function(c, p32, 3, Background=99, bbox=box)[0]
        ref[r[0] - 1:r[3], r[1] - 1:r[4], r[2] - 1:r[5]] = j
    ref = ref * OC.edt_erosion_mask(vol, 4).astype(np.uint16)
    assert len(bb) > 4
    np.testing.assert_array_equal(out, ref)


def _proj_masks(tmp_path, shape, x_cut):
    """xy / xz / yz masks (RLdecon_large_in_memory.m:31) that empty every x >= x_cut."""
    from petakit5d_b200 import zarrio as Z
    ny, nx, nz = shape
    xy = np.ones((ny, nx), np.uint8)
    xy[:, x_cut:] = 0
    xz = np.ones((nx, nz), np.uint8)
    xz[x_cut:, :] = 0
    paths = []
    for name, m in (("xy", xy), ("xz", xz), ("yz", np.ones((ny, nz), np.uint8))):
        paths.append(str(tmp_path / f"m_{name}.zarr"))
        Z.writezarr(m, paths[-1], blockSize=(64, 64, 1))
    return paths


def test_large_runner_zarr_io_and_masks(tmp_path):
    from petakit5d_b200 import zarrio as Z
    psf_true = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((150, 130, 64), 150, psf_true, seed=13)
    bead = synth.measured_psf((32, 32, 41), sigma_xy=1.3, sigma_z=3.0, seed=14)
    fin, zin, pfn = str(tmp_path / "raw.tif"), str(tmp_path / "raw.zarr"), str(tmp_path / "psf.tif")
    T.writetiff(vol, fin)
    Z.writezarr(vol, zin, blockSize=(64, 64, 32))
    T.writetiff(bead, pfn)
    kw = dict(DeconIter=2, batchSize=(64, 64, 64), EdgeErosion=4)
    full = K.RLdecon_large_in_memory(fin, pfn, str(tmp_path / "a" / "raw.tif"), 0.108, 0.3, **kw)
    paths = _proj_masks(tmp_path, vol.shape, 70)
    zout = str(tmp_path / "b" / "raw.zarr")
    got = K.RLdecon_large_in_memory(zin, pfn, zout, 0.108, 0.3, saveZarr=True, maskFullpaths=paths, **kw)
    np.testing.assert_array_equal(Z.readzarr(zout), got)
    g = P.psf_gen_new(bead, 0.1, 0.3)
    border = K.border_size(P.rldecon_psf_crop(g, g.shape, "simplified").shape)
    _, rb, _ = K.zarr_chunk_coordinates(vol.shape, batch_size=(64, 64, 64), block_size=(64, 64, 64),
                                        same_batch_size=False, border=border)
    ref = full.copy(order="F")
    skipped = 0
    for r in rb:
        if K.region_masked_out(paths, r):
            ref[r[0] - 1:r[3], r[1] - 1:r[4], r[2] - 1:r[5]] = 0
            skipped += 1
    assert 0 < skipped < len(rb)
    np.testing.assert_array_equal(got, ref)


def test_large_runner_deskew_rotate_sets_the_border_psf_only(tmp_path):
    psf_true = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((150, 130, 64), 150, psf_true, seed=15)
    bead = synth.measured_psf((32, 32, 41), sigma_xy=1.3, sigma_z=3.0, seed=16)
    fin, pfn = str(tmp_path / "raw.tif"), str(tmp_path / "psf.tif")
    T.writetiff(vol, fin)
    T.writetiff(bead, pfn)
    out = K.RLdecon_large_in_memory(fin, pfn, str(tmp_path / "d" / "raw.tif"), 0.108, 0.3, DeconIter=2,
                                    batchSize=(64, 64, 64), EdgeErosion=0, Deskew=True, Rotate=True)
    cpsf = P.psf_gen_new(bead, 0.1, 0.3 * np.sin(np.radians(32.45)))
    cpsf = P.rldecon_psf_crop(cpsf, cpsf.shape, "simplified")
    g = P.psf_gen_new(bead, 0.1, 0.3 * np.sin(np.radians(-32.45)))        # sind(SkewAngle), :102-106
    border = K.border_size(P.rldecon_psf_crop(g, g.shape, "simplified").shape)
    bb, rb, _ = K.zarr_chunk_coordinates(vol.shape, batch_size=(64, 64, 64), block_size=(64, 64, 64),
                                         same_batch_size=False, border=border)
    ref = np.zeros(vol.shape, np.uint16, order="F")
    for b, r in zip(bb, rb):
        c = np.asfortranarray(vol[b[0] - 1:b[3], b[1] - 1:b[4], b[2] - 1:b[5]])
        cp = P.rldecon_psf_crop(cpsf, c.shape, "omw")
        p32 = cp / np.float32(cp.sum(dtype=np.float32))
        box = [*(r[:3] - b[:3] + 1), *(r[3:] - b[:3] + 1)]
        ref[r[0] - 1:r[3], r[1] - 1:r[4], r[2] - 1:r[5]] = D.decon_lucy_function(c, p32, 2, Background=99, bbox=box)[0]
    np.testing.assert_array_equal(out, ref)


def test_large_runner_reuses_a_saved_common_mask(tmp_path):
    """RLdecon_large_in_memory.m:149-164: with SaveMaskfile, an existing Masks/<name>_eroded.tif (saved
    for another channel or time point) is applied instead of a mask computed from this frame."""
    psf_true = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((150, 130, 64), 150, psf_true, seed=17)
    bead = synth.measured_psf((32, 32, 41), sigma_xy=1.3, sigma_z=3.0, seed=18)
    fin, pfn = str(tmp_path / "raw.tif"), str(tmp_path / "psf.tif")
    T.writetiff(vol, fin)
    T.writetiff(bead, pfn)
    plain = K.RLdecon_large_in_memory(fin, pfn, str(tmp_path / "a" / "raw.tif"), 0.108, 0.3, DeconIter=2,
                                      batchSize=(64, 64, 64), EdgeErosion=0)
    common = np.zeros(vol.shape, np.uint8, order="F")
    common[20:120, 10:100, 5:60] = 1
    os.makedirs(tmp_path / "b" / "Masks")
    T.writetiff(common, str(tmp_path / "b" / "Masks" / "raw_eroded.tif"))
    out = K.RLdecon_large_in_memory(fin, pfn, str(tmp_path / "b" / "raw.tif"), 0.108, 0.3, DeconIter=2,
                                    batchSize=(64, 64, 64), EdgeErosion=4, SaveMaskfile=True)
    np.testing.assert_array_equal(out, plain * common.astype(bool))
