"""The in-place large-file runner (RLdecon_large_in_place) on a Zarr volume: region by region, the
same numbers as deconvolving each batch of the chunk grid and pasting its region."""
import os

import numpy as np
import pytest

from petakit5d_b200 import chunking as K
from petakit5d_b200 import decon as D
from petakit5d_b200 import psfgen as P
from petakit5d_b200 import synth
from petakit5d_b200 import tiff as T
from petakit5d_b200 import zarrio as Z

pytestmark = pytest.mark.gpu


def test_in_place_runner_matches_batch_composition(tmp_path):
    psf_true = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((130, 100, 60), 120, psf_true, seed=21)
    bead = synth.measured_psf((32, 32, 41), sigma_xy=1.3, sigma_z=3.0, seed=22)
    zin = str(tmp_path / "raw.zarr")
    Z.writezarr(vol, zin, blockSize=(32, 32, 32))
    pfn = str(tmp_path / "psf.tif")
    T.writetiff(bead, pfn)
    out = K.RLdecon_large_in_place(zin, pfn, str(tmp_path / "decon"), 0.108, 0.3, DeconIter=3,
                                   batchSize=(64, 64, 64), blockSize=(32, 32, 32), Background=100, EdgeErosion=2,
                                   groupSize=3)
    assert out.endswith("raw.zarr") and os.path.isdir(out)
    got = Z.readzarr(out)
    g = P.psf_gen_new(bead, 0.1, 0.3)
    border = K.border_size(P.rldecon_psf_crop(g, g.shape, "simplified").shape)
    cpsf = P.psf_gen_new(bead, 0.1, 0.3 * np.sin(np.radians(32.45)))
    cpsf = P.rldecon_psf_crop(cpsf, cpsf.shape, "simplified")
    bb, rb, _ = K.zarr_chunk_coordinates(vol.shape, batch_size=(64, 64, 64), block_size=(32, 32, 32),
                                         same_batch_size=True, border=border)
    ref = np.zeros(vol.shape, np.uint16, order="F")
    for b, r in zip(bb, rb):
        c = np.asfortranarray(vol[b[0] - 1:b[3], b[1] - 1:b[4], b[2] - 1:b[5]])
        cp = P.rldecon_psf_crop(cpsf, c.shape, "omw")
        p32 = cp / np.float32(cp.sum(dtype=np.float32))
        box = [*(r[:3] - b[:3] + 1), *(r[3:] - b[:3] + 1)]
        j = D.decon_lucy_function(c, p32, 3, Background=100, bbox=box, EdgeErosion=2)[0]
        ref[r[0] - 1:r[3], r[1] - 1:r[4], r[2] - 1:r[5]] = j
    assert len(bb) > 4
    np.testing.assert_array_equal(got, ref)
    # the output exists now: a second call returns at once
    assert K.RLdecon_large_in_place(zin, pfn, str(tmp_path / "decon"), 0.108, 0.3) == out


def test_in_place_runner_skips_masked_regions(tmp_path):
    psf_true = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((130, 100, 60), 120, psf_true, seed=23)
    bead = synth.measured_psf((32, 32, 41), sigma_xy=1.3, sigma_z=3.0, seed=24)
    zin = str(tmp_path / "raw.zarr")
    Z.writezarr(vol, zin, blockSize=(32, 32, 32))
    pfn = str(tmp_path / "psf.tif")
    T.writetiff(bead, pfn)
    kw = dict(DeconIter=2, batchSize=(64, 64, 64), blockSize=(32, 32, 32), Background=100, groupSize=3)
    full = Z.readzarr(K.RLdecon_large_in_place(zin, pfn, str(tmp_path / "a"), 0.108, 0.3, **kw))
    xy = np.ones((130, 100), np.uint8)
    xy[:, 64:] = 0
    paths = []
    for name, m in (("xy", xy), ("xz", np.ones((100, 60), np.uint8)), ("yz", np.ones((130, 60), np.uint8))):
        paths.append(str(tmp_path / f"m_{name}.zarr"))
        Z.writezarr(m, paths[-1], blockSize=(32, 32, 1))
    got = Z.readzarr(K.RLdecon_large_in_place(zin, pfn, str(tmp_path / "b"), 0.108, 0.3, maskFullpaths=paths, **kw))
    g = P.psf_gen_new(bead, 0.1, 0.3)
    border = K.border_size(P.rldecon_psf_crop(g, g.shape, "simplified").shape)
    _, rb, _ = K.zarr_chunk_coordinates(vol.shape, batch_size=(64, 64, 64), block_size=(32, 32, 32),
                                        same_batch_size=True, border=border)
    ref = full.copy(order="F")
    skipped = 0
    for r in rb:
        if K.region_masked_out(paths, r):
            ref[r[0] - 1:r[3], r[1] - 1:r[4], r[2] - 1:r[5]] = 0
            skipped += 1
    assert 0 < skipped < len(rb)
    np.testing.assert_array_equal(got, ref)
