"""Edge taper on the GPU (pk_edgetaper) against the oracle restatement of edgetaper and
fspecial('gaussian') (RLdecon.m:351-357).

The library sums in float32 and the oracle in float64 through the FFT: single results within 1e-5
of the image's range, uint16 results within 1 level and at least 99.9% identical."""
import os

import numpy as np
import pytest

from oracle import edgetaper as OE
from petakit5d_b200 import _lib
from petakit5d_b200 import decon as D
from petakit5d_b200 import psfgen as P
from petakit5d_b200 import synth
from petakit5d_b200 import taper as TP
from petakit5d_b200 import tiff as T
from petakit5d_b200.rldecon import RLdecon

pytestmark = pytest.mark.gpu


def _check(got, ref):
    assert got.shape == ref.shape and got.dtype == ref.dtype
    d = np.abs(got.astype(np.float64) - ref.astype(np.float64))
    if got.dtype == np.uint16:
        assert d.max() <= 1 and (d == 0).mean() >= 0.999
    else:
        assert d.max() <= 1e-5 * float(np.abs(ref).max())


def _vol(shape, dtype, seed):
    a = np.random.default_rng(seed).random(shape) * 3000 + 100
    return np.asfortranarray(a.astype(dtype))


@pytest.mark.parametrize("shape,nt", [((96, 80, 6), 5), ((70, 45, 3), 1), ((64, 41, 2), 10)])
@pytest.mark.parametrize("dtype", [np.uint16, np.float32])
def test_gaussian_taper_matches_oracle(shape, nt, dtype):
    vol = _vol(shape, dtype, nt)
    psf = TP.fspecial_gaussian(nt + 30, nt)                 # the kernel RLdecon passes
    _check(TP.edgetaper_slices(vol, psf), OE.edgetaper_slices(vol, psf))


@pytest.mark.parametrize("dtype", [np.uint16, np.float32])
def test_non_separable_psf_matches_oracle(dtype):
    rng = np.random.default_rng(9)
    psf = rng.random((5, 8))
    psf /= psf.sum()
    vol = _vol((33, 29, 4), dtype, 9)
    _check(TP.edgetaper_slices(vol, psf), OE.edgetaper_slices(vol, psf))


def test_two_d_image_and_in_place():
    img = _vol((48, 52), np.uint16, 11)[:, :]
    psf = TP.fspecial_gaussian(33, 3.0)
    _check(TP.edgetaper(img, psf), OE.edgetaper(img, psf))
    vol = _vol((48, 52, 2), np.float32, 12)
    ref = OE.edgetaper_slices(vol, psf)
    out = TP.edgetaper_slices(vol, psf, out=vol)
    assert out is vol
    _check(vol, ref)


def test_errors():
    vol = _vol((40, 40, 2), np.uint16, 13)
    with pytest.raises(_lib.PkError):
        TP.edgetaper_slices(vol, np.ones((40, 3)))           # PSF as tall as the image
    with pytest.raises(ValueError):
        TP.edgetaper_slices(vol, np.ones((3, 3, 3)))


def test_rldecon_tapers_before_deconvolution(tmp_path):
    psf_true = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((96, 80, 48), 60, psf_true, seed=5)
    bead = synth.measured_psf((32, 32, 41), sigma_xy=1.3, sigma_z=3.0, seed=6)
    raw, pfn = str(tmp_path / "frame_CamA.tif"), str(tmp_path / "psf_CamA.tif")
    T.writetiff(vol, raw)
    T.writetiff(bead, pfn)
    out = str(tmp_path / "o" / "frame_CamA.tif")
    J, _, _ = RLdecon(raw, out, pfn, 0.108, 0.3, 0.1, Background=100, DeconIter=3, RLMethod="simplified",
                      nTapering=5, save16bit=False)
    tapered = TP.edgetaper_slices(vol, TP.fspecial_gaussian(35, 5.0))
    assert not np.array_equal(tapered, vol)
    _check(tapered, OE.edgetaper_slices(vol, OE.fspecial_gaussian(35, 5.0)))
    psf = P.rldecon_psf_crop(P.psf_gen_new(bead, 0.1, 0.3 * np.sin(np.radians(32.45))), vol.shape, "simplified")
    p32 = psf / np.float32(psf.sum(dtype=np.float32))
    ref = D.decon_lucy_function(tapered, p32, 3, Background=100, save16bit=False)[0]
    np.testing.assert_array_equal(J, ref)
    assert os.path.exists(out)
