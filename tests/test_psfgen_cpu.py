"""psf_gen_new restatement (oracle) against independent implementations and analytic answers, and
the host-side PSF crops of RLdecon (no GPU)."""
import numpy as np
import pytest
import scipy.ndimage as ndi

from oracle import psfgen as OP
from petakit5d_b200 import synth


def test_medfilt3_matches_scipy_nearest():
    a = synth.measured_psf((20, 17, 12), seed=4)
    assert np.array_equal(OP.medfilt3(a), ndi.median_filter(a, size=3, mode="nearest"))


def test_medfilt2_matches_scipy_zero_padding():
    a = synth.measured_psf((23, 19, 1), seed=5)
    ref = ndi.median_filter(a[:, :, 0], size=3, mode="constant", cval=0.0)
    assert np.array_equal(OP.medfilt2(a)[:, :, 0], ref)


def test_resample_z_constant_volume_scales_by_size_ratio():
    # a z-constant PSF has only the DC plane: ifft over new_nz of nz*c gives c*nz/new_nz
    p = np.full((4, 3, 40), 2.0, np.float32)
    out = OP.resample_z(p, 0.1, 0.3)
    new_nz = int(np.floor(40 / 3 + 0.5))
    assert out.shape == (4, 3, new_nz)
    np.testing.assert_allclose(out, 2.0 * 40 / new_nz, rtol=1e-12)


def test_resample_z_odd_size_second_band_wins():
    # psf_gen_new.m:128-131 with uint16 arithmetic: nz = 41, ratio 2 -> new_nz = 21, new_nz/2 -> 11, so
    # plane 10 is written twice and keeps F[30]; a cos at frequency 10 keeps only its F[31] partner
    nz = 41
    z = np.arange(nz)
    p = np.broadcast_to(np.cos(2 * np.pi * 10 * z / nz), (2, 2, nz)).astype(np.float64)
    out = OP.resample_z(p.astype(np.float32), 1.0, 2.0)
    j = np.arange(21)
    expect = np.maximum((nz / 2) / 21 * np.cos(2 * np.pi * 11 * j / 21), 0.0)
    np.testing.assert_allclose(out[0, 0], expect, atol=2e-6)


def test_resample_skipped_when_data_step_not_coarser():
    p = synth.measured_psf((12, 12, 9), seed=1)
    np.testing.assert_array_equal(OP.resample_z(p, 0.2, 0.2), np.maximum(p, 0))


def test_centre_moves_peak_to_middle_without_cleanup():
    # no positive value in the first / last five slices: the cleanup is skipped (psf_gen_new.m:28)
    p = np.zeros((16, 15, 21), np.float32)
    p[3, 11, 9] = 5.0
    p[4, 11, 9] = 1.0
    out = OP.psf_gen_new(p, 0.1, 0.1)
    assert out.shape == p.shape
    k = np.unravel_index(np.argmax(out), out.shape)
    assert k == (int(np.floor(17 / 2 + 0.5)) - 1, int(np.floor(16 / 2 + 0.5)) - 1, 10)
    assert out.sum() == pytest.approx(6.0)


def test_centre_pads_after_a_peak_far_from_the_first_slice():
    p = synth.measured_psf((32, 32, 41), peak=(16, 16, 30), sigma_z=8.0, seed=2)
    raw, _ = OP.clean(p)
    zs = int(np.nonzero(raw.sum(axis=(0, 1)))[0][0]) + 1
    pz = int(np.argmax(raw.ravel(order="F"))) // (32 * 32) + 1
    assert pz - zs > 41 / 2
    c = OP.centre(raw)
    assert c.shape[2] == 41 + pz - zs - int(np.floor(20 + 0.5)) + 3


def test_centre_pads_before_a_peak_far_from_the_last_slice():
    p = synth.measured_psf((32, 32, 41), peak=(15, 17, 10), sigma_z=8.0, seed=3)
    raw, _ = OP.clean(p)
    zt = int(np.nonzero(raw.sum(axis=(0, 1)))[0][-1]) + 1
    pz = int(np.argmax(raw.ravel(order="F"))) // (32 * 32) + 1
    assert zt - pz > 41 / 2
    c = OP.centre(raw)
    pad = zt - pz - 20 + 3
    assert c.shape[2] == 41 + pad
    np.testing.assert_array_equal(np.sort(c.ravel()), np.sort(np.concatenate([raw.ravel(), np.zeros(32 * 32 * pad)])))


def test_masked_mask_is_the_peak_component():
    p = synth.measured_psf((40, 40, 41), seed=6)
    raw, BW = OP.clean(p)
    lab, n = OP._label(BW)
    assert n == 1 and BW[20, 20, 20]
    assert np.all(raw >= 0) and np.all(raw[~BW] == 0)


def test_peak_outside_components_selects_the_background():
    # L(peakInd) == 0 makes BW = (L == 0): every voxel outside the kept components
    BW = np.zeros((12, 12, 12), bool)
    BW[1:4, 1:4, 1:4] = True
    med = np.zeros(BW.shape, np.float32)
    med[9, 9, 9] = 1.0
    out = OP._peak_component(BW, med)
    np.testing.assert_array_equal(out, ~BW)


def test_input_checks():
    with pytest.raises(ValueError):
        OP.clean(np.ones((16, 16, 3), np.float32))
    with pytest.raises(ValueError):
        OP.clean(np.full((8, 16, 12), 200.0, np.float32))
    with pytest.raises(NotImplementedError):
        OP.clean(np.ones((16, 16), np.float32), method=OP.MEDIAN)


@pytest.mark.parametrize("omw", [True, False])
def test_rldecon_psf_crop_matches_oracle(omw):
    from petakit5d_b200.psfgen import rldecon_psf_crop
    rng = np.random.default_rng(7)
    for _ in range(6):
        psf = np.zeros(tuple(rng.integers(8, 20, size=3)), np.float32)
        lo = [int(rng.integers(0, s // 2)) for s in psf.shape]
        hi = [int(rng.integers(s // 2 + 1, s + 1)) for s in psf.shape]
        psf[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = rng.random((hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]))
        data = tuple(int(v) for v in rng.integers(6, 24, size=3))
        a = rldecon_psf_crop(psf, data, "omw" if omw else "simplified")
        b = OP.rldecon_psf_crop(psf, data, omw)
        np.testing.assert_array_equal(a, b)
