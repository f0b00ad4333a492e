"""The edge-taper oracle (fspecial('gaussian') and edgetaper of RLdecon.m:351-357) on its own
properties, and the host-side kernel builder of the library against it."""
import numpy as np
import pytest

from oracle import edgetaper as OE


def test_fspecial_gaussian_is_normalised_and_symmetric():
    for hs, s in [(31, 1.0), (35, 5.0), (40, 10.0)]:
        h = OE.fspecial_gaussian(hs, s)
        assert h.shape == (hs, hs) and abs(h.sum() - 1.0) < 1e-14
        np.testing.assert_array_equal(h, h.T)
        np.testing.assert_array_equal(h, h[::-1, ::-1])
        c = (hs - 1) // 2
        assert h.max() == h[c, c]


def test_fspecial_drops_values_below_eps_times_max():
    h = OE.fspecial_gaussian(31, 1.0)                       # corners at exp(-225) of the centre
    assert h[0, 0] == 0.0 and h[15, 15] > 0.0


def test_product_kernel_builder_matches_oracle():
    from petakit5d_b200 import taper as TP
    for hs, s in [(31, 1.0), (35, 5.0), (40, 10.0)]:
        np.testing.assert_array_equal(TP.fspecial_gaussian(hs, s), OE.fspecial_gaussian(hs, s))


@pytest.mark.parametrize("n", [32, 36, 64, 101])
def test_taper_weight_is_one_at_the_borders_and_zero_inside(n):
    psf = OE.fspecial_gaussian(31, 3.0)
    b = OE.taper_weight(psf, n, 0)
    assert b.shape == (n,)
    assert abs(b[0] - 1.0) < 1e-12 and abs(b[-1] - 1.0) < 1e-12
    np.testing.assert_allclose(b, b[::-1], atol=1e-12)
    if n - 1 > 2 * 30:                                      # lags beyond the PSF's width
        assert np.abs(b[31:n - 31]).max() < 1e-12


def test_fft_blur_equals_the_direct_circular_sum():
    rng = np.random.default_rng(3)
    img = rng.random((23, 19))
    for psf in (OE.fspecial_gaussian(7, 1.5), rng.random((5, 8)), rng.random((4, 3))):
        np.testing.assert_allclose(OE.circular_blur(img, psf), OE.circular_blur_direct(img, psf), atol=1e-12)


def test_delta_psf_and_constant_image_are_fixed_points():
    rng = np.random.default_rng(4)
    img = (rng.random((40, 33)) * 4000).astype(np.uint16)
    np.testing.assert_array_equal(OE.edgetaper(img, np.ones((1, 1))), img)
    c = np.full((40, 33), 1234, np.uint16)
    np.testing.assert_array_equal(OE.edgetaper(c, OE.fspecial_gaussian(31, 2.0)), c)


def test_taper_blends_to_the_blur_at_the_borders():
    rng = np.random.default_rng(5)
    img = rng.random((64, 64)) * 1000
    psf = OE.fspecial_gaussian(31, 3.0)
    j = OE.edgetaper(img, psf)
    b = OE.circular_blur(img, psf)
    np.testing.assert_allclose(j[0, :], b[0, :], atol=1e-9)
    np.testing.assert_allclose(j[:, -1], b[:, -1], atol=1e-9)
    np.testing.assert_allclose(j[31:33, 31:33], img[31:33, 31:33], atol=1e-9)


def test_uint16_keeps_its_class_with_matlab_rounding():
    img = np.full((40, 40), 7, np.uint16)
    img[0, 0] = 60000
    j = OE.edgetaper(img, OE.fspecial_gaussian(31, 2.0))
    assert j.dtype == np.uint16
    a = OE.taper_alpha(OE.fspecial_gaussian(31, 2.0), 40, 40)
    f = a * img + (1 - a) * OE.circular_blur(img.astype(np.float64), OE.fspecial_gaussian(31, 2.0))
    np.testing.assert_array_equal(j, np.floor(f + 0.5).astype(np.uint16))


def test_slices_are_independent():
    rng = np.random.default_rng(6)
    vol = np.asfortranarray((rng.random((36, 34, 3)) * 500).astype(np.float32))
    psf = OE.fspecial_gaussian(31, 1.0)
    out = OE.edgetaper_slices(vol, psf)
    for z in range(3):
        np.testing.assert_array_equal(out[:, :, z], OE.edgetaper(vol[:, :, z], psf))


def test_psf_larger_than_the_image_is_rejected():
    with pytest.raises(ValueError):
        OE.edgetaper(np.zeros((20, 40)), np.ones((20, 3)))
