"""Known-answer tests that pin the oracle restatement (no reference golden vectors exist).

Each case is an analytic property of the reference's algorithm (decon_psf2otf.m, decon_lucy_function.m,
decon_lucy_omw_function.m) or a table of the reference's integer helpers.
"""
import numpy as np
import pytest

from oracle import chunking as OC
from oracle import decon as O
from oracle import morph as OM


def _delta(shape=(5, 5, 7)):
    p = np.zeros(shape, np.float32)
    p[shape[0] // 2, shape[1] // 2, shape[2] // 2] = 1
    return p


def test_delta_psf_otf_is_one():
    otf = O.psf2otf_half(_delta(), (16, 12, 10), np.float64)
    assert np.allclose(otf, 1.0, atol=1e-12)


def test_otf_dc_is_one_after_normalisation():
    rng = np.random.default_rng(0)
    psf = rng.random((7, 9, 5)).astype(np.float32)
    otf = O.psf2otf_half(O.normalize_psf(psf, np.float64), (20, 18, 10), np.float64)
    assert abs(otf[0, 0, 0] - 1) < 1e-12


def test_blur_conserves_flux():
    rng = np.random.default_rng(1)
    psf = rng.random((5, 5, 5))
    otf = O.psf2otf_half(O.normalize_psf(psf, np.float64), (16, 16, 8), np.float64)
    J = rng.random((16, 16, 8))
    assert abs(O.conv_half(J, otf).sum() - J.sum()) < 1e-9 * J.sum()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_delta_psf_decon_is_identity(dtype):
    rng = np.random.default_rng(2)
    I = rng.integers(100, 4000, size=(16, 12, 10)).astype(np.uint16)
    J = O.decon_lucy_omw(I, _delta(), _delta(), 2, background=100, save16bit=False, dtype=dtype)
    Ipre, _ = O.preprocess(I, 100, False, dtype)
    assert O.rel_l2(J, Ipre) < (1e-6 if dtype == np.float32 else 1e-13)
    J2 = O.decon_lucy(I, _delta(), 5, background=100, save16bit=False, dtype=dtype)
    assert O.rel_l2(J2, Ipre) < (1e-5 if dtype == np.float32 else 1e-12)


def test_rl_fixed_point():
    """I = blur(J*) without noise: J* is stationary under the RL update."""
    rng = np.random.default_rng(3)
    psf = np.exp(-np.add.outer(np.add.outer(np.arange(-3, 4) ** 2, np.arange(-3, 4) ** 2), np.arange(-3, 4) ** 2) / 4.0)
    Js = rng.uniform(50, 500, size=(16, 16, 16))
    otf = O.psf2otf_half(O.normalize_psf(psf, np.float64), Js.shape, np.float64)
    I = O.conv_half(Js, otf)
    ratio = I / np.maximum(O.conv_half(Js, otf), O.EPS)
    Jn = O.conv_half(ratio, np.conj(otf)) * Js
    assert O.rel_l2(Jn, Js) < 1e-12


def test_uniform_image_is_stationary_for_omw():
    rng = np.random.default_rng(4)
    psf = rng.random((5, 5, 5)).astype(np.float32)
    I = np.full((12, 12, 12), 700.0)
    J = O.decon_lucy_omw(I, psf, psf[::-1, ::-1, ::-1], 2, background=0, save16bit=False, dtype=np.float64)
    assert np.allclose(J, 700.0, rtol=1e-10)


def test_uint16_conversion_table():
    x = np.array([0.5, 1.5, 2.5, 0.49999997, 65535.4, 65535.6, np.nan, -1.0, -0.5, 1e9, np.inf, -np.inf],
                 dtype=np.float32)
    want = np.array([1, 2, 3, 0, 65535, 65535, 0, 0, 0, 65535, 65535, 0], dtype=np.uint16)
    assert np.array_equal(O.to_uint16(x), want)


def test_uint16_background_rounding():
    assert O.round_background_u16(100.5) == 101
    assert O.round_background_u16(99.49) == 99
    assert O.round_background_u16(-3) == 0
    I = np.array([0, 50, 100, 101, 65535], dtype=np.uint16).reshape(5, 1, 1)
    out, mask = O.preprocess(I, 100, True, np.float32)
    assert out.ravel().tolist() == [0, 0, 0, 1, 65435]
    assert mask.ravel().tolist() == [False, True, True, True, True]


@pytest.mark.parametrize("n,good", [(352, 360), (416, 420), (544, 560), (31, 32), (41, 42), (101, 108), (1, 1),
                                    (7, 8), (14, 14), (224, 224), (288, 288), (1025, 1050)])
def test_find_good_factor_number(n, good):
    assert OC.find_good_factor_number(n) == good


def test_find_good_factor_number_options():
    assert OC.find_good_factor_number(7, allow_odd_seven=True) == 7
    assert OC.find_good_factor_number(13, direction=-1) == 12
    assert OC.find_good_factor_number(1025, allow_odd_seven=True) == 1029


def test_chunk_coordinates_table():
    # 10 x 7 x 5 volume, batch 4 x 4 x 5, block 2, border 1, sameBatchSize false
    b, r, l = OC.zarr_chunk_coordinates((10, 7, 5), batch_size=(4, 4, 5), block_size=(2, 2, 5), border=1,
                                        same_batch_size=False)
    assert r.tolist() == [[1, 1, 1, 4, 4, 5], [5, 1, 1, 8, 4, 5], [9, 1, 1, 10, 4, 5],
                          [1, 5, 1, 4, 7, 5], [5, 5, 1, 8, 7, 5], [9, 5, 1, 10, 7, 5]]
    assert b.tolist() == [[1, 1, 1, 5, 5, 5], [4, 1, 1, 9, 5, 5], [8, 1, 1, 10, 5, 5],
                          [1, 4, 1, 5, 7, 5], [4, 4, 1, 9, 7, 5], [8, 4, 1, 10, 7, 5]]
    assert l.tolist() == [[1, 1, 1, 4, 4, 5], [2, 1, 1, 5, 4, 5], [2, 1, 1, 3, 4, 5],
                          [1, 2, 1, 4, 4, 5], [2, 2, 1, 5, 4, 5], [2, 2, 1, 3, 4, 5]]
    # sameBatchSize: the last batch keeps the full batch size before the border
    b2, r2, _ = OC.zarr_chunk_coordinates((10, 7, 5), batch_size=(4, 4, 5), block_size=(2, 2, 5), border=1,
                                          same_batch_size=True)
    assert b2[2].tolist() == [6, 1, 1, 10, 5, 5]
    assert OC.border_size((31, 31, 41)) == [21, 21, 26]


def test_structuring_elements():
    assert len(OM.sphere_offsets(1)) == 7
    assert len(OM.sphere_offsets(2)) == 33
    d4 = O.disk_nhood(4).astype(int)
    want = np.array([[0, 0, 1, 1, 1, 0, 0], [0, 1, 1, 1, 1, 1, 0], [1, 1, 1, 1, 1, 1, 1], [1, 1, 1, 1, 1, 1, 1],
                     [1, 1, 1, 1, 1, 1, 1], [0, 1, 1, 1, 1, 1, 0], [0, 0, 1, 1, 1, 0, 0]])
    assert np.array_equal(d4, want)
    assert O.disk_nhood(1).astype(int).tolist() == [[0, 1, 0], [1, 1, 1], [0, 1, 0]]
    assert O.disk_nhood(0).astype(int).tolist() == [[1]]


def test_edge_erosion_full_mask():
    m = np.ones((8, 9, 10), bool)
    e = O.mask_edge_erosion(m, 2)
    assert e.sum() == (8 - 4) * (9 - 4) * (10 - 4)
    assert not e[:2].any() and not e[:, -2:].any() and not e[:, :, :2].any()


def test_edge_erosion_irregular_mask():
    m = np.ones((20, 20, 12), bool)
    m[:5, :5, :] = False            # a notch makes the mask irregular
    e = O.mask_edge_erosion(m, 2)
    assert not e[:, :, 0].any() and not e[:, :, -1].any()
    assert not e[4, 5, 5] and not e[5, 4, 5]   # eroded next to the notch (disk radius 1)
    assert e[5, 5, 5]                          # diagonal neighbour: the radius-1 disk is a cross
    assert e[10, 10, 5]


def test_damp_factor_tie_doubles():
    """decon_lucy_function.m:179: J == d*I yields 2J."""
    J = np.array([1.0, 2.0, 5.0], np.float32).reshape(3, 1, 1)
    I = np.array([1.0, 1.0, 1.0], np.float32).reshape(3, 1, 1)
    out = O.postprocess(J, I, None, damp=2.0, save16bit=False)
    assert out.ravel().tolist() == [1.0, 4.0, 2.0]


def test_single_plane_edge_erosion_takes_the_2d_steps():
    """decon_mask_edge_erosion.m on an [ny nx 1] array: ndims is 2, so no z faces and no z erosion."""
    from oracle.decon import mask_edge_erosion
    full = np.ones((20, 17, 1), bool)
    m = mask_edge_erosion(full, 3)
    ref = np.zeros((20, 17), bool)
    ref[3:17, 3:14] = True
    np.testing.assert_array_equal(m[:, :, 0], ref)
    np.testing.assert_array_equal(mask_edge_erosion(full[:, :, 0], 3), ref)
    irr = np.ones((20, 17), bool)
    irr[8, 8] = False
    m2 = mask_edge_erosion(irr, 2)                              # disk(1): the 4-neighbourhood
    assert m2.shape == (20, 17) and not m2[0].any() and not m2[:, -1].any()
    assert not m2[8, 8] and not m2[7, 8] and not m2[8, 9] and m2[7, 7] and m2[5, 5]
    np.testing.assert_array_equal(mask_edge_erosion(irr[:, :, None], 2)[:, :, 0], m2)
