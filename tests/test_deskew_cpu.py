"""deskewRotateFrame3D restatement (oracle) against an independent interpolator and analytic answers
(no GPU)."""
import math

import numpy as np
import pytest
import scipy.ndimage as ndi

from oracle import deskew as D


def _vol(shape=(40, 96, 48), seed=0):
    return (np.random.default_rng(seed).random(shape) * 1000).astype(np.float32)


@pytest.mark.parametrize("reverse", [False, True])
def test_direct_warp_matches_bilinear_map_coordinates(reverse):
    vol = _vol()
    p = D.plan(vol.shape, 32.45, 0.2, 0.108, reverse=reverse)
    assert not p["do_interp"]
    out = D.deskew_rotate_frame3d(vol, 32.45, 0.2, 0.108, reverse=reverse)
    tm = p["tmat"]
    ox, oy, oz = out.shape
    z = np.arange(oz, dtype=np.float64)[None, None, :]
    y = np.arange(oy, dtype=np.float64)[None, :, None]
    ty = np.broadcast_to(tm[1][2] * z + tm[1][3], out.shape)
    tz = np.broadcast_to(tm[2][1] * y + tm[2][2] * z + tm[2][3], out.shape)
    ii = np.broadcast_to(np.arange(ox, dtype=np.float64)[:, None, None], out.shape)
    ref = ndi.map_coordinates(vol, np.stack([ii, ty, tz]), order=1, mode="constant")
    inside = (ty >= 0) & (ty + 1 < vol.shape[1]) & (tz >= 0) & (tz + 1 < vol.shape[2])
    assert inside.mean() > 0.3
    np.testing.assert_allclose(out[inside], ref[inside], rtol=2e-6, atol=1e-3)
    assert not out[~inside].any()


def test_output_box_formula():
    # deskewRotateFrame3D.m:65-66: round([ny, (nx-1)cos + (nz-1) zAniso / sin, (nx-1) sin - 4])
    th = math.radians(32.45)
    za = math.sin(th) * 0.3 / 0.108
    p = D.plan((40, 96, 48), 32.45, 0.3, 0.108)
    assert p["out_size"] == [40, round(95 * math.cos(th) + 47 * za / math.sin(th)), round(95 * math.sin(th) - 4)]


def test_skewed_interpolation_step_and_slices():
    p = D.plan((40, 96, 48), 32.45, 0.3, 0.108, reverse=True)
    assert p["do_interp"] and p["stepsize"] == pytest.approx(0.5)
    assert p["nz_total"] == 95
    index, orig, nint = D.interp_indexing(95, 0.5)
    assert nint == 47 and orig[::2].all() and not orig[1::2].any()
    np.testing.assert_array_equal(index[::2], np.arange(48))
    # |dx| / xStepThresh >= 1.5: ndiv = ceil(|dx| / thresh) equal steps
    p = D.plan((40, 96, 48), 32.45, 0.65, 0.108)
    dx = math.cos(math.radians(32.45)) * 0.65 / 0.108
    assert p["stepsize"] == pytest.approx(1 / math.ceil(dx / 2.0))


@pytest.mark.parametrize("reverse", [False, True])
def test_skewed_slices_of_a_linear_volume(reverse):
    # for f = a x + b z + c the interpolated slice at zo + zw is exact: a (x + xstep (1 - 2 zw)) + ...
    # without reverse (the skew shift of the sheet), a x + ... with reverse (deskewRotateFrame3D geometry)
    ny, nx, nz = 8, 60, 10
    a, b, c = 3.0, 7.0, 100.0
    x = np.arange(nx)[None, :, None]
    z = np.arange(nz)[None, None, :]
    vol = np.broadcast_to(a * x + b * z + c, (ny, nx, nz)).astype(np.float32)
    xstep, step = 2.6, 0.5
    im_int, index, orig = D.skewed_interp(vol, xstep, step, reverse, False)
    xa = math.ceil(xstep)
    for i in np.flatnonzero(~orig):
        zout = step * i
        zo, zw = math.floor(zout), zout - math.floor(zout)
        shift = 0.0 if reverse else xstep * (1 - 2 * zw)
        for yy in range(xa + 1, nx - xa - 2):
            np.testing.assert_allclose(im_int[:, yy, index[i]], a * (yy + shift) + b * (zo + zw) + c, rtol=1e-5)


def test_uint16_rounding_of_blocks_and_tail():
    # x86 MEX: whole 16-element blocks round res + 0.5 to nearest even (so 2.25 -> 3), the tail
    # truncates res + 0.5 (2.25 -> 2)
    row = np.full(20, 9, np.uint16)
    out = D._blend([(row, 0.25), (row, 0.0)], True, True, 20)
    assert (out[:16] == 3).all() and (out[16:] == 2).all()


def test_uint16_input_association():
    # (a wa + b wb) + (c wc + d wd) in the blocks vs ((a wa + b wb) + c wc) + d wd in the tail
    vals = [np.full(17, v, np.uint16) for v in (1, 3, 65535, 7)]
    w = [np.float32(v) for v in (0.1, 0.2, 0.3, 0.4)]
    out = D._blend(list(zip(vals, w)), True, False, 17)
    p = [np.float32(v) * wk for v, wk in zip((1, 3, 65535, 7), w)]
    assert out[0] == (p[0] + p[1]) + (p[2] + p[3])
    assert out[16] == ((p[0] + p[1]) + p[2]) + p[3]
