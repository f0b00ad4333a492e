"""Deskew / rotate on the GPU (pk_deskew_rotate) against the oracle restatement of
deskewRotateFrame3D.m and its MEX files.

The kernels use the MEX files' float association, weights and rounding, so outputs agree bit for
bit except where the 4x4 inverse (LAPACK in the oracle, Gauss-Jordan in the library) moves a source
coordinate across an integer by a rounding step: float outputs within 1e-5 of the volume's range,
uint16 outputs within 1 level, and at least 99.9% of voxels identical."""
import numpy as np
import pytest

from oracle import deskew as OD
from petakit5d_b200 import deskew as G

pytestmark = pytest.mark.gpu


def _vol(dtype, shape=(40, 96, 48), seed=0):
    a = np.random.default_rng(seed).random(shape) * 3000 + 100
    return np.asfortranarray(a.astype(dtype))


def _check(got, ref):
    assert got.shape == ref.shape and got.dtype == ref.dtype
    if got.dtype == np.uint16:
        d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
        assert d.max() <= 1
    else:
        d = np.abs(got.astype(np.float64) - ref.astype(np.float64))
        assert d.max() <= 1e-5 * float(np.abs(ref).max())
    assert (d == 0).mean() >= 0.999


@pytest.mark.parametrize("dz", [0.2, 0.3, 0.65])          # direct warp; skewed step 1/2; skewed step 1/3
@pytest.mark.parametrize("reverse", [False, True])
@pytest.mark.parametrize("kind", ["f32", "u16_f32", "u16_u16"])
def test_deskew_rotate_matches_oracle(dz, reverse, kind):
    vol = _vol(np.float32 if kind == "f32" else np.uint16)
    s16 = kind == "u16_u16"
    got = G.deskewRotateFrame3D(vol, 32.45, dz, 0.108, reverse=reverse, save16bit=s16)
    ref = OD.deskew_rotate_frame3d(vol, 32.45, dz, 0.108, reverse=reverse, save16bit=s16)
    _check(got, ref)


@pytest.mark.parametrize("bbox", [(1, 20, 5, 40, 120, 30), (3, 1, 1, 37, 60, 47), (1, 1, 40, 40, 90, 60)])
def test_deskew_rotate_bbox(bbox):
    vol = _vol(np.uint16, (40, 80, 36), seed=1)
    got = G.deskewRotateFrame3D(vol, 32.45, 0.3, 0.108, reverse=True, bbox=bbox, save16bit=True)
    ref = OD.deskew_rotate_frame3d(vol, 32.45, 0.3, 0.108, reverse=True, bbox=bbox, save16bit=True)
    _check(got, ref)


def test_deskew_rotate_objective_scan():
    vol = _vol(np.float32, (24, 50, 30), seed=2)
    got = G.deskewRotateFrame3D(vol, 32.45, 0.3, 0.108, objectiveScan=True)
    ref = OD.deskew_rotate_frame3d(vol, 32.45, 0.3, 0.108, objective_scan=True)
    _check(got, ref)


def test_deskew_rotate_odd_row_length_and_other_angle():
    vol = _vol(np.uint16, (37, 70, 41), seed=3)
    for s16 in (False, True):
        got = G.deskewRotateFrame3D(vol, -31.3, 0.25, 0.104, reverse=False, save16bit=s16)
        ref = OD.deskew_rotate_frame3d(vol, -31.3, 0.25, 0.104, reverse=False, save16bit=s16)
        _check(got, ref)


def test_deskew_rotate_device_after_decon(cuda):
    """Deconvolve on the device and deskew the result without a host round trip."""
    import torch
    from petakit5d_b200 import decon, synth
    psf = synth.gaussian_psf((31, 31, 41))
    vol = synth.puncta_volume((64, 96, 48), 60, psf, seed=4)
    d_in = torch.from_numpy(vol.ravel(order="F").copy()).to(cuda)
    d_j = torch.empty(vol.size, dtype=torch.float32, device=cuda)
    decon.decon_device("omw", d_in, "uint16", vol.shape, psf, psf, numit=2, out=d_j, Background=100,
                       save16bit=False)
    dims = G.deskew_rotate_device(d_j, torch.float32, vol.shape, 32.45, 0.3, 0.108, reverse=True)
    d_o = torch.empty(int(np.prod(dims)), dtype=torch.float32, device=cuda)
    G.deskew_rotate_device(d_j, torch.float32, vol.shape, 32.45, 0.3, 0.108, d_out=d_o, reverse=True)
    torch.cuda.synchronize()
    J = d_j.cpu().numpy().reshape(vol.shape, order="F")
    got = d_o.cpu().numpy().reshape(dims, order="F")
    _check(got, OD.deskew_rotate_frame3d(J, 32.45, 0.3, 0.108, reverse=True))


def test_deskew_rotate_rejects_bad_input():
    from petakit5d_b200._lib import PkError
    with pytest.raises(PkError):
        G.deskewRotateFrame3D(_vol(np.float32), 32.45, 0.3, 0.108, bbox=(0, 1, 1, 10, 10, 10))
    with pytest.raises(PkError):
        G.deskewRotateFrame3D(_vol(np.float32), 32.45, 0.3, 0.108, bbox=(1, 1, 1, 41, 10, 10))
    with pytest.raises(NotImplementedError):
        G.deskewRotateFrame3D(_vol(np.float32), 32.45, 0.3, 0.108, interpMethod="cubic")
