"""The library's 3D real transform against numpy's, on the half-spectrum layout."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(16, 8, 4), (128, 128, 64), (64, 48, 40), (30, 22, 26), (31, 41, 17), (1, 1, 1), (2, 3, 5),
         (224, 36, 28), (360, 12, 10), (352, 20, 8), (416, 14, 6), (21, 35, 49), (288, 160, 8),
         # x and z lengths whose plans end in a direct odd radix (224 = 16*2*7, 288 = 16*2*9, ...)
         (16, 224, 8), (8, 12, 288), (4, 352, 6), (6, 4, 416), (4, 272, 4), (2, 210, 420)]


def _r2c(vol, cuda):
    import torch
    from petakit5d_b200 import decon as D
    ny, nx, nz = vol.shape
    d_in = torch.from_numpy(np.ascontiguousarray(vol.transpose(2, 1, 0))).to(cuda)
    spec = torch.empty((nz, nx, ny // 2 + 1), dtype=torch.complex64, device=cuda)
    D.fft3_r2c(d_in, vol.shape, spec)
    torch.cuda.synchronize()
    return spec.cpu().numpy().transpose(2, 1, 0), spec


@pytest.mark.parametrize("shape", SIZES)
def test_r2c_matches_numpy(shape, cuda):
    rng = np.random.default_rng(7)
    vol = rng.standard_normal(shape).astype(np.float32)
    got, _ = _r2c(vol, cuda)
    ref = np.fft.rfftn(vol.astype(np.float64), axes=(2, 1, 0))
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 2e-6, (shape, err)


@pytest.mark.parametrize("shape", SIZES)
def test_c2r_roundtrip(shape, cuda):
    import torch
    from petakit5d_b200 import decon as D
    rng = np.random.default_rng(11)
    vol = rng.standard_normal(shape).astype(np.float32)
    _, spec = _r2c(vol, cuda)
    out = torch.empty((shape[2], shape[1], shape[0]), dtype=torch.float32, device=cuda)
    D.fft3_c2r(spec, shape, out)
    torch.cuda.synchronize()
    back = out.cpu().numpy().transpose(2, 1, 0) / np.prod(shape)
    err = np.linalg.norm(back - vol) / np.linalg.norm(vol)
    assert err < 2e-6, (shape, err)
