"""OMW and Biggs-RL iterations of the CUDA library against the FP32 oracle (and the FP64 one)."""
import numpy as np
import pytest

from oracle import decon as O
from petakit5d_b200 import decon as D
from petakit5d_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    vol, psf = synth.single_volume_workload("rl_small", seed=1)
    return vol, psf


def test_psf2otf_matches_oracle(small):
    _, psf = small
    got = D.psf2otf_half(psf, (128, 128, 64))
    ref = O.psf2otf_half(O.normalize_psf(psf, np.float64), (128, 128, 64), np.float64)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6
    assert abs(got[0, 0, 0] - 1) < 1e-6                     # DC of a normalised PSF


def test_omw_two_iterations_fp32_parity(small):
    vol, psf = small
    psf_b = np.ascontiguousarray(psf[::-1, ::-1, ::-1])
    J, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 2, Background=100, save16bit=False)
    ref = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, save16bit=False, dtype=np.float32)
    ref64 = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, save16bit=False, dtype=np.float64)
    e32 = O.rel_l2(J, ref)
    e64 = O.rel_l2(J, ref64)
    print(f"OMW x2 rel-L2 vs FP32 oracle {e32:.2e}, vs FP64 oracle {e64:.2e}")
    assert e32 <= 1e-4
    assert e64 <= 1e-4


def test_rl_twenty_iterations_fp32_parity(small):
    vol, psf = small
    J, _, k = D.decon_lucy_function(vol, psf, 20, Background=100, save16bit=False)
    ref = O.decon_lucy(vol, psf, 20, background=100, save16bit=False, dtype=np.float32)
    ref64 = O.decon_lucy(vol, psf, 20, background=100, save16bit=False, dtype=np.float64)
    e32 = O.rel_l2(J, ref)
    e64 = O.rel_l2(J, ref64)
    print(f"RL x20 rel-L2 vs FP32 oracle {e32:.2e}, vs FP64 oracle {e64:.2e}")
    assert k == 20
    assert e32 <= 1e-3


def test_uint16_output_within_one_lsb(small):
    vol, psf = small
    psf_b = np.ascontiguousarray(psf[::-1, ::-1, ::-1])
    J, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 2, Background=100)
    ref = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, dtype=np.float32)
    assert J.dtype == np.uint16
    assert np.max(np.abs(J.astype(np.int64) - ref.astype(np.int64))) <= 1
