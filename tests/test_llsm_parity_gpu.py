"""Parity at the benchmarked size: the 512x512x256 light-sheet volume with the 64x64x101 lobed PSF
(the bench's default workload), and a Biggs-RL volume large enough for the 4096-point-tile kernels.

At these sizes the passes run the 4096-point-tile instantiations (`k_y<plan, mode, 4096>`,
`k_xz<plan, 4096>`), which the 128x128x64 tests never reach: a volume takes the 1024-point tiles only
when its y pass has fewer than 2 * 3 * (SM count) CTAs.  Every result is compared with the float32
oracle (decon_lucy_omw_function.m:105-113, decon_lucy_function.m:120-143) and its error against the
float64 oracle is printed.  Tolerances: rel-L2 <= 1e-4 for OMW x2 and <= 1e-3 for RL, uint16 within
1 LSB of the float32 oracle's uint16.
"""
import numpy as np
import pytest

from oracle import backprojector as OB
from oracle import decon as O
from petakit5d_b200 import backprojector as B
from petakit5d_b200 import decon as D
from petakit5d_b200 import synth

pytestmark = pytest.mark.gpu

BG = 100


@pytest.fixture(scope="module")
def llsm():
    return synth.single_volume_workload("omw_llsm", seed=1)


def _check_omw(vol, psf, pb_lib, pb_ref, label):
    J, _ = D.decon_lucy_omw_function(vol, psf, pb_lib, 2, Background=BG, save16bit=False)
    ref = O.decon_lucy_omw(vol, psf, pb_ref, 2, background=BG, save16bit=False, dtype=np.float32)
    e32 = O.rel_l2(J, ref)
    ref64 = O.decon_lucy_omw(vol, psf, np.asarray(pb_ref, np.float64), 2, background=BG, save16bit=False,
                             dtype=np.float64)
    e64 = O.rel_l2(J, ref64)
    o64 = O.rel_l2(ref, ref64)
    print(f"{label}: OMW x2 512x512x256 rel-L2 vs FP32 oracle {e32:.2e}, vs FP64 oracle {e64:.2e} "
          f"(FP32 oracle vs FP64 oracle {o64:.2e})")
    assert J.shape == vol.shape and J.dtype == np.float32
    assert e32 <= 1e-4
    J16, _ = D.decon_lucy_omw_function(vol, psf, pb_lib, 2, Background=BG)
    ref16 = O.to_uint16(ref)
    assert J16.dtype == np.uint16
    assert int(np.max(np.abs(J16.astype(np.int64) - ref16.astype(np.int64)))) <= 1


def test_omw_wiener_butterworth_llsm(llsm):
    """Wiener-Butterworth backprojector (alpha 0.005, beta 1e-3, order 8), each side generating its own."""
    vol, psf = llsm
    pb_lib, _ = B.BackProjector(psf, "wiener-butterworth", 0.005, 1e-3, 8, 1)
    pb_ref, _ = OB.wb_backprojector(psf, alpha=0.005, beta=1e-3, n=8, res_flag=1)
    assert O.rel_l2(pb_lib, pb_ref) < 1e-6
    _check_omw(vol, psf, pb_lib, pb_ref, "WB")


def test_omw_generator_llsm(llsm):
    """OMW backprojector (alpha 0.005, OTFCumThresh 0.6, not skewed), each side generating its own."""
    vol, psf = llsm
    b_lib, _, _, mask_lib = B.omw_backprojector_generation(psf, 0.005, False, OTFCumThresh=0.6)
    b_ref, _, _, mask_ref = OB.omw_backprojector_generation(psf, 0.005, False, otf_cum_thresh=0.6)
    assert np.array_equal(np.asarray(mask_lib, bool), np.asarray(mask_ref, bool))
    assert O.rel_l2(b_lib, b_ref) < 1e-5
    _check_omw(vol, psf, np.asarray(b_lib, np.float32), np.asarray(b_ref, np.float32), "OMW generator")


def test_rl_4096_tiles():
    """Biggs RL x10 on 512x128x128 (y, x, z): 16384 rows of 256 complex points, 1024 y-pass CTAs of
    16 rows (>= 2 * 3 * 148), so PRE, RLPRE, RATIO, RLUPD and RLFINAL all run the 4096-point-tile kernels
    (with the register-resident per-voxel phase of the 16x16 plan)."""
    psf = synth.gaussian_psf(**synth.SMALL_PSF)
    shape = (512, 128, 128)
    vol = synth.puncta_volume(shape, 1200, psf, seed=11, background=synth.sinusoid_background(shape))
    J, _, k = D.decon_lucy_function(vol, psf, 10, Background=BG, save16bit=False)
    ref = O.decon_lucy(vol, psf, 10, background=BG, save16bit=False, dtype=np.float32)
    ref64 = O.decon_lucy(vol, psf, 10, background=BG, save16bit=False, dtype=np.float64)
    e32, e64 = O.rel_l2(J, ref), O.rel_l2(J, ref64)
    print(f"RL x10 512x128x128 rel-L2 vs FP32 oracle {e32:.2e}, vs FP64 oracle {e64:.2e}")
    assert k == 10
    assert e32 <= 1e-3
    J16, _, _ = D.decon_lucy_function(vol, psf, 10, Background=BG)
    assert int(np.max(np.abs(J16.astype(np.int64) - O.to_uint16(ref).astype(np.int64)))) <= 1
