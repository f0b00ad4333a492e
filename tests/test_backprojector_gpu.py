"""OMW and Wiener-Butterworth backprojector generation against the oracle restatements."""
import numpy as np
import pytest

from oracle import backprojector as OB
from oracle import decon as O
from petakit5d_b200 import backprojector as B
from petakit5d_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def psf_small():
    return synth.gaussian_psf((31, 31, 41), 1.3, 3.0)


@pytest.mark.parametrize("alpha,thresh", [(0.005, 0.6), (0.005, 0.88), (0.01, 0.9)])
def test_omw_backprojector_matches_oracle(psf_small, alpha, thresh):
    b, omw, absc, mask = B.omw_backprojector_generation(psf_small, alpha, False, OTFCumThresh=thresh,
                                                        hannWinBounds=(0.8, 1.0))
    rb, romw, rabsc, rmask = OB.omw_backprojector_generation(psf_small, alpha, False, otf_cum_thresh=thresh,
                                                             hann_win_bounds=(0.8, 1.0))
    assert O.rel_l2(absc, rabsc) < 1e-6
    assert np.array_equal(mask.astype(bool), rmask.astype(bool)), int(np.sum(mask.astype(bool) != rmask.astype(bool)))
    assert O.rel_l2(omw, romw) < 1e-6
    assert O.rel_l2(b, rb) < 1e-5


def test_omw_backprojector_lobed_psf_auto_skew():
    psf = synth.gaussian_psf((33, 33, 45), 1.5, 4.0, lobes=(-12, 12), lobe_amp=0.15)
    b, _, _, mask = B.omw_backprojector_generation(psf, 0.005, None, OTFCumThresh=0.6)
    rb, _, _, rmask = OB.omw_backprojector_generation(psf, 0.005, None, otf_cum_thresh=0.6)
    assert np.array_equal(mask.astype(bool), rmask.astype(bool))
    assert O.rel_l2(b, rb) < 1e-5


def test_omw_backprojector_rejects_zero_psf():
    from petakit5d_b200._lib import PkError
    with pytest.raises(PkError):
        B.omw_backprojector_generation(np.zeros((9, 9, 9), np.float32), 0.005, False)


@pytest.mark.parametrize("order", [8, 10])
def test_wb_backprojector_matches_oracle(psf_small, order):
    pb, ob = B.BackProjector(psf_small, "wiener-butterworth", 0.005, 1e-3, order, 1)
    rpb, rob = OB.wb_backprojector(psf_small, alpha=0.005, beta=1e-3, n=order, res_flag=1)
    assert O.rel_l2(ob, rob) < 1e-9
    assert O.rel_l2(pb, rpb) < 1e-9


def test_omw_decon_with_generated_backprojector(psf_small):
    """End to end: generated b_omw feeds decon_lucy_omw_function (RLdecon.m:289-333,397-401)."""
    from petakit5d_b200 import decon as D
    vol = synth.puncta_volume((96, 96, 64), 120, psf_small, seed=9, background=100.0)
    b, _, _, _ = B.omw_backprojector_generation(psf_small, 0.005, False, OTFCumThresh=0.6)
    J, _ = D.decon_lucy_omw_function(vol, psf_small, b, 2, Background=100, save16bit=False)
    ref = O.decon_lucy_omw(vol, psf_small, b, 2, background=100, save16bit=False, dtype=np.float32)
    assert O.rel_l2(J, ref) <= 1e-4


@pytest.mark.parametrize("bp_type,tol", [("traditional", 1e-12), ("gaussian", 1e-6), ("butterworth", 1e-9),
                                         ("wiener", 1e-9)])
def test_other_backprojector_types_match_oracle(psf_small, bp_type, tol):
    """The non-default bp_types of BackProjector.m:163-191."""
    pb, ob = B.BackProjector(psf_small, bp_type, 0.005, 1e-3, 8, 1)
    rpb, rob = OB.back_projector(psf_small, bp_type, alpha=0.005, beta=1e-3, n=8, res_flag=1)
    assert pb.shape == rpb.shape and ob.shape == rob.shape
    assert O.rel_l2(ob, rob) < tol
    assert O.rel_l2(pb, rpb) < tol


def test_backprojector_alpha_beta_from_cutoff_gain(psf_small):
    """alpha = 1 / beta = 1 take the traditional back projector's cutoff gain (BackProjector.m:136-156)."""
    pb, ob = B.BackProjector(psf_small, "wiener", 1, 1, 8, 0)
    rpb, rob = OB.back_projector(psf_small, "wiener", alpha=1, beta=1, n=8, res_flag=0)
    assert O.rel_l2(ob, rob) < 1e-9
    assert O.rel_l2(pb, rpb) < 1e-9
