"""BackProjector's bp_type handling on the host, and the oracle's simple branches
(third_parties/WBDeconvolution/BackProjector.m:163-191, 232-233)."""
import numpy as np
import pytest

from oracle import backprojector as OB
from petakit5d_b200 import synth


@pytest.fixture(scope="module")
def psf():
    return synth.gaussian_psf((21, 21, 25), 1.2, 2.5)


def test_unknown_bp_type_is_rejected_like_the_reference(psf):
    from petakit5d_b200 import backprojector as B
    with pytest.raises(ValueError, match="does not match any back-projector type"):
        B.BackProjector(psf, "inverse")
    with pytest.raises(ValueError, match="does not match any back-projector type"):
        OB.back_projector(psf, "inverse")


def test_oracle_traditional_is_the_flipped_psf(psf):
    pb, ob = OB.back_projector(psf, "traditional")
    flipped = psf[::-1, ::-1, ::-1].astype(np.float64)
    assert np.array_equal(pb, flipped)
    assert np.allclose(ob, np.fft.fftn(np.fft.ifftshift(flipped)))


def test_oracle_butterworth_is_real_and_gains_beta_at_the_cutoff(psf):
    """OTF_bp is the Butterworth mask alone: real, 1 at zero frequency, <= 1 everywhere."""
    pb, ob = OB.back_projector(psf, "butterworth", beta=1e-3, n=8)
    assert np.all(ob.imag == 0)
    assert ob.real[0, 0, 0] == 1.0
    assert ob.real.max() <= 1.0


def test_oracle_wiener_butterworth_is_the_default_form(psf):
    a = OB.wb_backprojector(psf, alpha=0.005, beta=1e-3, n=8)
    b = OB.back_projector(psf, "wiener-butterworth", 0.005, 1e-3, 8)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
