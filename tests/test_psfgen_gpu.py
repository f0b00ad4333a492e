"""psf_gen_new on the GPU (pk_psf_gen) against the oracle restatement.

Without axial resampling every operation is a float32 operation in a fixed order (the medians are
exact, the border means are float64 sums in the same order), so the PSF must match bit for bit;
with resampling the float64 z-transform pair leaves float32 rounding differences only
(tolerance 1e-6 of the peak)."""
import numpy as np
import pytest

from oracle import psfgen as OP
from petakit5d_b200 import psfgen as G
from petakit5d_b200 import synth
from petakit5d_b200._lib import PkError

pytestmark = pytest.mark.gpu

CASES = [
    dict(size_yxz=(64, 64, 101), seed=0),                                     # the LLSM PSF size
    dict(size_yxz=(31, 31, 41), sigma_xy=1.3, sigma_z=3.0, seed=1),
    dict(size_yxz=(32, 32, 41), peak=(16, 16, 30), sigma_z=8.0, seed=2),      # z padding after
    dict(size_yxz=(32, 32, 41), peak=(15, 17, 10), sigma_z=8.0, seed=3),      # z padding before
    dict(size_yxz=(16, 24, 20), peak=(7, 12, 9), seed=4),                     # border rows overlap (ny < 20)
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("method", ["masked", "median"])
def test_psf_gen_bit_exact_without_resampling(case, method):
    p = synth.measured_psf(**CASES[case])
    got = G.psf_gen_new(p, 0.1, 0.1, 1.5, method)
    ref = OP.psf_gen_new(p, 0.1, 0.1, 1.5, OP.MASKED if method == "masked" else OP.MEDIAN)
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got, ref.astype(np.float32))


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("dz", [0.2, 0.3, 0.25])
def test_psf_gen_axial_resampling(case, dz):
    p = synth.measured_psf(**CASES[case])
    got = G.psf_gen_new(p, 0.1, dz)
    ref = OP.psf_gen_new(p, 0.1, dz)
    assert got.shape == ref.shape
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-6 * float(np.abs(ref).max()))


def test_psf_gen_without_cleanup_is_a_centring_shift():
    p = np.zeros((16, 15, 21), np.float32)
    p[3, 11, 9] = 5.0
    p[4, 12, 10] = -1.0
    got = G.psf_gen_new(p, 0.1, 0.1)
    np.testing.assert_array_equal(got, OP.psf_gen_new(p, 0.1, 0.1))


def test_psf_gen_2d_masked():
    p = synth.measured_psf((48, 40, 1), peak=(20, 22, 0), seed=8)[:, :, 0]
    got = G.psf_gen_new(p, 0.1, 0.1)
    ref = OP.psf_gen_new(p, 0.1, 0.1)
    assert got.shape == (48, 40)
    np.testing.assert_array_equal(got, ref[:, :, 0])


def test_psf_gen_errors():
    with pytest.raises(PkError):
        G.psf_gen_new(np.ones((16, 16, 3), np.float32), 0.1, 0.1)            # fewer than 5 slices
    with pytest.raises(PkError):
        G.psf_gen_new(np.full((8, 16, 12), 200.0, np.float32), 0.1, 0.1)      # fewer than 10 rows
    with pytest.raises(PkError):
        G.psf_gen_new(np.ones((16, 16), np.float32), 0.1, 0.1, 1.5, "median")  # medfilt is undefined
    with pytest.raises(PkError):
        G.psf_gen_new(np.zeros((16, 16, 9), np.float32), 0.1, 0.1)            # all zero


def test_psf_gen_feeds_backprojector_and_decon():
    """The prepared PSF goes straight into the OMW backprojector and a deconvolution call."""
    from petakit5d_b200 import backprojector as B
    from petakit5d_b200 import decon as D
    p = G.psf_gen_new(synth.measured_psf((31, 31, 41), sigma_xy=1.3, sigma_z=3.0, seed=9), 0.1, 0.1)
    b = B.omw_backprojector_generation(p, 0.005, False, OTFCumThresh=0.6)[0]
    vol = synth.puncta_volume((64, 64, 48), 50, synth.gaussian_psf((31, 31, 41)), seed=2)
    out, _ = D.decon_lucy_omw_function(vol, p, b, 2, Background=100)
    assert out.shape == vol.shape and np.isfinite(out.astype(np.float64)).all()
