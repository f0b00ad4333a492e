"""The CUDA library against the committed golden fixtures."""
import os

import numpy as np
import pytest

from oracle import decon as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def g():
    return dict(np.load(os.path.join(HERE, "golden", "golden.npz")))


def test_otf(g):
    from petakit5d_b200 import decon as D
    got = D.psf2otf_half(g["psf"], g["vol"].shape)
    assert O.rel_l2(got, g["otf_half"]) < 1e-6


def test_omw_and_rl(g):
    from petakit5d_b200 import decon as D
    J, _ = D.decon_lucy_omw_function(g["vol"], g["psf"], g["psf_b"], 2, Background=100, save16bit=False)
    assert O.rel_l2(J, g["omw2_f32"]) <= 1e-4
    J, _ = D.decon_lucy_omw_function(g["vol"], g["psf"], g["psf_b"], 2, Background=100, bbox=[3, 2, 4, 20, 18, 13])
    assert J.shape == g["omw2_u16_bbox"].shape
    assert np.max(np.abs(J.astype(np.int64) - g["omw2_u16_bbox"].astype(np.int64))) <= 1
    J, _, _ = D.decon_lucy_function(g["vol"], g["psf"], 5, Background=100, save16bit=False)
    assert O.rel_l2(J, g["rl5_f32"]) <= 1e-3
    J, _, _ = D.decon_lucy_function(g["vol"], g["psf"], 5, Background=100, dampFactor=1.5, scaleFactor=2.0)
    assert np.max(np.abs(J.astype(np.int64) - g["rl5_u16_damp_scale"].astype(np.int64))) <= 1
    J, _ = D.decon_lucy_omw_function(g["vol"], g["psf"], g["psf_b"], 2, Background=100, deconOffset=10.0,
                                     EdgeErosion=2, save16bit=False)
    ref = g["omw2_offset_erosion"]
    assert np.array_equal(J == 0, ref == 0)              # the eroded mask is bit-exact
    assert O.rel_l2(J, ref) <= 1e-4


def test_backprojectors(g):
    from petakit5d_b200 import backprojector as B
    b, _, absc, mask = B.omw_backprojector_generation(g["bpsf"], 0.005, False, OTFCumThresh=0.6)
    assert np.array_equal(mask.astype(np.uint8), g["otf_mask"])
    assert O.rel_l2(absc, g["abs_otf_c"]) < 1e-6
    assert O.rel_l2(b, g["b_omw"]) < 1e-5
    pb, _ = B.BackProjector(g["bpsf"], "wiener-butterworth", 0.005, 1e-3, 8, 1)
    assert O.rel_l2(pb, g["wb_psf_bp"]) < 1e-9


def test_tables(g):
    from petakit5d_b200 import chunking as K
    assert [K.find_good_factor_number(int(n)) for n in g["good_in"]] == g["good_out"].tolist()
    bb, rb, lb = K.zarr_chunk_coordinates((300, 257, 129), (128, 100, 64), (32, 32, 32), None, True, (21, 21, 26))
    assert np.array_equal(bb, g["chunk_batch"]) and np.array_equal(rb, g["chunk_region"])
    assert np.array_equal(lb, g["chunk_local"])
