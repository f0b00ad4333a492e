"""The library against the committed fixtures of the rows next to the path (psf_gen_new,
deskewRotateFrame3D, RLdecon's edge taper, the large-file runner's edge erosion)."""
import os

import numpy as np
import pytest

from petakit5d_b200 import chunking as K
from petakit5d_b200 import deskew as G
from petakit5d_b200 import psfgen as P
from petakit5d_b200 import taper as TP

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(os.path.join(HERE, "golden", "golden_next.npz")))


def test_psf_gen_fixtures(golden):
    b = golden["bead"]
    np.testing.assert_array_equal(P.psf_gen_new(b, 0.1, 0.1, 1.5, "masked"), golden["psfgen_masked"])
    np.testing.assert_array_equal(P.psf_gen_new(b, 0.1, 0.1, 1.5, "median"), golden["psfgen_median"])
    r = golden["psfgen_resampled"]
    np.testing.assert_allclose(P.psf_gen_new(b, 0.1, 0.25), r, rtol=0, atol=1e-6 * float(r.max()))


@pytest.mark.parametrize("key,dz,rev,s16,f32", [("dsr_direct_u16", 0.2, True, True, False),
                                                ("dsr_skewed_u16", 0.3, True, True, False),
                                                ("dsr_skewed_f32", 0.3, False, False, True)])
def test_deskew_fixtures(golden, key, dz, rev, s16, f32):
    vol = golden["dsr_vol"].astype(np.float32) if f32 else golden["dsr_vol"]
    got = G.deskewRotateFrame3D(vol, 32.45, dz, 0.108, reverse=rev, save16bit=s16)
    ref = golden[key]
    assert got.shape == ref.shape
    d = np.abs(got.astype(np.float64) - ref.astype(np.float64))
    assert d.max() <= (1 if s16 else 1e-5 * float(ref.max()))
    assert (d == 0).mean() >= 0.999


def test_edge_erosion_fixture(golden):
    m = K.edge_erosion_mask(golden["edt_im"], 4)
    np.testing.assert_array_equal(m.astype(np.uint8), golden["edt_mask_e4"])


def test_edge_taper_fixture(golden):
    got = TP.edgetaper_slices(golden["taper_vol"], TP.fspecial_gaussian(35, 5.0))
    d = np.abs(got.astype(np.int64) - golden["taper_u16_nt5"].astype(np.int64))
    assert d.max() <= 1 and (d == 0).mean() >= 0.999
