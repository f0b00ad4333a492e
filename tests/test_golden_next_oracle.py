"""The oracle reproduces the committed fixtures of the rows next to the path
(tests/golden/make_golden_next.py)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(os.path.join(HERE, "golden", "golden_next.npz")))


@pytest.fixture(scope="module")
def fresh():
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden_next
    return make_golden_next.make()


@pytest.mark.parametrize("key", ["bead", "psfgen_masked", "psfgen_median", "dsr_vol", "dsr_direct_u16",
                                 "dsr_skewed_u16", "dsr_skewed_f32", "edt_im", "edt_mask_e4", "taper_vol",
                                 "taper_u16_nt5"])
def test_exact_fixtures(golden, fresh, key):
    assert np.array_equal(np.asarray(fresh[key]), golden[key])


def test_resampled_fixture(golden, fresh):
    np.testing.assert_allclose(fresh["psfgen_resampled"], golden["psfgen_resampled"], rtol=0, atol=1e-6)
