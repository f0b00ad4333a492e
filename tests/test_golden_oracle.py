"""The oracle reproduces the committed golden fixtures (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(os.path.join(HERE, "golden", "golden.npz")))


@pytest.fixture(scope="module")
def fresh():
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden
    return make_golden.make()


@pytest.mark.parametrize("key", ["otf_half", "omw2_f32", "rl5_f32", "omw2_offset_erosion", "b_omw", "abs_otf_c",
                                 "wb_psf_bp"])
def test_float_fixtures(golden, fresh, key):
    from oracle import decon as O
    assert fresh[key].shape == golden[key].shape
    assert O.rel_l2(fresh[key], golden[key]) < 1e-6


@pytest.mark.parametrize("key", ["vol", "omw2_u16_bbox", "rl5_u16_damp_scale", "otf_mask", "good_out", "chunk_batch",
                                 "chunk_region", "chunk_local"])
def test_exact_fixtures(golden, fresh, key):
    assert np.array_equal(np.asarray(fresh[key]), golden[key])
