"""Edge erosion of a single plane (decon_mask_edge_erosion.m): MATLAB's ndims of an [ny nx 1] array is
2, so neither branch touches z.  The library against the oracle, both branches."""
import numpy as np
import pytest

from oracle import decon as O
from petakit5d_b200 import decon as D
from petakit5d_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("irregular", [False, True])
def test_single_plane_edge_erosion_matches_oracle(irregular):
    rng = np.random.default_rng(31)
    vol = np.asfortranarray((rng.random((64, 56, 1)) * 2000 + 150).astype(np.uint16))
    if irregular:
        vol[20:30, 10:25, 0] = 0
    psf = synth.gaussian_psf((15, 15, 1), sigma_xy=1.5, sigma_z=1.0)
    J = D.decon_lucy_function(vol, psf, 3, Background=100, deconOffset=5.0, EdgeErosion=3, save16bit=False)[0]
    ref = O.decon_lucy(vol, psf, 3, background=100, offset=5.0, edge_erosion=3, save16bit=False)
    assert J.shape == ref.shape == (64, 56, 1)
    assert np.array_equal(J == 0, ref == 0)                     # the mask is bit-exact
    assert J[40:54, 30:46, 0].all()                              # a plane is not cleared as a z face
    assert O.rel_l2(J, ref) <= 1e-3


@pytest.mark.parametrize("shape,hole", [((40, 36, 20), False), ((40, 36, 20), True), ((40, 36, 1), True),
                                        ((40, 36, 1), False)])
def test_mask_edge_erosion_entry_matches_oracle(shape, hole):
    """pk_mask_edge_erosion (decon_mask_edge_erosion(im > 0, E) on its own) against the oracle."""
    vol = np.asfortranarray((np.random.default_rng(5).random(shape) * 1000 + 1).astype(np.float32))
    if hole:
        vol[10:20, 5:15, :] = 0
    for E in (1, 3, 4):
        got = D.decon_mask_edge_erosion(vol, E)
        np.testing.assert_array_equal(got, O.mask_edge_erosion(vol > 0, E))
