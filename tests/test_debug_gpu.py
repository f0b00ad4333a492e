"""debug = true through the library: err_mat against the oracle's iterates, the uint16 snapshots
written as Iter_%04d.tif, and the deconvolved output unchanged by the debug bookkeeping."""
import os

import numpy as np
import pytest

from oracle import decon as O
from petakit5d_b200 import _lib
from petakit5d_b200 import decon as D
from petakit5d_b200 import synth
from petakit5d_b200.tiff import readtiff

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    vol, psf = synth.single_volume_workload("rl_small", seed=4)
    return vol, psf, np.ascontiguousarray(psf[::-1, ::-1, ::-1])


def _check_err(err, ref):
    assert err.shape == ref.shape
    assert np.array_equal(err[:, 0], ref[:, 0])
    np.testing.assert_allclose(err[:, 1], ref[:, 1], rtol=1e-4)
    np.testing.assert_allclose(err[:, 2], ref[:, 2], rtol=1e-4)
    np.testing.assert_allclose(err[:, 3], ref[:, 3], rtol=1e-2, atol=1e-5)


def test_omw_debug(small, tmp_path):
    vol, psf, psf_b = small
    folder = str(tmp_path / "dbg")
    J, err = D.decon_lucy_omw_function(vol, psf, psf_b, 4, Background=100, save16bit=False, debug=True,
                                       debug_folder=folder, saveStep=2)
    its = []
    O.decon_lucy_omw(vol, psf, psf_b, 4, background=100, save16bit=False, dtype=np.float32, iterates=its)
    Ipre, _ = O.preprocess(vol, 100, False, np.float32)
    _check_err(err, O.debug_err_mat(its, Ipre, 2, "omw"))
    for k in (2, 4):
        snap = readtiff(os.path.join(folder, f"Iter_{k:04d}.tif"))
        assert np.max(np.abs(snap.astype(np.int64) - O.to_uint16(its[k - 1]).astype(np.int64))) <= 1
    plain, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 4, Background=100, save16bit=False)
    assert np.array_equal(J, plain)


def test_rl_debug(small, tmp_path):
    vol, psf, _ = small
    folder = str(tmp_path / "dbg_rl")
    J, err, k = D.decon_lucy_function(vol, psf, 6, Background=100, save16bit=False, debug=True,
                                      debug_folder=folder, saveStep=2)
    assert k == 6
    its = []
    O.decon_lucy(vol, psf, 6, background=100, save16bit=False, dtype=np.float32, iterates=its)
    Ipre, _ = O.preprocess(vol, 100, False, np.float32)
    _check_err(err, O.debug_err_mat(its, Ipre, 2, "rl"))
    assert sorted(os.listdir(folder)) == ["Iter_0002.tif", "Iter_0004.tif", "Iter_0006.tif"]
    plain, _, _ = D.decon_lucy_function(vol, psf, 6, Background=100, save16bit=False)
    assert np.array_equal(J, plain)


def test_rl_debug_without_step_index_is_refused(small, tmp_path):
    vol, psf, _ = small
    with pytest.raises(_lib.PkError):
        D.decon_lucy_function(vol, psf, 5, Background=100, debug=True, debug_folder=str(tmp_path), saveStep=2)
