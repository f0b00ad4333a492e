"""RLdecon option handling that needs no GPU."""
import os

import numpy as np
import pytest

from petakit5d_b200 import tiff as T
from petakit5d_b200 import zarrio as Z
from petakit5d_b200.rldecon import RLdecon


@pytest.mark.parametrize("kw,err", [({"RLMethod": "original"}, NotImplementedError),
                                    ({"RLMethod": "cudagen"}, NotImplementedError),
                                    ({"Deskew": True, "DSRCombined": False, "Rotate": True}, NotImplementedError),
                                    ({"Deskew": True, "Rotate": False}, NotImplementedError),
                                    ({"notAnOption": 1}, TypeError),
                                    ({"RLMethod": "fancy"}, ValueError)])
def test_rejected_options(kw, err):
    with pytest.raises(err):
        RLdecon("in.tif", "out.tif", "psf.tif", 0.108, 0.3, 0.1, **kw)


@pytest.mark.parametrize("save_zarr", [False, True])
def test_zero_iterations_write_the_input_through_the_chosen_writer(tmp_path, save_zarr):
    """DeconIter = 0 passes the (cropped) data through (RLdecon.m:414-419); saveZarr picks the Zarr
    writer with the run's blockSize (:126-130, :560-562) and the maximum projections stay TIFF."""
    vol = np.asfortranarray(np.random.default_rng(0).integers(0, 5000, (40, 36, 12)).astype(np.uint16))
    out = str(tmp_path / "d" / ("frame.zarr" if save_zarr else "frame.tif"))
    bb = [3, 4, 2, 38, 30, 11]
    J, _, _ = RLdecon("", out, None, 0.108, 0.3, 0.1, rawdata=vol, DeconIter=0, saveZarr=save_zarr,
                      blockSize=[16, 16, 8], deconBbox=bb)
    ref = vol[2:38, 3:30, 1:11]
    np.testing.assert_array_equal(J, ref)
    if save_zarr:
        assert os.path.isdir(out) and Z.getZarrInfo(out)[1] == (16, 16, 8)
        np.testing.assert_array_equal(Z.readzarr(out), ref)
    else:
        np.testing.assert_array_equal(T.readtiff(out), ref)
    np.testing.assert_array_equal(T.readtiff(str(tmp_path / "d" / "MIPs" / "frame_MIP_z.tif")), ref.max(axis=2))
    assert sorted(os.listdir(tmp_path / "d")) == ["MIPs", os.path.basename(out)]   # no temporaries left


def test_frame3d_options_and_skips(tmp_path):
    """XR_RLdeconFrame3D.m:145-193: nothing to save is an error; missing frames and frames whose
    result exists (without Overwrite) are skipped before any GPU work."""
    import warnings
    from petakit5d_b200.rldecon import XR_RLdeconFrame3D
    with pytest.raises(ValueError):
        XR_RLdeconFrame3D(["a.tif"], 0.108, 0.3, str(tmp_path), save3Dstack=[False, False, False], mipAxis=[0, 0, 0])
    with pytest.raises(TypeError):
        XR_RLdeconFrame3D(["a.tif"], 0.108, 0.3, str(tmp_path), notAnOption=1)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        XR_RLdeconFrame3D([str(tmp_path / "missing.tif")], 0.108, 0.3, str(tmp_path))
    assert any("does not exist" in str(x.message) for x in w)
    raw = str(tmp_path / "frame.tif")
    T.writetiff(np.ones((8, 8, 4), np.uint16), raw)
    os.makedirs(tmp_path / "matlab_decon")
    T.writetiff(np.full((8, 8, 4), 3, np.uint16), str(tmp_path / "matlab_decon" / "frame.tif"))
    XR_RLdeconFrame3D([raw], 0.108, 0.3, "", PSFfile="psf.tif")       # the result exists: skipped
    assert T.readtiff(str(tmp_path / "matlab_decon" / "frame.tif")).max() == 3
