"""RLdecon option handling that needs no GPU."""
import pytest

from petakit5d_b200.rldecon import RLdecon


@pytest.mark.parametrize("kw,err", [({"saveZarr": True}, NotImplementedError),
                                    ({"RLMethod": "original"}, NotImplementedError),
                                    ({"RLMethod": "cudagen"}, NotImplementedError),
                                    ({"Deskew": True, "DSRCombined": False, "Rotate": True}, NotImplementedError),
                                    ({"notAnOption": 1}, TypeError),
                                    ({"RLMethod": "fancy"}, ValueError)])
def test_rejected_options(kw, err):
    with pytest.raises(err):
        RLdecon("in.tif", "out.tif", "psf.tif", 0.108, 0.3, 0.1, **kw)
