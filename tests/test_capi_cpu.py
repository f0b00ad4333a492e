"""The C ABI library loads and exports every symbol of include/pkdecon.h; host-only entry points
(no GPU work) agree with the oracle's tables."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import chunking as OC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "pkdecon.h")).read()
    return sorted(set(re.findall(r"^PK_API[^;(]*?\b(pk_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_drop_in_entry_points():
    names = _declared()
    for n in ("pk_decon_lucy", "pk_decon_lucy_omw", "pk_omw_backprojector", "pk_wb_backprojector", "pk_backprojector",
              "pk_batch_decon", "pk_server_submit", "pk_find_good_factor_number", "pk_chunk_coordinates"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from petakit5d_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_declared()) == set(_lib.EXPORTED), "ctypes signatures and header disagree"


def test_version_and_defaults():
    from petakit5d_b200 import _lib
    assert b"sm_100a" in _lib.lib.pk_version()
    p = _lib.DeconParams()
    _lib.lib.pk_params_default(p)
    assert (p.background, p.damp_factor, p.scale_factor, p.decon_offset, p.edge_erosion, p.save16bit, p.has_bbox) == \
        (0.0, 1.0, 1.0, 0.0, 0, 1, 0)


def test_output_dims_follow_bbox():
    from petakit5d_b200 import _lib
    p = _lib.DeconParams()
    _lib.lib.pk_params_default(p)
    od = _lib.i64x3([0, 0, 0])
    assert _lib.lib.pk_output_dims(_lib.i64x3([64, 48, 32]), p, od) == 0
    assert list(od) == [64, 48, 32]
    p.has_bbox = 1
    for i, v in enumerate([3, 4, 5, 20, 30, 31]):
        p.bbox[i] = v
    assert _lib.lib.pk_output_dims(_lib.i64x3([64, 48, 32]), p, od) == 0
    assert list(od) == [18, 27, 27]


@pytest.mark.parametrize("n", [1, 7, 14, 31, 41, 101, 352, 416, 544, 1025, 2049, 4097])
def test_good_factor_matches_oracle(n):
    from petakit5d_b200 import _lib
    for d in (1, -1):
        for odd7 in (0, 1):
            if d == -1 and n == 1:
                continue
            assert _lib.lib.pk_find_good_factor_number(n, d, odd7) == OC.find_good_factor_number(n, d, bool(odd7))


@pytest.mark.parametrize("vol,batch,block,border,same", [
    ((10, 7, 5), (4, 4, 5), (2, 2, 5), (1, 1, 1), 0),
    ((10, 7, 5), (4, 4, 5), (2, 2, 5), (1, 1, 1), 1),
    ((2048, 2048, 1024), (512, 512, 512), (512, 512, 512), (32, 32, 32), 0),
    ((300, 257, 129), (128, 100, 64), (32, 32, 32), (21, 21, 26), 1),
])
def test_chunk_coordinates_match_oracle(vol, batch, block, border, same):
    from petakit5d_b200 import _lib
    n = _lib.lib.pk_chunk_coordinates(_lib.i64x3(vol), _lib.i64x3(batch), _lib.i64x3(block), None, same,
                                      _lib.i64x3(border), None, None, None)
    bb = np.zeros((n, 6), np.int64)
    rb = np.zeros((n, 6), np.int64)
    lb = np.zeros((n, 6), np.int64)
    _lib.lib.pk_chunk_coordinates(_lib.i64x3(vol), _lib.i64x3(batch), _lib.i64x3(block), None, same,
                                  _lib.i64x3(border), bb.ctypes.data, rb.ctypes.data, lb.ctypes.data)
    b, r, l = OC.zarr_chunk_coordinates(vol, batch, block, None, bool(same), border)
    assert np.array_equal(bb, b) and np.array_equal(rb, r) and np.array_equal(lb, l)


def test_ctx_create_fails_cleanly_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from petakit5d_b200 import _lib
    assert not _lib.lib.pk_ctx_create(0)
    assert "device" in _lib.last_error()
