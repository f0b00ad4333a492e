"""Zarr v2 reader / writer of libpkdecon.so against the format restatement in oracle/zarrio.py
(no GPU)."""
import os

import numpy as np
import pytest

from oracle import zarrio as OZ
from petakit5d_b200 import zarrio as Z
from petakit5d_b200._lib import PkError


def _vol(dtype, shape, seed=0):
    rng = np.random.default_rng(seed)
    a = rng.random(shape) * 1000 if np.dtype(dtype).kind == "f" else rng.integers(0, 60000, shape)
    return np.asfortranarray(a.astype(dtype))


@pytest.mark.parametrize("dtype", [np.uint16, np.float32, np.uint8, np.float64])
@pytest.mark.parametrize("comp", ["zlib", "gzip", None])
def test_written_arrays_read_back_by_the_restatement(tmp_path, dtype, comp):
    v = _vol(dtype, (70, 53, 29))
    p = str(tmp_path / "nested" / "dir" / "a.zarr")
    Z.writezarr(v, p, blockSize=(32, 20, 16), compressor=comp)     # ragged edge chunks on every axis
    np.testing.assert_array_equal(OZ.read(p), v)
    np.testing.assert_array_equal(Z.readzarr(p), v)
    shape, chunks, dt = Z.getZarrInfo(p)
    assert shape == v.shape and chunks == (32, 20, 16) and dt == v.dtype


@pytest.mark.parametrize("order,sep,comp", [("F", ".", "zlib"), ("C", ".", "gzip"), ("F", "/", None),
                                            ("C", "/", "zlib")])
def test_reads_restatement_arrays_and_regions(tmp_path, order, sep, comp):
    v = _vol(np.uint16, (45, 38, 21), seed=1)
    p = str(tmp_path / "b.zarr")
    OZ.write(p, v, (16, 16, 8), order=order, compressor=comp, separator=sep)
    np.testing.assert_array_equal(Z.readzarr(p), v)
    bb = [3, 10, 2, 40, 33, 19]
    np.testing.assert_array_equal(Z.readzarr(p, inputBbox=bb), v[2:40, 9:33, 1:19])


def test_missing_chunks_read_as_fill_value(tmp_path):
    v = _vol(np.uint16, (20, 20, 20), seed=2)
    p = str(tmp_path / "c.zarr")
    OZ.write(p, v, (10, 10, 10), fill_value=7)
    os.remove(os.path.join(p, "1.0.1"))
    ref = v.copy()
    ref[10:20, 0:10, 10:20] = 7
    np.testing.assert_array_equal(Z.readzarr(p), ref)


def test_2d_arrays_and_errors(tmp_path):
    im = _vol(np.uint16, (33, 17), seed=3)
    p = str(tmp_path / "d.zarr")
    Z.writezarr(im, p, blockSize=(16, 16, 16))
    assert Z.getZarrInfo(p)[0] == (33, 17, 1)
    np.testing.assert_array_equal(Z.readzarr(p)[:, :, 0], im)
    with pytest.raises(PkError):
        Z.readzarr(str(tmp_path / "missing.zarr"))
    with pytest.raises(PkError):
        Z.readzarr(p, inputBbox=[1, 1, 1, 40, 17, 1])
    q = str(tmp_path / "e.zarr")
    OZ.write(q, im[:, :, None], (16, 16, 1), compressor="zlib")
    meta = open(os.path.join(q, ".zarray")).read().replace('"zlib"', '"blosc"')
    open(os.path.join(q, ".zarray"), "w").write(meta)
    with pytest.raises(PkError):                      # the reference's default codec: not in this build
        Z.readzarr(q)


def test_region_writes_cover_whole_chunks(tmp_path):
    v = _vol(np.uint16, (50, 40, 30), seed=4)
    p = str(tmp_path / "r.zarr")
    Z.writezarr(np.zeros_like(v), p, blockSize=(16, 16, 8))
    for bb in ([1, 1, 1, 32, 32, 16], [33, 1, 1, 50, 40, 30], [1, 33, 17, 32, 40, 30], [1, 1, 17, 32, 32, 30],
               [1, 33, 1, 32, 40, 16], [33, 1, 1, 50, 40, 30]):
        Z.writezarr_region(np.asfortranarray(v[bb[0] - 1:bb[3], bb[1] - 1:bb[4], bb[2] - 1:bb[5]]), p, bb)
    np.testing.assert_array_equal(Z.readzarr(p), v)
    np.testing.assert_array_equal(OZ.read(p), v)
    with pytest.raises(PkError):                       # not chunk aligned
        Z.writezarr_region(np.zeros((10, 10, 10), np.uint16), p, [2, 1, 1, 11, 10, 10])


@pytest.mark.parametrize("fill", [False, True])
def test_bool_masks_read_as_uint8(tmp_path, fill):
    m = np.asfortranarray(np.random.default_rng(5).random((30, 22, 9)) > 0.4)
    p = str(tmp_path / "m.zarr")
    OZ.write(p, m, (16, 16, 4), fill_value=fill)                   # dtype "|b1", fill_value false / true
    os.remove(os.path.join(p, "1.0.1"))
    ref = m.copy()
    ref[16:30, 0:16, 4:8] = fill
    got = Z.readzarr(p)
    assert got.dtype == np.uint8
    np.testing.assert_array_equal(got, ref.astype(np.uint8))


@pytest.mark.parametrize("comp", ["zlib", "gzip"])
def test_large_chunks_compressed_in_pieces_are_standard_streams(tmp_path, comp):
    """Fewer chunks than threads: each 2.6 MB chunk is deflated as parallel 1 MB pieces joined behind
    one header; Python's zlib / gzip decode every chunk file to the same bytes."""
    v = _vol(np.uint16, (300, 280, 20), seed=6)
    p = str(tmp_path / "big.zarr")
    Z.writezarr(v, p, blockSize=(300, 280, 16), compressor=comp, threads=8)
    np.testing.assert_array_equal(OZ.read(p), v)
    np.testing.assert_array_equal(Z.readzarr(p), v)
    import gzip
    import zlib
    raw = open(os.path.join(p, "0.0.0"), "rb").read()
    body = gzip.decompress(raw) if comp == "gzip" else zlib.decompress(raw)
    assert len(body) == 300 * 280 * 16 * 2


def test_uncompressed_reads_by_pieces_fill_swap_and_truncation(tmp_path):
    v = _vol(np.uint16, (50, 40, 30), seed=7)
    p = str(tmp_path / "u.zarr")
    OZ.write(p, v, (32, 32, 16), compressor=None, fill_value=7)
    os.remove(os.path.join(p, "1.0.1"))
    ref = v.copy()
    ref[32:50, 0:32, 16:30] = 7
    np.testing.assert_array_equal(Z.readzarr(p, threads=8), ref)               # 8 chunks, 8 threads
    np.testing.assert_array_equal(Z.readzarr(p, threads=32), ref)              # 4 z-pieces per chunk
    bb = [5, 3, 2, 47, 38, 29]
    np.testing.assert_array_equal(Z.readzarr(p, inputBbox=bb, threads=16), ref[4:47, 2:38, 1:29])
    pb = str(tmp_path / "be.zarr")
    OZ.write(pb, v.astype(">u2"), (32, 32, 16), compressor=None)
    np.testing.assert_array_equal(Z.readzarr(pb, threads=16), v)
    with open(os.path.join(p, "0.0.0"), "r+b") as f:                            # a truncated chunk
        f.truncate(100)
    with pytest.raises(PkError):
        Z.readzarr(p, threads=16)


def test_region_writes_with_nested_keys(tmp_path):
    """'/' chunk keys (the in-place runner's arrays of more than 10000 chunks): region writes create
    the chunk folders; Python's reading of the format agrees."""
    v = _vol(np.uint16, (40, 36, 20), seed=8)
    p = str(tmp_path / "n.zarr")
    OZ.write(p, np.zeros_like(v), (16, 16, 8), separator="/")
    import shutil
    for d in os.listdir(p):
        if not d.startswith("."):
            shutil.rmtree(os.path.join(p, d))                       # no chunk folders yet
    Z.writezarr_region(v[16:40, 0:32, 8:20], p, [17, 1, 9, 40, 32, 20])
    ref = np.zeros_like(v)
    ref[16:40, 0:32, 8:20] = v[16:40, 0:32, 8:20]
    np.testing.assert_array_equal(OZ.read(p), ref)
    assert os.path.isfile(os.path.join(p, "1", "0", "1"))


def test_runner_arrays_use_nested_keys_past_10000_chunks(tmp_path):
    import json
    from petakit5d_b200.chunking import _create_empty_zarr
    _create_empty_zarr(str(tmp_path / "a.zarr"), (200, 100, 10), (2, 2, 2), np.uint16)      # 25000 chunks
    _create_empty_zarr(str(tmp_path / "b.zarr"), (200, 100, 10), (20, 20, 10), np.uint16)
    sep = [json.load(open(str(tmp_path / f / ".zarray")))["dimension_separator"] for f in ("a.zarr", "b.zarr")]
    assert sep == ["/", "."]


@pytest.mark.parametrize("comp", ["zlib", None])
def test_writezarr_nested_keys(tmp_path, comp):
    """writezarr(..., 'dimSeparator', '/') (io/writezarr.m:21): nested chunk folders, read back by the
    format restatement and by the reader."""
    v = _vol(np.uint16, (50, 40, 30), seed=9)
    p = str(tmp_path / "s.zarr")
    Z.writezarr(v, p, blockSize=(32, 32, 16), compressor=comp, dimSeparator="/")
    assert os.path.isdir(os.path.join(p, "1", "1"))
    np.testing.assert_array_equal(OZ.read(p), v)
    np.testing.assert_array_equal(Z.readzarr(p), v)
    with pytest.raises(ValueError):
        Z.writezarr(v, p, dimSeparator="_")
