"""Blosc Zarr chunks (the reference's default codec, io/cpp-zarr/src/zarr.cpp:17): the library's
reader and writer against the blosc chunk restatement of oracle/blosc.py, whose LZ4 and zstd streams
come from pyarrow's bundled lz4 and zstd (implementations independent of csrc/blosc.cu)."""
import numpy as np
import pytest

from oracle import blosc as OB
from oracle import zarrio as OZ


def _vol(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    if np.dtype(dtype).kind == "f":
        return np.asfortranarray(rng.normal(100, 20, size=shape).astype(dtype))
    base = rng.poisson(120, size=shape) + (np.arange(shape[0])[:, None, None] % 7) * 30
    return np.asfortranarray(base.astype(dtype))


@pytest.mark.parametrize("cname", ["lz4", "zstd", "zlib"])
@pytest.mark.parametrize("split", [True, False])
def test_library_reads_restatement_blosc_chunks(tmp_path, cname, split):
    from petakit5d_b200 import zarrio as Z
    a = _vol((130, 70, 45), np.uint16, 1)
    p = str(tmp_path / "a.zarr")
    OZ.write(p, a, (64, 32, 20), compressor="blosc", cname=cname, split=split)
    assert np.array_equal(Z.readzarr(p), a)
    assert np.array_equal(Z.readzarr(p, inputBbox=[5, 9, 3, 100, 61, 40]), a[4:100, 8:61, 2:40])


@pytest.mark.parametrize("comp", ["blosc", "blosc-zstd", "blosc-zlib"])
@pytest.mark.parametrize("dtype", [np.uint16, np.float32, np.uint8])
def test_library_blosc_chunks_read_by_the_restatement(tmp_path, comp, dtype):
    from petakit5d_b200 import zarrio as Z
    a = _vol((96, 50, 33), dtype, 2)
    p = str(tmp_path / "b.zarr")
    Z.writezarr(a, p, blockSize=(64, 32, 16), compressor=comp)
    assert np.array_equal(OZ.read(p), a)
    assert np.array_equal(Z.readzarr(p), a)


def test_lz4_streams_against_pyarrow():
    """The library's LZ4 block encoder and decoder, through blosc chunks: chunks the library wrote
    decode with pyarrow's LZ4 (the restatement), and large repetitive and random data round-trip."""
    import json
    import os
    import tempfile
    from petakit5d_b200 import zarrio as Z
    rng = np.random.default_rng(3)
    cases = [np.zeros((300, 200, 2), np.uint16), rng.integers(0, 65535, (300, 200, 2)).astype(np.uint16),
             np.tile(np.arange(300, dtype=np.uint16)[:, None, None], (1, 200, 2))]
    for i, a in enumerate(cases):
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, f"c{i}.zarr")
            Z.writezarr(np.asfortranarray(a), p, blockSize=(300, 200, 2), compressor="blosc")
            with open(os.path.join(p, ".zarray")) as f:
                meta = json.load(f)
            assert meta["compressor"]["id"] == "blosc" and meta["compressor"]["cname"] == "lz4"
            with open(os.path.join(p, "0.0.0"), "rb") as f:
                raw = f.read()
            assert np.array_equal(np.frombuffer(OB.decompress(raw), np.uint16).reshape(a.shape, order="F"), a)
            assert np.array_equal(Z.readzarr(p), a)


def test_corrupt_and_unsupported_blosc_chunks(tmp_path):
    from petakit5d_b200 import _lib
    from petakit5d_b200 import zarrio as Z
    a = _vol((64, 32, 8), np.uint16, 4)
    p = str(tmp_path / "c.zarr")
    OZ.write(p, a, (64, 32, 8), compressor="blosc", cname="lz4")
    fn = str(tmp_path / "c.zarr" / "0.0.0")
    raw = bytearray(open(fn, "rb").read())
    bad = bytes(raw[:len(raw) // 2])                    # truncated
    open(fn, "wb").write(bad)
    with pytest.raises(_lib.PkError):
        Z.readzarr(p)
    raw[2] = (raw[2] & 0x1F) | (0 << 5)                 # codec 0 (blosclz): refused, not misread
    open(fn, "wb").write(bytes(raw))
    with pytest.raises(_lib.PkError):
        Z.readzarr(p)
