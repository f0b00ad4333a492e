"""TIFF reader / writer of libpkdecon.so against libtiff (through PIL and OpenCV) and the format
restatement in oracle/tiff.py (no GPU)."""
import struct

import numpy as np
import pytest

from oracle import tiff as OT
from petakit5d_b200 import tiff as T
from petakit5d_b200._lib import PkError

cv2 = pytest.importorskip("cv2")
Image = pytest.importorskip("PIL.Image")


def _vol(dtype, shape=(70, 53, 5), seed=0):
    rng = np.random.default_rng(seed)
    if np.dtype(dtype).kind == "f":
        a = rng.random(shape) * 1000
    else:
        # smooth ramps plus noise: long LZW strings, tables that fill and clear
        a = (np.cumsum(rng.integers(0, 3, shape), axis=1) + rng.integers(0, 4, shape)) % np.iinfo(dtype).max
    return np.asfortranarray(a.astype(dtype))


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32])
@pytest.mark.parametrize("comp", ["lzw", "none"])
def test_written_files_read_back_with_libtiff(tmp_path, dtype, comp):
    v = _vol(dtype, (700, 61, 3))               # 700 rows: two 512-row strips per page
    p = str(tmp_path / "a.tif")
    T.writetiff(v, p, Compression=comp)
    ok, pages = cv2.imreadmulti(p, flags=cv2.IMREAD_UNCHANGED)
    assert ok and len(pages) == 3
    for k in range(3):
        np.testing.assert_array_equal(pages[k], v[:, :, k])
    np.testing.assert_array_equal(OT.read_volume(p), v)
    np.testing.assert_array_equal(T.readtiff(p), v)
    assert T.getImageSize(p) == v.shape


@pytest.mark.parametrize("dtype,mode", [(np.uint16, "I;16"), (np.float32, "F"), (np.uint8, "L")])
def test_reads_libtiff_lzw_pages(tmp_path, dtype, mode):
    v = _vol(dtype, (300, 257, 1), seed=1)[:, :, 0]
    p = str(tmp_path / "p.tif")
    Image.fromarray(np.ascontiguousarray(v)).save(p, compression="tiff_lzw")
    np.testing.assert_array_equal(T.readtiff(p), v)


@pytest.mark.parametrize("comp,pred,rows", [(cv2.IMWRITE_TIFF_COMPRESSION_LZW, cv2.IMWRITE_TIFF_PREDICTOR_HORIZONTAL, 7),
                                            (cv2.IMWRITE_TIFF_COMPRESSION_LZW, cv2.IMWRITE_TIFF_PREDICTOR_NONE, 64),
                                            (cv2.IMWRITE_TIFF_COMPRESSION_DEFLATE, cv2.IMWRITE_TIFF_PREDICTOR_HORIZONTAL, 16),
                                            (cv2.IMWRITE_TIFF_COMPRESSION_NONE, cv2.IMWRITE_TIFF_PREDICTOR_NONE, 5)])
def test_reads_libtiff_multipage_strips_and_predictor(tmp_path, comp, pred, rows):
    v = _vol(np.uint16, (123, 97, 4), seed=2)
    p = str(tmp_path / "m.tif")
    assert cv2.imwritemulti(p, [np.ascontiguousarray(v[:, :, k]) for k in range(4)],
                            [cv2.IMWRITE_TIFF_COMPRESSION, comp, cv2.IMWRITE_TIFF_PREDICTOR, pred,
                             cv2.IMWRITE_TIFF_ROWSPERSTRIP, rows])
    np.testing.assert_array_equal(T.readtiff(p), v)
    np.testing.assert_array_equal(T.readtiff(p, range=[2, 3]), v[:, :, 1:3])


def _classic(path, pages, bo="<", strips=None, desc=None, raw_stack=False):
    """Hand-built classic TIFF: uint16 pages, one strip each (LZW strips when ``strips`` is given)."""
    h, w = pages[0].shape
    data = [strips[k] if strips else pages[k].astype(np.dtype(np.uint16).newbyteorder(bo)).tobytes()
            for k in range(len(pages))]
    if raw_stack:
        data = [b"".join(data)]
    out = bytearray(b"II*\0" if bo == "<" else b"MM\0*") + b"\0\0\0\0"
    offs = []
    for d in data:
        offs.append(len(out))
        out += d
    ifds = []
    for k, d in enumerate(data):
        if len(out) % 2:
            out += b"\0"
        ents = [(256, 4, 1, w), (257, 4, 1, h), (258, 3, 1, 16), (259, 3, 1, 5 if strips else 1), (262, 3, 1, 1),
                (273, 4, 1, offs[k]), (277, 3, 1, 1), (278, 4, 1, h), (279, 4, 1, len(d))]
        dpos = None
        if desc is not None:
            dpos = len(out)
            out += desc.encode() + b"\0"
            if len(out) % 2:
                out += b"\0"
            ents.append((270, 2, len(desc) + 1, dpos))
        ents.sort()
        ifds.append(len(out))
        out += struct.pack(bo + "H", len(ents))
        for tag, typ, cnt, val in ents:
            if typ == 3:
                out += struct.pack(bo + "HHIHH", tag, typ, cnt, val, 0)
            else:
                out += struct.pack(bo + "HHII", tag, typ, cnt, val)
        out += b"\0\0\0\0"
    for k in range(len(ifds) - 1):
        nxt = ifds[k + 1]
        n = struct.unpack(bo + "H", out[ifds[k]:ifds[k] + 2])[0]
        out[ifds[k] + 2 + 12 * n:ifds[k] + 6 + 12 * n] = struct.pack(bo + "I", nxt)
    out[4:8] = struct.pack(bo + "I", ifds[0])
    with open(path, "wb") as f:
        f.write(out)


def test_big_endian_and_oracle_lzw_strips(tmp_path):
    v = _vol(np.uint16, (40, 33, 3), seed=3)
    pages = [v[:, :, k] for k in range(3)]
    p = str(tmp_path / "be.tif")
    _classic(p, pages, bo=">")
    np.testing.assert_array_equal(T.readtiff(p), v)
    np.testing.assert_array_equal(np.asarray(Image.open(p)), v[:, :, 0])     # the hand-built file is valid
    # LZW strips from the oracle encoder, decoded by the library and by libtiff
    q = str(tmp_path / "lz.tif")
    _classic(q, pages, strips=[OT.lzw_encode(np.ascontiguousarray(pg).astype("<u2").tobytes()) for pg in pages])
    np.testing.assert_array_equal(T.readtiff(q), v)
    np.testing.assert_array_equal(np.asarray(Image.open(q)), v[:, :, 0])


def test_imagej_raw_stack(tmp_path):
    v = _vol(np.uint16, (20, 24, 6), seed=4)
    p = str(tmp_path / "ij.tif")
    _classic(p, [v[:, :, k] for k in range(6)], desc="ImageJ=1.54f\nimages=6\nslices=6\n", raw_stack=True)
    assert T.getImageSize(p) == (20, 24, 6)
    np.testing.assert_array_equal(T.readtiff(p), v)
    np.testing.assert_array_equal(T.readtiff(p, range=[3, 5]), v[:, :, 2:5])


def test_single_page_is_2d_and_lzw_round_trip_of_degenerate_rows(tmp_path):
    p = str(tmp_path / "s.tif")
    v = np.zeros((513, 1, 1), np.uint16)           # one column, a 1-row second strip, all zeros
    T.writetiff(v, p)
    back = T.readtiff(p)
    assert back.shape == (513, 1)
    np.testing.assert_array_equal(back, v[:, :, 0])
    w = _vol(np.float64, (9, 8, 2), seed=5)
    T.writetiff(w, p)
    np.testing.assert_array_equal(T.readtiff(p), w)


def test_errors(tmp_path):
    bad = tmp_path / "x.tif"
    bad.write_bytes(b"not a tiff at all")
    with pytest.raises(PkError):
        T.readtiff(bad)
    with pytest.raises(PkError):
        T.readtiff(tmp_path / "missing.tif")
    p = str(tmp_path / "r.tif")
    T.writetiff(_vol(np.uint16, (8, 8, 3)), p)
    with pytest.raises(PkError):
        T.readtiff(p, range=[2, 4])
    with pytest.raises(TypeError):
        T.writetiff(np.zeros((4, 4), np.int16), p)
