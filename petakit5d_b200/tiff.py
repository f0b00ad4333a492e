"""Minimal uncompressed multi-page TIFF writer for uint16 volumes (the debug runs' Iter_%04d.tif).

A MATLAB [ny nx nz] volume is written as nz pages of ny rows by nx columns (the layout writetiff in
the reference produces for its debug snapshots): little-endian, one strip per page, 16-bit
unsigned, min-is-black.  No compression and no ImageJ metadata.
"""
from __future__ import annotations

import struct

import numpy as np

_TAGS_PER_PAGE = 10


def write_tiff(path, vol):
    """Write ``vol`` ([ny, nx, nz] or [ny, nx], uint16) to ``path``."""
    v = np.asarray(vol)
    if v.dtype != np.uint16:
        raise TypeError("write_tiff takes uint16 volumes")
    if v.ndim == 2:
        v = v[:, :, None]
    ny, nx, nz = v.shape
    page_bytes = ny * nx * 2
    ifd_bytes = 2 + 12 * _TAGS_PER_PAGE + 4
    with open(path, "wb") as f:
        f.write(b"II" + struct.pack("<HI", 42, 8))
        pos = 8
        for z in range(nz):
            ifd_pos = pos
            data_pos = ifd_pos + ifd_bytes
            next_ifd = data_pos + page_bytes if z + 1 < nz else 0
            tags = [                                    # (tag, type, count, value); 3 = SHORT, 4 = LONG
                (256, 4, 1, nx),                        # ImageWidth (columns = x)
                (257, 4, 1, ny),                        # ImageLength (rows = y)
                (258, 3, 1, 16),                        # BitsPerSample
                (259, 3, 1, 1),                         # Compression: none
                (262, 3, 1, 1),                         # Photometric: min-is-black
                (273, 4, 1, data_pos),                  # StripOffsets
                (277, 3, 1, 1),                         # SamplesPerPixel
                (278, 4, 1, ny),                        # RowsPerStrip
                (279, 4, 1, page_bytes),                # StripByteCounts
                (339, 3, 1, 1),                         # SampleFormat: unsigned
            ]
            f.write(struct.pack("<H", len(tags)))
            for tag, typ, cnt, val in tags:
                f.write(struct.pack("<HHI", tag, typ, cnt))
                f.write(struct.pack("<HH", val, 0) if typ == 3 else struct.pack("<I", val))
            f.write(struct.pack("<I", next_ifd))
            f.write(np.ascontiguousarray(v[:, :, z]).astype("<u2").tobytes())   # row-major: rows = y
            pos = data_pos + page_bytes


def read_tiff(path):
    """Read a file written by write_tiff back into a [ny, nx, nz] uint16 array (for tests)."""
    with open(path, "rb") as f:
        b = f.read()
    if b[:4] != b"II*\x00":
        raise ValueError("not a little-endian TIFF")
    (off,) = struct.unpack_from("<I", b, 4)
    pages = []
    while off:
        (n,) = struct.unpack_from("<H", b, off)
        t = {}
        for i in range(n):
            tag, typ, cnt = struct.unpack_from("<HHI", b, off + 2 + 12 * i)
            val = struct.unpack_from("<H" if typ == 3 else "<I", b, off + 2 + 12 * i + 8)[0]
            t[tag] = val
        nx, ny = t[256], t[257]
        data = np.frombuffer(b, "<u2", ny * nx, t[273]).reshape(ny, nx)
        pages.append(data)
        (off,) = struct.unpack_from("<I", b, off + 2 + 12 * n)
    return np.stack(pages, axis=2)
