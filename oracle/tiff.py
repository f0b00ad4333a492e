"""TIFF restatement for the I/O either side of the deconvolution path (oracle; test infrastructure).

The reference reads and writes its volumes with parallelReadTiff / parallelWriteTiff
(microscopeDataProcessing/io/cpp-tiff/src/parallelreadtiff.cpp, parallelwritetiff.cpp, called
from io/readtiff.m and io/writetiff.m), which sit on libtiff.  What is restated here is the published
format those files use (TIFF 6.0 and BigTIFF), not their code:
  * LZW (TIFF 6.0 section 13): codes 0-255 literal, 256 Clear, 257 EndOfInformation, 258.. table
    entries; 9- to 12-bit codes packed most-significant bit first; the code width grows one code
    early ("early change": the decoder widens after adding entry 510, 1022, 2046); the encoder emits
    Clear when entry 4093 has been added.
  * Horizontal differencing (Predictor = 2) per row of samples.
  * The volume orientation of the MEX files: a MATLAB array [ny nx nz] is stored with ImageLength ny,
    ImageWidth nx, one page per z (so each page is the transpose of the column-major plane).
The CUDA library's C++ reader / writer is checked against this module and against libtiff itself
(through PIL and OpenCV) in tests/test_tiffio_cpu.py.
"""
from __future__ import annotations

import struct

import numpy as np

CLEAR, EOI, FIRST = 256, 257, 258


def lzw_encode(data: bytes) -> bytes:
    out = bytearray()
    acc = 0
    nacc = 0

    def put(code, width):
        nonlocal acc, nacc
        acc = (acc << width) | code
        nacc += width
        while nacc >= 8:
            nacc -= 8
            out.append((acc >> nacc) & 0xFF)
        acc &= (1 << nacc) - 1 if nacc else 0

    width = 9
    table = {}
    nxt = FIRST
    put(CLEAR, width)
    if not data:
        put(EOI, width)
        if nacc:
            out.append((acc << (8 - nacc)) & 0xFF)
        return bytes(out)
    w = data[0]
    for k in data[1:]:
        key = (w, k)
        if key in table:
            w = table[key]
            continue
        put(w, width)
        table[key] = nxt
        nxt += 1
        if nxt == 4094:
            put(CLEAR, width)
            table.clear()
            nxt = FIRST
            width = 9
        elif nxt > (1 << width) - 1:
            width += 1
        w = k
    put(w, width)
    nxt += 1
    if nxt == 4094:
        put(CLEAR, width)
        width = 9
    elif nxt > (1 << width) - 1:
        width += 1
    put(EOI, width)
    if nacc:
        out.append((acc << (8 - nacc)) & 0xFF)
    return bytes(out)


def lzw_decode(data: bytes, expected: int | None = None) -> bytes:
    out = bytearray()
    pos = 0            # bit position
    nbits = len(data) * 8
    width = 9
    table = [bytes([i]) for i in range(256)] + [b"", b""]
    prev = None

    def get(width):
        nonlocal pos
        if pos + width > nbits:
            return EOI
        v = 0
        for _ in range(width):
            byte = data[pos >> 3]
            v = (v << 1) | ((byte >> (7 - (pos & 7))) & 1)
            pos += 1
        return v

    while True:
        code = get(width)
        if code == EOI:
            break
        if code == CLEAR:
            table = table[:FIRST]
            width = 9
            prev = None
            code = get(width)
            if code == EOI:
                break
            out += table[code]
            prev = code
            continue
        if code < len(table):
            s = table[code]
            if prev is not None:
                table.append(table[prev] + s[:1])
        elif code == len(table) and prev is not None:
            s = table[prev] + table[prev][:1]
            table.append(s)
        else:
            raise ValueError("corrupt LZW stream")
        out += s
        prev = code
        if len(table) == (1 << width) - 1 and width < 12:
            width += 1
        if expected is not None and len(out) >= expected:
            break
    return bytes(out)


_TYPES = {1: "B", 2: "B", 3: "H", 4: "I", 5: "II", 6: "b", 7: "B", 8: "h", 9: "i", 11: "f", 12: "d", 16: "Q", 17: "q"}
_SIZE = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 6: 1, 7: 1, 8: 2, 9: 4, 11: 4, 12: 8, 16: 8, 17: 8}


def read_pages(path):
    """Parse every IFD of a classic or BigTIFF file: list of {tag: values}."""
    with open(path, "rb") as f:
        buf = f.read()
    bo = "<" if buf[:2] == b"II" else ">"
    magic = struct.unpack(bo + "H", buf[2:4])[0]
    big = magic == 43
    off = struct.unpack(bo + ("Q" if big else "I"), buf[8:16] if big else buf[4:8])[0]
    pages = []
    while off:
        n = struct.unpack(bo + ("Q" if big else "H"), buf[off:off + (8 if big else 2)])[0]
        p = off + (8 if big else 2)
        tags = {}
        for _ in range(n):
            if big:
                tag, typ, cnt = struct.unpack(bo + "HHQ", buf[p:p + 12])
                field = buf[p + 12:p + 20]
                p += 20
            else:
                tag, typ, cnt = struct.unpack(bo + "HHI", buf[p:p + 8])
                field = buf[p + 8:p + 12]
                p += 12
            size = _SIZE.get(typ, 1) * cnt
            if size > len(field):
                voff = struct.unpack(bo + ("Q" if big else "I"), field)[0]
                raw = buf[voff:voff + size]
            else:
                raw = field[:size]
            fmt = _TYPES.get(typ, "B")
            tags[tag] = list(struct.unpack(bo + fmt * (cnt if len(fmt) == 1 else cnt), raw)) if typ != 2 else raw
        pages.append(tags)
        off = struct.unpack(bo + ("Q" if big else "I"), buf[p:p + (8 if big else 4)])[0]
    return pages, buf, bo


def read_volume(path):
    """Pages of a strip TIFF as a MATLAB-ordered array [ny nx nz] (uncompressed or LZW, predictor 1/2)."""
    pages, buf, bo = read_pages(path)
    out = []
    for t in pages:
        w, h = t[256][0], t[257][0]
        bits = t.get(258, [1])[0]
        fmt = t.get(339, [1])[0]
        comp = t.get(259, [1])[0]
        pred = t.get(317, [1])[0]
        dt = {(8, 1): np.uint8, (16, 1): np.uint16, (32, 1): np.uint32, (32, 3): np.float32,
              (64, 3): np.float64}[(bits, fmt)]
        dt = np.dtype(dt).newbyteorder(bo)
        rows = t.get(278, [h])[0]
        page = bytearray()
        for k, (so, sc) in enumerate(zip(t[273], t[279])):
            nrow = min(rows, h - k * rows)
            raw = buf[so:so + sc]
            if comp == 5:
                raw = lzw_decode(raw, nrow * w * bits // 8)[:nrow * w * bits // 8]
            elif comp != 1:
                raise NotImplementedError(f"compression {comp}")
            page += raw
        a = np.frombuffer(bytes(page), dtype=dt).reshape(h, w).astype(dt.newbyteorder("="))
        if pred == 2:
            a = np.cumsum(a, axis=1, dtype=a.dtype)
        out.append(a)
    return np.stack(out, axis=2)
