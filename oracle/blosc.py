"""Blosc chunk format restated in numpy (oracle; test infrastructure).

PetaKit5D's Zarr writer compresses chunks with blosc (io/cpp-zarr/src/parallelwritezarr.cpp:332-345,
defaults cname "lz4", clevel 5, shuffle 1 from io/cpp-zarr/src/zarr.cpp:17) and reads them with
blosc2_decompress (io/cpp-zarr/src/parallelreadzarr.cpp:150-157).  Neither c-blosc nor a Python
binding of it is in this image; this module restates the published blosc chunk layout:

  16-byte header: version, codec version, flags, typesize, then little-endian uint32 nbytes,
  blocksize and cbytes; flags 0x01 byte shuffle, 0x02 stored raw after the header, 0x04 bit shuffle,
  0x10 blocks not split, bits 5-7 the codec (0 blosclz, 1 lz4, 2 snappy, 3 zlib, 4 zstd); one int32
  start offset per block; per block, typesize streams (when split: flag 0x10 clear, typesize <= 16,
  blocksize / typesize >= 128, not the short last block) or one, each an int32 size and the data
  (raw when the size equals the stream's length); the byte shuffle applies per block.

The codecs inside come from independent implementations: LZ4 block format and zstd from pyarrow
(Arrow's bundled lz4 and zstd), zlib from Python's zlib.  The library's own LZ4 codec
(petakit5d_b200/csrc/blosc.cu) is checked against these in tests/test_blosc_cpu.py.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

CODECS = {"blosclz": 0, "lz4": 1, "lz4hc": 1, "snappy": 2, "zlib": 3, "zstd": 4}


def _pa():
    import pyarrow as pa
    return pa


def _decode_stream(codec, data, n):
    if codec == 1:
        return _pa().decompress(data, decompressed_size=n, codec="lz4_raw", asbytes=True)
    if codec == 3:
        return zlib.decompress(data)
    if codec == 4:
        return _pa().decompress(data, decompressed_size=n, codec="zstd", asbytes=True)
    raise NotImplementedError(f"blosc codec {codec}")


def _encode_stream(codec, data, clevel):
    if codec == 1:
        return _pa().compress(data, codec="lz4_raw", asbytes=True)
    if codec == 3:
        return zlib.compress(data, clevel)
    if codec == 4:
        return _pa().compress(data, codec="zstd", asbytes=True)
    raise NotImplementedError(f"blosc codec {codec}")


def _splits(flags, typesize, bsize, leftover):
    return typesize if (not (flags & 0x10) and 1 < typesize <= 16 and bsize // typesize >= 128 and not leftover) else 1


def _shuffle(block, typesize):
    ne = len(block) // typesize
    a = np.frombuffer(block[:ne * typesize], np.uint8).reshape(ne, typesize)
    return a.T.tobytes() + block[ne * typesize:]


def _unshuffle(block, typesize):
    ne = len(block) // typesize
    a = np.frombuffer(block[:ne * typesize], np.uint8).reshape(typesize, ne)
    return a.T.tobytes() + block[ne * typesize:]


def decompress(chunk: bytes) -> bytes:
    """One blosc chunk -> its uncompressed bytes."""
    version, _, flags, typesize, nbytes, blocksize, cbytes = struct.unpack_from("<BBBBIII", chunk, 0)
    if flags & 0x02:
        return bytes(chunk[16:16 + nbytes])
    if flags & 0x04:
        raise NotImplementedError("bit shuffle")
    codec = flags >> 5
    nblocks = nbytes // blocksize + (1 if nbytes % blocksize else 0)
    starts = struct.unpack_from(f"<{nblocks}i", chunk, 16)
    out = bytearray()
    for b in range(nblocks):
        leftover = b == nblocks - 1 and nbytes % blocksize != 0
        bsize = nbytes % blocksize if leftover else blocksize
        ns = _splits(flags, typesize, bsize, leftover)
        ne = bsize // ns
        p = starts[b]
        parts = []
        for _ in range(ns):
            (cs,) = struct.unpack_from("<i", chunk, p)
            p += 4
            data = bytes(chunk[p:p + cs])
            p += cs
            parts.append(data if cs == ne else _decode_stream(codec, data, ne))
        block = b"".join(parts)
        if (flags & 0x01) and typesize > 1:
            block = _unshuffle(block, typesize)
        out += block
    return bytes(out)


def compress(data: bytes, typesize: int, cname: str = "lz4", clevel: int = 5, shuffle: bool = True,
             blocksize: int = 64 * 1024, split: bool = True) -> bytes:
    """Bytes -> one blosc chunk (version 2 layout; blocks split into typesize streams when `split`)."""
    codec = CODECS[cname]
    n = len(data)
    blocksize = min(n, blocksize) if n else 1
    if typesize > 1 and blocksize > typesize:
        blocksize -= blocksize % typesize
    nblocks = n // blocksize + (1 if n % blocksize else 0) if n else 0
    flags = (codec << 5) | (0x01 if shuffle and typesize > 1 else 0) | (0 if split else 0x10)
    body = bytearray()
    starts = []
    hdr_len = 16 + 4 * nblocks
    for b in range(nblocks):
        leftover = b == nblocks - 1 and n % blocksize != 0
        bsize = n % blocksize if leftover else blocksize
        block = data[b * blocksize:b * blocksize + bsize]
        if shuffle and typesize > 1:
            block = _shuffle(block, typesize)
        starts.append(hdr_len + len(body))
        ns = _splits(flags, typesize, bsize, leftover)
        ne = bsize // ns
        for j in range(ns):
            s = block[j * ne:(j + 1) * ne]
            c = _encode_stream(codec, s, clevel)
            if len(c) >= ne:
                c = s
            body += struct.pack("<i", len(c)) + c
    total = hdr_len + len(body)
    head = struct.pack("<BBBBIII", 2, 1, flags, typesize, n, blocksize, total)
    return head + struct.pack(f"<{nblocks}i", *starts) + bytes(body)
