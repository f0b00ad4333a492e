"""Zarr v2 restatement (oracle; test infrastructure).

Reads and writes Zarr v2 arrays from the published storage specification with json, zlib, gzip,
numpy and the blosc chunk restatement of oracle/blosc.py, to check libpkdecon.so's reader / writer
(tests/test_zarrio_cpu.py, tests/test_blosc_cpu.py): ``.zarray`` with
shape, chunks, dtype, order, compressor, fill_value and dimension_separator; one file per chunk named
by its chunk indices; every chunk stored at full chunk size, in order "F" or "C".
"""
from __future__ import annotations

import gzip
import json
import os
import zlib

import numpy as np

from . import blosc


def write(path, a, chunks, order="F", compressor="zlib", separator=".", fill_value=0, cname="lz4", split=True):
    a = np.asarray(a)
    os.makedirs(path, exist_ok=True)
    if compressor == "blosc":
        comp = {"blocksize": 0, "clevel": 5, "cname": cname, "id": "blosc", "shuffle": 1}
    else:
        comp = None if compressor is None else {"id": compressor, "level": 1}
    meta = {"chunks": list(chunks), "compressor": comp, "dimension_separator": separator,
            "dtype": a.dtype.str, "fill_value": fill_value, "filters": None, "order": order,
            "shape": list(a.shape), "zarr_format": 2}
    with open(os.path.join(path, ".zarray"), "w") as f:
        json.dump(meta, f)
    grid = [-(-s // c) for s, c in zip(a.shape, chunks)]
    for idx in np.ndindex(*grid):
        blk = np.full(chunks, fill_value, a.dtype)
        sl = tuple(slice(i * c, min((i + 1) * c, s)) for i, c, s in zip(idx, chunks, a.shape))
        part = a[sl]
        blk[tuple(slice(0, n) for n in part.shape)] = part
        raw = blk.tobytes(order=order)
        if compressor == "zlib":
            raw = zlib.compress(raw, 1)
        elif compressor == "gzip":
            raw = gzip.compress(raw, 1)
        elif compressor == "blosc":
            raw = blosc.compress(raw, a.dtype.itemsize, cname=cname, split=split)
        key = separator.join(str(i) for i in idx)
        fn = os.path.join(path, *key.split("/")) if separator == "/" else os.path.join(path, key)
        os.makedirs(os.path.dirname(fn), exist_ok=True)
        with open(fn, "wb") as f:
            f.write(raw)


def read(path):
    with open(os.path.join(path, ".zarray")) as f:
        meta = json.load(f)
    shape, chunks = meta["shape"], meta["chunks"]
    dt = np.dtype(meta["dtype"])
    order = meta.get("order", "C")
    sep = meta.get("dimension_separator", ".")
    comp = (meta.get("compressor") or {}).get("id")
    fill = meta.get("fill_value") or 0
    out = np.empty(shape, dt)
    grid = [-(-s // c) for s, c in zip(shape, chunks)]
    for idx in np.ndindex(*grid):
        fn = os.path.join(path, sep.join(str(i) for i in idx))
        if os.path.exists(fn):
            with open(fn, "rb") as f:
                raw = f.read()
            if comp == "zlib":
                raw = zlib.decompress(raw)
            elif comp == "gzip":
                raw = gzip.decompress(raw)
            elif comp == "blosc":
                raw = blosc.decompress(raw)
            blk = np.frombuffer(raw, dt).reshape(chunks, order=order)
        else:
            blk = np.full(chunks, fill, dt)
        sl = tuple(slice(i * c, min((i + 1) * c, s)) for i, c, s in zip(idx, chunks, shape))
        out[sl] = blk[tuple(slice(0, x.stop - x.start) for x in sl)]
    return out
