"""Chunk-grid and size-bucketing restatements (oracle; test infrastructure).

* ``find_good_factor_number`` follows utils/findGoodFactorNumber.m:1-26.
* ``zarr_chunk_coordinates`` follows microscopeDataProcessing/stitch/XR_zarrChunkCoordinatesExtraction.m:1-83.
* ``border_size`` follows RLdecon_large_in_memory.m:177 / RLdecon_large_in_place.m:175.
* ``edt_erosion_mask`` follows RLdecon_large_in_memory.m:153-157 (bwdist through scipy's exact EDT).
"""
from __future__ import annotations

import numpy as np


def _factor(n):
    fs, p = [], 2
    while p * p <= n:
        while n % p == 0:
            fs.append(p)
            n //= p
        p += 1
    if n > 1 or not fs:
        fs.append(n)
    return fs


def find_good_factor_number(n, direction=1, allow_odd_seven=False):
    """Nearest number (stepping by ``direction``) whose prime factors are in {2,3,5,7}; odd numbers
    with a factor 7 are rejected unless ``allow_odd_seven`` (findGoodFactorNumber.m:15-24)."""
    g = int(n)
    f = _factor(g)
    while f[-1] > 7 or (not allow_odd_seven and f[0] > 2 and f[-1] == 7):
        g += direction
        f = _factor(g)
    return g


def border_size(psf_size):
    """``round((size(psf) + 10) / 2)`` (RLdecon_large_in_memory.m:177)."""
    return [int(np.floor((s + 10) / 2.0 + 0.5)) for s in psf_size]


def zarr_chunk_coordinates(vol_size, batch_size=(1024, 1024, 1024), block_size=(256, 256, 256), bbox=None,
                           same_batch_size=True, border=50):
    """XR_zarrChunkCoordinatesExtraction.m:36-81 -> (batchBBoxes, regionBBoxes, localBBoxes), 1-based
    inclusive ``[y1 x1 z1 y2 x2 z2]`` rows, chunks enumerated with y fastest (ndgrid order)."""
    vol = np.array(vol_size, dtype=np.int64)
    if bbox is None or len(bbox) == 0:
        ws = np.array([1, 1, 1], dtype=np.int64)
        we = vol.copy()
    else:
        ws = np.array(bbox[:3], dtype=np.int64)
        we = np.array(bbox[3:], dtype=np.int64)
    wsz = we - ws + 1
    bs = np.minimum(wsz, np.array(batch_size, dtype=np.int64))
    blk = np.minimum(wsz, np.broadcast_to(np.array(block_size, dtype=np.int64), (3,)))
    bs = -(-bs // blk) * blk                                            # ceil(batch/block)*block
    nsub = -(-wsz // bs)
    border = np.broadcast_to(np.array(border, dtype=np.int64), (3,))
    subs = [(y, x, z) for z in range(nsub[2]) for x in range(nsub[1]) for y in range(nsub[0])]
    n = len(subs)
    region = np.zeros((n, 6), dtype=np.int64)
    S = np.array(subs, dtype=np.int64)
    region[:, :3] = S * bs + ws
    region[:, 3:] = np.minimum(region[:, :3] + bs - 1, we)
    batch = region.copy()
    if same_batch_size:
        batch[:, :3] = batch[:, 3:] - bs + 1
    batch[:, :3] = np.maximum(1, batch[:, :3] - border)
    batch[:, 3:] = np.minimum(vol, batch[:, 3:] + border)
    local = np.zeros((n, 6), dtype=np.int64)
    local[:, :3] = region[:, :3] - batch[:, :3] + 1
    local[:, 3:] = local[:, :3] + (region[:, 3:] - region[:, :3])
    region = region - np.concatenate([ws, ws]) + 1
    return batch, region, local


def edt_erosion_mask(im, E):
    """RLdecon_large_in_memory.m:153-157: mask = im > 0 with the six faces cleared, then
    bwdist(~mask) > E - 1 (Euclidean distance to the nearest cleared voxel; scipy's exact EDT)."""
    import scipy.ndimage as ndi
    m = np.asarray(im) > 0
    m[[0, -1], :, :] = False
    m[:, [0, -1], :] = False
    m[:, :, [0, -1]] = False
    if not m.any():
        return m
    return ndi.distance_transform_edt(m) > (E - 1)
