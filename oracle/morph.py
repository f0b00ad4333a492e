"""Binary morphology used by omw_backprojector_generation.m (oracle; test infrastructure).

Arrays are indexed ``m[y, x, z]``.  Conventions restated from the MATLAB Image Processing Toolbox
calls at omw_backprojector_generation.m:44-48,73-109,122:
  * ``strel('sphere', r)``: voxels with dy^2+dx^2+dz^2 <= r^2.
  * ``imerode``: AND over the neighbourhood, voxels outside the volume count as true.
  * ``imdilate``: OR over the neighbourhood, voxels outside the volume count as false.
  * ``imopen`` = dilate(erode(.)), ``imclose`` = erode(dilate(.)).
  * connectivity 26 for ``bwareaopen`` / ``bwconncomp`` / ``bwlabeln``; components are numbered in
    MATLAB linear (column-major, y fastest) order of their first voxel.
  * ``bwconvhull(slice, 'union')``: convex hull of the corners (+-0.5) of every foreground pixel;
    a pixel is set when its centre lies inside the hull or on its boundary.  (MATLAB's exact
    boundary rule is not pinned; the CUDA library uses this same rule.)
"""
from __future__ import annotations

import numpy as np
import scipy.ndimage as ndi


def sphere_offsets(r):
    g = np.arange(-r, r + 1)
    return [(a, b, c) for a in g for b in g for c in g if a * a + b * b + c * c <= r * r]


def _shift_and(mask, offsets, outside):
    """AND (erosion, outside=True) or OR (dilation, outside=False) of shifted copies."""
    sh = mask.shape
    acc = None
    for off in offsets:
        shifted = np.full_like(mask, outside)
        src = tuple(slice(max(0, o), sh[i] + min(0, o)) for i, o in enumerate(off))
        dst = tuple(slice(max(0, -o), sh[i] + min(0, -o)) for i, o in enumerate(off))
        shifted[dst] = mask[src]
        acc = shifted if acc is None else (acc & shifted if outside else acc | shifted)
    return acc


def erode(mask, r):
    return _shift_and(mask.astype(bool), sphere_offsets(r), True)


def dilate(mask, r):
    return _shift_and(mask.astype(bool), sphere_offsets(r), False)


def imopen(mask, r):
    return dilate(erode(mask, r), r)


def imclose(mask, r):
    return erode(dilate(mask, r), r)


def label26(mask):
    """Connected components (26-connectivity) numbered in MATLAB linear order; returns (labels, n)."""
    t = np.ascontiguousarray(mask.transpose(2, 1, 0))   # C-order raster == MATLAB linear order
    lab, n = ndi.label(t, structure=np.ones((3, 3, 3), dtype=bool))
    return lab.transpose(2, 1, 0), n


def bwareaopen(mask, P):
    lab, n = label26(mask)
    if n == 0:
        return mask.astype(bool)
    sizes = np.bincount(lab.ravel(), minlength=n + 1)
    keep = sizes >= P
    keep[0] = False
    return keep[lab]


def largest_component(mask):
    lab, n = label26(mask)
    if n == 0:
        return mask.astype(bool)
    sizes = np.bincount(lab.ravel(), minlength=n + 1)
    sizes[0] = -1
    best = int(np.argmax(sizes))            # first maximum == lowest label
    return lab == best


def convhull_fill2d(img):
    """bwconvhull(img, 'union') with the corner-hull / closed-boundary rule."""
    img = np.asarray(img, dtype=bool)
    ii, jj = np.nonzero(img)
    if ii.size == 0:
        return img.copy()
    # corners in doubled integer coordinates
    pts = set()
    for a, b in zip(ii.tolist(), jj.tolist()):
        for da in (-1, 1):
            for db in (-1, 1):
                pts.add((2 * a + da, 2 * b + db))
    pts = sorted(pts)

    def cross(o, a, b):
        return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])

    lower, upper = [], []
    for p in pts:
        while len(lower) >= 2 and cross(lower[-2], lower[-1], p) <= 0:
            lower.pop()
        lower.append(p)
    for p in reversed(pts):
        while len(upper) >= 2 and cross(upper[-2], upper[-1], p) <= 0:
            upper.pop()
        upper.append(p)
    hull = lower[:-1] + upper[:-1]        # counter-clockwise
    i0, i1 = ii.min(), ii.max()
    j0, j1 = jj.min(), jj.max()
    I, Jg = np.mgrid[i0:i1 + 1, j0:j1 + 1]
    X = 2 * I.astype(np.int64)
    Y = 2 * Jg.astype(np.int64)
    inside = np.ones(X.shape, dtype=bool)
    m = len(hull)
    for k in range(m):
        o = hull[k]
        a = hull[(k + 1) % m]
        inside &= ((a[0] - o[0]) * (Y - o[1]) - (a[1] - o[1]) * (X - o[0])) >= 0
    out = img.copy()
    out[i0:i1 + 1, j0:j1 + 1] |= inside
    return out
