"""CPU restatement of the combined deskew / rotate of PetaKit5D (oracle; test infrastructure).

Follows deskewRotateFrame3D.m:1-260 on its default ("fast") path -- linear interpolation, no
resampling, CPU -- which hands the work to two C++ MEX files:
  * volume_deskew_rotate_warp_mex.cpp:215-487 when the slice-to-slice shift |dx| <= xStepThresh;
  * skewed_space_interp_volume_deskew_rotate_warp_mex.cpp:430-1289 otherwise: intermediate slices
    are first interpolated in the skewed space (deskewRotateFrame3D.m:71-118), then warped.

Arrays are indexed ``a[y, x, z]`` (MATLAB ``[ny nx nz]``).  The warp keeps the first axis (y) as is
and interpolates bilinearly over (x, z); an output row of ny voxels is a weighted sum of four (or,
in the skewed interpolation, two) input rows.  The x86-64 build of those MEX files is restated, so
the float arithmetic follows its association and rounding exactly:
  * float input: ``((a*wa + b*wb) + c*wc) + d*wd`` everywhere;
  * uint16 input: ``(a*wa + b*wb) + (c*wc + d*wd)`` for the positions of whole 16-element blocks of
    a row, ``((a*wa + b*wb) + c*wc) + d*wd`` for the last ``len % 16``;
  * uint16 output: the block positions round ``res + 0.5`` to nearest-even (so the result is biased
    up by half a level), the last ``len % 16`` truncate ``res + 0.5``; both saturate at 65535;
  * weights are float32, from float64 coordinates as the MEX files compute them.
Rows whose source coordinates fall outside the volume stay zero.  Two defects of the MEX files are
not reproduced: the float kernel's last partial 8-element block writes past the end of its row
(into the next row, which is usually recomputed), and row indices that leave the volume in the
skewed interpolation read neighbouring memory (here they read as zero).
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32


def _mround(v):
    return math.floor(v + 0.5) if v >= 0 else math.ceil(v - 0.5)


def interp_step(dx, dz, xy_pixel_size, theta, xstep_thresh):
    """deskewRotateFrame3D.m:75-97: the interpolated slice step dzout (returned as dzout / dz)."""
    if abs(dx) / xstep_thresh < 1.5:
        thr = xy_pixel_size * xstep_thresh / math.cos(theta)
        dzout = dz / (math.ceil((dz / thr) / (1 / 1)) * (1 / 1))
        counter = 1
        while dzout / thr < 0.4:
            dzout = dz / (math.ceil((dz / thr) / (1 / (counter + 1))) * (1 / (counter + 1)))
            counter += 1
    else:
        dzout = dz / math.ceil(abs(dx) / xstep_thresh)
    return dzout / dz, dzout


def n_total(nz, stepsize):
    """Slices after skewed-space interpolation (skewed_space_interp_volume_deskew_rotate_warp_mex.cpp:1183)."""
    return int(math.floor(_mround((nz - 1) / stepsize * 100000) / 100000) + 1)


def interp_indexing(n, stepsize):
    """determine_interpolation_indexing (:1152-1170): slices at integer positions are originals."""
    index = np.zeros(n, np.int64)
    orig = np.zeros(n, bool)
    c = 0
    for i in range(n):
        s = i * stepsize
        r = _mround(s)
        if abs(s - r) < 1e-3:
            orig[i] = True
            index[i] = r
        else:
            index[i] = c
            c += 1
    return index, orig, c


def plan(dims, angle, dz, xy_pixel_size, reverse=False, objective_scan=False, xstep_thresh=2.0, bbox=None):
    """deskewRotateFrame3D.m:53-208 (fast path): output box, skewed interpolation step and the 4x4
    backward matrix the MEX files take."""
    ny, nx, nz = (int(v) for v in dims)
    theta = angle * math.pi / 180
    dx = math.cos(theta) * dz / xy_pixel_size
    zaniso = dz / xy_pixel_size if objective_scan else math.sin(abs(theta)) * dz / xy_pixel_size
    if not objective_scan:
        out_size = [_mround(v) for v in (ny, (nx - 1) * math.cos(theta) + (nz - 1) * zaniso / math.sin(abs(theta)),
                                          (nx - 1) * math.sin(abs(theta)) - 4)]
    else:
        out_size = [_mround(v) for v in (ny, nx * math.cos(theta) + nz * zaniso * math.sin(abs(theta)),
                                          nz * zaniso * math.cos(theta) + nx * math.sin(abs(theta)))]
    do_interp = (not objective_scan) and abs(dx) > xstep_thresh
    step = None
    dx_orig = dx
    if do_interp:
        step, dzout = interp_step(dx, dz, xy_pixel_size, theta, xstep_thresh)
        nz = n_total(nz, step)
        dz = dzout
        dx = math.cos(theta) * dz / xy_pixel_size
        zaniso = dz / xy_pixel_size if objective_scan else math.sin(abs(theta)) * dz / xy_pixel_size
    if not reverse:
        xshift, xstep = -dx, dx
    else:
        xshift, xstep = dx + math.ceil((nz - 1) * dx), -dx
    nx_ds = math.ceil((nz - 1) * dx) + nx
    if objective_scan:
        nx_ds = nx
        ds_S = np.eye(4)
    else:
        ds_S = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [xstep, 0, 1, 0], [xshift, 0, 0, 1]], float)
    if reverse:
        theta = -theta
    center = (np.array([ny, nx_ds, nz], float) + 1) / 2
    T1 = np.eye(4)
    T1[3, :3] = -center[[1, 0, 2]]
    S = np.diag([1.0, 1.0, zaniso, 1.0])
    c, s = math.cos(theta), math.sin(theta)
    R = np.array([[c, 0, -s, 0], [0, 1, 0, 0], [s, 0, c, 0], [0, 0, 0, 1]], float)
    T2 = np.eye(4)
    T2[3, :3] = (np.array(out_size, float)[[1, 0, 2]] + 1) / 2
    offset = np.zeros((4, 4))
    offset[3, :3] = 1
    if not objective_scan and reverse:
        ds_S[3, 0] -= dx
    M = ds_S @ ((T1 + offset) @ S @ R @ (T2 - offset))
    tmat = np.linalg.inv(M.T)
    tmat = tmat[[1, 0, 2, 3]][:, [1, 0, 2, 3]]
    box = list(bbox) if bbox is not None else [1, 1, 1] + out_size
    return dict(out_size=out_size, do_interp=do_interp, stepsize=step, xstep=abs(dx_orig), tmat=tmat, bbox=box,
                nz_total=nz)


def _blend(terms, u16_in, u16_out, length):
    """Weighted sum of 2 or 4 (row, weight) terms over one output row (see the module notes)."""
    prods = [r.astype(F32) * F32(w) for r, w in terms]
    if len(prods) == 2:
        res = prods[0] + prods[1]
        seq = res
    else:
        seq = ((prods[0] + prods[1]) + prods[2]) + prods[3]
        res = (prods[0] + prods[1]) + (prods[2] + prods[3]) if u16_in else seq
    body = length - length % 16
    if not u16_out:
        if u16_in and len(prods) == 4:
            res = np.concatenate([res[:body], seq[body:]])
        return res.astype(F32)
    h = F32(0.5)
    rb = np.rint((res + h).astype(np.float64))            # cvtps: round to nearest even
    rt = np.floor((seq + h).astype(np.float64))           # (uint16_t) cast of a non-negative float
    r = np.concatenate([rb[:body], rt[body:]])
    return np.clip(r, 0, 65535).astype(np.uint16)


def skewed_interp(im, xstep, stepsize, reverse, u16_out):
    """skewed_space_interp_defined_stepsize* (:430-884): the interpolated slices, in order."""
    ny, nx, nz = im.shape
    ntot = n_total(nz, stepsize)
    index, orig, nint = interp_indexing(ntot, stepsize)
    u16_in = im.dtype == np.uint16
    out = np.zeros((ny, nx, nint), np.uint16 if u16_out else F32)
    xa = math.ceil(xstep)
    zero = np.zeros(ny, im.dtype)

    def row(y, z):
        return im[:, y, z] if 0 <= y < nx and 0 <= z < nz else zero

    for i in range(ntot):
        if orig[i]:
            continue
        zi = int(index[i])
        zout = stepsize * i
        zw = zout - math.floor(zout)
        if reverse:
            s, t = math.ceil(xstep) - xstep * zw, xstep * (1 - zw)
        else:
            s, t = xstep * (1 - zw), math.ceil(xstep) - xstep * zw
        sw, tw = s - math.floor(s), t - math.floor(t)
        s, t = int(math.floor(s)), int(math.floor(t))
        zo = int(math.floor(zout))
        swf, twf, zwf = float(F32(sw)), float(F32(tw)), float(F32(zw))
        c00 = F32((1.0 - swf) * (1.0 - zwf))
        c01 = F32(swf * (1.0 - zwf))
        c10 = F32((1.0 - twf) * zwf)
        c11 = F32(F32(twf) * F32(zwf))
        for y in range(nx):
            if reverse:
                if y < xa - s:
                    terms = [(row(y + t, zo + 1), c10), (row(y + t + 1, zo + 1), c11)]
                elif y < nx - t - 1:
                    terms = [(row(y + s - xa, zo), c00), (row(y + s - xa + 1, zo), c01),
                             (row(y + t, zo + 1), c10), (row(y + t + 1, zo + 1), c11)]
                else:
                    terms = [(row(y + s - xa, zo), c00), (row(y + s - xa + 1, zo), c01)]
            else:
                if y < xa - s:
                    terms = [(row(y + s, zo), c00), (row(y + s + 1, zo), c01)]
                elif y < nx - t - 1:
                    terms = [(row(y + s, zo), c00), (row(y + s + 1, zo), c01),
                             (row(y + t - xa, zo + 1), c10), (row(y + t - xa + 1, zo + 1), c11)]
                else:
                    terms = [(row(y + t - xa, zo + 1), c10), (row(y + t - xa + 1, zo + 1), c11)]
            out[:, y, zi] = _blend(terms, u16_in, u16_out, ny)
    return out, index, orig


def _nudge(t, n):
    """The MEX files' edge rule: a coordinate exactly one below the last index is moved just inside."""
    counter = 1
    while math.floor(t) + 1 == n:
        t -= 1e-9 * counter
        counter *= 2
    return t


def warp(im, tmat, bbox, u16_out, im_int=None, index=None, orig=None):
    """transformVolume* (volume_deskew_rotate_warp_mex.cpp:215-380; the skewed variant :885-1150)."""
    ny, nx = im.shape[0], im.shape[1]
    nzt = im.shape[2] if im_int is None else len(orig)
    sx, sy, sz = (float(F32(bbox[k]) - F32(1)) for k in range(3))
    ex, ey, ez = (float(F32(bbox[k])) for k in range(3, 6))
    if min(sx, sy, sz) < 0 or sx > ex or sy > ey or sz > ez:
        raise ValueError("bbox is invalid")
    ox, oy, oz = int(F32(ex - sx)), int(F32(ey - sy)), int(F32(ez - sz))
    x0 = int(math.floor(sx))
    u16_in = im.dtype == np.uint16
    out = np.zeros((ox, oy, oz), np.uint16 if u16_out else F32)

    def plane_row(z, y):
        if im_int is None:
            return im[x0:x0 + ox, y, z], u16_in
        if orig[z]:
            return im[x0:x0 + ox, y, int(index[z])], u16_in
        return im_int[x0:x0 + ox, y, int(index[z])], im_int.dtype == np.uint16

    for z in range(oz):
        ty = tmat[1][2] * float(F32(z + F32(sz))) + tmat[1][3]
        if ty < 0 or ty + 1 >= nx:
            if ty + 1 == nx:
                ty = _nudge(ty, nx)
            else:
                continue
        y0 = int(math.floor(ty))
        wy = F32(ty - y0)
        for y in range(oy):
            tz = tmat[2][1] * float(F32(y + F32(sy))) + tmat[2][2] * float(F32(z + F32(sz))) + tmat[2][3]
            if tz < 0 or tz + 1 >= nzt:
                if tz + 1 == nzt:
                    tz = _nudge(tz, nzt)
                else:
                    continue
            z0 = int(math.floor(tz))
            wz = F32(tz - z0)
            w00 = F32(F32(1) - wy) * F32(F32(1) - wz)
            w01 = F32(F32(1) - wy) * wz
            w10 = wy * F32(F32(1) - wz)
            w11 = wy * wz
            a, ua = plane_row(z0, y0)
            b, ub = plane_row(z0 + 1, y0)
            c, _ = plane_row(z0, y0 + 1)
            d, _ = plane_row(z0 + 1, y0 + 1)
            if ua == ub:
                terms = [(a, w00), (b, w01), (c, w10), (d, w11)]
                uin = ua
            elif ua:                                       # uint16 slice z0, float slice z0 + 1
                terms = [(a, w00), (b, w01), (c, w10), (d, w11)]
                uin = True
            else:                                          # float slice z0, uint16 slice z0 + 1
                terms = [(b, w01), (a, w00), (d, w11), (c, w10)]
                uin = True
            out[:, y, z] = _blend(terms, uin, u16_out, ox)
    return out


def deskew_rotate_frame3d(vol, angle, dz, xy_pixel_size, reverse=False, bbox=None, objective_scan=False,
                          xstep_thresh=2.0, save16bit=False):
    """volout = deskewRotateFrame3D(vol, angle, dz, xyPixelSize, 'reverse', ..., 'bbox', ...,
    'objectiveScan', ..., 'xStepThresh', ..., 'save16bit', ...) on the fast path."""
    vol = np.asarray(vol)
    if vol.dtype not in (np.float32, np.uint16):
        vol = vol.astype(F32)
    u16_out = bool(save16bit) and vol.dtype == np.uint16
    p = plan(vol.shape, angle, dz, xy_pixel_size, reverse, objective_scan, xstep_thresh, bbox)
    if p["do_interp"]:
        im_int, index, orig = skewed_interp(vol, p["xstep"], p["stepsize"], reverse, u16_out)
        return warp(vol, p["tmat"], p["bbox"], u16_out, im_int, index, orig)
    return warp(vol, p["tmat"], p["bbox"], u16_out)
