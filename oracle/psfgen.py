"""CPU restatement of psf_gen_new.m (oracle; test infrastructure).

psf_gen_new.m:1-140 cleans a measured PSF before deconvolution: background subtraction, a mask of
the connected component that holds the peak, centring of the peak, and axial resampling to the
data's z step.  RLdecon.m:207-265 calls it for every PSF (``psfGen`` defaults to true) and then
crops the PSF for the non-OMW methods and to the data size; ``rldecon_psf_crop`` restates that.

Arrays are indexed ``a[y, x, z]`` (MATLAB ``[ny nx nz]``).  Conventions of the MATLAB calls:
  * ``medfilt3(A, [3 3 3])``: median of the 27-neighbourhood, 'symmetric' padding (for a 3-wide
    window the same as repeating the edge voxel).  ``medfilt2(A, [3 3])``: 9-neighbourhood,
    zero padding.
  * ``bwareaopen(BW, P, 26)`` / ``bwlabeln``: 26-connected components (8 in 2D), those with fewer
    than P voxels removed; ``L == L(peakInd)`` selects the component of the first maximum of the
    median-filtered PSF, or every voxel outside the components when the peak is not in one.
  * ``imclose(BW, strel('sphere', 3))``: dilation (outside = false) then erosion (outside = true)
    with the ball dy^2+dx^2+dz^2 <= 9; 2D: ``strel('disk', 3)`` as the decon path's disk.
  * ``mean`` over the 20 border rows (and z): float64 sum, divided, rounded to float32.
  * ``median`` of an even count: the mean of the two middle values in float64, rounded to float32.
  * ``uint16(new_nz)/2`` rounds half away from zero, so for odd ``new_nz`` the two kept bands of
    the axial spectrum share one plane and the second assignment wins (psf_gen_new.m:130-131).
  * The axial resampling keeps the x/y transform pair out: ``ifftn(trunc_z(fftn(P)))`` equals
    ``ifft_z(trunc_z(fft_z(P)))`` because the truncation acts on z only.
"""
from __future__ import annotations

import numpy as np

from .decon import disk_nhood
from .morph import label26 as _label26_3d, sphere_offsets, _shift_and

MASKED, MEDIAN = 0, 1


def _round_half_away(v):
    v = float(v)
    return int(np.floor(v + 0.5)) if v >= 0 else int(np.ceil(v - 0.5))


def _border_rows(ny):
    """``[1:10, end-9:end]`` as 0-based row indices (duplicates kept, as MATLAB indexing does)."""
    if ny < 10:
        raise ValueError("psf_gen_new needs at least 10 rows (index [1:10, end-9:end])")
    return np.r_[0:10, ny - 10:ny]


def medfilt3(a):
    """``medfilt3(a, [3 3 3])``: 27-neighbourhood median, edge voxels repeated."""
    p = np.pad(a, 1, mode="edge")
    ny, nx, nz = a.shape
    stack = np.stack([p[1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx, 1 + dz:1 + dz + nz]
                      for dz in (-1, 0, 1) for dx in (-1, 0, 1) for dy in (-1, 0, 1)])
    return np.sort(stack, axis=0)[13]


def medfilt2(a):
    """``medfilt2(a, [3 3])`` on each z plane (nz == 1): 9-neighbourhood median, zero padding."""
    p = np.pad(a, ((1, 1), (1, 1), (0, 0)), mode="constant")
    ny, nx, nz = a.shape
    stack = np.stack([p[1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx, :] for dx in (-1, 0, 1) for dy in (-1, 0, 1)])
    return np.sort(stack, axis=0)[4]


def _label(mask):
    return _label26_3d(mask)        # with nz == 1 the 26-neighbourhood is the 8-neighbourhood


def _bwareaopen(mask, P):
    lab, n = _label(mask)
    if n == 0:
        return np.zeros_like(mask, dtype=bool)
    sizes = np.bincount(lab.ravel(), minlength=n + 1)
    keep = sizes >= P
    keep[0] = False
    return keep[lab]


def _peak_component(BW, med):
    """``L = bwlabeln(BW); [~, peakInd] = max(med(:)); BW = L == L(peakInd)``."""
    lab, _ = _label(BW)
    pk = int(np.argmax(med.ravel(order="F")))            # first maximum in MATLAB linear order
    return lab == lab.ravel(order="F")[pk]


def _nhood_offsets(nz):
    if nz > 1:
        return sphere_offsets(3)
    d = disk_nhood(3)
    r = d.shape[0] // 2
    return [(a - r, b - r, 0) for a in range(d.shape[0]) for b in range(d.shape[1]) if d[a, b]]


def _imclose(BW, offs):
    return _shift_and(_shift_and(BW, offs, False), offs, True)


def _row_mean_f32(sub):
    """Mean over axis 0 of the border rows: float64 sum in row order, rounded to float32."""
    acc = np.zeros(sub.shape[1:], np.float64)
    for r in range(sub.shape[0]):
        acc += sub[r].astype(np.float64)
    return (acc / sub.shape[0]).astype(np.float32)


def _border_colmean_f32(raw, rows):
    """``mean(raw([1:10, end-9:end], :, :), [1, 3])`` per x: float64 sum, rows outer and z inner."""
    nx, nz = raw.shape[1], raw.shape[2]
    acc = np.zeros(nx, np.float64)
    for r in rows:
        for z in range(nz):
            acc += raw[r, :, z].astype(np.float64)
    return (acc / (len(rows) * nz)).astype(np.float32)


def _median_f32(v):
    v = np.sort(v.astype(np.float32))
    n = v.size
    if n == 0:
        return np.float32(np.nan)
    if n % 2:
        return v[n // 2]
    return np.float32((np.float64(v[n // 2 - 1]) + np.float64(v[n // 2])) / 2.0)


def clean(psf, med_factor=1.5, method=MASKED):
    """psf_gen_new.m:19-95: background subtraction and the peak-component mask.

    Returns (psf_raw, BW) with BW None when the cleanup is skipped (no positive value in the
    first/last slices, :27-29)."""
    psf = np.asarray(psf, dtype=np.float32)
    if psf.ndim == 2:
        psf = psf[:, :, None]
    ny, nx, nz = psf.shape
    raw = psf.copy()
    if nz > 1:
        if nz < 5:
            raise ValueError("psf_gen_new needs at least 5 slices (index [1:5, end-4:end])")
        fl = raw[:, :, np.r_[0:5, nz - 5:nz]]                                   # :26
        if not np.any(fl > 0):                                                  # :28
            return raw, None
        if method == MEDIAN:                                                    # :30-41
            m = _median_f32(fl[fl > 0])
            raw = raw - np.float32(med_factor) * m                             # single arithmetic
            raw = np.maximum(raw, np.float32(0))
            med = medfilt3(raw)
            BW = _bwareaopen(med > 0, 300)
            BW = _peak_component(BW, med)
            BW = _imclose(BW, _nhood_offsets(nz))
            return raw * BW, BW
        rows = _border_rows(ny)                                                 # :42-58
        med = medfilt3(psf)
        sub = med[rows]
        a = (np.sqrt(np.abs(sub - np.float32(100))).max(axis=0) * np.float32(3)
             + _row_mean_f32(sub)).astype(np.float32)
        BW = _bwareaopen(med > a[None], 300)
        BW = _peak_component(BW, med)
        BW = _imclose(BW, _nhood_offsets(nz))
        colmean = _border_colmean_f32(raw, rows)
        out = (raw * BW).astype(np.float32) - colmean[None, :, None]
        out[out < 0] = 0.0
        return out.astype(np.float32), BW
    if method == MEDIAN:                                                        # :62-74
        raise NotImplementedError("psf_gen_new.m:68 calls medfilt, which neither MATLAB nor the reference defines")
    rows = _border_rows(ny)                                                     # :75-89
    med = medfilt2(psf)
    sub = med[rows]
    if np.any(sub < 0):
        raise NotImplementedError("negative border rows make psf_gen_new.m:78 complex (sqrt of a negative)")
    a = (np.sqrt(sub).max(axis=0) * np.float32(3) + _row_mean_f32(sub)).astype(np.float32)
    BW = _bwareaopen(med > a[None], 50)
    BW = _peak_component(BW, med)
    BW = _imclose(BW, _nhood_offsets(1))
    colmean = _border_colmean_f32(raw, rows)
    out = (raw * BW).astype(np.float32) - colmean[None, :, None]
    out[out < 0] = 0.0
    return out.astype(np.float32), BW


def centre(raw):
    """psf_gen_new.m:97-124: z padding when the PSF reaches too far from the peak, then circshift
    of the peak to ``round(([ny nx nz] + 1) / 2)`` (1-based)."""
    ny, nx, nz = raw.shape
    flat = raw.ravel(order="F")
    pk = int(np.argmax(flat))
    py, px, pz = pk % ny + 1, (pk // ny) % nx + 1, pk // (ny * nx) + 1          # 1-based
    zsum = raw.astype(np.float32).sum(axis=(0, 1), dtype=np.float64)
    zst = np.nonzero(zsum)[0] + 1
    if zst.size == 0:
        raise ValueError("psf_gen_new: the cleaned PSF is all zero")
    zs, zt = int(zst[0]), int(zst[-1])
    if pz - zs > nz / 2:                                                        # :109-112
        pad = pz - zs - _round_half_away((nz - 1) / 2) + 3
        raw = np.concatenate([raw, np.zeros((ny, nx, pad), np.float32)], axis=2)
        nz = raw.shape[2]
    if zt - pz > nz / 2:                                                        # :113-117
        pad = zt - pz - _round_half_away((nz - 1) / 2) + 3
        raw = np.concatenate([np.zeros((ny, nx, pad), np.float32), raw], axis=2)
        pz = pz + pad
        nz = raw.shape[2]
    shift = [_round_half_away((n + 1) / 2 - p) for n, p in zip((ny, nx, nz), (py, px, pz))]
    return np.roll(raw, shift, axis=(0, 1, 2))


def resample_z(p, dz_psf, dz_data):
    """psf_gen_new.m:126-139: keep the low axial frequencies when the data's z step is coarser."""
    ratio = dz_data / dz_psf
    p = np.asarray(p, dtype=np.float32)
    if not ratio > 1:
        return np.maximum(p, np.float32(0))
    ny, nx, nz = p.shape
    new_nz = min(max(_round_half_away(nz / ratio), 0), 65535)                   # uint16(round(.))
    h = (new_nz + 1) // 2                                                       # uint16 new_nz/2
    F = np.fft.fft(p.astype(np.float64), axis=2)
    T = np.zeros((ny, nx, new_nz), np.complex128)
    T[:, :, 0:h] = F[:, :, 0:h]
    if h > 0:
        T[:, :, new_nz - h:new_nz] = F[:, :, nz - h:nz]
    out = np.real(np.fft.ifft(T, axis=2)) if new_nz > 0 else np.zeros((ny, nx, 0))
    return np.maximum(out, 0.0)


def psf_gen_new(psf, dz_psf, dz_data, med_factor=1.5, method=MASKED):
    """psf_gen_new.m:1-140.  Returns float64 after axial resampling, float32 otherwise (as MATLAB)."""
    raw, _ = clean(psf, med_factor, method)
    c = centre(raw)
    return resample_z(c, dz_psf, dz_data)


def rldecon_psf_crop(psf, data_size, omw):
    """RLdecon.m:249-265: for non-OMW methods crop to the nonzero bounding box keeping the centre
    (minus one voxel of margin); then crop a PSF larger than the data around its centre."""
    psf = np.asarray(psf)
    psz = np.array(psf.shape)
    if not omw:
        nzs = [np.nonzero(psf.sum(axis=tuple(a for a in range(3) if a != d)))[0] + 1 for d in range(3)]
        crop = np.array([min(n[0] - 1, psz[d] - n[-1]) for d, n in enumerate(nzs)]) - 1
        crop = np.maximum(0, crop)
        lo, hi = crop, psz - crop
        psf = psf[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        psz = np.array(psf.shape)
    im = np.array(data_size)
    if np.any(psz > im):
        s = np.maximum(0, (psz - im) // 2)
        t = s + np.minimum(psz, im)
        psf = psf[s[0]:t[0], s[1]:t[1], s[2]:t[2]]
    return psf
