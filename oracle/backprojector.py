"""CPU restatement of the OMW and Wiener-Butterworth backprojector generators (oracle; test infra).

* ``omw_backprojector_generation`` follows microscopeDataProcessing/decon/omw_backprojector_generation.m
* ``back_projector`` follows third_parties/WBDeconvolution/BackProjector.m (every bp_type;
  ``wb_backprojector`` is its 'wiener-butterworth' form)

Arithmetic choices shared with the CUDA library (the reference leaves them to MATLAB):
  * the PSF-size transforms are computed in float64 and, where the reference works in single,
    rounded to single afterwards; |OTF| is sqrt(re^2 + im^2) in float64 rounded to single;
  * the cumulative-OTF sum is a sequential float64 cumsum over the descending sort, and the total
    is its last element;
  * spherical directions are (X, Y, Z) / r with r = sqrt(X^2 + Y^2 + Z^2) (the value
    ``sph2cart(cart2sph(X, Y, Z), 1)`` has mathematically; (1, 0, 0) at r = 0);
  * knn (K = 2) ranks edge points by squared distance ((dy^2 + dx^2) + dz^2), ties by lower index.
"""
from __future__ import annotations

import numpy as np

from . import morph
from .decon import normalize_psf


def _fftn64(a):
    return np.fft.fftn(np.asarray(a, dtype=np.float64) if not np.iscomplexobj(a) else a.astype(np.complex128))


def _ifftn64(a):
    return np.fft.ifftn(a.astype(np.complex128))


def _to3(a):
    a = np.asarray(a)
    while a.ndim < 3:
        a = a[..., None]
    return a


def otf_at_psf_size(psf32):
    """decon_psf2otf(psf) with outSize = psfSize: circshift(-floor(psz/2)), fftn."""
    psz = np.array(psf32.shape)
    sh = np.roll(psf32.astype(np.float64), shift=tuple(-(psz // 2)), axis=(0, 1, 2))
    O = np.fft.fftn(sh).astype(np.complex64)
    absO = np.sqrt(O.real.astype(np.float64) ** 2 + O.imag.astype(np.float64) ** 2).astype(np.float32)
    return O, absO


def cum_threshold(absO, otf_thresh, min_int_thresh):
    """omw_backprojector_generation.m:35-41 -> dc_thresh (float64)."""
    vals = np.sort(absO.ravel().astype(np.float64))[::-1]
    cs = np.cumsum(vals)
    total = cs[-1]
    hit = np.nonzero(cs > total * otf_thresh)[0]
    tind = int(hit[0])
    dc = vals[tind] / np.float64(absO[0, 0, 0])
    return max(dc, float(min_int_thresh)), tind


def knn2_directions(P, Q, chunk=4096):
    """K=2 nearest rows of P for each row of Q (columns y, x, z); ties by lower index."""
    nq = Q.shape[0]
    inds = np.empty((nq, 2), dtype=np.int64)
    dmat = np.empty((nq, 2), dtype=np.float64)
    for s in range(0, nq, chunk):
        q = Q[s:s + chunk]
        dy = q[:, None, 0] - P[None, :, 0]
        dx = q[:, None, 1] - P[None, :, 1]
        dz = q[:, None, 2] - P[None, :, 2]
        d2 = dy * dy + dx * dx
        d2 = d2 + dz * dz
        i1 = np.argmin(d2, axis=1)
        rows = np.arange(q.shape[0])
        v1 = d2[rows, i1].copy()
        d2[rows, i1] = np.inf
        i2 = np.argmin(d2, axis=1)
        v2 = d2[rows, i2]
        inds[s:s + chunk, 0] = i1
        inds[s:s + chunk, 1] = i2
        dmat[s:s + chunk, 0] = np.sqrt(v1)
        dmat[s:s + chunk, 1] = np.sqrt(v2)
    return inds, dmat


def omw_mask_pipeline(absO, otf_thresh=0.9, area_thresh=100, min_int_thresh=1e-3, skewed=False):
    """Threshold, morphology, component selection and per-slice convex hulls
    (omw_backprojector_generation.m:33-109).  Returns (mask, skewed, dc_thresh)."""
    abs_c = np.fft.fftshift(absO)
    dc, _ = cum_threshold(absO, otf_thresh, min_int_thresh)
    m = abs_c > (np.float32(absO[0, 0, 0]) * np.float32(dc))            # :43
    m = morph.imopen(m, 2)                                              # :44
    m = morph.bwareaopen(m, area_thresh)
    m = morph.imclose(m, 2)
    m = morph.imopen(m, 2)
    m = morph.bwareaopen(m, area_thresh)                                # :48
    if not m.any():
        raise ValueError("The OTF mask is empty, check the PSF and OTF-related parameters!")
    if skewed is None:                                                  # :57-71
        skewed = False
        xz = m.sum(axis=0) > 0
        import scipy.ndimage as ndi
        _, ncc = ndi.label(np.ascontiguousarray(xz.T), structure=np.ones((3, 3), dtype=bool))
        if ncc > 1:
            line = xz.sum(axis=0)
            pind = int(np.argmax(line)) + 1
            if np.all(line > 0) and abs(pind - (line.size + 1) / 2.0) > 1:
                skewed = True
    if skewed:                                                          # :73-88
        L, n = morph.label26(m)
        if n + 1 > 4:
            sizes = np.bincount(L.ravel(), minlength=n + 1)[1:]
            order = np.argsort(-sizes, kind="stable")[:3]
            m = np.isin(L, order + 1)
            L, n = morph.label26(m)
        elif n + 1 == 2:
            L = (L + 1) * m
        m = np.concatenate([L == 3, L == 2, L == 1], axis=2)
    else:                                                               # :89-94
        m = morph.largest_component(m)
    zinds = np.nonzero(m.sum(axis=(0, 1)))[0]                           # :98-109
    xinds = np.nonzero(m.sum(axis=(0, 2)))[0]
    yinds = np.nonzero(m.sum(axis=(1, 2)))[0]
    for z in zinds:
        m[:, :, z] = morph.convhull_fill2d(m[:, :, z])
    for y in yinds:
        m[y, :, :] = morph.convhull_fill2d(m[y, :, :])
    for x in xinds:
        m[:, x, :] = morph.convhull_fill2d(m[:, x, :])
    return m, skewed, dc


def star_window(m, hann_bounds=(0.8, 1.0)):
    """Relative star distance to the mask edge and the cos^2 apodisation (:122-148)."""
    psz = np.array(m.shape)
    edge = m & ~morph.erode(m, 1)
    c = (psz + 1) / 2.0
    Y, X, Z = np.meshgrid(np.arange(1, psz[0] + 1) - c[0], np.arange(1, psz[1] + 1) - c[1],
                          np.arange(1, psz[2] + 1) - c[2], indexing="ij")
    rs = np.sqrt((X * X + Y * Y) + Z * Z)
    safe = np.where(rs > 0, rs, 1.0)
    Xn = np.where(rs > 0, X / safe, 1.0)
    Yn = np.where(rs > 0, Y / safe, 0.0)
    Zn = np.where(rs > 0, Z / safe, 0.0)
    F = lambda a: a.ravel(order="F")
    e = F(edge)
    P = np.stack([F(Yn)[e], F(Xn)[e], F(Zn)[e]], axis=1)
    Q = np.stack([F(Yn), F(Xn), F(Zn)], axis=1)
    inds, dmat = knn2_directions(P, Q)
    Rn = F(rs)[e]
    d1 = dmat[inds[:, 0], 0]                                            # :137 (indexes rows by edge index)
    d2 = dmat[inds[:, 1], 1]
    with np.errstate(invalid="ignore", divide="ignore"):
        rn = (Rn[inds[:, 0]] * d2 + Rn[inds[:, 1]] * d1) / (d1 + d2)
        bw = F(rs) / rn
    l, u = float(hann_bounds[0]), float(hann_bounds[1])
    with np.errstate(invalid="ignore"):
        cosv = np.cos(np.pi * (bw - l) / 2.0 / (u - l))
        win = (bw < l).astype(np.float64) + (cosv * cosv) * ((bw >= l) & (bw < u))
    return win.reshape(tuple(psz), order="F")


def omw_backprojector_generation(psf, alpha, skewed, otf_cum_thresh=0.9, otf_area_thresh=100,
                                 hann_win_bounds=(0.8, 1.0), min_int_thresh=1e-3):
    """omw_backprojector_generation.m:1-166 -> (b_omw, OTF_bp_omw, abs_OTF_c, OTF_mask)."""
    psf = _to3(np.asarray(psf))
    if psf.size == 0 or np.all(psf == 0):
        raise ValueError("A valid nonzero PSF needs to be provided!")
    p = normalize_psf(psf, np.float32)                                  # :29-30
    O, absO = otf_at_psf_size(p)                                        # :32-33
    abs_c = np.fft.fftshift(absO)                                       # :34
    m, skewed, _ = omw_mask_pipeline(absO, otf_cum_thresh, otf_area_thresh, min_int_thresh, skewed)
    mask = star_window(m, hann_win_bounds)
    psz = np.array(m.shape)
    if skewed:                                                          # :150-153
        mask = mask.reshape(psz[0], psz[1], psz[2] // 3, 3, order="F").sum(axis=3)
        m = m.reshape(psz[0], psz[1], psz[2] // 3, 3, order="F").sum(axis=3)
    om = np.fft.ifftshift(mask).astype(np.float32)                      # :155
    den = absO * absO + np.float32(alpha)                               # :158
    w = (O.real / den) - 1j * (O.imag / den)
    w = w.astype(np.complex64)
    omw = (om * w.real + 1j * (om * w.imag)).astype(np.complex64)       # :161
    b = np.fft.fftshift(np.real(_ifftn64(omw))).astype(np.float32)     # :163
    return b, omw, abs_c, m


# ---------------------------------------------------------------- Wiener-Butterworth
def _fwhm(y):
    """fwhm (BackProjector.m:443-483) in single precision with x = 1..N."""
    y = np.asarray(y, dtype=np.float32)
    y = y / y.max()
    N = y.size
    lev = np.float32(0.5)
    x = np.arange(1, N + 1, dtype=np.float64)
    if y[0] < lev:
        center = int(np.argmax(y))
    else:
        center = int(np.argmin(y))
    i = 1
    while np.sign(y[i] - lev) == np.sign(y[i - 1] - lev):
        i += 1
    interp = (lev - y[i - 1]) / (y[i] - y[i - 1])
    tlead = np.float32(x[i - 1]) + interp * np.float32(x[i] - x[i - 1])
    i = center + 1                                  # 0-based form of i = centerindex + 1
    while np.sign(y[i] - lev) == np.sign(y[i - 1] - lev) and i <= N - 2:
        i += 1
    if i != N - 1:
        interp = (lev - y[i - 1]) / (y[i] - y[i - 1])
        ttrail = np.float32(x[i - 1]) + interp * np.float32(x[i] - x[i - 1])
        return np.float32(ttrail - tlead)
    return np.float32(np.nan)


def fwhm_psf(psf32):
    """fwhm_PSF (BackProjector.m:260-396), cFlag = 0, fitFlag = 0, 3D input."""
    ind = int(np.argmax(psf32.ravel(order="F")))
    ix, iy, iz = np.unravel_index(ind, psf32.shape, order="F")
    return _fwhm(psf32[:, iy, iz]), _fwhm(psf32[ix, :, iz]), _fwhm(psf32[ix, iy, :])


def wb_backprojector(psf_fp, alpha=1e-4, beta=1e-3, n=10, res_flag=1, ires=(0.0, 0.0, 0.0)):
    """BackProjector(PSF_fp, 'wiener-butterworth', alpha, beta, n, resFlag, iRes) -> (PSF_bp, OTF_bp)."""
    return back_projector(psf_fp, "wiener-butterworth", alpha, beta, n, res_flag, ires)


def _gaussian_psf_3d(Sx, Sy, Sz, Fx, Fy, Fz):
    """gen_gaussianPSF_3D / gen_gaussian3D (BackProjector.m:485-514) with single-precision FWHMs: every
    product with a sigma is single, so the PSF is single."""
    sx, sy, sz = Fx / np.float32(2.3548), Fy / np.float32(2.3548), Fz / np.float32(2.3548)
    qx, qy, qz = sx * sx * np.float32(2), sy * sy * np.float32(2), sz * sz * np.float32(2)
    coef = np.float32(1) / (((np.float32((2 * np.pi) ** 1.5) * sx) * sy) * sz)
    i = np.arange(1, Sx + 1, dtype=np.float64)[:, None, None] - (Sx + 1) / 2.0
    j = np.arange(1, Sy + 1, dtype=np.float64)[None, :, None] - (Sy + 1) / 2.0
    k = np.arange(1, Sz + 1, dtype=np.float64)[None, None, :] - (Sz + 1) / 2.0
    d = ((i * i).astype(np.float32) / qx + (j * j).astype(np.float32) / qy) + (k * k).astype(np.float32) / qz
    return (coef * np.exp(-d.astype(np.float32))).astype(np.float32)


def back_projector(psf_fp, bp_type="wiener-butterworth", alpha=1e-4, beta=1e-3, n=10, res_flag=1,
                   ires=(0.0, 0.0, 0.0)):
    """BackProjector(PSF_fp, bp_type, alpha, beta, n, resFlag, iRes) -> (PSF_bp, OTF_bp)
    (BackProjector.m:67-233, every bp_type of :163-231)."""
    if bp_type not in ("traditional", "gaussian", "butterworth", "wiener", "wiener-butterworth"):
        raise ValueError("bp_type does not match any back-projector type")
    P = _to3(np.asarray(psf_fp)).astype(np.float32)
    Sx, Sy, Sz = P.shape
    Scx, Scy, Scz = (Sx + 1) / 2.0, (Sy + 1) / 2.0, (Sz + 1) / 2.0
    Soz = int(np.floor((Sz + 1) / 2.0 + 0.5))
    Fx, Fy, Fz = fwhm_psf(P)
    flipped = P[::-1, ::-1, ::-1].astype(np.float64)                   # flipPSF
    OTF_flip = np.fft.fftn(np.fft.ifftshift(flipped))
    OTF_abs = np.fft.fftshift(np.abs(OTF_flip))
    M = OTF_abs.max()
    if res_flag == 0:
        rx, ry, rz = Fx / np.float32(2 ** 0.5), Fy / np.float32(2 ** 0.5), Fz / np.float32(2 ** 0.5)
    elif res_flag == 1:
        rx, ry, rz = Fx, Fy, Fz
    elif res_flag == 2:
        rx, ry, rz = (np.float32(v) for v in ires)
    else:
        raise ValueError("Processing terminated, please set resFlag as 0, 1, or 2")
    tx = np.float32(np.float32(1) / rx) / np.float32(1.0 / Sx)
    ty = np.float32(np.float32(1) / ry) / np.float32(1.0 / Sy)
    tz = np.float32(np.float32(1) / rz) / np.float32(1.0 / Sz)
    if alpha == 1 or beta == 1:
        ON = OTF_abs / M
        tl = ON.max(axis=2).max(axis=1)
        bx = (tl[max(_mround(np.float32(Scx) - tx), 1) - 1] + tl[min(_mround(np.float32(Scx) + tx), Sx) - 1]) / 2
        tl = ON.max(axis=2).max(axis=0)
        by = (tl[max(_mround(np.float32(Scy) - ty), 1) - 1] + tl[min(_mround(np.float32(Scy) + ty), Sy) - 1]) / 2
        tl = ON.max(axis=0).max(axis=0)
        bz = (tl[max(_mround(np.float32(Scz) - tz), 1) - 1] + tl[min(_mround(np.float32(Scz) + tz), Sz) - 1]) / 2
        bfp = (bx + by + bz) / 3
        if alpha == 1:
            alpha = bfp
        if beta == 1:
            beta = bfp
    i = np.arange(1, Sx + 1, dtype=np.float32)[:, None, None]
    j = np.arange(1, Sy + 1, dtype=np.float32)[None, :, None]
    k = np.arange(1, Sz + 1, dtype=np.float32)[None, None, :]

    def butterworth(ee):                                              # :178-186, :214-227
        a = (i - np.float32(Scx)) / tx
        b = (j - np.float32(Scy)) / ty
        c = (k - np.float32(Scz)) / tz
        w = (a * a + b * b) + c * c
        wn = np.power(w.astype(np.float64), float(n)).astype(np.float32)
        mask = (np.float32(1) / np.sqrt(np.float32(1) + np.float32(ee) * wn)).astype(np.float64)
        return np.fft.ifftshift(mask)

    if bp_type == "traditional":                                      # :164-166
        return flipped, OTF_flip
    if bp_type == "gaussian":                                         # :168-171
        G = _gaussian_psf_3d(Sx, Sy, Sz, Fx, Fy, Fz)
        OTF = np.fft.fftn(np.fft.ifftshift(G.astype(np.float64)))
        return G.astype(np.float64), OTF.astype(np.complex64).astype(np.complex128)
    if bp_type == "butterworth":                                      # :173-187
        OTF_bp = butterworth(1 / beta ** 2 - 1).astype(np.complex128)
        return np.fft.fftshift(np.real(np.fft.ifftn(OTF_bp))), OTF_bp
    OTF_flip_norm = OTF_flip / M
    OTF_W = OTF_flip_norm / (np.abs(OTF_flip_norm) ** 2 + alpha)
    if bp_type == "wiener":                                           # :189-191
        return np.fft.fftshift(np.real(np.fft.ifftn(OTF_W))), OTF_W
    W_abs = np.fft.fftshift(np.abs(OTF_W))
    tplane = np.abs(W_abs[:, :, Soz - 1])
    tline = tplane.max(axis=1)
    to1 = max(_mround(np.float32(Scx) - tx), 1)
    to2 = min(_mround(np.float32(Scx) + tx), Sx)
    beta_wx = (tline[to1 - 1] + tline[to2 - 1]) / 2
    mask = butterworth(beta_wx / beta ** 2 - 1)
    OTF_bp = mask * OTF_W
    PSF_bp = np.fft.fftshift(np.real(np.fft.ifftn(OTF_bp)))
    return PSF_bp, OTF_bp


def _mround(v):
    """MATLAB round (half away from zero) to int."""
    v = float(v)
    return int(np.floor(v + 0.5)) if v >= 0 else int(np.ceil(v - 0.5))
