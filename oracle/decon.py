"""CPU restatement of PetaKit5D's RL / OMW deconvolution iterations (oracle; test infrastructure).

Volumes are numpy arrays indexed like MATLAB: ``a[y, x, z]`` (MATLAB size order ``[ny nx nz]``).
Every function takes ``dtype`` = ``np.float32`` (the reference's single-precision GPU path) or
``np.float64`` (the "FP64 host oracle").  FFTs are scipy.fft (pocketfft); a real transform over the
y axis plus complex transforms over x and z gives the half spectrum, which is mathematically the
same as the reference's ``real(ifftn(fftn(.) .* OTF))`` because every OTF here is the transform of a
real PSF (Hermitian).

Where this restatement deliberately fixes an order of operations that the reference leaves to
MATLAB, the CUDA library follows the same choice:
  * PSF normalisation: the sum is taken in float64 and each PSF value is divided in float64, then
    rounded to the working dtype (reference: single-precision ``PSF ./ sum(PSF(:))``).
  * ``a*s + o`` is evaluated as two rounded float operations (no fused multiply-add).
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

EPS = 2.0 ** -52  # MATLAB ``eps`` (double); ``max(single, eps)`` compares against single(eps) = 2^-52


def _workers():
    import os
    return os.cpu_count() or 1


def rfft3(a, workers=None):
    """Half spectrum: real transform over y (axis 0), complex over x and z."""
    return sfft.rfftn(a, axes=(2, 1, 0), workers=workers or _workers())


def irfft3(S, shape, workers=None):
    return sfft.irfftn(S, s=(shape[2], shape[1], shape[0]), axes=(2, 1, 0), workers=workers or _workers())


def pad3(sz):
    """decon_padlength (decon_psf2otf.m:49-58): pad a size vector with ones to 3 dims."""
    sz = list(sz)
    return tuple(sz + [1] * (3 - len(sz)))


def normalize_psf(psf, dtype=np.float32):
    """``PSF ./ sum(PSF(:))`` (decon_lucy_omw_function.m:70-71, decon_lucy_function.m:76,
    omw_backprojector_generation.m:29-30) with the sum and the division taken in float64."""
    p = np.asarray(psf).astype(dtype)
    s = np.sum(p.astype(np.float64))
    return (p.astype(np.float64) / s).astype(dtype)


def psf2otf_half(psf, out_size, dtype=np.float32):
    """decon_psf2otf.m:1-46 at the data size, returned as the half spectrum (y real axis).

    Zero-pad ``psf`` (post) to ``out_size``, circshift by ``-floor(psfSize/2)``, FFT.
    """
    psf = np.asarray(psf, dtype=dtype)
    if psf.ndim < 3:
        psf = psf.reshape(pad3(psf.shape))
    psz = np.array(psf.shape)
    osz = np.array(pad3(out_size))
    if np.any(osz < psz):
        raise ValueError("outSizeIsSmallerThanPsfSize")  # decon_psf2otf.m:20-22
    if np.all(psf == 0):
        return np.zeros((osz[0] // 2 + 1, osz[1], osz[2]), dtype=np.complex64 if dtype == np.float32 else np.complex128)
    big = np.zeros(tuple(osz), dtype=dtype)
    big[:psz[0], :psz[1], :psz[2]] = psf                       # padarray(psf, padSize, 'post')
    big = np.roll(big, shift=tuple(-(psz // 2)), axis=(0, 1, 2))  # circshift(psf, -floor(psfSize/2))
    return rfft3(big)


def conv_half(x, otf_half):
    """``real(ifftn(fftn(x) .* OTF))`` via the half spectrum."""
    return irfft3(rfft3(x) * otf_half, x.shape).astype(x.dtype, copy=False)


def round_background_u16(bg):
    """MATLAB ``uint16(Background)``: round half away from zero, saturate to [0, 65535]."""
    return int(to_uint16(np.array([bg], dtype=np.float64))[0])


def preprocess(I, background, need_mask, dtype=np.float32):
    """Input handling of the GPU branch (decon_lucy_omw_function.m:80-91; decon_lucy_function.m:85-95).

    uint16 input: ``I - uint16(Background)`` (saturating) then ``single``; other input:
    ``max(I - Background, 0)`` in the working dtype.  ``I_mask = I ~= 0`` is taken on the raw input.
    """
    bg = 0.0 if background is None else float(background)
    I = np.asarray(I)
    mask = (I != 0) if need_mask else None
    if I.dtype == np.uint16:
        b = round_background_u16(bg)
        out = np.where(I > b, I.astype(np.int64) - b, 0).astype(dtype)
    else:
        x = I.astype(dtype)
        out = np.fmax(x - dtype(bg), dtype(0))          # MATLAB max ignores NaN
    return out, mask


def to_uint16(J):
    """MATLAB ``uint16(J)``: round half away from zero, saturate, NaN -> 0."""
    x = np.asarray(J).astype(np.float64)
    r = np.where(x >= 0, np.floor(x + 0.5), np.ceil(x - 0.5))
    r = np.nan_to_num(r, nan=0.0, posinf=65535.0, neginf=0.0)
    return np.clip(r, 0, 65535).astype(np.uint16)


# ---------------------------------------------------------------- edge erosion
def disk_nhood(R):
    """``strel('disk', R)`` neighbourhood (default N=4).

    R < 3: exact disk ``x^2+y^2 <= R^2``.  R >= 3: the radial decomposition into four periodic lines
    (Adams 1993; Jones & Soille 1996): extent k = 2R/(cot(pi/8) + 1/sin(pi/8)); line q has
    repetition floor(k/|v_q|) along v_q in {(1,0),(1,1),(0,1),(-1,1)}; the Minkowski sum of the
    lines is then widened by a horizontal and a vertical line of length 2(R - r_got - 1) + 1 when
    that is >= 3.  Returned as a boolean (2r+1, 2r+1) array, rows = y.
    """
    R = int(R)
    if R < 3:
        yy, xx = np.mgrid[-R:R + 1, -R:R + 1]
        return (xx * xx + yy * yy) <= R * R
    theta = np.pi / 8.0
    k = 2.0 * R / (1.0 / np.tan(theta) + 1.0 / np.sin(theta))
    pts = {(0, 0)}
    for v in ((1, 0), (1, 1), (0, 1), (-1, 1)):
        rp = int(np.floor(k / np.hypot(*v)))
        pts = {(a + m * v[0], b + m * v[1]) for (a, b) in pts for m in range(-rp, rp + 1)}
    rmax = max(a for a, _ in pts)
    ln = 2 * (R - rmax - 1) + 1
    if ln >= 3:
        h = ln // 2
        pts = {(a, b + m) for (a, b) in pts for m in range(-h, h + 1)}
        pts = {(a + m, b) for (a, b) in pts for m in range(-h, h + 1)}
    r = max(max(abs(a), abs(b)) for a, b in pts)
    out = np.zeros((2 * r + 1, 2 * r + 1), dtype=bool)
    for a, b in pts:
        out[a + r, b + r] = True
    return out


def _erode_offsets(mask, offsets):
    """Binary erosion with the neighbourhood given as offsets; outside the image counts as true."""
    out = np.ones_like(mask)
    sh = mask.shape
    for off in offsets:
        shifted = np.ones_like(mask)
        src = tuple(slice(max(0, o), sh[i] + min(0, o)) for i, o in enumerate(off))
        dst = tuple(slice(max(0, -o), sh[i] + min(0, -o)) for i, o in enumerate(off))
        shifted[dst] = mask[src]
        out &= shifted
    return out


def mask_edge_erosion(mask, E):
    """decon_mask_edge_erosion.m:1-30.  MATLAB's ndims of an [ny nx 1] array is 2, so a single plane
    takes the 2-D steps: no z faces (:11-13) and no z erosion (:23-28)."""
    mask = np.asarray(mask) > 0
    shape = mask.shape
    if mask.ndim == 2:
        mask = mask[:, :, None]
    two_d = mask.shape[2] == 1
    return _mask_edge_erosion3(mask, int(E), two_d).reshape(shape)


def _mask_edge_erosion3(mask, E, two_d):
    if mask.all():                                             # :8-15 full rectangular mask
        m = mask.copy()
        for ax in range(2 if two_d else 3):
            idx = [slice(None)] * 3
            idx[ax] = slice(0, min(E, m.shape[ax]))
            m[tuple(idx)] = False
            idx[ax] = slice(max(m.shape[ax] - E, 0), m.shape[ax])
            m[tuple(idx)] = False
        return m
    m = mask.copy()                                            # :18-29 irregular mask
    m[[0, -1], :, :] = False
    m[:, [0, -1], :] = False
    if not two_d:
        m[:, :, [0, -1]] = False
    d = disk_nhood(E - 1)
    r = d.shape[0] // 2
    offs = [(a - r, b - r, 0) for a, b in zip(*np.nonzero(d))]
    m = _erode_offsets(m, offs)
    if not two_d:
        h = E - 1                                              # true(2E-1, 1) along z
        m = _erode_offsets(m, [(0, 0, o) for o in range(-h, h + 1)])
    return m


# ---------------------------------------------------------------- post-processing
def postprocess(J, I, I_mask, damp=1.0, scale=1.0, offset=0.0, edge_erosion=0, save16bit=True, bbox=None):
    """decon_lucy_omw_function.m:146-177 / decon_lucy_function.m:177-213."""
    dt = J.dtype.type
    if damp > 1:                                               # :147-149
        dI = dt(damp) * I
        J = J * (J <= dI) + np.minimum(J, dI * (J >= dI))
    if edge_erosion > 0:
        I_mask = mask_edge_erosion(I_mask, edge_erosion)
    if scale != 1 or offset != 0 or edge_erosion > 0:
        if offset != 0 or edge_erosion > 0:
            J = ((J * dt(scale)) + dt(offset)) * I_mask.astype(dt)
        else:
            J = J * dt(scale)
    if save16bit:
        J = to_uint16(J)
    if bbox is not None and len(bbox) == 6:
        b = [int(v) for v in bbox]
        J = J[b[0] - 1:b[3], b[1] - 1:b[4], b[2] - 1:b[5]]
    return J


# ---------------------------------------------------------------- the iterations
def decon_lucy_omw(I, psf_f, psf_b, numit, background=None, save16bit=True, damp=1.0, scale=1.0,
                   offset=0.0, edge_erosion=0, bbox=None, dtype=np.float32, return_float=False, iterates=None):
    """decon_lucy_omw_function.m:1-177 (GPU branch input handling, 2-iteration regime)."""
    need_mask = offset != 0 or edge_erosion > 0
    Ipre, I_mask = preprocess(I, background, need_mask, dtype)
    size = Ipre.shape
    otf_f = psf2otf_half(normalize_psf(psf_f, dtype), size, dtype)   # :70
    otf_b = psf2otf_half(normalize_psf(psf_b, dtype), size, dtype)   # :71
    eps = dtype(EPS)
    J = Ipre
    for _ in range(int(numit)):                                # :105-113
        CX = conv_half(J, otf_f)
        CX = np.fmax(CX, eps)
        J = conv_half(Ipre / CX, otf_b) * J
        J = np.fmax(J, dtype(0))
        if iterates is not None:                               # the debug branch's J (:114)
            iterates.append(J.copy())
    if return_float:
        return J
    return postprocess(J, Ipre, I_mask, damp, scale, offset, edge_erosion, save16bit, bbox)


def decon_lucy(I, psf, numit, background=None, save16bit=True, damp=1.0, scale=1.0, offset=0.0,
               edge_erosion=0, bbox=None, dtype=np.float32, return_float=False, lambdas=None, iterates=None):
    """decon_lucy_function.m:1-213: Biggs-Andrews accelerated RL ('simplified')."""
    need_mask = offset != 0 or edge_erosion > 0
    Ipre, I_mask = preprocess(I, background, need_mask, dtype)
    size = Ipre.shape
    H = psf2otf_half(normalize_psf(psf, dtype), size, dtype)         # :76
    Hc = np.conj(H)
    eps = dtype(EPS)
    J2 = Ipre
    J3 = np.zeros(size, dtype)
    J4 = np.zeros(size, dtype)
    Y = None
    lam = 0.0                                                  # :120  2*any(J_4~=0) = 0
    for k in range(1, int(numit) + 1):
        if k > 2:                                              # :124-128
            num = np.sum(((J2 - Y) * J4).astype(np.float64))
            den = np.sum((J4 * J4).astype(np.float64))
            lam = num / (den + EPS)
            lam = max(min(lam, 1.0), 0.0)
            J4 = J2 - Y
        elif k == 2:                                           # :129-130
            J4 = J2 - Y
        Y = np.fmax(J2 + dtype(lam) * (J2 - J3), dtype(0))      # :132
        RB = np.fmax(conv_half(Y, H), eps)                     # :136
        RB = Ipre / RB                                         # :138
        J3 = J2                                                # :141
        J2 = np.fmax(Y * conv_half(RB, Hc), dtype(0))           # :142
        if lambdas is not None:
            lambdas.append(lam)
        if iterates is not None:                               # the debug branch's J_2 (:144)
            iterates.append(J2.copy())
    if return_float:
        return J2
    return postprocess(J2, Ipre, I_mask, damp, scale, offset, edge_erosion, save16bit, bbox)


def err_mat_from_mse(mse, estep, method):
    """err_mat of the debug branch from the per-iteration mean((J - I).^2): decon_lucy_omw_function.m
    :115-127 with the trim at :142-144, decon_lucy_function.m:145-157 with the trim at :173-175.  The
    reference indexes rows by the step index istp (not by k) in the stopping measure, and RL's trim
    uses the last istp (an error in MATLAB when none was set); both are kept."""
    numit = len(mse)
    e = np.zeros((numit + 1, 4))                               # 1-based rows as in MATLAB
    istp = None
    for k in range(1, numit + 1):
        e[k, 0] = k
        e[k, 1] = mse[k - 1]
        e[k, 2] = e[k, 1] / e[1, 1]
        if k % estep == 0 and k > estep * 2:
            istp = k // estep
            e[k, 3] = min(abs(e[istp, 2] - e[istp - 1, 2]) / 10,
                          abs(e[istp, 2] + e[istp - 2, 2] - 2 * e[istp - 1, 2]) / 2)
        elif k < 3 * estep:
            e[k, 3] = 1
        else:
            e[k, 3] = e[istp * estep, 3]
    if method == "omw":
        rows = numit // estep
    else:
        if istp is None:
            raise ValueError("istp undefined: NUMIT < 3*saveStep (decon_lucy_function.m:174)")
        rows = istp
    return e[1:rows + 1]


def debug_err_mat(iterates, Ipre, estep, method):
    """err_mat of a debug run from its iterates (mean in float64 of the float64 difference, :115)."""
    I64 = np.asarray(Ipre, np.float64)
    mse = [float(np.mean((np.asarray(J, np.float64) - I64) ** 2)) for J in iterates]
    return err_mat_from_mse(mse, estep, method)


def rel_l2(a, b):
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    a = np.asarray(a, dtype=np.complex128 if cplx else np.float64)
    b = np.asarray(b, dtype=np.complex128 if cplx else np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
