"""CPU oracle (test infrastructure only) for the edge taper of RLdecon.m:351-357:

    taperKernel = fspecial('gaussian', nTapering+30, nTapering);
    for iz = 1:nz, rawdata(:,:,iz) = edgetaper(rawdata(:,:,iz), taperKernel); end

``fspecial`` and ``edgetaper`` are MATLAB Image Processing Toolbox functions, closed third-party code
that is not under the reference tree; this file restates their documented behaviour in float64:

* ``fspecial('gaussian', hsize, sigma)``: exp(-(x^2 + y^2) / (2 sigma^2)) on an hsize x hsize grid
  centred at (hsize - 1) / 2, values below eps * max set to 0, normalised to sum 1.
* ``edgetaper(I, PSF)``: J = alpha .* I + (1 - alpha) .* B, with B the circular blur of I by PSF
  (``real(ifft2(fft2(I) .* psf2otf(PSF, size(I))))``) and a weight alpha that is 1 in the interior and
  0 at the borders, built from the PSF's autocorrelation: per axis d, beta_d is the circular
  autocorrelation of the PSF's projection on d (period n_d - 1), normalised to 1 at lag 0 and
  extended by its lag-0 value to length n_d; alpha = (1 - beta_y) (1 - beta_x)^T.  J keeps I's class
  (uint16 by MATLAB's round-half-away and saturation).

Parity unpinned: no MATLAB here and no reference test covers the taper; the FFT form below is
cross-checked against a direct circular sum in the tests.
"""
import numpy as np


def fspecial_gaussian(hsize, sigma):
    """fspecial('gaussian', hsize, sigma) for a scalar hsize (float64, sum 1)."""
    r = np.arange(int(hsize), dtype=np.float64) - (int(hsize) - 1) / 2.0
    h = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / (2.0 * float(sigma) ** 2))
    h[h < np.finfo(np.float64).eps * h.max()] = 0.0
    return h / h.sum()


def taper_weight(psf, n, axis):
    """beta_d of the taper weight: circular autocorrelation of the PSF's projection on ``axis`` over a
    period of n - 1 samples, normalised by its maximum, lag 0 repeated at index n - 1."""
    p = np.asarray(psf, np.float64).sum(axis=1 - axis)
    if p.size > n - 1:
        raise ValueError("edgetaper: PSF larger than the image")
    z = np.real(np.fft.ifft(np.abs(np.fft.fft(p, n - 1)) ** 2))
    z = np.concatenate([z, z[:1]])
    return z / z.max()


def taper_alpha(psf, ny, nx):
    return np.outer(1.0 - taper_weight(psf, ny, 0), 1.0 - taper_weight(psf, nx, 1))


def circular_blur(img, psf):
    """real(ifft2(fft2(img) .* psf2otf(psf, size(img)))) in float64."""
    ny, nx = img.shape
    hy, hx = psf.shape
    pad = np.zeros((ny, nx))
    pad[:hy, :hx] = psf
    otf = np.fft.fft2(np.roll(pad, (-(hy // 2), -(hx // 2)), axis=(0, 1)))
    return np.real(np.fft.ifft2(np.fft.fft2(img) * otf))


def circular_blur_direct(img, psf):
    """The same blur as a direct sum: B(y, x) = sum_ij psf(i, j) img((y + hy//2 - i) mod ny,
    (x + hx//2 - j) mod nx).  Small cases only."""
    ny, nx = img.shape
    hy, hx = psf.shape
    out = np.zeros((ny, nx))
    for i in range(hy):
        for j in range(hx):
            out += psf[i, j] * np.roll(img, (i - hy // 2, j - hx // 2), axis=(0, 1))
    return out


def _to_class(j, dtype):
    if dtype == np.uint16:
        r = np.where(j >= 0, np.floor(j + 0.5), np.ceil(j - 0.5))
        return np.clip(np.nan_to_num(r), 0, 65535).astype(np.uint16)
    return j.astype(dtype)


def edgetaper(img, psf):
    """edgetaper(I, PSF) for one 2-D image (uint16 or floating)."""
    img = np.asarray(img)
    psf = np.asarray(psf, np.float64)
    a = img.astype(np.float64)
    alpha = taper_alpha(psf, *a.shape)
    j = alpha * a + (1.0 - alpha) * circular_blur(a, psf)
    return _to_class(j, img.dtype if img.dtype in (np.uint16, np.float32) else np.float64)


def edgetaper_slices(vol, psf):
    """RLdecon.m:354-356: edgetaper of every z slice of a [ny, nx, nz] volume."""
    vol = np.asarray(vol)
    out = np.empty(vol.shape, vol.dtype, order="F")
    for z in range(vol.shape[2]):
        out[:, :, z] = edgetaper(vol[:, :, z], psf)
    return out
