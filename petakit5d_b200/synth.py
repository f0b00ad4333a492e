"""Seeded synthetic volumes and PSFs for the deconvolution workloads.

The reference's demo runs on a light-sheet dataset that is downloaded at run time
(demos/demo_RL_deconvolution.m:43); these generators stand in for it.  Volumes are numpy arrays
indexed ``[y, x, z]`` (MATLAB order) in Fortran (column-major) memory order, so their bytes are
exactly what a MATLAB caller would hand to the C ABI.  All randomness comes from numpy's PCG64
with an explicit seed.

Workloads (sizes are x, y, z):
  * ``puncta_volume``        -- Gaussian puncta (sigma 1 voxel, amplitude U[200, 2000]) at uniform
                                positions plus a background, convolved with the PSF, Poisson noise.
  * ``gaussian_psf``         -- anisotropic Gaussian PSF, peak at the 1-based index floor(size/2)+1.
  * ``lobed_psf``            -- Gaussian PSF plus two side lobes at +-dz along z.
  * ``sinusoid_background``  -- smooth 3D sinusoid background (period, amplitude, offset).
  * ``chunk_workload``       -- uneven chunks with overlap borders and per-chunk PSF ids.
  * ``measured_psf``         -- a bead image as a microscope records it (camera offset, read noise,
                                hot pixels, peak anywhere): the input of psf_gen_new.
"""
from __future__ import annotations

import numpy as np

__all__ = ["gaussian_psf", "lobed_psf", "puncta_volume", "sinusoid_background", "chunk_workload",
           "single_volume_workload", "measured_psf", "LLSM_PSF", "SMALL_PSF"]


def _rng(seed):
    return np.random.Generator(np.random.PCG64(int(seed)))


def gaussian_psf(size_yxz=(31, 31, 41), sigma_xy=1.3, sigma_z=3.0, lobes=(), lobe_amp=0.0):
    """Normalised (sum 1, float32) Gaussian PSF; ``lobes`` are extra z offsets with ``lobe_amp``."""
    ny, nx, nz = size_yxz
    cy, cx, cz = ny // 2, nx // 2, nz // 2
    y = (np.arange(ny) - cy)[:, None, None].astype(np.float64)
    x = (np.arange(nx) - cx)[None, :, None].astype(np.float64)
    z = (np.arange(nz) - cz)[None, None, :].astype(np.float64)
    lat = np.exp(-(y * y + x * x) / (2 * sigma_xy ** 2))
    p = lat * np.exp(-(z * z) / (2 * sigma_z ** 2))
    for dz in lobes:
        p = p + lobe_amp * lat * np.exp(-((z - dz) ** 2) / (2 * sigma_z ** 2))
    p /= p.sum()
    return np.asfortranarray(p.astype(np.float32))


def lobed_psf(size_yxz=(64, 64, 101), sigma_xy=1.5, sigma_z=4.0, lobe_dz=12, lobe_amp=0.15):
    return gaussian_psf(size_yxz, sigma_xy, sigma_z, lobes=(-lobe_dz, lobe_dz), lobe_amp=lobe_amp)


def measured_psf(size_yxz=(64, 64, 101), peak=None, sigma_xy=1.5, sigma_z=4.0, amplitude=5000.0, offset=100.0,
                 read_noise=3.0, hot_pixels=6, seed=0):
    """Bead image: offset + amplitude * Gaussian(peak) + Gaussian read noise + isolated hot pixels,
    float32 in Fortran order.  ``peak`` is 0-based (y, x, z); default the array centre."""
    ny, nx, nz = size_yxz
    rng = _rng(seed)
    py, px, pz = peak if peak is not None else (ny // 2, nx // 2, nz // 2)
    y = (np.arange(ny) - py)[:, None, None].astype(np.float64)
    x = (np.arange(nx) - px)[None, :, None].astype(np.float64)
    z = (np.arange(nz) - pz)[None, None, :].astype(np.float64)
    img = offset + amplitude * np.exp(-(y * y + x * x) / (2 * sigma_xy ** 2) - (z * z) / (2 * sigma_z ** 2))
    img = img + rng.normal(0.0, read_noise, size=(ny, nx, nz))
    for _ in range(hot_pixels):
        img[rng.integers(ny), rng.integers(nx), rng.integers(nz)] += amplitude * 0.2
    return np.asfortranarray(img.astype(np.float32))


SMALL_PSF = dict(size_yxz=(31, 31, 41), sigma_xy=1.3, sigma_z=3.0)
LLSM_PSF = dict(size_yxz=(64, 64, 101), sigma_xy=1.5, sigma_z=4.0, lobe_dz=12, lobe_amp=0.15)


def sinusoid_background(shape_yxz, period=200.0, amplitude=300.0, offset=100.0):
    """offset + amplitude * (1 + sin(2 pi y/P) sin(2 pi x/P) sin(2 pi z/P)) / 2  (>= offset)."""
    ny, nx, nz = shape_yxz
    w = 2 * np.pi / period
    sy = np.sin(w * np.arange(ny))[:, None, None]
    sx = np.sin(w * np.arange(nx))[None, :, None]
    sz = np.sin(w * np.arange(nz))[None, None, :]
    return offset + amplitude * 0.5 * (1.0 + sy * sx * sz)


def _render_puncta(shape, n, rng, sigma=1.0, amp=(200.0, 2000.0), radius=4):
    ny, nx, nz = shape
    img = np.zeros(shape, dtype=np.float64)
    pos = rng.uniform(0.0, 1.0, size=(n, 3)) * np.array([ny, nx, nz], dtype=np.float64)
    a = rng.uniform(amp[0], amp[1], size=n)
    base = np.floor(pos).astype(np.int64)
    off = np.arange(-radius, radius + 1)
    oy, ox, oz = np.meshgrid(off, off, off, indexing="ij")
    oy, ox, oz = oy.ravel(), ox.ravel(), oz.ravel()
    step = 4096
    for s in range(0, n, step):
        b = base[s:s + step]
        p = pos[s:s + step]
        iy = b[:, 0:1] + oy[None, :]
        ix = b[:, 1:2] + ox[None, :]
        iz = b[:, 2:3] + oz[None, :]
        d2 = (iy - p[:, 0:1]) ** 2 + (ix - p[:, 1:2]) ** 2 + (iz - p[:, 2:3]) ** 2
        v = a[s:s + step, None] * np.exp(-d2 / (2 * sigma * sigma))
        np.add.at(img, (iy % ny, ix % nx, iz % nz), v)
    return img


def _circular_blur(img, psf):
    """Circular convolution with the PSF, centred the way decon_psf2otf centres it."""
    import scipy.fft as sfft
    shape = img.shape
    big = np.zeros(shape, dtype=np.float64)
    ps = psf.shape
    big[:ps[0], :ps[1], :ps[2]] = psf
    big = np.roll(big, shift=tuple(-(np.array(ps) // 2)), axis=(0, 1, 2))
    ax = (2, 1, 0)
    H = sfft.rfftn(big, axes=ax, workers=-1)
    out = sfft.irfftn(sfft.rfftn(img, axes=ax, workers=-1) * H, s=(shape[2], shape[1], shape[0]), axes=ax, workers=-1)
    return out


def puncta_volume(shape_yxz, n_puncta, psf, seed, background=100.0):
    """uint16 volume: puncta + background (scalar or array), blurred by ``psf``, Poisson noise."""
    rng = _rng(seed)
    img = _render_puncta(tuple(shape_yxz), int(n_puncta), rng)
    clean = _circular_blur(img, psf) + background
    clean = np.maximum(clean, 0.0)
    noisy = rng.poisson(clean)
    return np.asfortranarray(np.clip(noisy, 0, 65535).astype(np.uint16))


def single_volume_workload(kind, seed=1):
    """(volume, psf) for the single-volume workloads.

    ``kind='rl_small'``: 128x128x64 (x,y,z), 200 puncta, background 100, 31x31x41 Gaussian PSF.
    ``kind='omw_llsm'``: 512x512x256, 20 000 puncta over a sinusoid background, 64x64x101 lobed PSF.
    """
    if kind == "rl_small":
        psf = gaussian_psf(**SMALL_PSF)
        vol = puncta_volume((128, 128, 64), 200, psf, seed, background=100.0)
        return vol, psf
    if kind == "omw_llsm":
        psf = lobed_psf(**LLSM_PSF)
        shape = (512, 512, 256)
        vol = puncta_volume(shape, 20000, psf, seed, background=sinusoid_background(shape))
        return vol, psf
    raise ValueError(kind)


def chunk_workload(n_chunks=96, seed=3, border=16, core_xy=(192, 256, 320, 384), core_z=(96, 128, 192, 256),
                   sigmas=(1.3, 1.5, 1.8), density=200.0 / (128 * 128 * 64)):
    """Uneven chunks with ``border`` overlap voxels per side; returns (chunks, psfs, psf_ids, bboxes).

    Each chunk is core + 2*border per axis; its output region (1-based inclusive deconBbox,
    ``[y1 x1 z1 y2 x2 z2]``) is the core.  Content follows the small-volume generator (same puncta
    density, background 100) blurred by the chunk's PSF.
    """
    rng = _rng(seed)
    psfs = [gaussian_psf((31, 31, 41), s, 3.0) for s in sigmas]
    chunks, ids, bboxes = [], [], []
    for i in range(n_chunks):
        cy = int(rng.choice(core_xy))
        cx = int(rng.choice(core_xy))
        cz = int(rng.choice(core_z))
        pid = int(rng.integers(0, len(psfs)))
        shape = (cy + 2 * border, cx + 2 * border, cz + 2 * border)
        n = int(round(density * np.prod(shape)))
        chunks.append(puncta_volume(shape, n, psfs[pid], seed * 100003 + i, background=100.0))
        ids.append(pid)
        bboxes.append([border + 1, border + 1, border + 1, border + cy, border + cx, border + cz])
    return chunks, psfs, ids, bboxes


# ---------------------------------------------------------------- GPU generator for large workloads
def puncta_volume_torch(shape_yxz, n_puncta, psf, seed, background=100.0, device="cuda", sinusoid=None,
                        gaussian_psf_sigmas=None):
    """The same recipe as ``puncta_volume`` run with torch on ``device`` (for volumes too large to
    generate quickly on the host).  Returns an int16 tensor shaped (nz, nx, ny) whose bits are the
    uint16 voxels, i.e. the column-major [ny nx nz] volume.  ``sinusoid``: dict of
    ``sinusoid_background`` arguments added to ``background``.

    ``gaussian_psf_sigmas=(sigma_xy, sigma_z)``: the PSF is that Gaussian, so each blurred punctum is
    rendered directly (a sigma-1 Gaussian convolved with the PSF is the Gaussian with the variances
    added), which avoids a transform of the whole volume."""
    if gaussian_psf_sigmas is not None:
        return _blurred_puncta_torch(shape_yxz, n_puncta, gaussian_psf_sigmas, seed, background, device)
    import torch
    ny, nx, nz = (int(v) for v in shape_yxz)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    img = torch.zeros(nz * nx * ny, dtype=torch.float32, device=device)
    n = int(n_puncta)
    radius = 4
    off = torch.arange(-radius, radius + 1, device=device)
    oz, ox, oy = torch.meshgrid(off, off, off, indexing="ij")
    oy, ox, oz = oy.reshape(1, -1), ox.reshape(1, -1), oz.reshape(1, -1)
    dims = torch.tensor([ny, nx, nz], device=device, dtype=torch.float32)
    step = 1 << 16
    for s in range(0, n, step):
        m = min(step, n - s)
        pos = torch.rand((m, 3), generator=g, device=device) * dims
        amp = 200.0 + 1800.0 * torch.rand((m, 1), generator=g, device=device)
        b = torch.floor(pos).to(torch.int64)
        iy, ix, iz = b[:, 0:1] + oy, b[:, 1:2] + ox, b[:, 2:3] + oz
        d2 = (iy - pos[:, 0:1]) ** 2 + (ix - pos[:, 1:2]) ** 2 + (iz - pos[:, 2:3]) ** 2
        val = amp * torch.exp(-d2 / 2.0)
        idx = (iy % ny) + ny * ((ix % nx) + nx * (iz % nz))
        img.index_add_(0, idx.reshape(-1), val.reshape(-1))
        del pos, amp, b, iy, ix, iz, d2, val, idx
    img = img.view(nz, nx, ny)
    p = np.asarray(psf, np.float64)
    p = (p / p.sum()).astype(np.float32)
    py, px, pz = p.shape
    ker = torch.zeros((nz, nx, ny), dtype=torch.float32, device=device)
    ker[:pz, :px, :py] = torch.from_numpy(np.ascontiguousarray(p.transpose(2, 1, 0))).to(device)
    ker = torch.roll(ker, shifts=(-(pz // 2), -(px // 2), -(py // 2)), dims=(0, 1, 2))
    H = torch.fft.rfftn(ker)
    del ker
    F = torch.fft.rfftn(img)
    del img
    F *= H
    del H
    clean = torch.fft.irfftn(F, s=(nz, nx, ny))
    del F
    clean += float(background)
    if sinusoid is not None:
        period = float(sinusoid.get("period", 200.0))
        amp = float(sinusoid.get("amplitude", 300.0))
        offv = float(sinusoid.get("offset", 100.0))
        w = 2 * np.pi / period
        sy = torch.sin(w * torch.arange(ny, device=device, dtype=torch.float32)).view(1, 1, ny)
        sx = torch.sin(w * torch.arange(nx, device=device, dtype=torch.float32)).view(1, nx, 1)
        sz = torch.sin(w * torch.arange(nz, device=device, dtype=torch.float32)).view(nz, 1, 1)
        clean += offv + amp * 0.5 * (1.0 + sz * sx * sy)
    clean.clamp_(min=0)
    noisy = torch.poisson(clean, generator=g)
    del clean
    noisy.clamp_(0, 65535)
    v = noisy.to(torch.int32)
    del noisy
    v = torch.where(v > 32767, v - 65536, v).to(torch.int16)
    return v


def _blurred_puncta_torch(shape_yxz, n_puncta, sigmas, seed, background, device, slab=64):
    """Blurred Gaussian puncta rendered z-slab by z-slab (every tensor stays below 2^31 elements);
    puncta wrap around every axis, as the circular blur of the host generator does."""
    import torch
    ny, nx, nz = (int(v) for v in shape_yxz)
    sxy, sz = float(sigmas[0]), float(sigmas[1])
    vy = vx = 1.0 + sxy * sxy
    vz = 1.0 + sz * sz
    gain = 1.0 / np.sqrt(vy * vx * vz)                      # product of sigma_1 / sqrt(var) per axis
    ry, rz = int(np.ceil(4 * np.sqrt(vy))), int(np.ceil(4 * np.sqrt(vz)))
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    n = int(n_puncta)
    pos = torch.rand((n, 3), generator=g, device=device) * torch.tensor([ny, nx, nz], device=device, dtype=torch.float32)
    amp = (200.0 + 1800.0 * torch.rand((n,), generator=g, device=device)) * gain
    order = torch.argsort(pos[:, 2])
    pos, amp = pos[order], amp[order]
    zs = pos[:, 2].contiguous()
    out = torch.empty((nz, nx, ny), dtype=torch.int16, device=device)
    oy = torch.arange(-ry, ry + 1, device=device)
    oz = torch.arange(-rz, rz + 1, device=device)
    Z, X, Y = torch.meshgrid(oz, oy, oy, indexing="ij")
    Y, X, Z = Y.reshape(1, -1), X.reshape(1, -1), Z.reshape(1, -1)
    for z0 in range(0, nz, slab):
        z1 = min(nz, z0 + slab)
        img = torch.full(((z1 - z0) * nx * ny,), float(background), dtype=torch.float32, device=device)
        for shift in (0.0, float(nz), -float(nz)):          # wrap-around copies near the z ends
            lo = torch.searchsorted(zs, torch.tensor([z0 - rz - 1 - shift], device=device))
            hi = torch.searchsorted(zs, torch.tensor([z1 + rz + 1 - shift], device=device))
            i0, i1 = int(lo.item()), int(hi.item())
            for c0 in range(i0, i1, 1 << 13):
                c1 = min(i1, c0 + (1 << 13))
                p = pos[c0:c1]
                pz = p[:, 2:3] + shift
                b = torch.floor(torch.cat([p[:, 0:2], pz], dim=1)).to(torch.int64)
                iy, ix, iz = b[:, 0:1] + Y, b[:, 1:2] + X, b[:, 2:3] + Z
                e = (iy - p[:, 0:1]) ** 2 / (2 * vy) + (ix - p[:, 1:2]) ** 2 / (2 * vx) + (iz - pz) ** 2 / (2 * vz)
                val = amp[c0:c1, None] * torch.exp(-e)
                keep = (iz >= z0) & (iz < z1)
                idx = (iy % ny) + ny * ((ix % nx) + nx * (iz - z0))
                img.index_add_(0, idx[keep], val[keep])
                del p, pz, b, iy, ix, iz, e, val, keep, idx
        img.clamp_(min=0)
        noisy = torch.poisson(img, generator=g).clamp_(0, 65535).to(torch.int32)
        del img
        out[z0:z1] = torch.where(noisy > 32767, noisy - 65536, noisy).to(torch.int16).view(z1 - z0, nx, ny)
        del noisy
    return out
