"""Region skipping by 2-D Zarr masks in the large-file runners (RLdecon_large_in_memory.m:201-216,
RLdecon_for_zarr_block.m:111-128), on the host."""
import os

import numpy as np
import pytest

from petakit5d_b200 import chunking as K
from petakit5d_b200 import tiff as T
from petakit5d_b200 import zarrio as Z


def _masks(tmp_path, ny, nx, nz, xy=None, xz=None, yz=None):
    paths = []
    for name, shape, m in (("xy", (ny, nx), xy), ("xz", (nx, nz), xz), ("yz", (ny, nz), yz)):
        a = np.ones(shape, np.uint8) if m is None else m.astype(np.uint8)
        p = str(tmp_path / f"mask_{name}.zarr")
        Z.writezarr(a, p, blockSize=(16, 16, 1))
        paths.append(p)
    return paths


def test_region_is_skipped_when_any_projection_window_is_empty(tmp_path):
    ny, nx, nz = 40, 36, 20
    xy = np.zeros((ny, nx), bool)
    xy[5:15, 20:30] = True
    yz = np.ones((ny, nz), bool)
    yz[:, 12:] = False
    paths = _masks(tmp_path, ny, nx, nz, xy=xy, yz=yz)
    rng = np.random.default_rng(0)
    for _ in range(60):
        lo = rng.integers(1, [ny, nx, nz], endpoint=True)
        hi = np.array([rng.integers(l, n, endpoint=True) for l, n in zip(lo, (ny, nx, nz))])
        r = [*lo, *hi]
        want = not (xy[lo[0] - 1:hi[0], lo[1] - 1:hi[1]].any() and yz[lo[0] - 1:hi[0], lo[2] - 1:hi[2]].any())
        assert K.region_masked_out(paths, r) == want, r
    assert not K.region_masked_out((), [1, 1, 1, 4, 4, 4])
    assert not K.region_masked_out([""], [1, 1, 1, 4, 4, 4])


def test_in_place_runner_writes_zeros_for_masked_regions_without_deconvolving(tmp_path):
    vol = np.asfortranarray(np.random.default_rng(1).integers(100, 3000, (70, 60, 40)).astype(np.uint16))
    zin = str(tmp_path / "raw.zarr")
    Z.writezarr(vol, zin, blockSize=(32, 32, 32))
    pfn = str(tmp_path / "psf.tif")
    T.writetiff(np.ones((9, 9, 11), np.float32), pfn)
    paths = _masks(tmp_path, 70, 60, 40, xy=np.zeros((70, 60), bool))
    dpath = str(tmp_path / "decon")
    os.makedirs(dpath)
    stale = str(tmp_path / "decon" / "raw.zarr_7")              # an interrupted run's temporary array
    Z.writezarr(np.full(vol.shape, 9, np.uint16), stale, blockSize=(32, 32, 32))
    out = K.RLdecon_large_in_place(zin, pfn, dpath, 0.108, 0.3, batchSize=(64, 64, 64), blockSize=(32, 32, 32),
                                   maskFullpaths=paths, psfGen=False, flipZstack=True, uuid="7")
    got = Z.readzarr(out)
    assert got.shape == vol.shape and got.dtype == np.uint16 and not got.any()
    assert not os.path.exists(stale)
    assert not os.path.exists(os.path.join(dpath, "zarr_flag", "raw_7"))       # flags removed at the end
    for ax, shape in (("y", (60, 40)), ("x", (70, 40)), ("z", (70, 60))):       # XR_MIP_zarr, axis [1 1 1]
        mip = T.readtiff(os.path.join(dpath, "MIPs", f"raw_MIP_{ax}.tif"))
        assert mip.shape == shape and not mip.any()


def test_in_place_runner_resumes_flagged_tasks(tmp_path):
    """A second call with the same uuid skips the tasks whose flag exists (RLdecon_large_in_place.m:217-221):
    here the only task, so the temporary array is moved into place as it stands."""
    vol = np.asfortranarray(np.random.default_rng(2).integers(100, 3000, (70, 60, 40)).astype(np.uint16))
    zin = str(tmp_path / "raw.zarr")
    Z.writezarr(vol, zin, blockSize=(32, 32, 32))
    pfn = str(tmp_path / "psf.tif")
    T.writetiff(np.ones((9, 9, 11), np.float32), pfn)
    dpath = str(tmp_path / "decon")
    os.makedirs(dpath)
    part = np.asfortranarray(np.arange(70 * 60 * 40, dtype=np.uint32).reshape(70, 60, 40) % 5000).astype(np.uint16)
    Z.writezarr(part, os.path.join(dpath, "raw.zarr_9"), blockSize=(32, 32, 32))
    _, rb, _ = K.zarr_chunk_coordinates((70, 60, 40), batch_size=(64, 64, 64), block_size=(32, 32, 32),
                                        same_batch_size=True, border=K.border_size((9, 9, 11)))
    flags = os.path.join(dpath, "zarr_flag", "raw_9")
    os.makedirs(flags)
    open(os.path.join(flags, f"blocks_1_{len(rb)}.mat"), "wb").close()
    out = K.RLdecon_large_in_place(zin, pfn, dpath, 0.108, 0.3, batchSize=(64, 64, 64), blockSize=(32, 32, 32),
                                   psfGen=False, uuid="9")
    np.testing.assert_array_equal(Z.readzarr(out), part)
    np.testing.assert_array_equal(T.readtiff(os.path.join(dpath, "MIPs", "raw_MIP_z.tif")), part.max(axis=2))
    assert not os.path.exists(flags)


def test_mask_list_must_have_three_paths():
    with pytest.raises(ValueError):
        K.RLdecon_large_in_place("a.zarr", "p.tif", "d", 0.108, 0.3, maskFullpaths=["a.zarr", "b.zarr"])


def test_in_memory_runner_refuses_deskew_without_rotate():
    with pytest.raises(NotImplementedError):
        K.RLdecon_large_in_memory("a.tif", "p.tif", "d/a.tif", 0.108, 0.3, Deskew=True, Rotate=False)


def test_in_place_runner_accepts_deskew(tmp_path):
    vol = np.zeros((40, 40, 20), np.uint16)
    zin = str(tmp_path / "raw.zarr")
    Z.writezarr(vol, zin, blockSize=(32, 32, 32))
    pfn = str(tmp_path / "psf.tif")
    T.writetiff(np.ones((9, 9, 11), np.float32), pfn)
    paths = _masks(tmp_path, 40, 40, 20, xy=np.zeros((40, 40), bool))
    out = K.RLdecon_large_in_place(zin, pfn, str(tmp_path / "d"), 0.108, 0.3, batchSize=(32, 32, 32),
                                   blockSize=(32, 32, 32), maskFullpaths=paths, psfGen=False, Deskew=True)
    assert not Z.readzarr(out).any()


def test_frame3d_sends_large_frames_to_the_in_place_runner_and_returns(tmp_path):
    """XR_RLdeconFrame3D.m:164-168, 245-262: a frame over CPUMaxMem goes to RLdecon_large_in_place, after
    which the call returns (the next frame is not processed), as in the reference."""
    from petakit5d_b200.rldecon import XR_RLdeconFrame3D
    vol = np.asfortranarray(np.random.default_rng(3).integers(100, 3000, (40, 36, 20)).astype(np.uint16))
    frames = [str(tmp_path / "f1.zarr"), str(tmp_path / "f2.zarr")]
    for f in frames:
        Z.writezarr(vol, f, blockSize=(32, 32, 32))
    pfn = str(tmp_path / "psf.tif")
    T.writetiff(np.ones((9, 9, 11), np.float32), pfn)
    paths = _masks(tmp_path, 40, 36, 20, xy=np.zeros((40, 36), bool))
    dpath = str(tmp_path / "decon")
    XR_RLdeconFrame3D(frames, 0.108, 0.3, dpath, PSFfile=pfn, CPUMaxMem=0, largeMethod="inplace",
                      batchSize=[32, 32, 32], blockSize=[32, 32, 32], maskFullpaths=paths, psfGen=False, uuid="5")
    assert os.path.isdir(os.path.join(dpath, "f1.zarr")) and not Z.readzarr(os.path.join(dpath, "f1.zarr")).any()
    assert not os.path.exists(os.path.join(dpath, "f2.zarr"))
    assert os.path.exists(os.path.join(dpath, "MIPs", "f1_MIP_z.tif"))
