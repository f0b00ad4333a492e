"""Batched chunk deconvolution: shared launches must reproduce the per-chunk drop-in calls."""
import numpy as np
import pytest

from oracle import decon as O
from petakit5d_b200 import chunking as K
from petakit5d_b200 import decon as D
from petakit5d_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workload():
    rng = np.random.default_rng(5)
    psfs = [synth.gaussian_psf((15, 15, 21), s, 3.0) for s in (1.3, 1.5, 1.8)]
    psfs_b = [np.asfortranarray(p[::-1, ::-1, ::-1]) for p in psfs]
    shapes = [(48, 40, 32), (64, 64, 24), (40, 56, 40), (36, 36, 30), (64, 48, 32), (50, 44, 22)]
    chunks, ids, boxes = [], [], []
    for i, sh in enumerate(shapes):
        pid = int(rng.integers(0, 3))
        chunks.append(synth.puncta_volume(sh, 20, psfs[pid], seed=100 + i, background=100.0))
        ids.append(pid)
        boxes.append([4, 4, 4, sh[0] - 3, sh[1] - 3, sh[2] - 3])
    return chunks, psfs, psfs_b, ids, boxes


@pytest.mark.parametrize("method,numit", [("omw", 2), ("rl", 5)])
def test_batch_equals_single_calls(workload, method, numit):
    chunks, psfs, psfs_b, ids, boxes = workload
    outs = K.batch_decon(chunks, psfs, ids, numit, method, psfs_b if method == "omw" else None, boxes,
                         Background=100, save16bit=False)
    for c, pid, bb, o in zip(chunks, ids, boxes, outs):
        if method == "omw":
            ref, _ = D.decon_lucy_omw_function(c, psfs[pid], psfs_b[pid], numit, Background=100, save16bit=False, bbox=bb)
        else:
            ref, _, _ = D.decon_lucy_function(c, psfs[pid], numit, Background=100, save16bit=False, bbox=bb)
        assert o.shape == ref.shape
        assert np.array_equal(o, ref)


def test_batch_uint16_matches_oracle(workload):
    chunks, psfs, psfs_b, ids, boxes = workload
    outs = K.batch_decon(chunks, psfs, ids, 2, "omw", psfs_b, boxes, Background=100)
    for c, pid, bb, o in zip(chunks, ids, boxes, outs):
        ref = O.decon_lucy_omw(c, psfs[pid], psfs_b[pid], 2, background=100, bbox=bb)
        assert np.max(np.abs(o.astype(np.int64) - ref.astype(np.int64))) <= 1


def test_batch_padded_to_good_sizes_matches_oracle_on_padded_input(workload):
    _, psfs, psfs_b, _, _ = workload
    chunks = [synth.puncta_volume(sh, 15, psfs[0], seed=7 + i, background=100.0)
              for i, sh in enumerate([(44, 26, 22), (34, 38, 26)])]
    outs = K.batch_decon(chunks, psfs[:1], [0, 0], 2, "omw", psfs_b[:1], None, pad_good=True, Background=100,
                         save16bit=False)
    for c, o in zip(chunks, outs):
        pdims = [K.find_good_factor_number(v) for v in c.shape]
        Ipre, _ = O.preprocess(c, 100, False, np.float32)
        Ip = np.zeros(pdims, np.float32)
        Ip[:c.shape[0], :c.shape[1], :c.shape[2]] = Ipre
        ref = O.decon_lucy_omw(Ip, psfs[0], psfs_b[0], 2, background=0, save16bit=False)
        ref = ref[:c.shape[0], :c.shape[1], :c.shape[2]]
        assert o.shape == c.shape
        assert O.rel_l2(o, ref) <= 1e-4


def test_large_in_memory_chunked_matches_per_chunk_oracle():
    psf = synth.gaussian_psf((11, 11, 15), 1.3, 3.0)
    psf_b = np.asfortranarray(psf[::-1, ::-1, ::-1])
    vol = synth.puncta_volume((96, 80, 48), 60, psf, seed=21, background=100.0)
    out = K.decon_large_in_memory(vol, psf, 2, "omw", psf_b, batch_size=(48, 40, 24), Background=100, save16bit=False)
    border = K.border_size(psf.shape)
    bb, rb, _ = K.zarr_chunk_coordinates(vol.shape, (48, 40, 24), (48, 40, 24), None, False, border)
    ref = np.zeros(vol.shape, np.float32)
    for b, r in zip(bb, rb):
        c = vol[b[0] - 1:b[3], b[1] - 1:b[4], b[2] - 1:b[5]]
        st = r[:3] - b[:3] + 1
        en = r[3:] - b[:3] + 1
        o = O.decon_lucy_omw(c, psf, psf_b, 2, background=100, save16bit=False, bbox=[*st, *en])
        ref[r[0] - 1:r[3], r[1] - 1:r[4], r[2] - 1:r[5]] = o
    assert O.rel_l2(out, ref) <= 1e-4
