"""Serving with continuous batching: each result equals the plain drop-in call's, alone and mixed."""
import threading

import numpy as np
import pytest

from petakit5d_b200 import decon as D
from petakit5d_b200 import serve as SV
from petakit5d_b200 import synth
from petakit5d_b200._lib import PK_ERR_CANCELLED, PK_ERR_TIMEOUT, PkError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    psfs = [synth.gaussian_psf((15, 15, 21), s, 3.0) for s in (1.3, 1.5, 1.8)]
    psfs_b = [np.asfortranarray(p[::-1, ::-1, ::-1]) for p in psfs]
    rng = np.random.default_rng(11)
    reqs = []
    shapes = [(48, 40, 32), (64, 64, 24), (40, 56, 40), (36, 36, 30), (64, 48, 32), (50, 44, 22), (96, 96, 48)]
    for i in range(14):
        sh = shapes[i % len(shapes)]
        pid = int(rng.integers(0, 3))
        method = "omw" if rng.random() < 0.7 else "rl"
        numit = 2 if method == "omw" else 6
        vol = synth.puncta_volume(sh, 15, psfs[pid], seed=300 + i, background=100.0)
        reqs.append((vol, pid, method, numit))
    return psfs, psfs_b, reqs


def _alone(psfs, psfs_b, vol, pid, method, numit):
    if method == "omw":
        return D.decon_lucy_omw_function(vol, psfs[pid], psfs_b[pid], numit, Background=100)[0]
    return D.decon_lucy_function(vol, psfs[pid], numit, Background=100)[0]


def test_served_results_equal_alone_in_the_mix(setup):
    psfs, psfs_b, reqs = setup
    with SV.Server(budget_bytes=4e9, max_batch=8) as srv:
        for i in range(3):
            srv.add_psf(i, psfs[i], psfs_b[i])
        ids = []
        # requests arrive from two client threads while others run
        def client(sub):
            for vol, pid, method, numit in sub:
                ids.append((srv.submit(vol, pid, method, numit, Background=100), (vol, pid, method, numit)))
        t1 = threading.Thread(target=client, args=(reqs[::2],))
        t2 = threading.Thread(target=client, args=(reqs[1::2],))
        t1.start(); t2.start(); t1.join(); t2.join()
        lat = []
        for rid, (vol, pid, method, numit) in ids:
            out, ms = srv.wait(rid)
            lat.append(ms)
            assert np.array_equal(out, _alone(psfs, psfs_b, vol, pid, method, numit))
        st = srv.stats()
        assert st["completed"] == len(reqs)
        assert st["rounds"] > 0
        assert all(v > 0 for v in lat)


def test_served_tiny_budget_still_completes(setup):
    psfs, psfs_b, reqs = setup
    with SV.Server(budget_bytes=1, max_batch=4) as srv:
        srv.add_psf(0, psfs[0], psfs_b[0])
        ids = [srv.submit(v, 0, "omw", 2, Background=100) for v, _, _, _ in reqs[:4]]
        outs = [srv.wait(r)[0] for r in ids]
        for (v, _, _, _), o in zip(reqs[:4], outs):
            assert np.array_equal(o, _alone(psfs, psfs_b, v, 0, "omw", 2))
        # one request in flight at a time: the peak is one request's buffers
        assert srv.stats()["peak_inflight_bytes"] < 64 * 1024 * 1024


def test_served_cancel_and_timeout(setup):
    psfs, psfs_b, reqs = setup
    with SV.Server(budget_bytes=4e9, max_batch=2) as srv:
        srv.add_psf(0, psfs[0], psfs_b[0])
        vol = reqs[6][0]
        r1 = srv.submit(vol, 0, "rl", 20, Background=100)
        with pytest.raises(PkError) as e:
            srv.wait(r1, timeout_ms=0)
        assert e.value.status == PK_ERR_TIMEOUT
        r2 = srv.submit(vol, 0, "omw", 2, Background=100)
        srv.cancel(r1)
        with pytest.raises(PkError) as e:
            srv.wait(r1)
        assert e.value.status == PK_ERR_CANCELLED
        out, _ = srv.wait(r2)
        assert np.array_equal(out, _alone(psfs, psfs_b, vol, 0, "omw", 2))


def test_served_rejects_bad_requests(setup):
    psfs, psfs_b, reqs = setup
    with SV.Server() as srv:
        srv.add_psf(0, psfs[0], None)
        with pytest.raises(PkError):
            srv.submit(reqs[0][0], 0, "omw", 2)        # no backprojector registered for OMW
        with pytest.raises(PkError):
            srv.submit(reqs[0][0], 7, "rl", 2)         # unknown PSF id
