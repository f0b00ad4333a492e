"""Serving with continuous batching: each result equals the plain drop-in call's, alone and mixed.

Every scenario runs on both request loops: the host scheduler's rounds of shared pass launches and
the device-resident loop (a dispatcher kernel launching each request's pass graph from the device).
"""
import threading
import time

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


LOOPS = [pytest.param(False, id="host-loop"), pytest.param(True, id="device-loop")]


@pytest.mark.parametrize("device_loop", LOOPS)
def test_served_results_equal_alone_in_the_mix(setup, device_loop):
    psfs, psfs_b, reqs = setup
    with SV.Server(budget_bytes=4e9, max_batch=8, device_loop=device_loop) as srv:
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


@pytest.mark.parametrize("device_loop", LOOPS)
def test_served_tiny_budget_still_completes(setup, device_loop):
    psfs, psfs_b, reqs = setup
    with SV.Server(budget_bytes=1, max_batch=4, device_loop=device_loop) as srv:
        srv.add_psf(0, psfs[0], psfs_b[0])
        ids = [srv.submit(v, 0, "omw", 2, Background=100) for v, _, _, _ in reqs[:4]]
        outs = [srv.wait(r)[0] for r in ids]
        for (v, _, _, _), o in zip(reqs[:4], outs):
            assert np.array_equal(o, _alone(psfs, psfs_b, v, 0, "omw", 2))
        # one request in flight at a time: the peak is one request's buffers
        assert srv.stats()["peak_inflight_bytes"] < 64 * 1024 * 1024


@pytest.mark.parametrize("device_loop", LOOPS)
def test_served_cancel_and_timeout(setup, device_loop):
    psfs, psfs_b, reqs = setup
    with SV.Server(budget_bytes=4e9, max_batch=2, device_loop=device_loop) as srv:
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


def test_device_loop_wait_is_bounded(setup):
    """The dispatcher's waits are bounded.  Idle, it returns after idle_us (exit code 4).  With the
    idle bound out of the way and the scheduler's heartbeat stopped, it returns within heartbeat_ms
    (exit code 3); with the heartbeat back a new instance serves the next request."""
    psfs, psfs_b, reqs = setup
    vol = reqs[0][0]
    ref = _alone(psfs, psfs_b, vol, 0, "omw", 2)       # plain calls before any dispatcher runs
    with SV.Server(budget_bytes=4e9, max_batch=4, device_loop=True, idle_us=2000) as srv:
        srv.add_psf(0, psfs[0], psfs_b[0])
        out, _ = srv.wait(srv.submit(vol, 0, "omw", 2, Background=100))
        assert np.array_equal(out, ref)
        t0 = time.time()
        while srv.loop_status()["running"] and time.time() - t0 < 5.0:
            time.sleep(0.001)
        st = srv.loop_status()
        assert st["running"] == 0 and st["exit_code"] == 4, st
    with SV.Server(budget_bytes=4e9, max_batch=4, device_loop=True, heartbeat_ms=200, idle_us=60_000_000) as srv:
        srv.add_psf(0, psfs[0], psfs_b[0])
        out, _ = srv.wait(srv.submit(vol, 0, "omw", 2, Background=100))
        assert np.array_equal(out, ref)
        st = srv.loop_status()
        assert st["instances"] >= 1 and st["running"] == 1     # waiting for the next request
        srv.pause_heartbeat(True)
        t0 = time.time()
        while srv.loop_status()["running"] and time.time() - t0 < 5.0:
            time.sleep(0.01)
        st = srv.loop_status()
        assert st["running"] == 0 and st["exit_code"] == 3, st
        assert time.time() - t0 < 2.0
        srv.pause_heartbeat(False)
        out, _ = srv.wait(srv.submit(vol, 0, "omw", 2, Background=100))
        assert np.array_equal(out, ref)
        assert srv.loop_status()["instances"] >= 2


def test_device_loop_hands_over_after_its_launch_budget(setup):
    """A dispatcher launches at most 112 request graphs (the device runtime allows 120 fire-and-forget
    launches per launching graph); 130 requests need a second instance, and every one completes."""
    psfs, psfs_b, reqs = setup
    vol = reqs[3][0]                                            # 36 x 36 x 30
    ref = _alone(psfs, psfs_b, vol, 0, "omw", 2)
    with SV.Server(budget_bytes=4e9, max_batch=16, device_loop=True) as srv:
        srv.add_psf(0, psfs[0], psfs_b[0])
        ids = [srv.submit(vol, 0, "omw", 2, Background=100) for _ in range(130)]
        for rid in ids:
            out, _ = srv.wait(rid)
            assert np.array_equal(out, ref)
        st = srv.loop_status()
        assert st["instances"] >= 2
        assert srv.stats()["completed"] == 130


def test_host_loop_has_no_loop_status(setup):
    with SV.Server() as srv:
        with pytest.raises(PkError):
            srv.loop_status()
