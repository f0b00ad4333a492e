"""Served deconvolution with continuous batching (pk_server_* of libpkdecon.so).

    srv = Server(budget_bytes=150e9)
    srv.add_psf(0, psf, psf_b)
    rid = srv.submit(volume_u16, psf_id=0, method="omw", numit=2, Background=100)
    out, latency_ms = srv.wait(rid)

Requests that arrive while others are on the GPU are admitted at the next round as memory frees
up; their passes share launches with the running requests.  With device_loop=True the request loop
is device-resident: a dispatcher kernel launches each admitted request's whole pass program (a
device-launchable graph) from the device as soon as its input is on the GPU.  A result is bitwise
the same as the plain drop-in call's on the same inputs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import PkError, ServerConfig, check, i64x3, lib, ptr
from .decon import _params, _parse


class Server:
    def __init__(self, ctx=None, budget_bytes=150e9, max_batch=64, queue_capacity=1024, borrow_inputs=False,
                 device_loop=False, heartbeat_ms=2000, idle_us=2000):
        """borrow_inputs: read each submitted array in place (keep it alive and unchanged, ideally in
        pinned memory, until wait() returns) instead of copying it at submit.  device_loop: run the
        device-resident request loop (a dispatcher kernel launches each admitted request's pass graph
        from the device) instead of the host scheduler's rounds; heartbeat_ms and idle_us bound the
        dispatcher's waits on the host."""
        self.ctx = ctx or _lib.default_context()
        cfg = ServerConfig(int(budget_bytes), int(max_batch), int(queue_capacity), 1 if borrow_inputs else 0,
                           1 if device_loop else 0, int(heartbeat_ms), int(idle_us))
        self._borrowed = {}
        h = lib.pk_server_create(self.ctx.handle, cfg)
        if not h:
            raise PkError(_lib.PK_ERR_INVALID, _lib.last_error())
        self.handle = h
        self._meta = {}

    def add_psf(self, psf_id, psf_f, psf_b=None):
        pf = np.asfortranarray(np.asarray(psf_f, np.float32))
        pb = None if psf_b is None else np.asfortranarray(np.asarray(psf_b, np.float32))
        if pb is not None and pb.shape != pf.shape:
            raise ValueError("PSF_f and PSF_b must have the same size")
        check(lib.pk_server_add_psf(self.handle, int(psf_id), ptr(pf), ptr(pb), i64x3(pf.shape)))

    def submit(self, vol, psf_id, method="omw", numit=2, **kw):
        v = np.asfortranarray(np.asarray(vol))
        if v.dtype != np.uint16:
            raise TypeError("served requests take uint16 volumes")
        opts, _ = _parse(dict(kw))
        p = _params(opts)
        rid = lib.pk_server_submit(self.handle, ptr(v), i64x3(v.shape), int(psf_id), {"omw": 1, "rl": 0}[method],
                                   int(numit), p)
        if rid < 0:
            raise PkError(-rid, _lib.last_error())
        if self._borrowed is not None:
            self._borrowed[rid] = v            # keep the borrowed buffer alive until wait()
        od = i64x3([0, 0, 0])
        check(lib.pk_output_dims(i64x3(v.shape), p, od))
        self._meta[rid] = (tuple(od), np.uint16 if p.save16bit else np.float32)
        return rid

    def wait(self, rid, timeout_ms=600000, out=None):
        """Wait for request ``rid``; returns (result, latency_ms).  ``out`` (optional) receives the
        result (pinned memory makes the copy faster)."""
        shape, dt = self._meta[rid]
        if out is None:
            out = np.empty(shape, dt, order="F")
        elif out.shape != shape or out.dtype != dt:
            raise ValueError("out has the wrong shape or dtype")
        lat = C.c_double(0)
        st = lib.pk_server_wait(self.handle, int(rid), ptr(out), int(timeout_ms), C.byref(lat))
        if st != _lib.PK_ERR_TIMEOUT:
            self._meta.pop(rid, None)
            self._borrowed.pop(rid, None)
        check(st)
        return out, lat.value

    def cancel(self, rid):
        check(lib.pk_server_cancel(self.handle, int(rid)))

    def loop_status(self):
        """Device loop: {"running", "exit_code" (0 none, 1 stopped, 2 launch budget, 3 heartbeat
        stalled, 4 idle), "instances"}."""
        run, code, inst = C.c_int32(0), C.c_int32(0), C.c_int64(0)
        check(lib.pk_server_loop_status(self.handle, C.byref(run), C.byref(code), C.byref(inst)))
        return {"running": run.value, "exit_code": code.value, "instances": inst.value}

    def pause_heartbeat(self, pause=True):
        """Test hook: stop (or resume) the scheduler's heartbeat that bounds the dispatcher's wait."""
        check(lib.pk_server_pause_heartbeat(self.handle, 1 if pause else 0))

    def stats(self):
        s = (C.c_int64 * 4)()
        check(lib.pk_server_stats(self.handle, s))
        return {"completed": s[0], "rejected": s[1], "peak_inflight_bytes": s[2], "rounds": s[3]}

    def close(self):
        if self.handle:
            lib.pk_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
