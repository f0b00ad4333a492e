"""ctypes binding of libpkdecon.so (the C ABI in include/pkdecon.h).

The library is the product path: there is no CPU fallback.  Importing this module loads the
in-tree ``petakit5d_b200/lib/libpkdecon.so``; if it is missing the import fails with the build
command to run.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

# PK_LIB names another build of the library (the bounds-checked lib/libpkdecon_check.so, for one)
LIB_PATH = os.environ.get("PK_LIB") or os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libpkdecon.so")

PK_OK, PK_ERR_INVALID, PK_ERR_UNSUPPORTED, PK_ERR_CUDA, PK_ERR_NOMEM, PK_ERR_BUSY, PK_ERR_TIMEOUT, \
    PK_ERR_CANCELLED, PK_ERR_EMPTY_OTF_MASK, PK_ERR_INTERNAL = range(10)
PK_U16, PK_F32, PK_F64 = 0, 1, 2

STATUS_NAMES = {0: "ok", 1: "invalid", 2: "unsupported", 3: "cuda", 4: "nomem", 5: "busy", 6: "timeout",
                7: "cancelled", 8: "emptyOTFMask", 9: "internal"}


class PkError(RuntimeError):
    """Error raised by the library; ``.status`` is the pk_status code, ``.identifier`` the
    ``pkdecon:<name>`` identifier a MEX gateway reports."""

    def __init__(self, status, msg):
        self.status = int(status)
        self.identifier = "pkdecon:" + STATUS_NAMES.get(self.status, "unknown")
        super().__init__(f"{self.identifier}: {msg}")


class DeconParams(C.Structure):
    _fields_ = [("background", C.c_double), ("damp_factor", C.c_double), ("scale_factor", C.c_double),
                ("decon_offset", C.c_double), ("edge_erosion", C.c_int32), ("save16bit", C.c_int32),
                ("has_bbox", C.c_int32), ("bbox", C.c_int64 * 6)]


class Chunk(C.Structure):
    _fields_ = [("in_", C.c_void_p), ("dims", C.c_int64 * 3), ("psf_id", C.c_int32), ("has_bbox", C.c_int32),
                ("bbox", C.c_int64 * 6), ("out", C.c_void_p)]


class ServerConfig(C.Structure):
    _fields_ = [("budget_bytes", C.c_int64), ("max_batch", C.c_int32), ("queue_capacity", C.c_int32),
                ("borrow_inputs", C.c_int32), ("device_loop", C.c_int32), ("heartbeat_ms", C.c_int32),
                ("idle_us", C.c_int32)]


I64x3 = C.c_int64 * 3
P = C.c_void_p

_SIGS = {
    "pk_params_default": (None, [C.POINTER(DeconParams)]),
    "pk_ctx_create": (P, [C.c_int]),
    "pk_ctx_destroy": (None, [P]),
    "pk_ctx_reset": (C.c_int, [P]),
    "pk_last_error": (C.c_char_p, []),
    "pk_version": (C.c_char_p, []),
    "pk_ctx_stream": (P, [P]),
    "pk_ctx_kernel_launches": (C.c_int64, [P]),
    "pk_ctx_profile": (C.c_int, [P, C.c_int32]),
    "pk_ctx_profile_read": (C.c_int32, [P, C.c_char_p, C.c_int32]),
    "pk_selftest_device_wait": (C.c_int, [P, C.c_int64]),
    "pk_checked_build": (C.c_int32, []),
    "pk_ctx_tune_read": (C.c_int32, [P, C.c_char_p, C.c_int32]),
    "pk_output_dims": (C.c_int, [I64x3, C.POINTER(DeconParams), I64x3]),
    "pk_decon_lucy": (C.c_int, [P, P, C.c_int, I64x3, P, I64x3, C.c_int32, C.POINTER(DeconParams), P,
                                C.POINTER(C.c_int32)]),
    "pk_decon_lucy_omw": (C.c_int, [P, P, C.c_int, I64x3, P, I64x3, P, I64x3, C.c_int32,
                                    C.POINTER(DeconParams), P]),
    "pk_decon_debug": (C.c_int, [P, C.c_int32, P, C.c_int, I64x3, P, I64x3, P, I64x3, C.c_int32,
                                 C.POINTER(DeconParams), C.c_int32, P, P, C.POINTER(C.c_int32), P]),
    "pk_decon_submit": (C.c_int, [P, C.c_int32, P, C.c_int, I64x3, P, I64x3, P, I64x3, C.c_int32,
                                  C.POINTER(DeconParams), P, C.POINTER(C.c_int64)]),
    "pk_decon_wait": (C.c_int, [P, C.c_int64, C.c_int32]),
    "pk_ctx_join": (C.c_int, [P]),
    "pk_decon_lucy_device": (C.c_int, [P, P, C.c_int, I64x3, P, I64x3, C.c_int32, C.POINTER(DeconParams), P, P]),
    "pk_decon_lucy_omw_device": (C.c_int, [P, P, C.c_int, I64x3, P, I64x3, P, I64x3, C.c_int32,
                                           C.POINTER(DeconParams), P, P]),
    "pk_decon_lucy_omw_noalloc": (C.c_int, [P, C.c_int, I64x3, P, I64x3, P, I64x3, C.c_int32,
                                            C.POINTER(DeconParams), P, P]),
    "pk_psf2otf": (C.c_int, [P, P, I64x3, I64x3, P]),
    "pk_fft3_r2c_device": (C.c_int, [P, P, I64x3, P, P]),
    "pk_fft3_c2r_device": (C.c_int, [P, P, I64x3, P, P]),
    "pk_omw_backprojector": (C.c_int, [P, P, I64x3, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double, P, P, P, P]),
    "pk_wb_backprojector": (C.c_int, [P, P, I64x3, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                      C.POINTER(C.c_double), P, P]),
    "pk_backprojector": (C.c_int, [P, P, I64x3, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                   C.POINTER(C.c_double), P, P]),
    "pk_psf_gen": (C.c_int, [P, P, I64x3, C.c_double, C.c_double, C.c_double, C.c_int32, P, C.c_int64,
                             C.POINTER(C.c_int64)]),
    "pk_deskew_rotate": (C.c_int, [P, P, C.c_int, I64x3, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                   C.c_double, P, C.c_int32, P, C.POINTER(C.c_int64)]),
    "pk_deskew_rotate_device": (C.c_int, [P, P, C.c_int, I64x3, C.c_double, C.c_double, C.c_double, C.c_int32,
                                          C.c_int32, C.c_double, P, C.c_int32, P, C.POINTER(C.c_int64), P]),
    "pk_tiff_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "pk_tiff_read": (C.c_int, [C.c_char_p, P, P, C.c_int64, C.c_int32]),
    "pk_tiff_write": (C.c_int, [C.c_char_p, P, I64x3, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "pk_zarr_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                               C.POINTER(C.c_int32)]),
    "pk_zarr_read": (C.c_int, [C.c_char_p, P, P, C.c_int64, C.c_int32]),
    "pk_zarr_write": (C.c_int, [C.c_char_p, P, I64x3, C.c_int32, C.c_int32, I64x3, C.c_int32, C.c_int32]),
    "pk_zarr_write_region": (C.c_int, [C.c_char_p, P, P, C.c_int32]),
    "pk_host_alloc": (C.c_int, [C.c_int64, C.POINTER(C.c_void_p)]),
    "pk_host_free": (C.c_int, [P]),
    "pk_edge_erosion_edt": (C.c_int, [P, P, C.c_int, I64x3, C.c_int32, P, C.c_int, P]),
    "pk_edgetaper": (C.c_int, [P, P, C.c_int, I64x3, P, P, P]),
    "pk_mask_edge_erosion": (C.c_int, [P, P, C.c_int, I64x3, C.c_int32, P]),
    "pk_find_good_factor_number": (C.c_int64, [C.c_int64, C.c_int32, C.c_int32]),
    "pk_chunk_coordinates": (C.c_int64, [I64x3, I64x3, I64x3, P, C.c_int32, I64x3, P, P, P]),
    "pk_batch_decon": (C.c_int, [P, C.c_int32, C.c_int32, C.POINTER(Chunk), C.c_int, C.c_int32, P, P, P,
                                 C.c_int32, C.POINTER(DeconParams), C.c_int32, C.c_int32]),
    "pk_server_create": (P, [P, C.POINTER(ServerConfig)]),
    "pk_server_add_psf": (C.c_int, [P, C.c_int32, P, P, I64x3]),
    "pk_server_submit": (C.c_int64, [P, P, I64x3, C.c_int32, C.c_int32, C.c_int32, C.POINTER(DeconParams)]),
    "pk_server_wait": (C.c_int, [P, C.c_int64, P, C.c_int32, C.POINTER(C.c_double)]),
    "pk_server_cancel": (C.c_int, [P, C.c_int64]),
    "pk_server_stats": (C.c_int, [P, C.c_int64 * 4]),
    "pk_server_destroy": (None, [P]),
    "pk_server_loop_status": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "pk_server_pause_heartbeat": (C.c_int, [P, C.c_int32]),
}

EXPORTED = tuple(_SIGS)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m petakit5d_b200.build` "
                          "(nvcc, sm_100a); this package has no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error():
    m = lib.pk_last_error()
    return m.decode() if m else ""


def check(status):
    if status != PK_OK:
        raise PkError(status, last_error())


def i64x3(v):
    v = list(v)
    while len(v) < 3:
        v.append(1)
    return I64x3(*[int(x) for x in v[:3]])


def ptr(a):
    """Data pointer of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)


_ctx_lock = threading.Lock()
_ctx = {}


class Context:
    """A pk_ctx bound to one CUDA device (OTF caches, streams and work buffers live here)."""

    def __init__(self, device=0):
        h = lib.pk_ctx_create(int(device))
        if not h:
            raise PkError(PK_ERR_CUDA, last_error())
        self.handle = h
        self.device = device

    @property
    def stream(self):
        return lib.pk_ctx_stream(self.handle)

    @property
    def kernel_launches(self):
        return int(lib.pk_ctx_kernel_launches(self.handle))

    def profile(self, enable=True):
        check(lib.pk_ctx_profile(self.handle, 1 if enable else 0))

    def profile_read(self):
        import json
        cap = 1 << 20
        buf = C.create_string_buffer(cap)
        n = lib.pk_ctx_profile_read(self.handle, buf, cap)
        if n >= cap:
            raise PkError(PK_ERR_INVALID, "profile record larger than the read buffer")
        return json.loads(buf.value.decode())

    def tune_read(self):
        """The autotuner's decisions on this context (a list of dicts)."""
        import json
        cap = 1 << 20
        buf = C.create_string_buffer(cap)
        n = lib.pk_ctx_tune_read(self.handle, buf, cap)
        if n >= cap:
            raise PkError(PK_ERR_INVALID, "tune record larger than the read buffer")
        return json.loads(buf.value.decode())

    def reset(self):
        check(lib.pk_ctx_reset(self.handle))

    def close(self):
        if self.handle:
            lib.pk_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_context(device=0):
    with _ctx_lock:
        c = _ctx.get(device)
        if c is None:
            c = Context(device)
            _ctx[device] = c
        return c
