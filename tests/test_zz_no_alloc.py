"""pk_decon_lucy_omw_noalloc: the OMW deconvolution for callers that cannot allocate GPU memory.

Code that runs under another runtime's device-memory manager, or inside an allocation-free section
such as an instrument's acquisition loop, cannot call cudaMalloc.  This entry point takes every work
buffer from an array compiled into the library instead.  These tests call it through the C ABI and
check, on two calls in a row with different volumes, that its output matches the regular
device-pointer entry point's (pk_decon_lucy_omw_device) within the tolerance of the other parity
tests; that a call leaves the device's free memory unchanged; and that a volume larger than the
array's 1,048,576-voxel limit is refused.  The file is named so pytest collects it last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(cuda, shape, seed):
    import torch
    from petakit5d_b200 import synth
    psf = synth.gaussian_psf((15, 15, 21), 1.3, 3.0)
    psf_b = np.asfortranarray(psf[::-1, ::-1, ::-1])
    vol = synth.puncta_volume(shape, 30, psf, seed=seed, background=100.0)
    d_in = torch.from_numpy(np.ascontiguousarray(vol.T).view(np.int16)).to(cuda)
    return vol, psf, psf_b, d_in


def _params(save16bit, bbox=None, damp=1.0, scale=1.0):
    from petakit5d_b200 import _lib
    p = _lib.DeconParams()
    _lib.lib.pk_params_default(p)
    p.background = 100.0
    p.save16bit = 1 if save16bit else 0
    p.damp_factor = damp
    p.scale_factor = scale
    if bbox is not None:
        p.has_bbox = 1
        for i in range(6):
            p.bbox[i] = int(bbox[i])
    return p


def _run(fn_name, vol, psf, psf_b, d_in, save16bit, cuda, **post):
    import torch
    from petakit5d_b200 import _lib
    p = _params(save16bit, **post)
    od = _lib.i64x3([0, 0, 0])
    _lib.check(_lib.lib.pk_output_dims(_lib.i64x3(vol.shape), p, od))
    ny, nx, nz = (int(v) for v in od)
    out = torch.empty((nz, nx, ny), dtype=torch.int16 if save16bit else torch.float32, device=cuda)
    pf = np.asfortranarray(psf, np.float32)
    pb = np.asfortranarray(psf_b, np.float32)
    stream = torch.cuda.current_stream().cuda_stream
    args = (d_in.data_ptr(), _lib.PK_U16, _lib.i64x3(vol.shape), pf.ctypes.data, _lib.i64x3(pf.shape),
            pb.ctypes.data, _lib.i64x3(pb.shape), 2, p, out.data_ptr(), stream)
    if fn_name == "device":
        ctx = _lib.default_context()
        st = _lib.lib.pk_decon_lucy_omw_device(ctx.handle, *args)
    else:
        st = _lib.lib.pk_decon_lucy_omw_noalloc(*args)
    _lib.check(st)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    return (o.view(np.uint16) if save16bit else o).transpose(2, 1, 0)


@pytest.mark.parametrize("save16bit", [False, True])
def test_noalloc_matches_device_entry_point_on_two_calls(cuda, save16bit):
    from oracle import decon as O
    first = _setup(cuda, (64, 64, 32), seed=41)
    second = _setup(cuda, (48, 40, 36), seed=42)   # another size: the shared array is rewritten
    got = [_run("noalloc", *case, save16bit, cuda) for case in (first, second)]
    ref = [_run("device", *case, save16bit, cuda) for case in (first, second)]
    for g, r in zip(got, ref):
        assert g.shape == r.shape
        if save16bit:
            assert int(np.max(np.abs(g.astype(np.int64) - r.astype(np.int64)))) <= 1
        else:
            assert O.rel_l2(g, r) <= 1e-4


@pytest.mark.parametrize("post", [dict(bbox=[3, 5, 2, 40, 33, 30], damp=1.5, scale=2.0), dict(scale=0.5)])
def test_noalloc_post_processing_and_odd_rows(cuda, post):
    """Crop box, damping and scaling (the final pass's post-processing), on an odd-ny volume (no
    real/half-spectrum split table) and an even one, against the device entry point."""
    from oracle import decon as O
    for shape, seed in (((47, 40, 36), 44), ((64, 48, 32), 45)):
        case = _setup(cuda, shape, seed=seed)
        for save16bit in (False, True):
            g = _run("noalloc", *case, save16bit, cuda, **post)
            r = _run("device", *case, save16bit, cuda, **post)
            assert g.shape == r.shape
            if save16bit:
                assert int(np.max(np.abs(g.astype(np.int64) - r.astype(np.int64)))) <= 1
            else:
                assert O.rel_l2(g, r) <= 1e-4


def test_noalloc_call_leaves_free_memory_unchanged(cuda):
    import torch
    case = _setup(cuda, (64, 64, 32), seed=43)
    _run("noalloc", *case, True, cuda)                # warm-up: kernels are loaded on first use
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    _run("noalloc", *case, True, cuda)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_volumes_over_the_limit(cuda):
    import torch
    from petakit5d_b200 import _lib
    ny, nx, nz = 128, 128, 128                       # 2,097,152 voxels > 1,048,576
    d_in = torch.zeros((nz, nx, ny), dtype=torch.int16, device=cuda)
    out = torch.empty_like(d_in)
    psf = np.ones((3, 3, 3), np.float32, order="F")
    st = _lib.lib.pk_decon_lucy_omw_noalloc(d_in.data_ptr(), _lib.PK_U16, _lib.i64x3((ny, nx, nz)), psf.ctypes.data,
                                            _lib.i64x3(psf.shape), psf.ctypes.data, _lib.i64x3(psf.shape), 2,
                                            _params(True), out.data_ptr(), None)
    assert st == _lib.PK_ERR_UNSUPPORTED
    assert "1048576" in _lib.last_error()
    # an extent that would wrap to a small int (2^32 + 16) is refused before any conversion
    st = _lib.lib.pk_decon_lucy_omw_noalloc(d_in.data_ptr(), _lib.PK_U16, _lib.i64x3((2 ** 32 + 16, 1, 1)),
                                            psf.ctypes.data, _lib.i64x3((1, 1, 1)), psf.ctypes.data,
                                            _lib.i64x3((1, 1, 1)), 2, _params(True), out.data_ptr(), None)
    assert st == _lib.PK_ERR_UNSUPPORTED
    # NUMIT = 0 is refused with the unsupported status (the device entry point takes it)
    st = _lib.lib.pk_decon_lucy_omw_noalloc(d_in.data_ptr(), _lib.PK_U16, _lib.i64x3((32, 32, 16)), psf.ctypes.data,
                                            _lib.i64x3(psf.shape), psf.ctypes.data, _lib.i64x3(psf.shape), 0,
                                            _params(True), out.data_ptr(), None)
    assert st == _lib.PK_ERR_UNSUPPORTED
