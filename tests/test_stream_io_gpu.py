"""Host-buffer calls stream their copies by z-slab (first passes behind the upload, download behind
the last passes); their results must equal the device-pointer call on the same input, bit for bit,
including uneven slabs, both methods, float and uint16 output and the offset mask."""
import numpy as np
import pytest
import torch

from petakit5d_b200 import _lib
from petakit5d_b200 import decon as D
from petakit5d_b200 import synth

pytestmark = pytest.mark.gpu


def _device_call(method, vol, psf, psf_b, numit, ctx, **kw):
    dev = torch.device("cuda", 0)
    d_in = torch.from_numpy(np.ascontiguousarray(vol.T).view(np.int16)).to(dev)
    save16 = kw.get("save16bit", True)
    d_out = torch.empty(vol.T.shape, dtype=torch.int16 if save16 else torch.float32, device=dev)
    D.decon_device(method, d_in, "uint16", vol.shape, psf, psf_b, numit, out=d_out, ctx=ctx, **kw)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy()
    return (out.view(np.uint16) if save16 else out).T


@pytest.mark.parametrize("method,numit,kw", [
    ("omw", 2, {"Background": 100, "save16bit": True}),
    ("omw", 1, {"Background": 100, "save16bit": False, "deconOffset": 5.0}),
    ("rl", 3, {"Background": 100, "save16bit": False}),
])
def test_streamed_host_call_equals_device_call(method, numit, kw):
    vol, psf = synth.single_volume_workload("rl_small", seed=5)
    vol = np.asfortranarray(vol[:, :96, :61])          # nz = 61: slabs of uneven depth
    psf_b = np.ascontiguousarray(psf[::-1, ::-1, ::-1])
    ctx = _lib.Context(0)
    try:
        if method == "omw":
            got, _ = D.decon_lucy_omw_function(vol, psf, psf_b, numit, ctx=ctx, **kw)
        else:
            got, _, _ = D.decon_lucy_function(vol, psf, numit, ctx=ctx, **kw)
        want = _device_call(method, vol, psf, psf_b if method == "omw" else None, numit, ctx, **kw)
        assert got.shape == want.shape
        assert np.array_equal(got, want)
    finally:
        ctx.close()
