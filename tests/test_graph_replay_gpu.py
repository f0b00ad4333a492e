"""A context replays a CUDA graph of a call's launches from the second identical call on; the
replayed calls must give exactly what first calls on fresh contexts give."""
import numpy as np
import pytest

from petakit5d_b200 import _lib
from petakit5d_b200 import decon as D
from petakit5d_b200 import synth

pytestmark = pytest.mark.gpu


def _run(method, vol, psf, psf_b, ctx):
    if method == "omw":
        J, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 2, Background=100, save16bit=False, ctx=ctx)
    else:
        J, _, _ = D.decon_lucy_function(vol, psf, 5, Background=100, save16bit=False, ctx=ctx)
    return J


@pytest.mark.parametrize("method", ["omw", "rl"])
def test_repeated_calls_equal_first_calls(method):
    psf = synth.single_volume_workload("rl_small", seed=1)[1]
    psf_b = np.ascontiguousarray(psf[::-1, ::-1, ::-1])
    vols = [synth.single_volume_workload("rl_small", seed=s)[0] for s in (1, 2, 3, 4)]
    ctx = _lib.Context(0)
    try:
        launches = []
        for v in vols:            # 1st call direct, 2nd captured, 3rd and 4th replayed
            before = ctx.kernel_launches
            got = _run(method, v, psf, psf_b, ctx)
            launches.append(ctx.kernel_launches - before)
            fresh = _lib.Context(0)
            try:
                want = _run(method, v, psf, psf_b, fresh)
            finally:
                fresh.close()
            assert np.array_equal(got, want)
        assert len(set(launches[1:])) == 1      # replays count the same kernels as a direct call
    finally:
        ctx.close()
