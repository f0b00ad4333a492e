"""The context's OTF cache must tell apart PSFs that agree on the values its key samples: a PSF that
differs from a cached one anywhere gives the result a fresh context gives."""
import numpy as np
import pytest

from petakit5d_b200 import _lib
from petakit5d_b200 import decon as D
from petakit5d_b200 import synth

pytestmark = pytest.mark.gpu


def test_psf_differing_outside_the_sampled_values_is_not_a_cache_hit():
    vol, psf = synth.single_volume_workload("rl_small", seed=2)
    n = psf.size
    sampled = {(n - 1) * k // 255 for k in range(256)}
    flat = np.asfortranarray(psf, np.float32).ravel(order="F").copy()
    i = next(k for k in range(n // 2, n) if k not in sampled)
    flat[i] *= 1.5                                       # same sampled values, different PSF
    psf2 = flat.reshape(psf.shape, order="F")
    ctx = _lib.Context(0)
    try:
        J1, _, _ = D.decon_lucy_function(vol, psf, 3, Background=100, save16bit=False, ctx=ctx)
        J2, _, _ = D.decon_lucy_function(vol, psf2, 3, Background=100, save16bit=False, ctx=ctx)
        J1b, _, _ = D.decon_lucy_function(vol, psf, 3, Background=100, save16bit=False, ctx=ctx)
    finally:
        ctx.close()
    fresh = _lib.Context(0)
    try:
        W2, _, _ = D.decon_lucy_function(vol, psf2, 3, Background=100, save16bit=False, ctx=fresh)
    finally:
        fresh.close()
    assert np.array_equal(J2, W2)
    assert np.array_equal(J1, J1b)
    assert not np.array_equal(J1, J2)
