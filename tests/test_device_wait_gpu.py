"""Failure detection on the device without a fault: every wait in the persistent pass kernels is
bounded by a deadline, and a wait that runs out is recorded in the context's status word and turned
into PK_ERR_TIMEOUT on the host.  The self-test makes one such wait run out (a barrier that nothing
completes) and checks the status, then that the same context still deconvolves correctly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_device_wait_reports_timeout_and_context_survives(cuda):
    from oracle import decon as O
    from petakit5d_b200 import _lib
    from petakit5d_b200 import decon as D
    from petakit5d_b200 import synth
    ctx = _lib.Context(0)
    st = _lib.lib.pk_selftest_device_wait(ctx.handle, 2_000_000)      # 2 ms
    assert st == _lib.PK_ERR_TIMEOUT
    assert "bounded wait" in _lib.last_error()
    # the status was consumed: the next call on the context runs and is correct
    psf = synth.gaussian_psf((15, 15, 21), 1.3, 3.0)
    vol = synth.puncta_volume((64, 64, 32), 40, psf, seed=9, background=100.0)
    psf_b = np.asfortranarray(psf[::-1, ::-1, ::-1])
    J, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 2, Background=100, save16bit=False, ctx=ctx)
    ref = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, save16bit=False, dtype=np.float32)
    assert O.rel_l2(J, ref) <= 1e-4
    assert _lib.lib.pk_selftest_device_wait(ctx.handle, 10) == _lib.PK_ERR_INVALID   # limit out of range
