"""Asynchronous host-buffer calls (pk_decon_submit / pk_decon_wait): several calls in flight on the
two staging slots give the same results as synchronous calls, bit for bit."""
import numpy as np
import pytest

from petakit5d_b200 import decon as D
from petakit5d_b200 import synth
from petakit5d_b200 import tiff as T
from petakit5d_b200._lib import PkError

pytestmark = pytest.mark.gpu


def test_submitted_calls_match_synchronous_calls():
    psf = synth.gaussian_psf((31, 31, 41))
    vols = [synth.puncta_volume((96, 80, 48), 80, psf, seed=s) for s in range(5)]
    ins = []
    for v in vols:                                   # page-locked inputs and outputs
        h = T.pinned_empty(v.shape, np.uint16)
        h[...] = v
        ins.append(h)
    outs = [T.pinned_empty(v.shape, np.uint16) for v in vols]
    tickets = []
    for k, h in enumerate(ins):
        method = "omw" if k % 2 == 0 else "rl"
        tickets.append(D.decon_submit(method, h, psf, psf if method == "omw" else None, 3, outs[k], Background=100))
    for t in reversed(tickets):                      # collected in any order
        D.decon_wait(t)
    for k, v in enumerate(vols):
        if k % 2 == 0:
            ref, _ = D.decon_lucy_omw_function(v, psf, psf, 3, Background=100)
        else:
            ref = D.decon_lucy_function(v, psf, 3, Background=100)[0]
        np.testing.assert_array_equal(outs[k], ref)


def test_wait_errors_and_timeout():
    psf = synth.gaussian_psf((31, 31, 41))
    v = synth.puncta_volume((64, 64, 48), 40, psf, seed=9)
    out = T.pinned_empty(v.shape, np.uint16)
    t = D.decon_submit("omw", v, psf, psf, 2, out, Background=100)
    try:
        D.decon_wait(t, timeout_ms=0)                # finished already or PK_ERR_TIMEOUT; the ticket stays
    except PkError:
        pass
    D.decon_wait(t)
    with pytest.raises(PkError):
        D.decon_wait(t)                              # already collected
    with pytest.raises(ValueError):
        D.decon_submit("omw", v, psf, psf, 2, np.empty((3, 3, 3), np.uint16), Background=100)
