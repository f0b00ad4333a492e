"""The fused x-z-x convolution pass (pass_conv3.cuh) against the three separate passes.

Per k-column the fused kernel runs the same radix stages, twiddles and OTF multiply as the
separate TMA x / z passes; the separate passes may run on the register-IO kernels instead (the
autotuner's choice), whose operation order differs in the last bits, so a deconvolution with the
fused pass is compared with one without it (PK_CONV3=0) at rel-L2 1e-6.
Each run is a child process (the kernel table is read once per process).  The shapes cover the
(x, z) length pairs the fused kernel is built for (on volumes large enough for the 4096-point tiles: a
volume whose y pass gives fewer than two waves of CTAs runs the 1024-point-tile kernels, which are not
fused), OMW x2 and RL x6, and the run with the fused
kernel checks that it ran (`xzx_conv` in the per-pass profile).  One shape is also checked against
the FP32 oracle restatement of decon_lucy_omw_function.m.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, sys, numpy as np
from petakit5d_b200 import _lib, decon as D, synth
shape = tuple(json.loads(sys.argv[1])); method = sys.argv[2]; out = sys.argv[3]
rng = np.random.default_rng(5)
vol = np.asfortranarray(rng.integers(90, 3000, size=shape).astype(np.uint16))
psf = synth.gaussian_psf((15, 15, 21), 1.4, 2.5)
psf_b = np.asfortranarray(psf[::-1, ::-1, ::-1])
ctx = _lib.Context(0)
ctx.profile(True)
if method == "omw":
    J, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 2, Background=100, save16bit=False, ctx=ctx)
else:
    J = D.decon_lucy_function(vol, psf, 6, Background=100, save16bit=False, ctx=ctx)[0]
ctx.profile(False)
np.save(out, J)
print(json.dumps(sorted(ctx.profile_read().keys())))
'''


def _run(shape, method, tag, env):
    out = f"/tmp/conv3_{tag}.npy"
    e = dict(os.environ, PYTHONPATH=ROOT, **env)
    r = subprocess.run([sys.executable, "-c", CHILD, json.dumps(list(shape)), method, out], env=e,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out), json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("shape,method", [((64, 512, 256), "omw"), ((40, 256, 512), "omw"), ((64, 512, 512), "omw"),
                                          ((128, 256, 256), "omw"), ((64, 512, 256), "rl"), ((512, 512, 256), "omw")])
def test_fused_convolution_equals_separate_passes(shape, method):
    ref, kinds_ref = _run(shape, method, "sep", {"PK_CONV3": "0"})
    got, kinds = _run(shape, method, "fused", {"PK_CONV3": "1"})
    assert "xzx_conv" in kinds and "xzx_conv" not in kinds_ref, (kinds, kinds_ref)
    err = float(np.linalg.norm((got - ref).ravel()) / np.linalg.norm(ref.ravel()))
    assert err < 1e-6, (err, float(np.abs(got - ref).max()))


def test_fused_convolution_vs_oracle():
    from oracle import decon as O
    shape = (64, 512, 256)
    got, _ = _run(shape, "omw", "oracle", {"PK_CONV3": "1"})
    rng = np.random.default_rng(5)
    vol = np.asfortranarray(rng.integers(90, 3000, size=shape).astype(np.uint16))
    from petakit5d_b200 import synth
    psf = synth.gaussian_psf((15, 15, 21), 1.4, 2.5)
    psf_b = np.asfortranarray(psf[::-1, ::-1, ::-1])
    R = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, save16bit=False, dtype=np.float32)
    err = float(np.linalg.norm((got - R).ravel()) / np.linalg.norm(R.ravel()))
    assert err < 1e-4, err
