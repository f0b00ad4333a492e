"""The bounds-checked build (lib/libpkdecon_check.so, -DPK_CHECK) in place of compute-sanitizer:
every checked pass kernel tests the indices of its global-memory accesses and its shared-memory
layout against the launch, records a failure and skips the access (the call returns
PK_ERR_INTERNAL).  Small OMW and RL cases that reach the 1024-point-tile kernels, the
register-packing y kernel, the persistent TMA x/z kernels and the batched path run on it in a
child process (the library is chosen at import); none may trip a check, and the results must
match the oracle.  (A check that fires is not provoked on the GPU: a kernel given out-of-range
indices on purpose is not run; the checks' host side is the same status word as the device waits'
tested in tests/test_device_wait_gpu.py.)"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "petakit5d_b200", "lib", "libpkdecon_check.so")

CHILD = r"""
import numpy as np
from oracle import decon as O
from petakit5d_b200 import _lib, synth
from petakit5d_b200 import decon as D
from petakit5d_b200 import chunking as K
assert _lib.lib.pk_checked_build() == 1
psf = synth.gaussian_psf((15, 15, 21), 1.3, 3.0)
psf_b = np.asfortranarray(psf[::-1, ::-1, ::-1])
worst = 0.0
for shape in [(64, 64, 32), (512, 64, 48), (512, 128, 112), (47, 40, 36)]:
    vol = synth.puncta_volume(shape, 40, psf, seed=7, background=100.0)
    J, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 2, Background=100, save16bit=False)
    ref = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, save16bit=False, dtype=np.float32)
    worst = max(worst, O.rel_l2(J, ref))
    J, _, _ = D.decon_lucy_function(vol, psf, 4, Background=100, save16bit=False)
    ref = O.decon_lucy(vol, psf, 4, background=100, save16bit=False, dtype=np.float32)
    worst = max(worst, O.rel_l2(J, ref))
    J, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 2, Background=100, bbox=[3, 2, 4, 30, 28, 20])
chunks = [synth.puncta_volume(s, 30, psf, seed=i, background=100.0) for i, s in enumerate([(96, 80, 48), (64, 96, 40)])]
outs = K.batch_decon(chunks, [psf], [0, 0], 2, "omw", [psf_b], [None, None], Background=100)
for c, o in zip(chunks, outs):
    ref = O.decon_lucy_omw(c, psf, psf_b, 2, background=100, dtype=np.float32)
    assert int(np.max(np.abs(o.astype(np.int64) - ref.astype(np.int64)))) <= 1
print("worst rel-L2", worst)
assert worst <= 1e-3
"""


def test_checked_build_runs_clean(cuda):
    assert os.path.exists(CHECK_LIB), "build it with `python -m petakit5d_b200.build --check`"
    # PK_TUNE=0: the fallback variants, so the 512x128x112 volume runs the TMA x/z kernels and the
    # smaller ones the register-IO kernels, whatever a timing would pick
    env = dict(os.environ, PK_LIB=CHECK_LIB, PYTHONPATH=ROOT, PK_TUNE="0")
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, cwd=ROOT, capture_output=True, text=True, timeout=600)
    print(r.stdout[-2000:], r.stderr[-4000:])
    assert r.returncode == 0
