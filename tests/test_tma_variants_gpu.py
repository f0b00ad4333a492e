"""Every x / z pass kernel candidate the autotuner may pick gives the same deconvolution.

The autotuner times the register-IO kernel and the persistent TMA variants of a plan and keeps the
fastest (petakit5d_b200/csrc/passes.cu, choose_variant); a variant that is never the fastest on the
test volumes would otherwise go untested.  PK_TMA_VARIANT forces one candidate wherever the plan
has it; the shapes cover the 4096-point tiles and the 16-column, two- and three-buffer variants
of lines of 160..512 points (x: nx, z convolution: nz).  Reference: the register-IO kernels, and the
FP32 oracle restatement of decon_lucy_omw_function.m for one shape.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(64, 288, 416), (64, 416, 288), (64, 224, 160), (64, 512, 256), (64, 352, 224)]


def _run(shape, variant):
    from petakit5d_b200 import _lib
    from petakit5d_b200 import decon as D
    from petakit5d_b200 import synth
    os.environ["PK_TMA_VARIANT"] = str(variant)
    try:
        ctx = _lib.Context(0)
        rng = np.random.default_rng(11)
        vol = np.asfortranarray(rng.integers(90, 3000, size=shape).astype(np.uint16))
        psf = synth.gaussian_psf((15, 15, 21), 1.4, 2.5)
        psf_b = np.asfortranarray(psf[::-1, ::-1, ::-1])
        J, _ = D.decon_lucy_omw_function(vol, psf, psf_b, 2, Background=100, save16bit=False, ctx=ctx)
        tune = ctx.tune_read()
        del ctx
        return J, vol, psf, psf_b, tune
    finally:
        del os.environ["PK_TMA_VARIANT"]


@pytest.mark.parametrize("shape", SHAPES)
def test_tma_variants_match_register_io(shape):
    ref = _run(shape, -1)[0]
    for v in (0, 1, 2):
        J = _run(shape, v)[0]
        err = float(np.linalg.norm((J - ref).ravel()) / np.linalg.norm(ref.ravel()))
        assert err < 1e-6, (shape, v, err)


def test_tma_variant_vs_oracle():
    from oracle import decon as O
    J, vol, psf, psf_b, _ = _run((64, 288, 416), 1)
    R = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, save16bit=False, dtype=np.float32)
    err = float(np.linalg.norm((J - R).ravel()) / np.linalg.norm(R.ravel()))
    assert err < 1e-4, err
