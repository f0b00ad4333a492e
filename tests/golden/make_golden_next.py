"""Generate tests/golden/golden_next.npz from the oracle (run: python tests/golden/make_golden_next.py).

Fixtures for the rows on either side of the deconvolution (the reference ships no golden vectors for
them either): psf_gen_new on a seeded bead image (both methods, with and without axial resampling),
deskewRotateFrame3D on a seeded volume (direct warp and skewed-space interpolation, uint16 and single),
RLdecon's edge taper (edgetaper with fspecial('gaussian', 35, 5)) and the large-file runner's bwdist
edge erosion.  They pin the oracle against regressions (tests/test_golden_next_oracle.py) and give
the GPU tests fixed expected values (tests/test_golden_next_gpu.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import chunking as OC  # noqa: E402
from oracle import deskew as OD  # noqa: E402
from oracle import edgetaper as OE  # noqa: E402
from oracle import psfgen as OP  # noqa: E402
from petakit5d_b200 import synth  # noqa: E402


def make():
    g = {}
    bead = synth.measured_psf((28, 26, 33), peak=(13, 12, 20), sigma_xy=1.3, sigma_z=3.0, seed=77)
    g["bead"] = bead
    g["psfgen_masked"] = OP.psf_gen_new(bead, 0.1, 0.1, 1.5, OP.MASKED).astype(np.float32)
    g["psfgen_median"] = OP.psf_gen_new(bead, 0.1, 0.1, 1.5, OP.MEDIAN).astype(np.float32)
    g["psfgen_resampled"] = OP.psf_gen_new(bead, 0.1, 0.25, 1.5, OP.MASKED).astype(np.float32)
    rng = np.random.default_rng(78)
    vol = np.asfortranarray((rng.random((24, 40, 22)) * 3000 + 100).astype(np.uint16))
    g["dsr_vol"] = vol
    g["dsr_direct_u16"] = OD.deskew_rotate_frame3d(vol, 32.45, 0.2, 0.108, reverse=True, save16bit=True)
    g["dsr_skewed_u16"] = OD.deskew_rotate_frame3d(vol, 32.45, 0.3, 0.108, reverse=True, save16bit=True)
    g["dsr_skewed_f32"] = OD.deskew_rotate_frame3d(vol.astype(np.float32), 32.45, 0.3, 0.108, reverse=False)
    im = (rng.random((30, 28, 20)) > 0.05).astype(np.uint16) * 7
    g["edt_im"] = im
    g["edt_mask_e4"] = OC.edt_erosion_mask(im, 4).astype(np.uint8)
    tv = np.asfortranarray((rng.random((44, 40, 3)) * 3000 + 100).astype(np.uint16))
    g["taper_vol"] = tv
    g["taper_u16_nt5"] = OE.edgetaper_slices(tv, OE.fspecial_gaussian(35, 5.0))
    return g


if __name__ == "__main__":
    g = make()
    np.savez_compressed(os.path.join(HERE, "golden_next.npz"), **g)
    print("wrote", os.path.join(HERE, "golden_next.npz"), sum(v.nbytes for v in g.values()), "bytes")
