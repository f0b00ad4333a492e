"""Generate tests/golden/golden.npz from the oracle (run: python tests/golden/make_golden.py).

The reference ships no golden vectors for this path, so these fixtures are the oracle's outputs on
small seeded inputs: they pin the oracle against regressions (tests/test_golden_oracle.py) and give
the GPU tests fixed expected values (tests/test_golden_gpu.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import backprojector as OB  # noqa: E402
from oracle import chunking as OC  # noqa: E402
from oracle import decon as O  # noqa: E402
from petakit5d_b200 import synth  # noqa: E402


def make():
    psf = synth.gaussian_psf((7, 7, 9), 1.3, 2.0)
    psf_b = np.asfortranarray(psf[::-1, ::-1, ::-1])
    vol = synth.puncta_volume((24, 20, 16), 12, psf, seed=2024, background=100.0)
    bpsf = synth.gaussian_psf((19, 19, 25), 1.3, 2.6)
    g = {}
    g["vol"] = vol
    g["psf"] = psf
    g["psf_b"] = psf_b
    g["otf_half"] = O.psf2otf_half(O.normalize_psf(psf, np.float32), vol.shape, np.float32)
    g["omw2_f32"] = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, save16bit=False, dtype=np.float32)
    g["omw2_u16_bbox"] = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, bbox=[3, 2, 4, 20, 18, 13])
    g["rl5_f32"] = O.decon_lucy(vol, psf, 5, background=100, save16bit=False, dtype=np.float32)
    g["rl5_u16_damp_scale"] = O.decon_lucy(vol, psf, 5, background=100, damp=1.5, scale=2.0)
    g["omw2_offset_erosion"] = O.decon_lucy_omw(vol, psf, psf_b, 2, background=100, offset=10.0, edge_erosion=2,
                                                save16bit=False)
    b, omw, absc, mask = OB.omw_backprojector_generation(bpsf, 0.005, False, otf_cum_thresh=0.6)
    g["bpsf"] = bpsf
    g["b_omw"] = b
    g["otf_mask"] = mask.astype(np.uint8)
    g["abs_otf_c"] = absc
    pb, _ = OB.wb_backprojector(bpsf, alpha=0.005, beta=1e-3, n=8, res_flag=1)
    g["wb_psf_bp"] = pb
    g["good_in"] = np.array([1, 7, 31, 41, 101, 352, 416, 544, 1025], np.int64)
    g["good_out"] = np.array([OC.find_good_factor_number(int(n)) for n in g["good_in"]], np.int64)
    bb, rb, lb = OC.zarr_chunk_coordinates((300, 257, 129), (128, 100, 64), (32, 32, 32), None, True, (21, 21, 26))
    g["chunk_batch"], g["chunk_region"], g["chunk_local"] = bb, rb, lb
    return g


if __name__ == "__main__":
    g = make()
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **g)
    print("wrote", os.path.join(HERE, "golden.npz"), sum(v.nbytes for v in g.values()), "bytes")
