"""The oracle's bwdist edge erosion against a brute-force Euclidean distance on a small volume."""
import itertools

import numpy as np

from oracle import chunking as OC


def test_edt_erosion_mask_brute_force():
    rng = np.random.default_rng(0)
    im = (rng.random((9, 8, 7)) > 0.15).astype(np.uint16)
    for E in (1, 2, 3):
        m = im > 0
        m[[0, -1], :, :] = m[:, [0, -1], :] = m[:, :, [0, -1]] = False
        zeros = np.argwhere(~m)
        ref = np.zeros_like(m)
        for v in itertools.product(*[range(s) for s in m.shape]):
            d2 = ((zeros - np.array(v)) ** 2).sum(axis=1).min()
            ref[v] = np.sqrt(d2) > E - 1
        np.testing.assert_array_equal(OC.edt_erosion_mask(im, E), ref)
