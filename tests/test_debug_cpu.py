"""debug = true: the err_mat recurrence of the reference (restated in the oracle) on known inputs, and
the TIFF writer the debug snapshots go through."""
import numpy as np
import pytest

from oracle import decon as O


def test_err_mat_every_iteration():
    # saveStep 1: the stopping measure starts at k = 3 and uses rows k, k-1, k-2
    e = O.err_mat_from_mse([8, 4, 2, 1.5, 1.25], 1, "omw")
    want = np.array([[1, 8, 1, 1], [2, 4, 0.5, 1], [3, 2, 0.25, 0.025], [4, 1.5, 0.1875, 0.00625],
                     [5, 1.25, 0.15625, 0.003125]])
    np.testing.assert_allclose(e, want, rtol=0, atol=1e-15)


def test_err_mat_save_step_two_keeps_the_reference_indexing():
    # saveStep 2: at k = 6 the measure reads rows istp = 3, 2, 1 (step indices used as rows), k = 7
    # repeats row 6's; OMW keeps floor(7/2) = 3 rows, RL keeps istp = 3 rows
    mse = [8, 4, 2, 1.5, 1.25, 1.1, 1.05]
    full = O.err_mat_from_mse(mse, 2, "omw")
    assert full.shape == (3, 4)
    np.testing.assert_allclose(full, [[1, 8, 1, 1], [2, 4, 0.5, 1], [3, 2, 0.25, 1]], atol=1e-15)
    assert O.err_mat_from_mse(mse, 2, "rl").shape == (3, 4)
    e12 = O.err_mat_from_mse(mse + [1.0] * 5, 2, "omw")      # k = 6 row now inside the trim
    assert e12.shape == (6, 4)
    assert e12[5, 3] == pytest.approx(min(abs(0.25 - 0.5) / 10, abs(0.25 + 1 - 2 * 0.5) / 2))


def test_err_mat_rl_without_step_index_fails_like_the_reference():
    with pytest.raises(ValueError):
        O.err_mat_from_mse([4, 2, 1, 0.5, 0.25], 2, "rl")


