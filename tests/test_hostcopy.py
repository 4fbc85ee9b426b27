"""The threaded host copy used for large results (CPU only)."""
import numpy as np

from eemd4cuda_b200 import hostcopy as H


def test_fresh_copy_small_and_large():
    rng = np.random.default_rng(0)
    for shape in [(0,), (5,), (3, 7), (11, (H.PARALLEL_BYTES // 8) // 11 + 13)]:
        a = rng.standard_normal(shape)
        b = H.fresh_copy(a)
        assert b.shape == a.shape and b.dtype == a.dtype
        assert np.array_equal(a, b)
        assert not np.shares_memory(a, b)


def test_fresh_copy_non_contiguous():
    a = np.arange(4 * (H.PARALLEL_BYTES // 8), dtype=np.float64).reshape(4, -1)[:, ::2]
    b = H.fresh_copy(a)
    assert np.array_equal(a, b) and b.flags.c_contiguous
