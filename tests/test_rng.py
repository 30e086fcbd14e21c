"""The host rand() stream: identical to glibc rand() after srand(seed),
including the polynomial jump-ahead used to skip the F_cw draws."""
import ctypes

import pytest

from baccolonygrowth_b200.colony import Rng

libc = ctypes.CDLL("libc.so.6")


@pytest.mark.parametrize("seed", [1, 0, 12345, 2 ** 31 + 7, 2 ** 32 - 1])
def test_matches_glibc(seed):
    g = Rng(seed)
    libc.srand(ctypes.c_uint(seed))
    assert all(g.next() == libc.rand() for _ in range(5000))


@pytest.mark.parametrize("k", [1, 33, 4095, 4096, 100003, 2_500_001])
def test_skip(k):
    g = Rng(777)
    libc.srand(ctypes.c_uint(777))
    for _ in range(17):
        assert g.next() == libc.rand()
    g.skip(k)
    for _ in range(k):
        libc.rand()
    assert [g.next() for _ in range(50)] == [libc.rand() for _ in range(50)]


def test_frand_matches_float_cast():
    g = Rng(5)
    libc.srand(5)
    vals = g.frand(100)
    import numpy as np
    ref = np.array([np.float32(libc.rand()) / np.float32(2147483647) for _ in range(100)], dtype=np.float32)
    assert np.array_equal(vals, ref)
