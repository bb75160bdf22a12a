"""Rate (Poisson) coding on CPU: the library's inter-spike interval table
against the reference's (cpu/init.cpp:120-149, compiled in oracle/_ref), row
by row as multisets (the reference shuffles each row with std::random_shuffle,
whose order is implementation-defined); the NumPy-free port restatements of
rate fire / gather / pool against the reference build."""

import ctypes

import numpy as np
import pytest

from spyker_b200 import _lib


@pytest.mark.parametrize("time", [1, 2, 15, 30, 64, 100])
def test_interval_table_rows_are_the_reference_multisets(ref, time):
    got = np.zeros((time, 1024), dtype=np.uint16)
    _lib.lib.spk_rate_interval_table(time, got.ctypes.data_as(ctypes.c_void_p))
    want = ref.poisson_table(time)
    assert np.array_equal(np.sort(got, axis=1), np.sort(want, axis=1))
    assert got.min() >= 1


def test_port_rate_ops_match_reference(port, ref):
    rng = np.random.default_rng(4)
    pot = np.cumsum(rng.random((3, 9, 2, 5, 6)).astype(np.float32), axis=1)
    for dt in (np.uint8, np.float32):
        assert np.array_equal(port.rate_fire(pot, 0.4, dt), ref.rate_fire(pot, 0.4, dt))
    counts = ref.rate_fire(pot, 0.4, np.float32)
    assert np.array_equal(port.rate_gather(counts, np.float32), ref.rate_gather(counts, np.float32))
    rates = rng.integers(0, 4, size=(3, 2, 5, 6)).astype(np.float32)  # ties
    for k, st in (((2, 2), (2, 2)), ((3, 2), (1, 2))):
        assert np.array_equal(port.rate_pool(counts, rates, k, st), ref.rate_pool(counts, rates, k, st))
