"""Bounded device-side waits: an expired wait latches its bit in the device
error word, its kernel returns, and the context stays usable.

No GPU fault, trap or hang is involved: the expiry is reached by a look-back
on a state that nothing publishes (lnt_diag_expired_wait) under a short poll
budget, and by a real multi-tile sort run with a one-poll budget.
"""
import numpy as np
import pytest

import oracle
from test_gpu_sort import to_dev, to_host

pytestmark = pytest.mark.gpu

REDUCE_LOOKBACK_BIT = 1 << 1
SORT_LOOKBACK_BIT = 1 << 0


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


@pytest.fixture
def default_budget(cuda):
    cuda.device_status(clear=True)
    yield
    cuda.set_spin_limit(0)
    cuda.device_status(clear=True)


def _sort_case(n=1 << 22, seed=5):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 1 << 36, n, dtype=np.uint64), rng.uniform(-1, 1, n)


def test_expired_wait_reports_timeout(cuda, torch, default_budget):
    """A look-back on an unpublished state gives up after its budget, latches
    the reduce look-back bit, and later calls still run correctly."""
    import libnt_b200 as L
    cuda.set_spin_limit(1000)
    cuda.diag_expired_wait()
    word = cuda.device_status(clear=False)
    assert word & REDUCE_LOOKBACK_BIT
    st = L.lib().lnt_device_status(0, None, None)
    assert st == 6  # LNT_TIMEOUT
    assert cuda.device_status(clear=True) & REDUCE_LOOKBACK_BIT
    assert cuda.device_status(clear=False) == 0  # cleared
    cuda.set_spin_limit(0)
    keys, vals = _sort_case(1 << 20)
    k, v = cuda.sort_pairs(to_dev(keys, torch), to_dev(vals, torch), max_key=1 << 36)
    ek, ev = oracle.sort_pairs(keys, vals)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0


def test_sort_with_one_poll_budget(cuda, torch, default_budget):
    """A 2^22-pair sort (1024 tiles per digit pass) with a one-poll look-back
    budget: a tile that finds a predecessor unpublished twice gives up with a
    partial prefix, which keeps every write inside the output.  The call
    either latched the sort look-back bit or sorted correctly; with the
    default budget restored the same sort is exact."""
    keys, vals = _sort_case()
    ek, ev = oracle.sort_pairs(keys, vals)
    dk, dv = to_dev(keys, torch), to_dev(vals, torch)
    cuda.set_spin_limit(1)
    for _ in range(3):
        k, v = cuda.sort_pairs(dk, dv, max_key=1 << 36)
        word = cuda.device_status(clear=True)
        if word:
            assert word & SORT_LOOKBACK_BIT and not (word & ~SORT_LOOKBACK_BIT)
        else:
            np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    cuda.set_spin_limit(0)
    k, v = cuda.sort_pairs(dk, dv, max_key=1 << 36)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0
