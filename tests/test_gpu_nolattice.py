"""GPU parity of products without contracted indices (noLatticeMult, the
reference's SparseMIABase.h:1716-1826) through the C ABI: keys, order and
values bit-exact against the oracle (every output entry is a single product)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from test_gpu_sort import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def operand(rng, outer, d, n, dup=False):
    total = outer * d
    if dup:
        keys = np.sort(rng.integers(0, total, n, dtype=np.uint64))
    else:
        keys = np.sort(rng.choice(total, size=min(n, total), replace=False).astype(np.uint64))
    return keys, rng.uniform(-1, 1, keys.size)


@pytest.mark.parametrize("h,wB,d,na,nb", [
    (5, 4, 6, 12, 10),          # outer x outer per inter index
    (1, 1, 1, 1, 1),
    (1, 1, 5000, 3000, 3000),   # element-wise only
    (300, 200, 1, 250, 150),    # pure outer (one tab)
    (700, 90, 64, 20000, 5000),
    (3, 2000, 4000, 9000, 200000),
    (7, 3, 5, 0, 10),
    (7, 3, 5, 10, 0),
])
@pytest.mark.parametrize("dup", [False, True])
def test_nolattice_mult_matches_oracle(cuda, torch, rng, h, wB, d, na, nb, dup):
    ak, av = operand(rng, h, d, na, dup)
    bk, bv = operand(rng, wB, d, nb, dup)
    k, v = cuda.nolattice_mult(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch), h, wB, d)
    ek, ev = oracle.nolattice_mult(ak, av, h, d, bk, bv, wB)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0


def test_nolattice_mult_bad_dims(cuda, torch):
    import libnt_b200 as L
    z = to_dev(np.zeros(1, np.uint64), torch)
    zv = to_dev(np.zeros(1), torch)
    A = L.Lattice.of(z, zv, 4, 2, 3)  # cols(A) must be 1
    B = L.Lattice.of(z, zv, 2, 5, 3)
    b = C.c_size_t(0)
    assert L.lib().lnt_nolattice_mult_workspace(C.byref(A), C.byref(B), C.byref(b)) == 2
    A = L.Lattice.of(z, zv, 4, 1, 3)
    B = L.Lattice.of(z, zv, 1, 5, 2)  # tab counts differ
    assert L.lib().lnt_nolattice_mult_workspace(C.byref(A), C.byref(B), C.byref(b)) == 2
