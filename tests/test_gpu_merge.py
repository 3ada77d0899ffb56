"""GPU parity of the scan merge (outside_merge_sparse_storage_containers) and
of re-key + sort (sort(seq)) against the oracle, through the C ABI."""
import numpy as np
import pytest

import oracle
from test_gpu_sort import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def sorted_operand(rng, n, hi, dup=False):
    if dup:
        k = np.sort(rng.integers(0, hi, n, dtype=np.uint64))
    else:
        k = np.sort(rng.choice(hi, size=min(n, hi), replace=False).astype(np.uint64))
    return k, rng.uniform(-1, 1, k.size)


@pytest.mark.parametrize("na,nb,hi", [(0, 0, 10), (0, 5, 10), (7, 0, 10), (1, 1, 2), (1000, 1000, 1500),
                                      (2047, 2049, 10 ** 6), (100000, 30000, 200000), (1 << 20, 1 << 20, 1 << 36),
                                      (50000, 50000, 60000)])
@pytest.mark.parametrize("op", [0, 1])
def test_merge_sorted_unique(cuda, torch, rng, na, nb, hi, op):
    ak, av = sorted_operand(rng, na, hi)
    bk, bv = sorted_operand(rng, nb, hi)
    k, v = cuda.merge_sorted(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch), op)
    ek, ev = oracle.merge_sorted(ak, av, bk, bv, op)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)  # one op per output: exact


@pytest.mark.parametrize("na,nb,hi", [(5000, 7000, 100), (20000, 3000, 50), (3000, 3000, 2), (4100, 4100, 1)])
@pytest.mark.parametrize("op", [0, 1])
def test_merge_sorted_with_duplicate_runs(cuda, torch, rng, na, nb, hi, op):
    """Runs of equal keys inside an operand pair positionally (j-th A with j-th B),
    including runs that cross merge tiles."""
    ak, av = sorted_operand(rng, na, hi, dup=True)
    bk, bv = sorted_operand(rng, nb, hi, dup=True)
    k, v = cuda.merge_sorted(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch), op)
    ek, ev = oracle.merge_sorted(ak, av, bk, bv, op)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)


@pytest.mark.parametrize("dims,cur,new", [([512] * 4, [0, 1, 2, 3], [3, 2, 1, 0]),
                                          ([5, 8, 5, 8], [2, 0, 3, 1], [1, 3, 0, 2]),
                                          ([100, 100, 100], [0, 1, 2], [2, 0, 1])])
@pytest.mark.parametrize("n", [10, 2999, 3001, 200000])
def test_permute_sort_bit_exact(cuda, torch, rng, dims, cur, new, n):
    import libnt_b200 as L
    total = int(np.prod(dims))
    keys = rng.integers(0, total, n, dtype=np.uint64)
    vals = rng.standard_normal(n)
    k, v = cuda.permute_sort(to_dev(keys, torch), to_dev(vals, torch), max_key=total,
                             rekey=L.RekeySpec.make(dims, cur, new))
    ek, ev = oracle.sort_pairs(oracle.rekey(keys, dims, cur, new), vals)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)


@pytest.mark.parametrize("a_sorted,b_sorted", [(True, False), (False, True), (True, True)])
@pytest.mark.parametrize("na,nb", [(40000, 40000), (40000, 30000), (30000, 40000)])
def test_scan_merge_mia_level(cuda, torch, rng, a_sorted, b_sorted, na, nb):
    """c(i,j,k,l) = a(i,j,k,l) - b(l,k,j,i) through outside_scanMerge: the operand
    to be re-sorted is chosen by the reference's rule; GPU = permute_sort + merge."""
    import libnt_b200 as L
    dims = [16, 32, 8, 24]
    bdims = dims[::-1]
    total = int(np.prod(dims))
    ak = rng.choice(total, na, replace=False).astype(np.uint64)
    bk = rng.choice(total, nb, replace=False).astype(np.uint64)
    av, bv = rng.uniform(-1, 1, na), rng.uniform(-1, 1, nb)
    a = oracle.SparseMIA(dims, ak, av, sorted=False)
    b = oracle.SparseMIA(bdims, bk, bv, sorted=False)
    if a_sorted:
        a.sort()
    if b_sorted:
        b.sort()
    a0, b0 = a.copy(), b.copy()
    order = [3, 2, 1, 0]
    c = oracle.merge(a, b, order, op=1)
    # GPU: which operand gets sorted into the other's order (SparseMIABase.h:1429-1443)
    if b0.sorted and not a0.sorted or (a0.sorted and b0.sorted and not b0.size < a0.size):
        seq = oracle.reorder_from(oracle.reverse_order(order), b0.seq)
        ka, va = cuda.permute_sort(to_dev(a0.keys, torch), to_dev(a0.vals, torch), max_key=total,
                                   rekey=L.RekeySpec.make(dims, a0.seq, seq))
        kb, vb = to_dev(b0.keys, torch), to_dev(b0.vals, torch)
    else:
        seq = oracle.reorder_from(order, a0.seq)
        kb, vb = cuda.permute_sort(to_dev(b0.keys, torch), to_dev(b0.vals, torch), max_key=total,
                                   rekey=L.RekeySpec.make(bdims, b0.seq, seq))
        ka, va = to_dev(a0.keys, torch), to_dev(a0.vals, torch)
    k, v = cuda.merge_sorted(ka, va, kb, vb, 1)
    np.testing.assert_array_equal(to_host(k, np.uint64), c.keys)
    np.testing.assert_array_equal(to_host(v), c.vals)
