"""Empty, single-element and degenerate operands through the C ABI, as the
reference's containers allow them (an empty SparseMIA sorts, merges and
multiplies to an empty result; SparseMIA.h:628-665, FunctionUtil.h:373-419,
SparseLatticeBase.h:1854-1990).  Results against the oracle."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def to_dev(x, torch):
    x = np.ascontiguousarray(x)
    return torch.from_numpy(x.view(np.int64) if x.dtype == np.uint64 else x).cuda()


def to_host(t, dtype=None):
    a = t.cpu().numpy()
    return a.view(dtype) if dtype is not None else a


def _pairs(rng, n, max_key):
    return rng.integers(0, max_key, n, dtype=np.uint64), rng.uniform(-1, 1, n)


@pytest.mark.parametrize("n", [0, 1, 2, 33])
def test_sort_pairs_tiny(cuda, torch, rng, n):
    k, v = _pairs(rng, n, 1000)
    gk, gv = cuda.sort_pairs(to_dev(k, torch), to_dev(v, torch), max_key=1000)
    ek, ev = oracle.sort_pairs(k, v)
    np.testing.assert_array_equal(to_host(gk, np.uint64), ek)
    np.testing.assert_array_equal(to_host(gv), ev)


@pytest.mark.parametrize("na,nb", [(0, 0), (0, 7), (7, 0), (1, 1), (0, 1)])
def test_sort_reduce_empty_operands(cuda, torch, rng, na, nb):
    """sortMerge with an empty side: the result is the other side sorted and
    folded; both empty gives an empty result."""
    ak, av = _pairs(rng, na, 50)
    bk, bv = _pairs(rng, nb, 50)
    k, v = cuda.sort_reduce(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch), max_key=50)
    sk, sv = oracle.sort_pairs(np.concatenate([ak, bk]), np.concatenate([av, bv]))
    ek, ev = oracle.collect_duplicates(sk, sv)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0


def test_sort_reduce_all_zero_values(cuda, torch):
    """Every addend exactly zero: only the pair at position 0 survives the
    zero-head rule (SparseMIA.h:645-655)."""
    keys = np.array([5, 3, 3, 9, 1, 1, 5], dtype=np.uint64)
    vals = np.zeros(keys.size)
    k, v = cuda.sort_reduce(to_dev(keys, torch), to_dev(vals, torch), max_key=10)
    sk, sv = oracle.sort_pairs(keys, vals)
    ek, ev = oracle.collect_duplicates(sk, sv)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert ek.tolist() == [1]


@pytest.mark.parametrize("na,nb", [(0, 0), (0, 9), (9, 0), (1, 1)])
@pytest.mark.parametrize("op", [0, 1])
def test_merge_sorted_empty_operands(cuda, torch, rng, na, nb, op):
    ak = np.sort(rng.choice(40, na, replace=False).astype(np.uint64))
    bk = np.sort(rng.choice(40, nb, replace=False).astype(np.uint64))
    av, bv = rng.uniform(-1, 1, na), rng.uniform(-1, 1, nb)
    k, v = cuda.merge_sorted(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch), op=op)
    ek, ev = oracle.merge_sorted(ak, av, bk, bv, op)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)


def test_rekey_and_permute_sort_empty(cuda, torch):
    e = to_dev(np.zeros(0, np.uint64), torch)
    ev = to_dev(np.zeros(0), torch)
    assert cuda.rekey(e, [4, 5, 6], [0, 1, 2], [2, 0, 1]).numel() == 0
    k, v = cuda.permute_sort(e, ev, max_key=120)
    assert k.numel() == 0 and v.numel() == 0
    k, v = cuda.collect_duplicates(e, ev)
    assert k.numel() == 0 and v.numel() == 0


@pytest.mark.parametrize("na,nb", [(0, 20), (20, 0), (0, 0), (1, 1)])
def test_lattice_mult_empty_operand(cuda, torch, rng, na, nb):
    """C = A B with an empty A or B is empty (and the product count 0)."""
    h, w, wB = 6, 5, 4
    ak = np.sort(rng.choice(h * w, na, replace=False).astype(np.uint64))
    bk = np.sort(rng.choice(w * wB, nb, replace=False).astype(np.uint64))
    av, bv = rng.uniform(-1, 1, na), rng.uniform(-1, 1, nb)
    k, v, products = cuda.lattice_mult(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch),
                                       h, w, wB, 1)
    ek, ev = oracle.lattice_mult(ak, av, h, w, 1, bk, bv, wB)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_allclose(to_host(v), ev, rtol=0, atol=1e-15)
    if na == 0 or nb == 0:
        assert products == 0 and k.numel() == 0


def test_dense_crt_one_by_one(cuda, torch):
    """The smallest dense product (1 x 1 x 1) and a single row / column."""
    for h, w, wB in [(1, 1, 1), (1, 7, 1), (5, 1, 3)]:
        A = np.arange(1, h * w + 1, dtype=np.float64) * 0.5
        B = np.arange(1, w * wB + 1, dtype=np.float64) * -0.25
        C = to_host(cuda.dense_mult_crt(to_dev(A, torch), to_dev(B, torch), h, w, wB, 1, moduli=13))
        ref = (A.reshape(w, h).T @ B.reshape(wB, w).T).T.ravel()
        np.testing.assert_array_equal(C, ref)
