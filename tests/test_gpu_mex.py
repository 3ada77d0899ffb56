"""GPU: the mex-format host gateways (include/lnt_mex.h) against the oracle,
with host numpy arrays in the reference's wire formats (int64 keys, 1-based
uint8 orders, [h w d] shapes).  Results allocated through a Python allocator
callback and, once, through malloc (freed with libc's free)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from test_oracle import mixed_case, rowmajor_keys

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(cuda):
    import libnt_b200 as L
    return L.lib()


def ptr(a):
    return a.ctypes.data


def call_out(fn, *args, use_malloc=False):
    """Calls a gateway that allocates its result; returns (keys, vals)."""
    import libnt_b200 as L
    keep = []

    def alloc(nbytes):
        a = np.empty(max(nbytes, 1), np.uint8)
        keep.append(a)
        return a.ctypes.data

    cb = L.HostAlloc() if use_malloc else L.HostAlloc(alloc)
    cv, ck, nc = C.c_void_p(), C.c_void_p(), C.c_size_t()
    st = fn(*args, cb, C.byref(cv), C.byref(ck), C.byref(nc))
    assert st == 0, st
    n = nc.value
    vals = np.array((C.c_double * n).from_address(cv.value)) if n else np.zeros(0)
    keys = np.array((C.c_int64 * n).from_address(ck.value)) if n else np.zeros(0, np.int64)
    if use_malloc:
        libc = C.CDLL(None)
        libc.free.argtypes = [C.c_void_p]
        libc.free(cv)
        libc.free(ck)
    return keys.astype(np.uint64), vals


def test_mex_sort(lib, rng):
    keys = rng.choice(1 << 40, 100_000, replace=False).astype(np.int64)
    vals = rng.uniform(-1, 1, keys.size)
    ek, ev = oracle.sort_pairs(keys.astype(np.uint64), vals)
    assert lib.lnt_mex_sparse_sort(ptr(vals), ptr(keys), keys.size) == 0
    np.testing.assert_array_equal(keys.astype(np.uint64), ek)
    np.testing.assert_array_equal(vals, ev)


@pytest.mark.parametrize("dims,cur,desired", [([30, 40, 50], [1, 2, 3], [3, 1, 2]), ([7, 5, 9, 4], [2, 4, 1, 3], [4, 3, 2, 1])])
def test_mex_change_linidx_and_permute(lib, rng, dims, cur, desired):
    """SparseChangeLinIdxMex then SparsePermuteMex: the toolbox's re-sort of a
    sorted tensor under a new order."""
    total = int(np.prod(dims))
    keys = np.sort(rng.choice(total, min(total, 20_000), replace=False)).astype(np.int64)
    vals = rng.uniform(-1, 1, keys.size)
    c1, d1 = np.array(cur, np.uint8), np.array(desired, np.uint8)
    dm = np.array(dims, np.int64)
    ek = oracle.rekey(keys.astype(np.uint64), dims, [x - 1 for x in cur], [x - 1 for x in desired])
    assert lib.lnt_mex_sparse_change_linidx(ptr(keys), keys.size, len(dims), ptr(c1), ptr(d1), ptr(dm)) == 0
    np.testing.assert_array_equal(keys.astype(np.uint64), ek)
    sk, sv = oracle.sort_pairs(ek, vals)
    assert lib.lnt_mex_sparse_permute(ptr(vals), ptr(keys), keys.size, len(dims), ptr(c1), ptr(d1), ptr(dm)) == 0
    np.testing.assert_array_equal(keys.astype(np.uint64), sk)
    np.testing.assert_array_equal(vals, sv)


@pytest.mark.parametrize("op", [0, 1])
@pytest.mark.parametrize("use_malloc", [False, True])
def test_mex_merge(lib, rng, op, use_malloc):
    ak = np.sort(rng.choice(1 << 30, 50_000, replace=False)).astype(np.int64)
    bk = np.sort(np.concatenate([rng.choice(ak, 20_000, replace=False),
                                 rng.choice(1 << 30, 30_000, replace=False)])).astype(np.int64)
    av, bv = rng.uniform(-1, 1, ak.size), rng.uniform(-1, 1, bk.size)
    k, v = call_out(lib.lnt_mex_sparse_merge, ptr(av), ptr(ak), ak.size, ptr(bv), ptr(bk), bk.size, op,
                    use_malloc=use_malloc)
    ek, ev = oracle.merge_sorted(ak.astype(np.uint64), av, bk.astype(np.uint64), bv, op)
    np.testing.assert_array_equal(k, ek)
    np.testing.assert_array_equal(v, ev)


@pytest.mark.parametrize("alg", [0, 1, 2, 3])
def test_mex_sparselattice_mult(lib, rng, alg):
    """Algorithms 0 (operator*), 1 (csc_times), 2 (DCSC) and 3 (csc_no_accum)
    give the same product and pattern; 1 and 2 are also checked against the
    csc_times restatement."""
    h, w, wB, d = 60, 50, 40, 3
    ak = np.unique(rng.integers(0, h * w * d, 3000)).astype(np.int64)
    bk = np.unique(rng.integers(0, w * wB * d, 2000)).astype(np.int64)
    av, bv = rng.uniform(-1, 1, ak.size), rng.uniform(-1, 1, bk.size)
    ad, bd = np.array([h, w, d], np.int64), np.array([w, wB, d], np.int64)
    k, v = call_out(lib.lnt_mex_sparselattice_mult, ptr(av), ptr(ak), ak.size, ptr(ad), ptr(bv), ptr(bk), bk.size,
                    ptr(bd), alg)
    ek, ev, ea = oracle.lattice_mult(ak.astype(np.uint64), av, h, w, d, bk.astype(np.uint64), bv, wB, with_abs=True)
    np.testing.assert_array_equal(k, ek)
    assert np.all(np.abs(v - ev) <= 1e-12 * ea)
    if alg in (1, 2):
        ck, cv = oracle.csc_times(ak.astype(np.uint64), av, h, w, d, bk.astype(np.uint64), bv, wB)
        np.testing.assert_array_equal(k, ck)
        assert np.all(np.abs(v - cv) <= 1e-12 * ea)


@pytest.mark.parametrize("alg", [4, 5, -1, 6])
def test_mex_sparselattice_mult_unavailable_algorithms(lib, alg):
    """4 and 5 reach the reference's unfinished mtt_times; out-of-range values
    are rejected too: LNT_UNSUPPORTED, nothing allocated or returned."""
    import ctypes as C
    ak = np.array([0, 5], np.int64)
    av = np.array([1.0, 2.0])
    ad = np.array([3, 4, 1], np.int64)
    bd = np.array([4, 2, 1], np.int64)
    cv, ck, nc = C.c_void_p(), C.c_void_p(), C.c_size_t(7)
    import libnt_b200 as L
    st = lib.lnt_mex_sparselattice_mult(ptr(av), ptr(ak), 2, ptr(ad), ptr(av), ptr(ak), 2, ptr(bd), alg,
                                        L.HostAlloc(), C.byref(cv), C.byref(ck), C.byref(nc))
    assert st == 8


@pytest.mark.parametrize("dense_first", [True, False])
def test_mex_sparse_denselattice_mult(lib, rng, dense_first):
    """The reference's mixedlatticemulttests.cpp operands (20 x 20 x 20 x 20),
    the sparse operand passed unsorted, as MATLAB may hold it."""
    m1 = n1 = n2 = p = 20
    A, B = mixed_case(rng, m1, n1, n2, p)
    if dense_first:   # C = A (dense) * S, S = B's non-zeros (n1 x n2 x p)
        sk = rng.permutation(np.flatnonzero(B)).astype(np.int64)
        sv = B[sk]
        sd, dd, D = np.array([n1, n2, p], np.int64), np.array([m1, n1, p], np.int64), A
        oks = np.sort(sk).astype(np.uint64)
        ek, ev = oracle.dense_sparse_mult(A, oks, B[oks.astype(np.int64)], m1, n1, n2, p)
    else:             # C = S * B (dense), S = A's non-zeros (m1 x n1 x p)
        sk = rng.permutation(np.flatnonzero(A)).astype(np.int64)
        sv = A[sk]
        sd, dd, D = np.array([m1, n1, p], np.int64), np.array([n1, n2, p], np.int64), B
        rk = rowmajor_keys(sk, m1, n1)
        order = np.argsort(rk)
        ek, ev = oracle.sparse_dense_mult(rk[order].astype(np.uint64), sv[order], B, m1, n1, n2, p)
    k, v = call_out(lib.lnt_mex_sparse_denselattice_mult, ptr(sv), ptr(sk), sk.size, ptr(sd), ptr(D), ptr(dd),
                    int(dense_first))
    np.testing.assert_array_equal(k, ek)
    np.testing.assert_array_equal(v, ev)


def test_mex_empty_operands(lib, rng):
    """Empty operands: sort / change_linidx / permute are no-ops; merges and
    products return what the non-empty side gives (or nothing)."""
    e64, ef = np.zeros(0, np.int64), np.zeros(0)
    dims = np.array([4, 5], np.int64)
    o12, o21 = np.array([1, 2], np.uint8), np.array([2, 1], np.uint8)
    assert lib.lnt_mex_sparse_sort(ptr(ef), ptr(e64), 0) == 0
    assert lib.lnt_mex_sparse_change_linidx(ptr(e64), 0, 2, ptr(o12), ptr(o21), ptr(dims)) == 0
    assert lib.lnt_mex_sparse_permute(ptr(ef), ptr(e64), 0, 2, ptr(o12), ptr(o21), ptr(dims)) == 0
    bk = np.array([2, 5, 9], np.int64)
    bv = np.array([1.0, -2.0, 3.0])
    for op in (0, 1):
        k, v = call_out(lib.lnt_mex_sparse_merge, ptr(ef), ptr(e64), 0, ptr(bv), ptr(bk), 3, op)
        ek, ev = oracle.merge_sorted(e64.astype(np.uint64), ef, bk.astype(np.uint64), bv, op)
        np.testing.assert_array_equal(k, ek)
        np.testing.assert_array_equal(v, ev)
    k, v = call_out(lib.lnt_mex_sparse_merge, ptr(ef), ptr(e64), 0, ptr(ef), ptr(e64), 0, 0)
    assert k.size == 0
    d3 = np.array([3, 4, 2], np.int64)
    e3 = np.array([4, 5, 2], np.int64)
    k, v = call_out(lib.lnt_mex_sparselattice_mult, ptr(ef), ptr(e64), 0, ptr(d3), ptr(bv), ptr(bk), 3, ptr(e3), 0)
    assert k.size == 0
    B = rng.uniform(-1, 1, 4 * 5 * 2)
    for dense_first, sd, dd in ((0, d3, e3), (1, np.array([5, 6, 2], np.int64), np.array([3, 5, 2], np.int64))):
        k, v = call_out(lib.lnt_mex_sparse_denselattice_mult, ptr(ef), ptr(e64), 0, ptr(sd), ptr(B), ptr(dd),
                        dense_first)
        assert k.size == 0
