"""Pins the oracle (CPU restatement) against the reference: its own compiled
kernels (oracle/_ref, when the reference tree was present at build time),
its golden fixtures and its known-answer / property tests.  CPU only."""
import itertools
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference kernels not compiled (no reference tree)")


# ---------------------------------------------------------------------------
# against the reference's own compiled kernels
# ---------------------------------------------------------------------------

@needs_ref
@pytest.mark.parametrize("order", [2, 3, 4, 5, 6, 8])
def test_rekey_matches_reference_kernel(order, rng):
    for trial in range(4):
        dims = [int(x) for x in rng.integers(1, 40 if order < 6 else 9, order)]
        total = int(np.prod(dims))
        keys = rng.integers(0, total, 5000, dtype=np.uint64)
        cur = list(rng.permutation(order))
        new = list(rng.permutation(order))
        np.testing.assert_array_equal(oracle.rekey(keys, dims, cur, new), oracle.ref_rekey(keys, dims, cur, new))


@needs_ref
def test_rekey_512_4_reversal_matches_reference():
    rng = np.random.default_rng(1)
    dims = [512] * 4
    keys = rng.integers(0, 2 ** 36, 200000, dtype=np.uint64)
    got = oracle.rekey(keys, dims, [0, 1, 2, 3], [3, 2, 1, 0])
    np.testing.assert_array_equal(got, oracle.ref_rekey(keys, dims, [0, 1, 2, 3], [3, 2, 1, 0]))


def _multiset_equal_per_key(k1, v1, k2, v2):
    """keys identical; values equal as a multiset within each key run."""
    np.testing.assert_array_equal(k1, k2)
    o1 = np.lexsort((v1, k1))
    o2 = np.lexsort((v2, k2))
    np.testing.assert_array_equal(v1[o1], v2[o2])


@needs_ref
@pytest.mark.parametrize("n,bits", [(0, 8), (1, 8), (49, 10), (50, 10), (2999, 20), (3000, 20), (3001, 36),
                                    (100000, 36), (250000, 22), (70000, 11), (70000, 12)])
def test_sort_matches_reference_radix(n, bits, rng):
    keys = rng.integers(0, 2 ** bits, n, dtype=np.uint64)
    if n > 10:
        keys[: n // 10] = keys[n // 3]  # heavy duplicates
    vals = rng.standard_normal(n)
    k_ref, v_ref = oracle.ref_radix_sort(keys, vals, 2 ** bits)
    k, v = oracle.sort_pairs(keys, vals)
    assert np.all(k[1:] >= k[:-1])
    _multiset_equal_per_key(k, v, k_ref, v_ref)


@needs_ref
def test_introsort_matches_reference(rng):
    keys = rng.integers(0, 1000, 2500, dtype=np.uint64)
    vals = rng.standard_normal(2500)
    k_ref, v_ref = oracle.ref_introsort(keys, vals)
    k, v = oracle.sort_pairs(keys, vals)
    _multiset_equal_per_key(k, v, k_ref, v_ref)


# ---------------------------------------------------------------------------
# the reference's golden fixtures and KATs
# ---------------------------------------------------------------------------

def test_dense_golden_fixture_bit_exact():
    """DenseLattice data/test1.bin x test2.bin == multtest_ddd.bin
    (denselatticemulttests.cpp:19-49)."""
    z = np.load(GOLDEN / "dense_lattice_5x5x10.npz")
    h, w, wB, d = (int(x) for x in z["shape"])
    np.testing.assert_array_equal(oracle.dense_lattice_mult(z["A"], z["B"], h, w, wB, d), z["C"])


def test_dense_closed_form_kat():
    """dense_mia_mult_test.cpp:44-74: a increments 1..dim2^2 along the inner
    modes, b = 1, so every c = dim2^2 (dim2^2 + 1) / 2."""
    dim1, dim2 = 3, 4
    h, w, wB = dim1 * dim1, dim2 * dim2, dim1 * dim1
    # lattice A: rows (i,k), cols (j,l) with value incrementing over (j,l)
    A = np.empty((h, w))
    A[:, :] = np.arange(1, w + 1)[None, :]
    B = np.ones((w, wB))
    Cm = oracle.dense_lattice_mult(A.ravel(order="F"), B.ravel(order="F"), h, w, wB, 1)
    assert np.all(Cm == w * (w + 1) / 2)


def test_collect_duplicates_plus_kat(rng):
    """sparse_mia_functions.cpp:66-92: keys {2,1} then random 1/2 keys with
    value 1; collecting with + gives the two counts."""
    n = 40
    keys = np.empty(n, np.uint64)
    vals = np.ones(n)
    keys[0], keys[1] = 2, 1
    coin = rng.random(n - 2) >= 0.5
    keys[2:] = np.where(coin, 1, 2)
    c1 = 1 + int(coin.sum())
    c2 = 1 + int((~coin).sum())
    k, v = oracle.sort_pairs(keys, vals)
    k, v = oracle.collect_duplicates(k, v)
    np.testing.assert_array_equal(k, [1, 2])
    np.testing.assert_array_equal(v, [c1, c2])


def test_collect_duplicates_zero_quirk():
    """SparseMIA.h:645-655: a run starting with exact zeros starts at its first
    non-zero; all-zero runs vanish except the one at position 0; cancelled
    sums stay."""
    keys = np.array([1, 1, 3, 3, 3, 5, 7, 7, 9], np.uint64)
    vals = np.array([0.0, 0.0, 0.0, 2.0, 0.0, 0.0, 1.5, -1.5, -0.0])
    k, v = oracle.collect_duplicates(keys, vals, skip_zero_heads=True)
    np.testing.assert_array_equal(k, [1, 3, 7])
    np.testing.assert_array_equal(v, [0.0, 2.0, 0.0])
    k, v = oracle.collect_duplicates(keys, vals, skip_zero_heads=False)
    np.testing.assert_array_equal(k, [1, 3, 5, 7, 9])
    np.testing.assert_array_equal(v, [0.0, 2.0, 0.0, 0.0, -0.0])


@pytest.mark.parametrize("seq", [[2, 0, 3, 1], [1, 2, 3, 0], [0, 1, 2, 3], [2, 3, 0, 1]])
def test_sort_seq_equals_rekey_then_sort(seq, rng):
    """sparse_mia_functions.cpp:101-215: sort(seq) on sorted data equals
    change_linIdx_sequence(seq) followed by sort(), element by element."""
    dims = [3, 3, 3, 3]
    total = int(np.prod(dims))
    m = oracle.SparseMIA(dims, rng.integers(0, total, total // 2, dtype=np.uint64), rng.uniform(-5, 5, total // 2),
                         sorted=False)
    m.collect_duplicates()
    m2 = m.copy()
    m.sort(seq)
    m2.change_linIdx_sequence(seq)
    m2.sort()
    np.testing.assert_array_equal(m.keys, m2.keys)
    np.testing.assert_array_equal(m.vals, m2.vals)


# ---------------------------------------------------------------------------
# differential tests (sparse vs dense), as the reference's suites do
# ---------------------------------------------------------------------------

def _random_sparse(rng, dims, density=0.3, ones=False, seq=None, sorted_=False):
    total = int(np.prod(dims))
    dense = rng.uniform(0, 20, dims)
    dense[dense < 20 * (1 - density)] = 0  # reference: randu(0,20), threshold
    if ones:
        dense[dense != 0] = 1.0
    nz = np.flatnonzero(dense.ravel(order="F"))
    m = oracle.SparseMIA(list(dims), nz.astype(np.uint64), dense.ravel(order="F")[nz], sorted=True)
    if seq is not None:
        m.change_linIdx_sequence(seq)
        if sorted_:
            m.sort()
    return m, dense


@pytest.mark.parametrize("a_state,b_state", list(itertools.product(["unsorted", "sorted", "sorted_other"], repeat=2)))
@pytest.mark.parametrize("op", [0, 1])
def test_merge_branches_match_dense(a_state, b_state, op, rng):
    """sparse_mia_add_sub_tests.cpp:23-488 pattern: c(i,j,k,l) = a(i,j,k,l) +/- b(l,k,j,i)
    through the scan and the sort merge branches, against dense arithmetic."""
    dims = [5, 8, 5, 8]
    bd = [dims[3], dims[2], dims[1], dims[0]]
    a, da = _random_sparse(rng, dims)
    b, db = _random_sparse(rng, bd)
    for m, st in ((a, a_state), (b, b_state)):
        if st == "unsorted":
            m.change_linIdx_sequence([2, 0, 3, 1])
        elif st == "sorted_other":
            m.sort([1, 3, 0, 2])
    order = oracle.merge_index_order(list("ijkl"), list("lkji"))
    assert order == [3, 2, 1, 0]
    c = oracle.merge(a, b, order, op)
    expect = da + (1 if op == 0 else -1) * db.transpose(3, 2, 1, 0)
    np.testing.assert_allclose(c.to_dense(), expect, rtol=0, atol=1e-12)
    # the result is key-sorted under its own sequence
    assert np.all(c.keys[1:] > c.keys[:-1])


def test_sort_merge_sequence_rule():
    """sortMerge with |A| == |B| re-keys A to B's order: the result carries
    linIdxSequence {3,2,1,0} for c(i,j,k,l)=a(i,j,k,l)+b(l,k,j,i)."""
    rng = np.random.default_rng(3)
    dims = [4, 5, 6, 7]
    a = oracle.SparseMIA(dims, rng.integers(0, 840, 50, dtype=np.uint64), rng.standard_normal(50), sorted=False)
    b = oracle.SparseMIA(dims[::-1], rng.integers(0, 840, 50, dtype=np.uint64), rng.standard_normal(50),
                         sorted=False)
    c = oracle.merge(a, b, [3, 2, 1, 0])
    assert c.seq == [3, 2, 1, 0] and c.sorted
    # |A| > |B|: B is re-keyed into A's order, C keeps A's default sequence
    a2 = oracle.SparseMIA(dims, rng.integers(0, 840, 60, dtype=np.uint64), rng.standard_normal(60), sorted=False)
    b2 = oracle.SparseMIA(dims[::-1], rng.integers(0, 840, 50, dtype=np.uint64), rng.standard_normal(50),
                          sorted=False)
    c2 = oracle.merge(a2, b2, [3, 2, 1, 0])
    assert c2.seq == [0, 1, 2, 3] and b2.seq == [3, 2, 1, 0] and not b2.sorted


@pytest.mark.parametrize("a_lab,b_lab", [("ijk", "klj"), ("ijk", "jkl"), ("ij", "jk"), ("ikj", "jlk")])
def test_product_matches_dense(a_lab, b_lab, rng):
    """sparse_mia_mult_test.cpp:19-168 pattern: sparse product vs dense einsum."""
    dimmap = {"i": 8, "j": 5, "k": 6, "l": 7}
    a, da = _random_sparse(rng, [dimmap[c] for c in a_lab])
    b, db = _random_sparse(rng, [dimmap[c] for c in b_lab])
    c, c_lab = oracle.product(a, list(a_lab), b, list(b_lab))
    expect = np.einsum(f"{a_lab},{b_lab}->{''.join(c_lab)}", da, db)
    np.testing.assert_allclose(c.to_dense(), expect, rtol=0, atol=1e-10)
    assert np.all(c.keys[1:] > c.keys[:-1])


def test_product_with_elementwise_index(rng):
    """Inter (element-wise '!') index becomes the tab: c(i,l,n) = a(i,j,!n) * b(j,l,!n)."""
    a, da = _random_sparse(rng, [6, 5, 4])
    b, db = _random_sparse(rng, [5, 7, 4])
    c, lab = oracle.product(a, ["i", "j", "!n"], b, ["j", "l", "!n"])
    assert lab == ["i", "l", "!n"]
    np.testing.assert_allclose(c.to_dense(), np.einsum("ijn,jln->iln", da, db), atol=1e-10)


def test_lattice_mult_cross_check_dense(rng):
    """csc_no_accum restatement vs a dense per-tab product on hypersparse
    lattices (sparse_lattice_mult_test_specialized.cpp:16-88 cross-checks)."""
    h, w, wB, d = 30, 40, 20, 5
    for density in (0.01, 0.1, 0.5):
        A = np.where(rng.random((h, w, d)) < density, rng.standard_normal((h, w, d)), 0.0)
        B = np.where(rng.random((w, wB, d)) < density, rng.standard_normal((w, wB, d)), 0.0)
        ak = np.flatnonzero(A.ravel(order="F")).astype(np.uint64)
        bk = np.flatnonzero(B.ravel(order="F")).astype(np.uint64)
        ck, cv = oracle.lattice_mult(ak, A.ravel(order="F")[ak.astype(np.int64)], h, w, d, bk,
                                     B.ravel(order="F")[bk.astype(np.int64)], wB)
        Cd = np.zeros(h * wB * d)
        Cd[ck.astype(np.int64)] = cv
        np.testing.assert_allclose(Cd, np.einsum("rkt,kct->rct", A, B).ravel(order="F"), atol=1e-12)


# ---- noLatticeMult (pure outer / element-wise products) ---------------------

def _sparse_operand(rng, dims, density=0.4):
    dense = np.where(rng.random(dims) < density, rng.uniform(-1, 1, dims), 0.0)
    idx = np.nonzero(dense.reshape(dims, order="F").ravel(order="F"))[0]  # LCO key, first mode fastest
    return dense, idx.astype(np.uint64), dense.ravel(order="F")[idx]


@pytest.mark.parametrize("a_lab,b_lab", [
    (["i", "!k"], ["j", "!k"]),            # outer i, j with element-wise k
    (["i", "j"], ["k", "l"]),              # pure outer
    (["!i", "!j"], ["!i", "!j"]),          # element-wise only
    (["i", "!k", "!m"], ["!m", "j", "!k"]),  # two inter modes, permuted in b
])
def test_nolattice_product_vs_dense(a_lab, b_lab):
    """c = a * b without contracted indices (noLatticeMult, SparseMIABase.h:1716-1826):
    C dims [a outer, b outer, inter], sorted, values = products of the dense operands."""
    rng = np.random.default_rng(5)
    size = {"i": 5, "j": 4, "k": 6, "l": 3, "m": 2}
    a_dims = [size[l.lstrip("!")] for l in a_lab]
    b_dims = [size[l.lstrip("!")] for l in b_lab]
    Ad, ak, av = _sparse_operand(rng, a_dims)
    Bd, bk, bv = _sparse_operand(rng, b_dims)
    a = oracle.SparseMIA(a_dims, ak, av, sorted=False)
    b = oracle.SparseMIA(b_dims, bk, bv, sorted=False)
    c, c_lab = oracle.product(a, list(a_lab), b, list(b_lab))
    assert c.sorted and np.all(np.diff(c.keys.astype(np.int64)) > 0)
    letters = {l.lstrip("!"): chr(ord("a") + n) for n, l in enumerate(sorted(size))}
    sub = lambda labs: "".join(letters[l.lstrip("!")] for l in labs)
    Cd = np.einsum(f"{sub(a_lab)},{sub(b_lab)}->{sub(c_lab)}", Ad, Bd)
    got = np.zeros(int(np.prod(c.dims)))
    got[c.keys.astype(np.int64)] = c.vals
    np.testing.assert_array_equal(got.reshape(c.dims, order="F"), Cd)
    # every pair of non-zeros with equal inter indices is an entry (values are non-zero)
    assert c.keys.size == np.count_nonzero(Cd)
    o = oracle.product_orders(list(a_lab), list(b_lab))
    assert a.seq == o["l_outer"] + o["l_inter"] and b.seq == o["r_outer"] + o["r_inter"]


def test_nolattice_keeps_duplicate_products():
    """Operands that are not sets: every product is its own entry (no fold)."""
    a = oracle.SparseMIA([3, 2], np.array([0, 0, 4], np.uint64), np.array([1.0, 2.0, 3.0]), sorted=False)
    b = oracle.SparseMIA([2, 2], np.array([1, 1], np.uint64), np.array([5.0, 7.0]), sorted=False)
    c, _ = oracle.product(a, ["i", "!k"], b, ["j", "!k"])   # k = 0 for all entries except a key 4 (k = 1)
    np.testing.assert_array_equal(c.keys, np.array([3, 3, 3, 3], np.uint64))
    np.testing.assert_array_equal(c.vals, np.array([5.0, 10.0, 7.0, 14.0]))


# ---- unary contraction / attraction (contract_attract) -----------------------

@pytest.mark.parametrize("labels,sub", [
    (["i", "j", "i", "j", "k"], "ijijk->k"),        # double trace
    (["!i", "j", "!i", "k", "j"], "ijikj->ki"),     # attraction of i, contraction of j
    (["!i", "k", "!i"], "iki->ki"),                  # attraction only (diagonal kept)
])
def test_contract_attract_vs_dense(labels, sub):
    rng = np.random.default_rng(11)
    size = {"i": 4, "j": 3, "k": 5}
    dims = [size[l.lstrip("!")] for l in labels]
    Ad, ak, av = _sparse_operand(rng, dims, density=0.6)
    m = oracle.SparseMIA(dims, ak, av, sorted=False)
    c, lab = oracle.unary(m, labels)
    o = oracle.unary_orders(labels)
    assert lab == o["labels"]
    Cd = np.einsum(sub, Ad)
    got = np.zeros(int(np.prod(c.dims)))
    got[c.keys.astype(np.int64)] = c.vals
    np.testing.assert_allclose(got.reshape(c.dims, order="F"), Cd, rtol=0, atol=1e-12)
    assert c.keys.size == np.count_nonzero(Cd)
    assert m.seq == o["contract"] + o["attract"] + o["other"]          # the operand is sorted in place
    assert c.sorted == bool(np.all(np.diff(c.keys.astype(np.int64)) >= 0))


def test_contract_attract_drops_zero_sums():
    """A group whose diagonal entries cancel exactly is not pushed (if (sum))."""
    m = oracle.SparseMIA([2, 2, 3], np.array([0, 3, 10], np.uint64), np.array([1.0, -1.0, 5.0]), sorted=False)
    c, lab = oracle.unary(m, ["i", "i", "k"])   # k = 0: (0,0,0) and (1,1,0) cancel; (0,1,2) is off the diagonal
    assert lab == ["k"] and c.keys.size == 0


# ---- mixed sparse / dense lattice products ------------------------------------

MIXED_SHAPES = [(20, 20, 20, 20), (1, 20, 1, 20), (20, 1, 20, 20), (20, 20, 20, 1), (20, 1, 1, 20)]


def mixed_case(rng, m1, n1, n2, p):
    """The reference's mixedlatticemulttests.cpp:13-40 set-up: dense lattices
    with entries U[0,10), those below 7 zeroed; the sparse operands hold their
    non-zeros."""
    A = rng.uniform(0, 10, m1 * n1 * p)
    B = rng.uniform(0, 10, n1 * n2 * p)
    A[A < 7] = 0.0
    B[B < 7] = 0.0
    return A, B


def dense_tabs(A, B, m1, n1, n2, p):
    """(p, m1, n2) per-tab products of column-major flat lattices."""
    return np.stack([A.reshape(p, n1, m1)[t].T @ B.reshape(p, n2, n1)[t].T for t in range(p)])


def rowmajor_keys(flat_colmajor_idx, rows, cols):
    r, c, t = flat_colmajor_idx % rows, (flat_colmajor_idx // rows) % cols, flat_colmajor_idx // (rows * cols)
    return c + cols * (r + rows * t)


@pytest.mark.parametrize("m1,n1,n2,p", MIXED_SHAPES)
def test_mixed_products_match_dense(rng, m1, n1, n2, p):
    """mixedlatticemulttests.cpp: sparse x dense and dense x sparse equal the
    dense product (fuzzy); every non-empty line of the sparse operand gives a
    full line of the result, other entries are absent."""
    A, B = mixed_case(rng, m1, n1, n2, p)
    Cd = dense_tabs(A, B, m1, n1, n2, p)
    # dense x sparse: B sparse, column-major keys
    bk = np.flatnonzero(B).astype(np.uint64)
    k, v = oracle.dense_sparse_mult(A, bk, B[bk.astype(np.int64)], m1, n1, n2, p)
    assert np.all(k[1:] > k[:-1])
    expect_cols = np.unique(bk // np.uint64(n1))
    assert k.size == expect_cols.size * m1
    flat = np.transpose(Cd, (0, 2, 1)).reshape(-1)
    np.testing.assert_allclose(v, flat[k.astype(np.int64)], rtol=1e-12, atol=1e-9)
    # sparse x dense: A sparse, row-major keys (col + n1 (row + m1 tab))
    nz = np.flatnonzero(A)
    rk = rowmajor_keys(nz, m1, n1)
    order = np.argsort(rk, kind="stable")
    k2, v2 = oracle.sparse_dense_mult(rk[order].astype(np.uint64), A[nz][order], B, m1, n1, n2, p)
    assert np.all(k2[1:] > k2[:-1])
    assert k2.size == np.unique(rk // n1).size * n2
    np.testing.assert_allclose(v2, Cd.reshape(-1)[k2.astype(np.int64)], rtol=1e-12, atol=1e-9)


def test_mixed_products_keep_zero_lines():
    """A line of the sparse operand whose products cancel still gives a full
    line of exact zeros (the reference writes every entry of the line)."""
    A = np.array([1.0, 2.0, 1.0, 2.0])              # 2 x 2 x 1: A(:,0) = A(:,1) = (1, 2)
    bk = np.array([0, 1], np.uint64)                # S(0,0) = 3, S(1,0) = -3 (2 x 1 x 1)
    k, v = oracle.dense_sparse_mult(A, bk, np.array([3.0, -3.0]), 2, 2, 1, 1)
    np.testing.assert_array_equal(k, np.array([0, 1], np.uint64))
    np.testing.assert_array_equal(v, np.array([0.0, 0.0]))


@pytest.mark.parametrize("s_dims,s_lab,d_dims,d_lab,dense_first,sub", [
    ([6, 5, 4], ["i", "j", "k"], [5, 4, 7], ["j", "k", "l"], False, "ijk,jkl->il"),
    ([6, 5, 3], ["i", "j", "!n"], [5, 7, 3], ["j", "l", "!n"], False, "ijn,jln->iln"),
    ([4, 7, 5], ["k", "l", "j"], [6, 5, 4], ["i", "j", "k"], True, "ijk,klj->il"),
    ([7, 5, 3], ["l", "j", "!n"], [6, 5, 3], ["i", "j", "!n"], True, "ijn,ljn->iln"),
])
def test_mixed_product_vs_dense(rng, s_dims, s_lab, d_dims, d_lab, dense_first, sub):
    """MIA-level mixed products against einsum: values of the kept lines, every
    other entry of the dense result zero; the sorted flag per side."""
    total = int(np.prod(s_dims))
    keys = rng.choice(total, 40, replace=False).astype(np.uint64)
    s = oracle.SparseMIA(s_dims, keys, rng.uniform(-1, 1, 40), sorted=False)
    D = rng.uniform(-1, 1, int(np.prod(d_dims)))
    Sd = np.zeros(total)
    Sd[keys.astype(np.int64)] = s.vals
    Sd = Sd.reshape(s_dims[::-1]).transpose()          # column-major: first mode fastest
    Dd = D.reshape(d_dims[::-1]).transpose()
    Cd = np.einsum(sub, Dd, Sd) if dense_first else np.einsum(sub, Sd, Dd)
    c, labels = oracle.mixed_product(s.copy(), s_lab, D, d_dims, d_lab, dense_first)
    assert c.seq == list(range(c.order)) and c.sorted == dense_first
    flat = Cd.transpose().reshape(-1)
    np.testing.assert_allclose(c.vals, flat[c.keys.astype(np.int64)], rtol=1e-12, atol=1e-12)
    rest = np.ones(flat.size, bool)
    rest[c.keys.astype(np.int64)] = False
    assert np.all(flat[rest] == 0.0)



@pytest.mark.parametrize("m1,n1,n2,p,hyper", [(20, 20, 20, 20, 1.0), (20, 20, 20, 20, 0.5), (40, 20, 20, 20, 1.0),
                                              (20, 20, 40, 20, 0.5)])
def test_lattice_product_second_oracles(rng, m1, n1, n2, p, hyper):
    """sparse_lattice_mult_test_specialized.cpp:13-53: the product by
    csc_no_accum (the oracle's restatement), csc_times and outer_times agree
    on random lattices of ceil(p m1 hyper) / ceil(p n2 hyper) entries with
    values U[1,10), duplicates collected: same keys, values within 1e-12."""
    na, nb = int(np.ceil(p * m1 * hyper)), int(np.ceil(p * n2 * hyper))
    ak = np.unique(rng.integers(0, m1 * n1 * p, na).astype(np.uint64))
    bk = np.unique(rng.integers(0, n1 * n2 * p, nb).astype(np.uint64))
    av, bv = rng.uniform(1, 10, ak.size), rng.uniform(1, 10, bk.size)
    ck, cv, ca = oracle.lattice_mult(ak, av, m1, n1, p, bk, bv, n2, with_abs=True)
    for k2, v2 in (oracle.csc_times(ak, av, m1, n1, p, bk, bv, n2), oracle.outer_times(ak, av, m1, n1, p, bk, bv, n2)):
        np.testing.assert_array_equal(k2, ck)
        assert np.all(np.abs(v2 - cv) <= 1e-12 * ca)


def _sparse_of(dense):
    """SparseMIA of a dense array's non-zeros (default sequence, column-major keys)."""
    flat = np.ravel(dense, order="F")
    keys = np.flatnonzero(flat).astype(np.uint64)
    return oracle.SparseMIA(list(dense.shape), keys, flat[keys.astype(np.int64)], sorted=True)


def _dense_of(m):
    keys = oracle.rekey(m.keys, m.dims, m.seq, list(range(m.order))) if m.seq != list(range(m.order)) else m.keys
    flat = np.zeros(int(np.prod(m.dims)))
    np.add.at(flat, keys.astype(np.int64), m.vals)
    return flat.reshape(m.dims, order="F")


def _thresholded(rng, shape):
    """The reference tests' differential data: randu(0,20), entries below 15 set to 0."""
    x = rng.uniform(0, 20, shape)
    x[x < 15] = 0.0
    return x


def test_reference_mult_test_expressions_vs_dense(rng):
    """sparse_mia_mult_test.cpp:123-148 at the oracle: element-wise results
    assigned to plain labels (matched by identity), '~' decrementing the inter
    labels of a product result, '!!' levels; against einsum on the dense data."""
    A = _thresholded(rng, (5, 8, 5, 8))
    B = _thresholded(rng, (8, 8, 5, 6))
    B2 = _thresholded(rng, (8, 8))
    D2 = _thresholded(rng, (8, 8))
    D = _thresholded(rng, (8,))
    a, b, b2, d2, d = map(_sparse_of, (A, B, B2, D2, D))
    # c(i,j,k,l) = a(i,!j,k,!l) * b2(!j,!l)
    c, lc = oracle.product(a.copy(), ["i", "!j", "k", "!l"], b2.copy(), ["!j", "!l"])
    c = oracle.assign(["i", "j", "k", "l"], c, lc)
    np.testing.assert_allclose(_dense_of(c), np.einsum("ijkl,jl->ijkl", A, B2), rtol=1e-12)
    # c(i,k,m,n) = ~(a(i,!j,k,!l) * b(!j,!l,m,n)) * d2(j,l)
    t, lt = oracle.product(a.copy(), ["i", "!j", "k", "!l"], b.copy(), ["!j", "!l", "m", "n"])
    assert lt == ["i", "k", "m", "n", "!j", "!l"]
    c, lc = oracle.product(t, oracle.decrement(lt, 2), d2.copy(), ["j", "l"])
    c = oracle.assign(["i", "k", "m", "n"], c, lc)
    np.testing.assert_allclose(_dense_of(c), np.einsum("ijkl,jlmn,jl->ikmn", A, B, D2), rtol=1e-12)
    # c(i,j,k,l) = ~(a(i,!j,k,!!l) * b2(!j,!!l)) * d(!l)
    t, lt = oracle.product(a.copy(), ["i", "!j", "k", "!!l"], b2.copy(), ["!j", "!!l"])
    c, lc = oracle.product(t, oracle.decrement(lt, 2), d.copy(), ["!l"])
    assert lc == ["i", "k", "j", "!l"]
    c = oracle.assign(["i", "j", "k", "l"], c, lc)
    np.testing.assert_allclose(_dense_of(c), np.einsum("ijkl,jl,l->ijkl", A, B2, D), rtol=1e-12)
