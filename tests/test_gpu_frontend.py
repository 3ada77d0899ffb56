"""GPU: the C++ index-label front end (lnt::SparseNT / DenseNT with lnt::Index
labels) against the oracle's restatement of the reference's expression layer,
including the side effects on the operands (linIdxSequence, sorted flag,
re-keyed / re-sorted storage)."""
import subprocess

import numpy as np
import pytest

import oracle
from frontend_build import build

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def driver(cuda):
    return build()


def write(d, name, m):
    (d / f"{name}.keys").write_bytes(np.ascontiguousarray(m.keys, np.uint64).tobytes())
    (d / f"{name}.vals").write_bytes(np.ascontiguousarray(m.vals, np.float64).tobytes())
    (d / f"{name}.meta").write_text(f"{m.order} {' '.join(map(str, m.dims))} {' '.join(map(str, m.seq))} "
                                    f"{int(m.sorted)}\n")


def read(d, name):
    meta = (d / f"{name}.meta").read_text().split()
    order = int(meta[0])
    dims = [int(x) for x in meta[1:1 + order]]
    seq = [int(x) for x in meta[1 + order:1 + 2 * order]]
    return oracle.SparseMIA(dims, np.frombuffer((d / f"{name}.keys").read_bytes(), np.uint64),
                            np.frombuffer((d / f"{name}.vals").read_bytes(), np.float64), seq,
                            bool(int(meta[1 + 2 * order])))


def run(driver, scenario, d):
    r = subprocess.run([str(driver), scenario, str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr


def same(got, exp, atol=1e-12):
    assert got.dims == exp.dims and got.seq == exp.seq and got.sorted == exp.sorted, \
        (got.dims, exp.dims, got.seq, exp.seq, got.sorted, exp.sorted)
    np.testing.assert_array_equal(got.keys, exp.keys)
    np.testing.assert_allclose(got.vals, exp.vals, rtol=0, atol=atol)


def rand_mia(rng, dims, n, sorted_=False, seq=None, unique=True):
    total = int(np.prod(dims))
    keys = (rng.choice(total, n, replace=False) if unique else rng.integers(0, total, n)).astype(np.uint64)
    m = oracle.SparseMIA(dims, keys, rng.uniform(-1, 1, n), sorted=False)
    if seq is not None:
        m.change_linIdx_sequence(seq)
    if sorted_:
        m.sort()
    return m


@pytest.mark.parametrize("scenario", ["product", "product_assign"])
@pytest.mark.parametrize("n", [2000, 10000])
def test_product(driver, tmp_path, rng, scenario, n):
    """c(i,l) = a(i,j,k) * b(k,l,j) (and c(l,i) = ...): toStraightLattice /
    toLatticeSort side effects on a and b, sorted default-sequence result."""
    a = rand_mia(rng, [100, 30, 40], n)
    b = rand_mia(rng, [40, 50, 30], n, sorted_=(n == 2000))
    write(tmp_path, "a", a)
    write(tmp_path, "b", b)
    run(driver, scenario, tmp_path)
    ea, eb = a.copy(), b.copy()
    c, lab = oracle.product(ea, list("ijk"), eb, list("klj"))
    if scenario == "product_assign":
        c = oracle.assign(list("li"), c, lab)
    same(read(tmp_path, "c"), c)
    same(read(tmp_path, "a_after"), ea, atol=0)
    same(read(tmp_path, "b_after"), eb, atol=0)


def test_elementwise_product(driver, tmp_path, rng):
    a = rand_mia(rng, [30, 20, 6], 800)
    b = rand_mia(rng, [20, 25, 6], 800)
    write(tmp_path, "a", a)
    write(tmp_path, "b", b)
    run(driver, "elementwise", tmp_path)
    c, _ = oracle.product(a.copy(), ["i", "j", "!n"], b.copy(), ["j", "l", "!n"])
    same(read(tmp_path, "c"), c)


def test_elementwise_product_decremented(driver, tmp_path, rng):
    """d(i,l,n) = ~(a(i,j,!n) * b(j,l,!n)): the same entries as the element-wise
    product, assigned to a target whose n is a plain label."""
    a = rand_mia(rng, [30, 20, 6], 800)
    b = rand_mia(rng, [20, 25, 6], 800)
    write(tmp_path, "a", a)
    write(tmp_path, "b", b)
    run(driver, "elementwise_decrement", tmp_path)
    c, _ = oracle.product(a.copy(), ["i", "j", "!n"], b.copy(), ["j", "l", "!n"])
    same(read(tmp_path, "c"), c)


@pytest.mark.parametrize("scenario,a_lab,b_lab,a_dims,b_dims", [
    ("outer_inter", ["i", "!n"], ["!n", "l"], [40, 9], [9, 30]),
    ("outer", ["i", "j"], ["k", "l"], [15, 12], [12, 14]),
])
def test_nolattice_product(driver, tmp_path, rng, scenario, a_lab, b_lab, a_dims, b_dims):
    """d(i,l,!n) = a(i,!n) * b(!n,l) and d(i,j,k,l) = a(i,j) * b(k,l): noLatticeMult,
    with both operands sorted in place under [outer, inter] as side effect."""
    a = rand_mia(rng, a_dims, 150)
    b = rand_mia(rng, b_dims, 120)
    write(tmp_path, "a", a)
    write(tmp_path, "b", b)
    run(driver, scenario, tmp_path)
    ea, eb = a.copy(), b.copy()
    c, _ = oracle.product(ea, a_lab, eb, b_lab)
    same(read(tmp_path, "c"), c, atol=0)
    same(read(tmp_path, "a_after"), ea, atol=0)
    same(read(tmp_path, "b_after"), eb, atol=0)


@pytest.mark.parametrize("scenario,labels,dims,c_labels", [
    ("trace", ["i", "j", "i", "j", "k"], [6, 5, 6, 5, 7], ["k"]),
    ("attract", ["!i", "j", "!i", "k", "j"], [6, 5, 6, 7, 5], ["k", "!i"]),
])
def test_unary_contract_attract(driver, tmp_path, rng, scenario, labels, dims, c_labels):
    """c(k) = a(i,j,i,j,k) and c(k,!i) = a(!i,j,!i,k,j): contract_attract, the
    operand sorted in place under [contract, attract, other], the result's
    sorted flag as push_back leaves it."""
    a = rand_mia(rng, dims, 4000)
    write(tmp_path, "a", a)
    run(driver, scenario, tmp_path)
    ea = a.copy()
    c, lab = oracle.unary(ea, labels)
    assert lab == c_labels
    same(read(tmp_path, "c"), c)
    same(read(tmp_path, "a_after"), ea, atol=0)


@pytest.mark.parametrize("a_state,b_state", [("unsorted", "unsorted"), ("sorted", "unsorted"),
                                             ("unsorted", "sorted"), ("sorted", "sorted"),
                                             ("sorted_other", "unsorted"), ("unsorted", "sorted_other")])
@pytest.mark.parametrize("na,nb", [(5000, 5000), (6000, 4000), (2000, 2500)])
@pytest.mark.parametrize("scenario", ["merge_add", "merge_sub"])
def test_merge_branches(driver, tmp_path, rng, a_state, b_state, na, nb, scenario):
    """c(i,j,k,l) = a(i,j,k,l) +/- b(l,k,j,i) through every branch of
    perform_outside_merge, with the operands' post-states."""
    dims = [12, 10, 14, 9]
    a = rand_mia(rng, dims, na, unique=False)
    b = rand_mia(rng, dims[::-1], nb, unique=False)
    for m, st in ((a, a_state), (b, b_state)):
        if st == "sorted":
            m.collect_duplicates()
        elif st == "sorted_other":
            m.collect_duplicates()
            m.sort([1, 3, 0, 2])
    write(tmp_path, "a", a)
    write(tmp_path, "b", b)
    run(driver, scenario, tmp_path)
    ea, eb = a.copy(), b.copy()
    c = oracle.merge(ea, eb, [3, 2, 1, 0], 0 if scenario == "merge_add" else 1)
    same(read(tmp_path, "c"), c)
    same(read(tmp_path, "a_after"), ea, atol=0)
    same(read(tmp_path, "b_after"), eb, atol=0)


def test_self_merge_and_plus_equals(driver, tmp_path, rng):
    dims = [8, 8, 8, 8]
    a = rand_mia(rng, dims, 1500)
    b = rand_mia(rng, dims, 1500)
    write(tmp_path, "a", a)
    write(tmp_path, "b", b)
    run(driver, "merge_self", tmp_path)
    c = oracle.merge(a.copy(), a.copy(), [3, 2, 1, 0])
    same(read(tmp_path, "c"), c)
    run(driver, "plus_equals", tmp_path)
    c = oracle.merge(a.copy(), b.copy(), [3, 2, 1, 0])
    same(read(tmp_path, "c"), c)


@pytest.mark.parametrize("n,sorted_", [(2000, True), (5000, True), (5000, False)])
def test_sort_seq_and_collect(driver, tmp_path, rng, n, sorted_):
    dims = [9, 11, 7, 13]
    a = rand_mia(rng, dims, n, sorted_=sorted_)
    write(tmp_path, "a", a)
    run(driver, "sort_seq", tmp_path)
    e = a.copy()
    e.sort([2, 0, 3, 1])  # incl. the < 3000 branch that leaves the flag cleared
    same(read(tmp_path, "c"), e, atol=0)
    a2 = rand_mia(rng, dims, n, unique=False)
    a2.vals[rng.random(n) < 0.3] = 0.0
    write(tmp_path, "a", a2)
    run(driver, "collect", tmp_path)
    e2 = a2.copy()
    e2.collect_duplicates()
    same(read(tmp_path, "c"), e2)


@pytest.mark.parametrize("slices", [-1, 0, 7])
def test_dense_product(driver, tmp_path, rng, slices):
    """c(i,j,m,n) = a(i,j,k,l) * b(k,l,m,n) on DenseNT<4>: plain float64 (-1),
    the default emulated scheme II (0) and scheme I slices (7)."""
    d1, d2 = 6, 5
    A = rng.uniform(-1, 1, d1 * d1 * d2 * d2)
    B = rng.uniform(-1, 1, d2 * d2 * d1 * d1)
    (tmp_path / "A.vals").write_bytes(A.tobytes())
    (tmp_path / "B.vals").write_bytes(B.tobytes())
    (tmp_path / "dense.meta").write_text(f"{d1} {d2} {slices}\n")
    run(driver, "dense", tmp_path)
    got = np.frombuffer((tmp_path / "C.vals").read_bytes(), np.float64)
    ref = oracle.dense_lattice_mult(A, B, d1 * d1, d2 * d2, d1 * d1, 1)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13)


@pytest.mark.parametrize("scenario,s_dims,s_lab,d_dims,d_lab,dense_first", [
    ("mixed_sd", [30, 20, 10], ["i", "j", "k"], [20, 10, 40], ["j", "k", "l"], False),
    ("mixed_sd_inter", [30, 20, 6], ["i", "j", "!n"], [20, 40, 6], ["j", "l", "!n"], False),
    ("mixed_ds", [10, 40, 20], ["k", "l", "j"], [30, 20, 10], ["i", "j", "k"], True),
    ("mixed_ds_inter", [40, 20, 6], ["l", "j", "!n"], [30, 20, 6], ["i", "j", "!n"], True),
])
def test_mixed_products(driver, tmp_path, rng, scenario, s_dims, s_lab, d_dims, d_lab, dense_first):
    """c(i,l) = s(i,j,k) * D(j,k,l) and c(i,l) = D(i,j,k) * s(k,l,j) (with and
    without an element-wise index): keys, sequence, sorted flag and values of
    the result, and the sparse operand's post-state, against the oracle."""
    s = rand_mia(rng, s_dims, 1500)
    D = rng.uniform(-1, 1, int(np.prod(d_dims)))
    write(tmp_path, "a", s)
    (tmp_path / "D.vals").write_bytes(D.tobytes())
    (tmp_path / "D.meta").write_text(" ".join(map(str, d_dims)) + "\n")
    run(driver, scenario, tmp_path)
    es = s.copy()
    c, _ = oracle.mixed_product(es, s_lab, D, d_dims, d_lab, dense_first)
    same(read(tmp_path, "c"), c, atol=0)
    same(read(tmp_path, "a_after"), es, atol=0)


def colmajor_permute(x, dims, perm):
    """Mode k of the result is mode perm[k] of x (column-major flat arrays)."""
    return np.ravel(np.asarray(x).reshape(dims, order="F").transpose(perm), order="F")


@pytest.mark.parametrize("slices", [-1, 0, 7])
def test_dense_product_permuted_operands(driver, tmp_path, rng, slices):
    """c(i,j,m,n) = a(k,i,l,j) * b(m,k,n,l): neither operand in lattice order,
    so both go through a permuted copy (latticeCopy) first."""
    d1, d2 = 6, 5
    A = rng.uniform(-1, 1, d2 * d1 * d2 * d1)
    B = rng.uniform(-1, 1, d1 * d2 * d1 * d2)
    (tmp_path / "A.vals").write_bytes(A.tobytes())
    (tmp_path / "B.vals").write_bytes(B.tobytes())
    (tmp_path / "dense.meta").write_text(f"{d1} {d2} {slices}\n")
    run(driver, "dense_perm", tmp_path)
    got = np.frombuffer((tmp_path / "C.vals").read_bytes(), np.float64)
    An = A.reshape([d2, d1, d2, d1], order="F")
    Bn = B.reshape([d1, d2, d1, d2], order="F")
    ref = np.ravel(np.einsum("kilj,mknl->ijmn", An, Bn), order="F")
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13)


@pytest.mark.parametrize("scenario,s_dims,s_lab,d_dims,perm,d_lab,dense_first", [
    # c(i,l) = s(i,j,k) * D(l,k,j): D's lattice order is (j, k, l) = modes [2, 1, 0]
    ("mixed_sd_perm", [30, 20, 10], ["i", "j", "k"], [40, 10, 20], [2, 1, 0], ["j", "k", "l"], False),
    # c(i,l) = D(j,i,k) * s(k,l,j): D's lattice order is (i, j, k) = modes [1, 0, 2]
    ("mixed_ds_perm", [10, 40, 20], ["k", "l", "j"], [20, 30, 10], [1, 0, 2], ["i", "j", "k"], True),
])
def test_mixed_products_permuted_dense(driver, tmp_path, rng, scenario, s_dims, s_lab, d_dims, perm, d_lab,
                                       dense_first):
    """Mixed products whose dense operand is not in lattice order: the result
    equals the product with the dense operand permuted first."""
    s = rand_mia(rng, s_dims, 1500)
    D = rng.uniform(-1, 1, int(np.prod(d_dims)))
    write(tmp_path, "a", s)
    (tmp_path / "D.vals").write_bytes(D.tobytes())
    (tmp_path / "D.meta").write_text(" ".join(map(str, d_dims)) + "\n")
    run(driver, scenario, tmp_path)
    es = s.copy()
    Dp = colmajor_permute(D, d_dims, perm)
    c, _ = oracle.mixed_product(es, s_lab, Dp, [d_dims[q] for q in perm], d_lab, dense_first)
    same(read(tmp_path, "c"), c, atol=0)
    same(read(tmp_path, "a_after"), es, atol=0)


@pytest.mark.parametrize("ascending", [True, False])
def test_push_back(driver, tmp_path, rng, ascending):
    """SparseMIA::push_back: entries kept in push order, the sorted flag
    dropping at the first key below its predecessor; sort(); more entries
    pushed after the storage was read (compared with the last stored key)."""
    dims = [30, 20, 10]
    a = rand_mia(rng, dims, 700)
    if ascending:
        a.keys, a.vals = oracle.sort_pairs(a.keys, a.vals)
    b = rand_mia(rng, dims, 50)
    write(tmp_path, "a", a)
    write(tmp_path, "b", b)
    run(driver, "push_back", tmp_path)
    c = read(tmp_path, "c")
    np.testing.assert_array_equal(c.keys, a.keys)
    np.testing.assert_array_equal(c.vals, a.vals)
    assert c.sorted == bool(np.all(a.keys[1:] >= a.keys[:-1]))
    cs = read(tmp_path, "c_sorted")
    sk, sv = oracle.sort_pairs(a.keys, a.vals)
    np.testing.assert_array_equal(cs.keys, sk)
    np.testing.assert_array_equal(cs.vals, sv)
    assert cs.sorted
    c3 = read(tmp_path, "c3")
    allk = np.concatenate([sk, b.keys])
    np.testing.assert_array_equal(c3.keys, allk)
    np.testing.assert_array_equal(c3.vals, np.concatenate([sv, b.vals]))
    assert c3.sorted == bool(np.all(allk[1:] >= allk[:-1]))


@pytest.mark.parametrize("scenario", ["ternary", "elem_assign", "repeated_elem"])
def test_reference_mult_test_expressions(driver, tmp_path, rng, scenario):
    """Expressions of sparse_mia_mult_test.cpp:123-148: element-wise indices
    assigned to plain labels (matched by identity), '!!' levels, and '~' on a
    product result feeding a further product."""
    a = rand_mia(rng, [5, 8, 5, 8], 900)
    b = rand_mia(rng, [8, 8, 5, 6], 900)
    b2 = rand_mia(rng, [8, 8], 40)
    d2 = rand_mia(rng, [8, 8], 40)
    d = rand_mia(rng, [8], 6)
    for name, m in (("a", a), ("b", b), ("b2", b2), ("d2", d2), ("d", d)):
        write(tmp_path, name, m)
    run(driver, scenario, tmp_path)
    if scenario == "ternary":
        t, lt = oracle.product(a.copy(), ["i", "!j", "k", "!l"], b.copy(), ["!j", "!l", "m", "n"])
        c, lc = oracle.product(t, oracle.decrement(lt, 2), d2.copy(), ["j", "l"])
        c = oracle.assign(["i", "k", "m", "n"], c, lc)
    elif scenario == "elem_assign":
        c, lc = oracle.product(a.copy(), ["i", "!j", "k", "!l"], b2.copy(), ["!j", "!l"])
        c = oracle.assign(["i", "j", "k", "l"], c, lc)
    else:
        t, lt = oracle.product(a.copy(), ["i", "!j", "k", "!!l"], b2.copy(), ["!j", "!!l"])
        c, lc = oracle.product(t, oracle.decrement(lt, 2), d.copy(), ["!l"])
        c = oracle.assign(["i", "j", "k", "l"], c, lc)
    same(read(tmp_path, "c"), c)


def test_dense_assignment_permutes(driver, tmp_path, rng):
    """c(n,m,j,i) = a(i,j,k,l) * b(k,l,m,n): the product's modes (i,j,m,n) are
    permuted into the target's label order."""
    d1, d2 = 6, 5
    A = rng.uniform(-1, 1, d1 * d1 * d2 * d2)
    B = rng.uniform(-1, 1, d2 * d2 * d1 * d1)
    (tmp_path / "A.vals").write_bytes(A.tobytes())
    (tmp_path / "B.vals").write_bytes(B.tobytes())
    (tmp_path / "dense.meta").write_text(f"{d1} {d2} 0\n")
    run(driver, "dense_assign_perm", tmp_path)
    got = np.frombuffer((tmp_path / "C.vals").read_bytes(), np.float64)
    An = A.reshape([d1, d1, d2, d2], order="F")
    Bn = B.reshape([d2, d2, d1, d1], order="F")
    ref = np.ravel(np.einsum("ijkl,klmn->nmji", An, Bn), order="F")
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13)
