"""GPU parity of the sparse lattice product (csc_no_accum) against the
oracle, through the C ABI: keys/pattern bit-exact (explicit zero sums
included), values within 1e-12 * sum|products| per output key."""
import numpy as np
import pytest

import oracle
from conftest import rel_ok
from test_gpu_sort import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def random_lattice(rng, rows, cols, tabs, nnz, dup=False, zero_frac=0.0):
    total = rows * cols * tabs
    if dup:
        keys = np.sort(rng.integers(0, total, nnz, dtype=np.uint64))
    else:
        keys = np.sort(rng.choice(total, size=min(nnz, total), replace=False).astype(np.uint64))
    vals = rng.uniform(-1, 1, keys.size)
    if zero_frac:
        vals[rng.random(keys.size) < zero_frac] = 0.0
    return keys, vals


def check(cuda, torch, ak, av, bk, bv, h, w, wB, d):
    k, v, products = cuda.lattice_mult(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch),
                                       h, w, wB, d)
    ek, ev, ea = oracle.lattice_mult(ak, av, h, w, d, bk, bv, wB, with_abs=True)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    assert rel_ok(to_host(v), ev, ea)
    assert cuda.device_status() == 0
    return products


@pytest.mark.parametrize("h,w,wB,d,na,nb", [
    (100, 10000, 100, 1, 10000, 10000),  # plain contraction 100^3 shape (SPA)
    (30, 40, 20, 5, 300, 300),           # element-wise tabs
    (512, 512, 512, 1, 20000, 20000),
    (1024, 64, 64, 3, 5000, 4000),
    (1, 1, 1, 1, 1, 1),
    (7, 3, 5, 2, 0, 10),
    (7, 3, 5, 2, 10, 0),
])
@pytest.mark.parametrize("zero_frac", [0.0, 0.3])
def test_lattice_mult_spa_shapes(cuda, torch, rng, h, w, wB, d, na, nb, zero_frac):
    ak, av = random_lattice(rng, h, w, d, na, zero_frac=zero_frac)
    bk, bv = random_lattice(rng, w, wB, d, nb, zero_frac=zero_frac)
    check(cuda, torch, ak, av, bk, bv, h, w, wB, d)


@pytest.mark.parametrize("h,w,wB,d,na,nb", [
    (3000, 500, 200, 2, 40000, 40000),           # h beyond the accumulator: ESC
    (5000, 1 << 26, 3, 4, 30000, 30000),          # w*d beyond dense column pointers: binary search
    (20000, 64, 2000, 1, 200000, 100000),         # ~10^6 products, heavy duplicates per output key
])
def test_lattice_mult_esc_shapes(cuda, torch, rng, h, w, wB, d, na, nb):
    ak, av = random_lattice(rng, h, w, d, na)
    bk, bv = random_lattice(rng, w, wB, d, nb)
    check(cuda, torch, ak, av, bk, bv, h, w, wB, d)


def test_lattice_mult_duplicate_keys(cuda, torch, rng):
    """Operands that are not sets: duplicate keys contribute every product."""
    for h in (64, 4096):
        ak, av = random_lattice(rng, h, 50, 2, 3000, dup=True)
        bk, bv = random_lattice(rng, 50, 40, 2, 3000, dup=True)
        check(cuda, torch, ak, av, bk, bv, h, 50, 40, 2)


def test_lattice_mult_bad_dims(cuda, torch):
    import ctypes as C

    import libnt_b200 as L
    z = to_dev(np.zeros(1, np.uint64), torch)
    zv = to_dev(np.zeros(1), torch)
    A = L.Lattice.of(z, zv, 4, 5, 1)
    B = L.Lattice.of(z, zv, 6, 5, 1)  # rows(B) != cols(A)
    b = C.c_size_t(0)
    assert L.lib().lnt_lattice_mult_plan_workspace(C.byref(A), C.byref(B), C.byref(b)) == 2


def test_plain_contraction_mia_level(cuda, torch):
    """c(i,l) = a(i,j,k) * b(k,l,j), dims 100^3, 10^4 distinct coordinates each,
    seed 0, both unsorted: toStraightLattice(A) + toLatticeSort(B) + csc_no_accum."""
    import libnt_b200 as L
    rng = np.random.default_rng(0)
    dims = [100, 100, 100]
    ak = rng.choice(10 ** 6, 10 ** 4, replace=False).astype(np.uint64)
    bk = rng.choice(10 ** 6, 10 ** 4, replace=False).astype(np.uint64)
    av, bv = rng.uniform(-1, 1, 10 ** 4), rng.uniform(-1, 1, 10 ** 4)
    a = oracle.SparseMIA(dims, ak, av, sorted=False)
    b = oracle.SparseMIA(dims, bk, bv, sorted=False)
    c, labels = oracle.product(a.copy(), list("ijk"), b.copy(), list("klj"))
    assert labels == ["i", "l"]
    o = oracle.product_orders(list("ijk"), list("klj"))
    a_seq = o["l_outer"] + o["l_inner"] + o["l_inter"]   # [0,1,2]: straight lattice, default sort
    b_seq = o["r_inner"] + o["r_outer"] + o["r_inter"]   # [2,0,1]
    ka, va = cuda.permute_sort(to_dev(ak, torch), to_dev(av, torch), max_key=10 ** 6,
                               rekey=L.RekeySpec.make(dims, [0, 1, 2], a_seq))
    kb, vb = cuda.permute_sort(to_dev(bk, torch), to_dev(bv, torch), max_key=10 ** 6,
                               rekey=L.RekeySpec.make(dims, [0, 1, 2], b_seq))
    k, v, _ = cuda.lattice_mult(ka, va, kb, vb, 100, 10 ** 4, 100, 1)
    np.testing.assert_array_equal(to_host(k, np.uint64), c.keys)
    np.testing.assert_allclose(to_host(v), c.vals, rtol=0, atol=1e-12)
