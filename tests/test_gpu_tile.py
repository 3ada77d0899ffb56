"""GPU parity of the tile engine of the sparse lattice product (dense or
nearly dense outputs) against the oracle's csc_no_accum, through the C ABI:
keys/pattern bit-exact, values within 1e-12 * sum|products| per output key."""
import numpy as np
import pytest

import oracle
from test_gpu_spgemm import check, random_lattice

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


@pytest.fixture
def force_tile(monkeypatch):
    monkeypatch.setenv("LNT_SPGEMM_ENGINE", "tile")


def zipf_coords(rng, n, dim, s=1.1):
    """Rank r (1-based) with probability ~ r^-s, truncated to dim ranks; rank r -> coordinate r - 1."""
    p = np.arange(1, dim + 1, dtype=np.float64) ** -s
    return rng.choice(dim, size=n, p=p / p.sum())


def skewed_operands(rng, di, dj, dk, dl, dm, na, nb):
    """a(i,j,k,l) and b(k,l,m) with Zipf (k,l) aligned in both, the other modes
    uniform, duplicate coordinates collapsed; returned as key-sorted lattices
    A (rows (i,j), cols (k,l)) and B (rows (k,l), cols m)."""
    i, j = rng.integers(0, di, na), rng.integers(0, dj, na)
    k, l = zipf_coords(rng, na, dk), zipf_coords(rng, na, dl)
    ak = np.unique((i + di * j) + (di * dj) * (k + dk * l).astype(np.int64)).astype(np.uint64)
    kb, lb, m = zipf_coords(rng, nb, dk), zipf_coords(rng, nb, dl), rng.integers(0, dm, nb)
    bk = np.unique((kb + dk * lb) + (dk * dl) * m.astype(np.int64)).astype(np.uint64)
    return ak, rng.standard_normal(ak.size), bk, rng.standard_normal(bk.size)


@pytest.mark.parametrize("dm", [64, 300, 1000])
def test_skewed_contraction_selects_tile(cuda, torch, rng, dm):
    """c(i,j,m) = a(i,j,k,l) * b(k,l,m) at reduced sizes: dims 64x32x16x16 and
    16x16xdm; the default engine choice takes the tile engine here."""
    import libnt_b200 as L
    ak, av, bk, bv = skewed_operands(rng, 64, 32, 16, 16, dm, 1 << 15, 1 << 14)
    L.profile_enable(True)
    L.profile_reset()
    try:
        check(cuda, torch, ak, av, bk, bv, 64 * 32, 256, dm, 1)
        assert L.profile_query("tile_numeric")[1] > 0
    finally:
        L.profile_enable(False)


@pytest.mark.parametrize("h,w,wB,d,na,nb", [
    (100, 10000, 100, 1, 10000, 10000),
    (30, 40, 20, 5, 300, 300),
    (512, 512, 512, 1, 20000, 20000),
    (1024, 64, 64, 3, 5000, 4000),
    (1, 1, 1, 1, 1, 1),
    (7, 3, 5, 2, 0, 10),
    (7, 3, 5, 2, 10, 0),
    (3000, 500, 200, 2, 40000, 40000),
    (20000, 64, 2000, 1, 200000, 100000),
    (129, 17, 65, 3, 2000, 1000),     # partial panel and partial tile
])
@pytest.mark.parametrize("zero_frac", [0.0, 0.3])
def test_tile_engine_shapes(cuda, torch, rng, force_tile, h, w, wB, d, na, nb, zero_frac):
    ak, av = random_lattice(rng, h, w, d, na, zero_frac=zero_frac)
    bk, bv = random_lattice(rng, w, wB, d, nb, zero_frac=zero_frac)
    check(cuda, torch, ak, av, bk, bv, h, w, wB, d)


def test_tile_engine_dense_and_sparse_rows(cuda, torch, rng, force_tile, monkeypatch):
    """B rows on both sides of a dense-row threshold of a quarter of the
    columns (LNT_TILE_DENSE_DIV=4): full rows, rows at the threshold, just below
    it, single-entry rows, empty rows."""
    monkeypatch.setenv("LNT_TILE_DENSE_DIV", "4")
    h, w, wB = 700, 40, 257
    rows = []
    for c in range(w):
        n = {0: wB, 1: (wB + 3) // 4, 2: (wB + 3) // 4 - 1, 3: 1, 4: 0}[c % 5]
        cols = np.sort(rng.choice(wB, n, replace=False))
        rows.append(c + w * cols.astype(np.int64))
    bk = np.sort(np.concatenate(rows)).astype(np.uint64)
    bv = rng.uniform(-1, 1, bk.size)
    ak, av = random_lattice(rng, h, w, 1, 5000)
    check(cuda, torch, ak, av, bk, bv, h, w, wB, 1)


def test_tile_engine_duplicate_keys(cuda, torch, rng, force_tile):
    """Operands that are not sets: duplicate keys contribute every product."""
    for h in (64, 4096):
        ak, av = random_lattice(rng, h, 50, 2, 3000, dup=True)
        bk, bv = random_lattice(rng, 50, 130, 2, 3000, dup=True)
        check(cuda, torch, ak, av, bk, bv, h, 50, 130, 2)


def test_tile_engine_exact_zero_sums_kept(cuda, torch, force_tile):
    """Products that cancel exactly stay in the pattern (csc_no_accum keeps zeros)."""
    h, w, wB = 2, 2, 70
    ak = np.array([0, 1, 2], np.uint64)             # A(0,0), A(1,0), A(0,1) = 1
    av = np.array([1.0, 1.0, 1.0])
    bk = np.array([0, 1, 2 * 69, 1 + 2 * 69], np.uint64)  # B(0,0)=1, B(1,0)=-1, B(0,69)=2, B(1,69)=-2
    bv = np.array([1.0, -1.0, 2.0, -2.0])
    check(cuda, torch, ak, av, bk, bv, h, w, wB, 1)
    ek, ev, _ = oracle.lattice_mult(ak, av, h, w, 1, bk, bv, wB, with_abs=True)
    assert ek.size == 4 and np.count_nonzero(ev == 0.0) == 2
