"""GPU parity of re-key, sort, collect_duplicates and the fused sort merge
against the oracle, through the C ABI.  Keys and sparsity pattern must be
bit-exact; values within 1e-12 * sum|terms| where summation order may differ."""
import numpy as np
import pytest

import oracle
from conftest import rel_ok

pytestmark = pytest.mark.gpu


def to_dev(a, torch):
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        a = a.view(np.int64)
    return torch.from_numpy(a).cuda()


def to_host(t, dtype=None):
    a = t.cpu().numpy()
    if dtype == np.uint64:
        a = a.view(np.uint64)
    return a


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


@pytest.mark.parametrize("order,dims,cur,new", [
    (4, [512] * 4, [0, 1, 2, 3], [3, 2, 1, 0]),
    (3, [100, 100, 100], [0, 1, 2], [2, 0, 1]),
    (5, [7, 13, 5, 11, 3], [2, 0, 3, 1, 4], [4, 2, 0, 1, 3]),
    (2, [1 << 20, 1 << 20], [0, 1], [1, 0]),
    (6, [3, 1, 7, 2, 9, 5], [5, 4, 3, 2, 1, 0], [0, 2, 4, 1, 3, 5]),
])
@pytest.mark.parametrize("n", [1, 7, 100003])
def test_rekey_bit_exact(cuda, torch, rng, order, dims, cur, new, n):
    total = int(np.prod(dims))
    keys = rng.integers(0, total, n, dtype=np.uint64)
    got = to_host(cuda.rekey(to_dev(keys, torch), dims, cur, new), np.uint64)
    np.testing.assert_array_equal(got, oracle.rekey(keys, dims, cur, new))


def test_rekey_in_place_unaligned(cuda, torch, rng):
    dims = [9, 10, 11]
    keys = rng.integers(0, 990, 1001, dtype=np.uint64)
    d = to_dev(keys, torch)
    sub = d[1:]  # 8-byte aligned, not 16
    cuda.rekey(sub, dims, [0, 1, 2], [1, 2, 0], out=sub)
    np.testing.assert_array_equal(to_host(d, np.uint64)[1:], oracle.rekey(keys[1:], dims, [0, 1, 2], [1, 2, 0]))


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 12289, 100000, 1 << 20, (1 << 22) + 7])
@pytest.mark.parametrize("bits", [1, 8, 9, 17, 36, 40, 63])
def test_sort_pairs_bit_exact(cuda, torch, rng, n, bits):
    if n > (1 << 20) and bits not in (36, 63):
        pytest.skip("large sizes only at the workload key widths")
    keys = rng.integers(0, 2 ** bits, n, dtype=np.uint64)
    vals = rng.standard_normal(n)
    k, v = cuda.sort_pairs(to_dev(keys, torch), to_dev(vals, torch), max_key=2 ** bits)
    ek, ev = oracle.sort_pairs(keys, vals)  # stable: the GPU sort is stable too
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0


@pytest.mark.parametrize("variant", range(12))
@pytest.mark.parametrize("n,bits", [(1, 9), (3071, 36), (12289, 20), (300007, 36), (200000, 63), (65537, 10)])
def test_every_sort_variant_bit_exact(cuda, torch, rng, monkeypatch, variant, n, bits):
    """Each compiled kernel variant (the autotuner may pick any) is stable and exact."""
    import libnt_b200 as L
    if variant >= L.lib().lnt_sort_variant_count():
        pytest.skip("variant not compiled")
    monkeypatch.setenv("LNT_SORT_VARIANT", str(variant))
    keys = rng.integers(0, 2 ** bits, n, dtype=np.uint64)
    keys[: n // 3] = keys[n // 2]
    vals = rng.standard_normal(n)
    k, v = cuda.sort_pairs(to_dev(keys, torch), to_dev(vals, torch), max_key=2 ** bits)
    ek, ev = oracle.sort_pairs(keys, vals)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0


def test_sort_pairs_in_place_and_duplicates(cuda, torch, rng):
    n = 300001
    keys = rng.integers(0, 1000, n, dtype=np.uint64)  # heavy duplicates
    vals = rng.standard_normal(n)
    for max_key in (1000, 1 << 20, 1 << 27):  # odd and even pass counts
        dk, dv = to_dev(keys, torch), to_dev(vals, torch)
        cuda.sort_pairs(dk, dv, max_key=max_key, out_keys=dk, out_vals=dv)
        ek, ev = oracle.sort_pairs(keys, vals)
        np.testing.assert_array_equal(to_host(dk, np.uint64), ek)
        np.testing.assert_array_equal(to_host(dv), ev)


def test_sort_all_equal_keys(cuda, torch, rng):
    n = 50000
    keys = np.full(n, 77, np.uint64)
    vals = rng.standard_normal(n)
    k, v = cuda.sort_pairs(to_dev(keys, torch), to_dev(vals, torch), max_key=1 << 36)
    np.testing.assert_array_equal(to_host(v), vals)


@pytest.mark.parametrize("skip", [True, False])
def test_collect_duplicates_quirk(cuda, torch, skip):
    keys = np.array([1, 1, 3, 3, 3, 5, 7, 7, 9], np.uint64)
    vals = np.array([0.0, 0.0, 0.0, 2.0, 0.0, 0.0, 1.5, -1.5, -0.0])
    k, v = cuda.collect_duplicates(to_dev(keys, torch), to_dev(vals, torch), skip_zero_heads=skip)
    ek, ev = oracle.collect_duplicates(keys, vals, skip_zero_heads=skip)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    np.testing.assert_array_equal(np.signbit(to_host(v)), np.signbit(ev))


@pytest.mark.parametrize("n,distinct", [(5000, 5000), (100000, 3), (100000, 1), (1 << 20, 40000), (200000, 190000)])
@pytest.mark.parametrize("zero_frac", [0.0, 0.5])
def test_collect_duplicates_runs_cross_tiles(cuda, torch, rng, n, distinct, zero_frac):
    keys = np.sort(rng.integers(0, distinct, n, dtype=np.uint64))
    vals = rng.standard_normal(n)
    vals[rng.random(n) < zero_frac] = 0.0
    for skip in (True, False):
        k, v = cuda.collect_duplicates(to_dev(keys, torch), to_dev(vals, torch), skip_zero_heads=skip)
        ek, ev, ea = oracle.collect_duplicates(keys, vals, skip_zero_heads=skip, with_abs=True)
        np.testing.assert_array_equal(to_host(k, np.uint64), ek)
        assert rel_ok(to_host(v), ev, ea)


def _merge_case(rng, dims, na, nb, zero_frac=0.0, replace=True):
    total = int(np.prod(dims))
    ak = rng.integers(0, total, na, dtype=np.uint64)
    bk = rng.integers(0, total, nb, dtype=np.uint64)
    av = rng.uniform(-1, 1, na)
    bv = rng.uniform(-1, 1, nb)
    if zero_frac:
        av[rng.random(na) < zero_frac] = 0.0
        bv[rng.random(nb) < zero_frac] = 0.0
    return ak, av, bk, bv


@pytest.mark.parametrize("dims,na,nb", [([512] * 4, 1 << 20, 1 << 20), ([5, 8, 5, 8], 700, 700),
                                        ([16, 16, 16, 16], 30000, 30000), ([512] * 4, 1 << 18, 1 << 19),
                                        ([6, 6, 6, 6], 3000, 10)])
@pytest.mark.parametrize("op", [0, 1])
def test_sort_merge_matches_oracle(cuda, torch, rng, dims, na, nb, op):
    """c(i,j,k,l) = a(i,j,k,l) +/- b(l,k,j,i), both unsorted: SparseMIA::sortMerge."""
    ak, av, bk, bv = _merge_case(rng, dims, na, nb, zero_frac=0.05)
    bdims = dims[::-1]
    a = oracle.SparseMIA(dims, ak, av, sorted=False)
    b = oracle.SparseMIA(bdims, bk, bv, sorted=False)
    c = oracle.merge(a.copy(), b.copy(), [3, 2, 1, 0], op)
    # The GPU call: which operand is re-keyed follows the same size rule.
    import libnt_b200 as L
    if na > nb:
        a_spec = None
        b_spec = L.RekeySpec.make(bdims, [0, 1, 2, 3], oracle.reorder_from([3, 2, 1, 0], [0, 1, 2, 3]))
    else:
        a_spec = L.RekeySpec.make(dims, [0, 1, 2, 3], oracle.reorder_from(oracle.reverse_order([3, 2, 1, 0]),
                                                                           [0, 1, 2, 3]))
        b_spec = None
    k, v = cuda.sort_reduce(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch),
                            max_key=int(np.prod(dims)), a_rekey=a_spec, b_rekey=b_spec,
                            b_scale=-1.0 if op else 1.0)
    np.testing.assert_array_equal(to_host(k, np.uint64), c.keys)
    # summation-error scale per output key from the oracle's own fold
    allk = np.concatenate([oracle.rekey(ak, dims, [0, 1, 2, 3], [3, 2, 1, 0]) if na <= nb else ak,
                           bk if na <= nb else oracle.rekey(bk, bdims, [0, 1, 2, 3], [3, 2, 1, 0])])
    allv = np.concatenate([av, -bv if op else bv])
    sk, sv = oracle.sort_pairs(allk, allv)
    ek, ev, ea = oracle.collect_duplicates(sk, sv, with_abs=True)
    np.testing.assert_array_equal(ek, c.keys)
    assert rel_ok(to_host(v), c.vals, ea)
    assert cuda.device_status() == 0


@pytest.mark.parametrize("path", ["bucketed", "bucketed_small", "lsd"])
@pytest.mark.parametrize("dims,n_each,dup_frac", [([512] * 4, 1 << 20, 0.0), ([64] * 4, 1 << 20, 0.0),
                                                   ([512] * 4, 3 << 19, 0.0), ([512] * 4, 1 << 20, 0.5)])
def test_sort_merge_both_paths(cuda, torch, rng, monkeypatch, path, dims, n_each, dup_frac):
    """The bucketed sort+collect (hist, 2 passes, per-bucket shared-memory sort
    with fused collect) and the LSD path give identical results; heavily
    duplicated keys overflow a bucket and fall back to the LSD path."""
    import libnt_b200 as L
    if path == "lsd":
        monkeypatch.setenv("LNT_NO_BUCKETS", "1")
    monkeypatch.setenv("LNT_BUCKET_SMALL", "1" if path == "bucketed_small" else "0")
    ak, av, bk, bv = _merge_case(rng, dims, n_each, n_each, zero_frac=0.1)
    if dup_frac:
        ak[: int(n_each * dup_frac)] = ak[0]
    # the smallest key gets only zero values: it must survive (position 0)
    total = int(np.prod(dims))
    ak[1], av[1] = 0, 0.0
    bk[1], bv[1] = 0, 0.0
    spec = L.RekeySpec.make(dims, [0, 1, 2, 3], [3, 2, 1, 0])
    k, v = cuda.sort_reduce(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch),
                            max_key=total, a_rekey=spec)
    allk = np.concatenate([oracle.rekey(ak, dims, [0, 1, 2, 3], [3, 2, 1, 0]), bk])
    allv = np.concatenate([av, bv])
    sk, sv = oracle.sort_pairs(allk, allv)
    ek, ev, ea = oracle.collect_duplicates(sk, sv, with_abs=True)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    if dup_frac:  # a run spanning many tiles is summed tile-wise on the LSD fallback
        assert rel_ok(to_host(v), ev, ea)
    else:  # same stable order and sequential fold: identical sums
        np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0


def test_sort_reduce_clustered_buckets(cuda, torch, rng):
    """36-bit keys, 2 x 2^20 pairs (512 buckets of about 4096): in even buckets
    every pair shares the next 12 key bits, so one sub-bucket holds the whole
    bucket and the local LSD passes sort it (with about 250 duplicate keys per
    bucket); odd buckets take the counting rank.  Keys and values exact."""
    n = 1 << 20
    top = rng.integers(0, 1 << 9, 2 * n).astype(np.uint64)
    mid = rng.integers(0, 1 << 12, 2 * n).astype(np.uint64)
    mid[top % 2 == 0] = 0
    keys = (top << np.uint64(27)) | (mid << np.uint64(15)) | rng.integers(0, 1 << 15, 2 * n).astype(np.uint64)
    vals = rng.uniform(-1, 1, 2 * n)
    vals[rng.random(2 * n) < 0.1] = 0.0
    k, v = cuda.sort_reduce(to_dev(keys[:n], torch), to_dev(vals[:n], torch), to_dev(keys[n:], torch),
                            to_dev(vals[n:], torch), max_key=1 << 36)
    sk, sv = oracle.sort_pairs(keys, vals)
    ek, ev = oracle.collect_duplicates(sk, sv)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0
