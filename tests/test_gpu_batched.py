"""GPU parity of the batched lattice products (one set of launches for
thousands of uneven contractions, capturable in a CUDA graph) against the
oracle's per-problem csc_no_accum restatement."""
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


def make_batch(rng, count, dim_lo, dim_hi, nnz_lo, nnz_hi):
    """Problems shaped like a(i,j,k) * b(k,l,j) as lattices: A is dim_i x (dim_j
    dim_k), B is (dim_j dim_k) x dim_l, nnz log-uniform, both key-sorted."""
    dims, ak, av, bk, bv = [], [], [], [], []
    for _ in range(count):
        i, j, k, l = (int(x) for x in rng.integers(dim_lo, dim_hi + 1, 4))
        h, w, wB = i, j * k, l
        na = min(int(round(10 ** rng.uniform(np.log10(nnz_lo), np.log10(nnz_hi)))), h * w)
        nb = min(int(round(10 ** rng.uniform(np.log10(nnz_lo), np.log10(nnz_hi)))), w * wB)
        a = np.sort(rng.choice(h * w, na, replace=False)).astype(np.uint64)
        b = np.sort(rng.choice(w * wB, nb, replace=False)).astype(np.uint64)
        dims.append((h, w, wB, 1))
        ak.append(a)
        bk.append(b)
        av.append(rng.uniform(-1, 1, na))
        bv.append(rng.uniform(-1, 1, nb))
    a_off = np.concatenate([[0], np.cumsum([x.size for x in ak])]).astype(np.uint64)
    b_off = np.concatenate([[0], np.cumsum([x.size for x in bk])]).astype(np.uint64)
    return np.array(dims, np.int64), a_off, b_off, ak, av, bk, bv


def check_batch(cuda, torch, batch, dims, ak, av, bk, bv):
    for p in range(len(dims)):
        h, w, wB, d = (int(x) for x in dims[p])
        k, v = batch.result(p)
        ek, ev, ea = oracle.lattice_mult(ak[p], av[p], h, w, d, bk[p], bv[p], wB, with_abs=True)
        np.testing.assert_array_equal(to_host(k, np.uint64), ek)
        assert rel_ok(to_host(v), ev, ea)


@pytest.mark.parametrize("chunk", ["1", "8", "64"])
def test_batched_matches_per_problem_oracle(cuda, torch, rng, monkeypatch, chunk):
    import libnt_b200 as L
    monkeypatch.setenv("LNT_BATCH_CHUNK", chunk)
    dims, a_off, b_off, ak, av, bk, bv = make_batch(rng, 96, 4, 40, 3, 3000)
    batch = L.Batch(dims, a_off, b_off, to_dev(np.concatenate(ak), torch), to_dev(np.concatenate(av), torch),
                    to_dev(np.concatenate(bk), torch), to_dev(np.concatenate(bv), torch))
    batch.run()
    check_batch(cuda, torch, batch, dims, ak, av, bk, bv)
    assert cuda.device_status() == 0


def test_batched_cuda_graph_replay(cuda, torch, rng):
    import libnt_b200 as L
    dims, a_off, b_off, ak, av, bk, bv = make_batch(rng, 200, 16, 128, 50, 5000)
    batch = L.Batch(dims, a_off, b_off, to_dev(np.concatenate(ak), torch), to_dev(np.concatenate(av), torch),
                    to_dev(np.concatenate(bk), torch), to_dev(np.concatenate(bv), torch))
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        batch.run()  # warm-up outside capture (sets kernel attributes)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        batch.run()
    batch.c_keys.zero_()
    batch.c_vals.zero_()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    check_batch(cuda, torch, batch, dims, ak, av, bk, bv)


def test_batched_rows_beyond_one_accumulator(cuda, torch, rng):
    """Problems with more than 512 rows are accumulated in blocks of 512 rows
    (a binary search per A column and block): same results as the oracle,
    at the block boundary (512, 513 rows) and well beyond it."""
    import libnt_b200 as L
    dims, ak, av, bk, bv = [], [], [], [], []
    for h, w, wB, na, nb in [(3000, 40, 30, 20000, 500), (1025, 8, 9, 4000, 50), (2048, 1, 3, 2048, 3),
                             (5000, 16, 4, 0, 30), (1500, 20, 20, 6000, 0), (512, 8, 9, 3000, 40),
                             (513, 8, 9, 3000, 40)]:
        a = np.sort(rng.choice(h * w, na, replace=False)).astype(np.uint64)
        b = np.sort(rng.choice(w * wB, nb, replace=False)).astype(np.uint64)
        dims.append((h, w, wB, 1))
        ak.append(a)
        bk.append(b)
        av.append(rng.uniform(-1, 1, na))
        bv.append(rng.uniform(-1, 1, nb))
    a_off = np.concatenate([[0], np.cumsum([x.size for x in ak])]).astype(np.uint64)
    b_off = np.concatenate([[0], np.cumsum([x.size for x in bk])]).astype(np.uint64)
    dims = np.array(dims, np.int64)
    batch = L.Batch(dims, a_off, b_off, to_dev(np.concatenate(ak), torch), to_dev(np.concatenate(av), torch),
                    to_dev(np.concatenate(bk), torch), to_dev(np.concatenate(bv), torch))
    batch.run()
    check_batch(cuda, torch, batch, dims, ak, av, bk, bv)
    assert cuda.device_status() == 0


def _unsorted_batch(rng, count, dim_lo, dim_hi, nnz_lo, nnz_hi, tall=()):
    """Problems c(i,l) = a(j,i,k) * b(k,l,j) as unsorted tensors: a's keys run j
    fastest (re-key {1,0,2} puts i first), b's keys k fastest (re-key {2,0,1});
    `tall` problems get i beyond the 512-row accumulator."""
    import libnt_b200 as L
    dims, specs_a, specs_b, ak, av, bk, bv = [], [], [], [], [], [], []
    for p in range(count):
        i, j, k, l = (int(x) for x in rng.integers(dim_lo, dim_hi + 1, 4))
        if p in tall:
            i = 1500 + 37 * p
        na = min(int(round(10 ** rng.uniform(np.log10(nnz_lo), np.log10(nnz_hi)))), i * j * k)
        nb = min(int(round(10 ** rng.uniform(np.log10(nnz_lo), np.log10(nnz_hi)))), k * l * j)
        if p % 17 == 5:
            na = 0  # empty operands
        if p % 19 == 7:
            nb = 0
        ak.append(rng.permutation(rng.choice(j * i * k, na, replace=False)).astype(np.uint64))
        bk.append(rng.permutation(rng.choice(k * l * j, nb, replace=False)).astype(np.uint64))
        av.append(rng.uniform(-1, 1, na))
        bv.append(rng.uniform(-1, 1, nb))
        dims.append((i, j * k, l, 1))
        specs_a.append(((j, i, k), [0, 1, 2], [1, 0, 2]))
        specs_b.append(((k, l, j), [0, 1, 2], [2, 0, 1]))
    a_off = np.concatenate([[0], np.cumsum([x.size for x in ak])]).astype(np.uint64)
    b_off = np.concatenate([[0], np.cumsum([x.size for x in bk])]).astype(np.uint64)
    ra = [L.RekeySpec.make(*x) for x in specs_a]
    rb = [L.RekeySpec.make(*x) for x in specs_b]
    return np.array(dims, np.int64), a_off, b_off, ak, av, bk, bv, specs_a, specs_b, ra, rb


def _expected_unsorted(p, dims, ak, av, bk, bv, specs_a, specs_b):
    h, w, wB, _ = (int(x) for x in dims[p])
    ka = oracle.rekey(ak[p], *specs_a[p])
    kb = oracle.rekey(bk[p], *specs_b[p])
    oa, ob = np.argsort(ka, kind="stable"), np.argsort(kb, kind="stable")
    return oracle.lattice_mult(ka[oa], av[p][oa], h, w, 1, kb[ob], bv[p][ob], wB, with_abs=True)


def test_batched_contract_unsorted_matches_oracle(cuda, torch, rng):
    """lnt_batched_contract on unsorted tensors: every problem re-keyed into its
    lattice order and sorted inside the call (one radix sort over keys prefixed
    with the problem), then multiplied; replayed from a CUDA graph on new
    values.  Each problem equals re-key + sort + csc_no_accum on the host."""
    import libnt_b200 as L
    dims, a_off, b_off, ak, av, bk, bv, sa, sb, ra, rb = _unsorted_batch(rng, 150, 4, 60, 3, 4000, tall=(3, 77))
    dk = [to_dev(np.concatenate(x), torch) for x in (ak, av, bk, bv)]
    batch = L.Batch(dims, a_off, b_off, *dk, a_rekey=ra, b_rekey=rb)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        batch.run()
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    for p in range(len(dims)):
        ek, ev, ea = _expected_unsorted(p, dims, ak, av, bk, bv, sa, sb)
        k, v = batch.result(p)
        np.testing.assert_array_equal(to_host(k, np.uint64), ek)
        assert rel_ok(to_host(v), ev, ea)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        batch.run()
    av = [rng.uniform(-1, 1, x.size) for x in av]
    dk[1].copy_(to_dev(np.concatenate(av), torch))
    batch.c_vals.zero_()
    g.replay()
    torch.cuda.synchronize()
    for p in range(len(dims)):
        ek, ev, ea = _expected_unsorted(p, dims, ak, av, bk, bv, sa, sb)
        k, v = batch.result(p)
        np.testing.assert_array_equal(to_host(k, np.uint64), ek)
        assert rel_ok(to_host(v), ev, ea)
    assert cuda.device_status() == 0
    del g


def test_batched_contract_full_workload(cuda, torch):
    """The benchmarked batch: 4096 problems c(i,l) = a(i,j,k) * b(k,l,j), dims
    U{16..512}, nnz log-U[1e2, 1e5], both operands unsorted; every problem
    checked against the oracle (keys exact, values within 1e-12 of the sum of
    |products| per key)."""
    import bench
    import libnt_b200 as L
    dims, tdims, a_off, b_off, ak, av, bk, bv = bench.batched_inputs()
    count = len(dims)
    dk = [to_dev(np.concatenate(x), torch) for x in (ak, av, bk, bv)]
    rb = [L.RekeySpec.make(tdims[p][1], [0, 1, 2], [2, 0, 1]) for p in range(count)]
    batch = L.Batch(dims, a_off, b_off, *dk, a_rekey=[None] * count, b_rekey=rb)
    batch.run()
    torch.cuda.synchronize()
    assert cuda.device_status() == 0
    off = batch.c_off.cpu().numpy()
    ck = batch.c_keys[: int(off[-1])].cpu().numpy().view(np.uint64)
    cv = batch.c_vals[: int(off[-1])].cpu().numpy()
    del dk, batch
    torch.cuda.empty_cache()
    for p in range(count):
        ek, ev, ea = bench.batched_expected(p, dims, tdims, ak, av, bk, bv, with_abs=True)
        np.testing.assert_array_equal(ck[off[p]:off[p + 1]], ek)
        assert rel_ok(cv[off[p]:off[p + 1]], ev, ea), p
