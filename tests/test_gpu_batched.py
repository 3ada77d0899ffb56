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


def test_batched_rejects_tall_problems(cuda, torch):
    import ctypes as C

    import libnt_b200 as L
    dims = np.array([[2048, 4, 4, 1]], np.int64)  # beyond the 1024-row accumulator
    off = np.array([0, 0], np.uint64)
    nb, cap = C.c_size_t(0), C.c_uint64(0)
    st = L.lib().lnt_batched_workspace(1, dims.ctypes.data, off.ctypes.data, off.ctypes.data, C.byref(nb),
                                       C.byref(cap))
    assert st == 8  # LNT_UNSUPPORTED
