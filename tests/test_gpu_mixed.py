"""GPU parity of the mixed sparse / dense lattice products
(SparseDenseLatticeMultMex; DenseLatticeBase.h:436-500 and
SparseLatticeBase.h:1148-1162) through the C ABI against the oracle: keys,
order and values bit-exact (both accumulate c = c + v * d in key order)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from test_gpu_sort import to_dev, to_host
from test_oracle import MIXED_SHAPES, mixed_case, rowmajor_keys

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def run_dense_first(cuda, torch, A, bk, bv, h, w, wB, d):
    k, v = cuda.sparse_dense_mult(to_dev(A, torch), to_dev(bk, torch), to_dev(bv, torch), w, wB, d, h, True)
    ek, ev = oracle.dense_sparse_mult(A, bk, bv, h, w, wB, d)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0


def run_sparse_first(cuda, torch, rk, av, B, h, w, wB, d):
    k, v = cuda.sparse_dense_mult(to_dev(B, torch), to_dev(rk, torch), to_dev(av, torch), h, w, d, wB, False)
    ek, ev = oracle.sparse_dense_mult(rk, av, B, h, w, wB, d)
    np.testing.assert_array_equal(to_host(k, np.uint64), ek)
    np.testing.assert_array_equal(to_host(v), ev)
    assert cuda.device_status() == 0


@pytest.mark.parametrize("m1,n1,n2,p", MIXED_SHAPES)
def test_mixed_reference_shapes(cuda, torch, rng, m1, n1, n2, p):
    """The shapes of the reference's mixedlatticemulttests.cpp (full, repeated
    inner, repeated outer, no depth, outer with one operand)."""
    A, B = mixed_case(rng, m1, n1, n2, p)
    bk = np.flatnonzero(B).astype(np.uint64)
    run_dense_first(cuda, torch, A, bk, B[bk.astype(np.int64)], m1, n1, n2, p)
    nz = np.flatnonzero(A)
    rk = rowmajor_keys(nz, m1, n1)
    order = np.argsort(rk, kind="stable")
    run_sparse_first(cuda, torch, rk[order].astype(np.uint64), A[nz][order], B, m1, n1, n2, p)


@pytest.mark.parametrize("h,w,wB,d,nnz", [
    (3000, 40, 50, 2, 900),      # several 1024-output chunks per line, ragged last chunk
    (257, 700, 3, 1, 2000),      # lines with more than 256 entries (batched staging)
    (1, 1, 1, 1, 1),
    (5, 9, 7, 3, 0),             # empty sparse operand
    (64, 1000, 64, 4, 30000),
])
def test_mixed_shapes(cuda, torch, rng, h, w, wB, d, nnz):
    A = rng.standard_normal(h * w * d)
    B = rng.standard_normal(w * wB * d)
    # dense x sparse: S is w x wB x d, duplicate keys allowed (every entry contributes)
    bk = np.sort(rng.integers(0, w * wB * d, nnz)).astype(np.uint64)
    bv = rng.standard_normal(nnz)
    bv[rng.random(nnz) < 0.1] = 0.0
    run_dense_first(cuda, torch, A, bk, bv, h, w, wB, d)
    # sparse x dense: S is h x w x d with row-major keys
    rk = np.sort(rng.integers(0, h * w * d, nnz)).astype(np.uint64)
    run_sparse_first(cuda, torch, rk, rng.standard_normal(nnz), B, h, w, wB, d)


def test_mixed_zero_line_kept(cuda, torch):
    A = np.array([1.0, 2.0, 1.0, 2.0])
    run_dense_first(cuda, torch, A, np.array([0, 1], np.uint64), np.array([3.0, -3.0]), 2, 2, 1, 1)


def test_mixed_bad_dims(cuda, torch):
    import libnt_b200 as L
    z = to_dev(np.zeros(1, np.uint64), torch)
    zv = to_dev(np.zeros(1), torch)
    S = L.Lattice.of(z, zv, 4, 0, 3)
    b = C.c_size_t(0)
    assert L.lib().lnt_sparse_dense_mult_workspace(C.byref(S), 5, 1, C.byref(b)) == 2
    S = L.Lattice.of(z, zv, 4, 2, 3)
    assert L.lib().lnt_sparse_dense_mult_workspace(C.byref(S), 0, 0, C.byref(b)) == 2
