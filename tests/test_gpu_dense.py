"""GPU dense lattice products (DenseLatticeBase::operator*): the plain FP64
path and the split-precision INT8 tensor-core path against the reference's
golden fixture, its closed-form known answer and the oracle's compensated
FP64 entries."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from test_gpu_sort import to_dev, to_host

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def test_golden_fixture_fp64_and_split(cuda, torch):
    """data/test1.bin x data/test2.bin = data/multtest_ddd.bin (5x5x10)."""
    z = np.load(GOLDEN / "dense_lattice_5x5x10.npz")
    h, w, wB, d = (int(x) for x in z["shape"])
    A, B = to_dev(z["A"], torch), to_dev(z["B"], torch)
    mag = np.abs(oracle.dense_lattice_mult(np.abs(z["A"]), np.abs(z["B"]), h, w, wB, d))
    # the fixture is Eigen's summation order; a fused-multiply-add GEMM may differ by a rounding
    c64 = to_host(cuda.dense_mult_fp64(A, B, h, w, wB, d))
    assert np.all(np.abs(c64 - z["C"]) <= 4 * 2.0 ** -52 * mag)
    cs = to_host(cuda.dense_mult_split(A, B, h, w, wB, d, slices=7))
    assert np.all(np.abs(cs - z["C"]) <= 1e-13 * mag)


def test_closed_form_kat_exact(cuda, torch):
    """dense_mia_mult_test.cpp:44-74: a increments along the inner modes, b = 1:
    every entry is dim2^2 (dim2^2 + 1) / 2 exactly on both paths."""
    dim1, dim2 = 3, 4
    h, w, wB = dim1 * dim1, dim2 * dim2, dim1 * dim1
    A = np.empty((h, w))
    A[:, :] = np.arange(1, w + 1)[None, :]
    B = np.ones((w, wB))
    Ad, Bd = to_dev(A.ravel(order="F"), torch), to_dev(B.ravel(order="F"), torch)
    for Cm in (cuda.dense_mult_fp64(Ad, Bd, h, w, wB), cuda.dense_mult_split(Ad, Bd, h, w, wB)):
        assert np.all(to_host(Cm) == w * (w + 1) / 2)


# componentwise bound on |C - C_ref| / (|A||B|): uniform data loses nothing to the
# row/column scaling; data spanning 2^+-20 inside a row keeps fewer bits in its
# small entries, one more slice (7 more bits) restores them
TOL = {("uniform", 7): 1e-13, ("uniform", 8): 1e-13, ("wide_exponent", 7): 2e-11, ("wide_exponent", 8): 1e-13}


@pytest.mark.parametrize("h,w,wB,d", [(100, 300, 70, 3), (257, 1000, 129, 1), (64, 4096, 64, 1)])
@pytest.mark.parametrize("variant", ["uniform", "wide_exponent"])
@pytest.mark.parametrize("slices", [7, 8])
def test_split_error_vs_compensated_fp64(cuda, torch, rng, h, w, wB, d, variant, slices):
    if variant == "uniform":
        A = rng.uniform(-1, 1, h * w * d)
        B = rng.uniform(-1, 1, w * wB * d)
    else:  # mantissa U[1,2) * 2^e, e in [-20, 20], random sign
        A = rng.uniform(1, 2, h * w * d) * 2.0 ** rng.integers(-20, 21, h * w * d) * rng.choice([-1, 1], h * w * d)
        B = rng.uniform(1, 2, w * wB * d) * 2.0 ** rng.integers(-20, 21, w * wB * d) * rng.choice([-1, 1], w * wB * d)
    Cs = to_host(cuda.dense_mult_split(to_dev(A, torch), to_dev(B, torch), h, w, wB, d, slices=slices))
    for t in range(d):
        At = A[t * h * w:(t + 1) * h * w]
        Bt = B[t * w * wB:(t + 1) * w * wB]
        rows, cols = np.meshgrid(np.arange(h), np.arange(wB), indexing="ij")
        ref, mag = oracle.dense_entries(At, Bt, h, w, rows.ravel(), cols.ravel())
        got = Cs[t * h * wB:(t + 1) * h * wB].reshape(wB, h).T.ravel()
        err = np.abs(got - ref) / np.maximum(mag, 1e-300)
        assert err.max() <= TOL[(variant, slices)], err.max()


# scheme II (moduli + Chinese remaindering): error about 2^(2-beta) |A||B|
CRT_TOL = {("uniform", 13): 1e-12, ("uniform", 16): 1e-13, ("wide_exponent", 13): 1e-8,
           ("wide_exponent", 16): 1e-12}


def test_crt_golden_fixture_and_kat(cuda, torch):
    z = np.load(GOLDEN / "dense_lattice_5x5x10.npz")
    h, w, wB, d = (int(x) for x in z["shape"])
    mag = np.abs(oracle.dense_lattice_mult(np.abs(z["A"]), np.abs(z["B"]), h, w, wB, d))
    c = to_host(cuda.dense_mult_crt(to_dev(z["A"], torch), to_dev(z["B"], torch), h, w, wB, d, moduli=13))
    assert np.all(np.abs(c - z["C"]) <= 1e-13 * mag)
    dim1, dim2 = 3, 4
    hh, ww, wwB = dim1 * dim1, dim2 * dim2, dim1 * dim1
    A = np.empty((hh, ww))
    A[:, :] = np.arange(1, ww + 1)[None, :]
    B = np.ones((ww, wwB))
    c = to_host(cuda.dense_mult_crt(to_dev(A.ravel(order="F"), torch), to_dev(B.ravel(order="F"), torch), hh, ww,
                                    wwB, 1, moduli=13))
    assert np.all(c == ww * (ww + 1) / 2)


@pytest.mark.parametrize("h,w,wB", [(600, 2000, 700), (256, 256, 256), (1, 130, 513), (300, 64, 3),
                                    (513, 4100, 257)])
@pytest.mark.parametrize("moduli", [13, 16])
def test_crt_integer_operands_exact(cuda, torch, rng, h, w, wB, moduli):
    """Integer operands (|a|, |b| <= 1000) are scaled by powers of two into
    integers without rounding, so scheme II must return A B exactly: every
    residue product tile of the tensor-core GEMM (partial row, column and K
    tiles included) is checked bit for bit."""
    A = rng.integers(-1000, 1001, h * w).astype(np.float64)
    B = rng.integers(-1000, 1001, w * wB).astype(np.float64)
    C = to_host(cuda.dense_mult_crt(to_dev(A, torch), to_dev(B, torch), h, w, wB, 1, moduli=moduli))
    ref = (A.reshape(w, h).T @ B.reshape(wB, w).T).T.ravel()  # column-major C, exact in float64
    np.testing.assert_array_equal(C, ref)


@pytest.mark.parametrize("variant,w,expect", [("uniform", 16384, 14), ("uniform", 4096, 13),
                                              ("wide_exponent", 16384, 15)])
def test_crt_moduli_choice_meets_tolerance(cuda, torch, rng, variant, w, expect):
    """lnt_dense_crt_moduli: the smallest count whose bound 2^(2-beta) R keeps
    every entry within 1e-12 of |A||B|, R the largest max / mean magnitude
    ratio of a row of A or column of B; the product with that count meets it."""
    h, wB = 48, 40
    if variant == "uniform":
        A, B = rng.uniform(-1, 1, h * w), rng.uniform(-1, 1, w * wB)
    else:
        A = rng.uniform(1, 2, h * w) * 2.0 ** rng.integers(-20, 21, h * w) * rng.choice([-1, 1], h * w)
        B = rng.uniform(1, 2, w * wB) * 2.0 ** rng.integers(-20, 21, w * wB) * rng.choice([-1, 1], w * wB)
    Ad, Bd = to_dev(A, torch), to_dev(B, torch)
    m = cuda.dense_crt_moduli(Ad, Bd, h, w, wB)
    assert m == expect
    Cs = to_host(cuda.dense_mult_crt(Ad, Bd, h, w, wB, 1, moduli=m))
    rows, cols = np.meshgrid(np.arange(h), np.arange(wB), indexing="ij")
    ref, mag = oracle.dense_entries(A, B, h, w, rows.ravel(), cols.ravel())
    got = Cs.reshape(wB, h).T.ravel()
    assert np.max(np.abs(got - ref) / mag) <= 1e-12


@pytest.mark.parametrize("h,w,wB,d", [(100, 300, 70, 3), (257, 1000, 129, 1), (64, 4096, 64, 1)])
@pytest.mark.parametrize("variant", ["uniform", "wide_exponent"])
@pytest.mark.parametrize("moduli", [13, 16])
def test_crt_error_vs_compensated_fp64(cuda, torch, rng, h, w, wB, d, variant, moduli):
    if variant == "uniform":
        A = rng.uniform(-1, 1, h * w * d)
        B = rng.uniform(-1, 1, w * wB * d)
    else:
        A = rng.uniform(1, 2, h * w * d) * 2.0 ** rng.integers(-20, 21, h * w * d) * rng.choice([-1, 1], h * w * d)
        B = rng.uniform(1, 2, w * wB * d) * 2.0 ** rng.integers(-20, 21, w * wB * d) * rng.choice([-1, 1], w * wB * d)
    Cs = to_host(cuda.dense_mult_crt(to_dev(A, torch), to_dev(B, torch), h, w, wB, d, moduli=moduli))
    for t in range(d):
        At = A[t * h * w:(t + 1) * h * w]
        Bt = B[t * w * wB:(t + 1) * w * wB]
        rows, cols = np.meshgrid(np.arange(h), np.arange(wB), indexing="ij")
        ref, mag = oracle.dense_entries(At, Bt, h, w, rows.ravel(), cols.ravel())
        got = Cs[t * h * wB:(t + 1) * h * wB].reshape(wB, h).T.ravel()
        err = np.abs(got - ref) / np.maximum(mag, 1e-300)
        assert err.max() <= CRT_TOL[(variant, moduli)], err.max()



@pytest.mark.parametrize("dims,perm", [
    ([7, 9, 11], [1, 2, 0]), ([40, 33, 5], [1, 0, 2]), ([5, 6, 7, 8], [0, 3, 1, 2]), ([64, 3, 70, 2], [2, 0, 3, 1]),
    ([3, 4, 5, 6, 7], [4, 2, 0, 3, 1]), ([1000, 1000], [1, 0]), ([8, 9], [0, 1]), ([1, 1, 5], [2, 0, 1]),
])
def test_dense_permute_matches_numpy(cuda, rng, dims, perm):
    """lnt_dense_permute: mode k of the result is mode perm[k] (column-major),
    bit-exact against numpy; both the contiguous-run and the tiled kernel."""
    import torch
    x = rng.standard_normal(int(np.prod(dims)))
    y = cuda.dense_permute(torch.from_numpy(x).cuda(), dims, perm)
    ref = np.ravel(x.reshape(dims, order="F").transpose(perm), order="F")
    np.testing.assert_array_equal(y.cpu().numpy(), ref)


def test_dense_permute_rejects_bad_perm(cuda):
    import ctypes as C

    import torch

    import libnt_b200 as L
    x = torch.zeros(12, dtype=torch.float64, device="cuda")
    y = torch.zeros(12, dtype=torch.float64, device="cuda")
    d = np.array([3, 4], np.int64)
    bad = np.array([1, 1], np.int32)
    assert L.lib().lnt_dense_permute(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), 2, d.ctypes.data,
                                     bad.ctypes.data, None) == 3
    assert L.lib().lnt_dense_permute(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr() + 8), 2, d.ctypes.data,
                                     np.array([1, 0], np.int32).ctypes.data, None) == 1   # overlapping
