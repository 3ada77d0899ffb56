"""CPU checks of the C ABI: the library loads, exports every function that
include/*.h declare, and rejects bad arguments before touching a GPU."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import libnt_b200 as L

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = "".join(h.read_text() for h in sorted((ROOT / "include").glob("*.h")))
    return sorted(set(re.findall(r"LNT_API\s+[\w\s\*]+?\b(lnt_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = header_symbols()
    assert "lnt_sort_pairs" in syms and "lnt_rekey" in syms and len(syms) >= 10


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    for s in header_symbols():
        assert hasattr(lib, s), f"{s} declared in include/*.h but not exported"


def test_python_bindings_cover_header():
    assert set(header_symbols()) <= set(L.declared_symbols()) | set(getattr(L, "EXTRA_SYMBOLS", []))


def test_status_strings():
    lib = L.lib()
    assert lib.lnt_status_string(0) == b"ok"
    assert lib.lnt_status_string(5) == b"workspace too small"
    assert lib.lnt_version() >= 100


def test_rekey_argument_errors_without_gpu():
    lib = L.lib()
    dims = (C.c_int64 * 3)(4, 5, 6)
    good = (C.c_int32 * 3)(0, 1, 2)
    bad = (C.c_int32 * 3)(0, 0, 2)
    dummy = C.c_void_p(256)  # never dereferenced: validation fails first
    assert lib.lnt_rekey(dummy, dummy, 10, 3, dims, good, bad, None) == 3  # LNT_BAD_SEQ
    zero = (C.c_int64 * 3)(4, 0, 6)
    assert lib.lnt_rekey(dummy, dummy, 10, 3, zero, good, good, None) == 2  # LNT_BAD_DIMS
    huge = (C.c_int64 * 3)(2 ** 31, 2 ** 31, 4)
    assert lib.lnt_rekey(dummy, dummy, 10, 3, huge, good, good, None) == 4  # LNT_OVERFLOW_KEYBITS
    assert lib.lnt_rekey(None, dummy, 10, 3, dims, good, good, None) == 1  # LNT_BAD_ARG
    assert lib.lnt_rekey(None, None, 0, 3, dims, good, good, None) == 0  # empty is a no-op


def test_workspace_queries():
    lib = L.lib()
    b = C.c_size_t(0)
    assert lib.lnt_sort_pairs_workspace(1 << 20, 1 << 36, C.byref(b)) == 0
    assert b.value >= 2 * (1 << 20) * 16
    assert lib.lnt_sort_pairs_workspace(1 << 30, 1 << 36, C.byref(b)) == 8  # beyond 2^30 pairs
    assert lib.lnt_sort_reduce_workspace(1 << 20, 1 << 20, 1 << 36, C.byref(b)) == 0
    assert b.value >= 2 * (2 << 20) * 16
    assert lib.lnt_collect_duplicates_workspace(12345, C.byref(b)) == 0 and b.value > 0


def test_sort_rejects_small_workspace_without_gpu():
    lib = L.lib()
    d = C.c_void_p(256)
    assert lib.lnt_sort_pairs(d, d, d, d, 1000, 1 << 20, d, 16, None) == 5  # LNT_WORKSPACE


def test_mex_gateways_reject_bad_arguments_without_gpu():
    """The mex-format host gateways (include/lnt_mex.h) check their arguments
    before any device work: 1-based orders, non-negative keys, the lattice
    product algorithm and shapes."""
    lib = L.lib()
    keys = np.array([3, 1, 2], np.int64)
    vals = np.ones(3)
    dims = np.array([4, 5], np.int64)
    bad = np.array([1, 1], np.uint8)    # not a permutation
    zero = np.array([0, 1], np.uint8)   # 0 is not a 1-based index
    ok = np.array([1, 2], np.uint8)
    assert lib.lnt_mex_sparse_change_linidx(keys.ctypes.data, 3, 2, bad.ctypes.data, ok.ctypes.data,
                                            dims.ctypes.data) == 3
    assert lib.lnt_mex_sparse_permute(vals.ctypes.data, keys.ctypes.data, 3, 2, ok.ctypes.data, zero.ctypes.data,
                                      dims.ctypes.data) == 3
    neg = np.array([3, -1, 2], np.int64)
    assert lib.lnt_mex_sparse_sort(vals.ctypes.data, neg.ctypes.data, 3) == 1
    cv, ck, nc = C.c_void_p(), C.c_void_p(), C.c_size_t()
    d3 = np.array([4, 5, 1], np.int64)
    e3 = np.array([6, 2, 1], np.int64)   # rows(B) != cols(A)
    args = (vals.ctypes.data, keys.ctypes.data, 3, d3.ctypes.data, vals.ctypes.data, keys.ctypes.data, 3)
    assert lib.lnt_mex_sparselattice_mult(*args, d3.ctypes.data, 5, L.HostAlloc(), C.byref(cv), C.byref(ck),
                                          C.byref(nc)) == 8   # mtt_times: the reference computes nothing
    assert lib.lnt_mex_sparselattice_mult(*args, e3.ctypes.data, 0, L.HostAlloc(), C.byref(cv), C.byref(ck),
                                          C.byref(nc)) == 2
    B = np.ones(12)
    assert lib.lnt_mex_sparse_denselattice_mult(vals.ctypes.data, keys.ctypes.data, 3, d3.ctypes.data,
                                                B.ctypes.data, e3.ctypes.data, 0, L.HostAlloc(), C.byref(cv), C.byref(ck),
                                                C.byref(nc)) == 2


def test_dense_permute_checks_arguments_without_gpu():
    lib = L.lib()
    d = np.array([3, 4], np.int64)
    assert lib.lnt_dense_permute(None, None, 2, d.ctypes.data, np.array([1, 1], np.int32).ctypes.data, None) == 3
    assert lib.lnt_dense_permute(None, None, 2, np.array([3, 0], np.int64).ctypes.data,
                                 np.array([1, 0], np.int32).ctypes.data, None) == 2
