"""The allocation-free sort entry point (lnt_sort_pairs_noalloc), for callers
that cannot call cudaMalloc: loops that must not synchronise the device on an
allocation, and plugins or foreign-function hosts with no device allocator to
hand over a workspace.  Collected last on purpose.

Called straight through the C ABI: calls in a row on different inputs, each
compared with lnt_sort_pairs on the same input (both sorts are stable, so the
results must be identical), covering an even and an odd number of digit
passes and the copy-only case, plus the size and overlap limits."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PAIRS = 262144  # LNT_SORT_NOALLOC_MAX_PAIRS in include/lnt.h


def _sort_reference(L, torch, k, v, max_key):
    """The existing entry point, lnt_sort_pairs, with a torch-allocated workspace."""
    ok, ov = torch.empty_like(k), torch.empty_like(v)
    nb = C.c_size_t(0)
    assert L.lib().lnt_sort_pairs_workspace(k.numel(), max_key, C.byref(nb)) == 0
    ws = torch.empty(nb.value, dtype=torch.uint8, device=k.device)
    st = L.lib().lnt_sort_pairs(C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()), C.c_void_p(ok.data_ptr()),
                                C.c_void_p(ov.data_ptr()), k.numel(), max_key, C.c_void_p(ws.data_ptr()),
                                nb.value, None)
    assert st == 0
    return ok, ov


def _sort_noalloc(L, torch, k, v, max_key):
    ok, ov = torch.empty_like(k), torch.empty_like(v)
    st = L.lib().lnt_sort_pairs_noalloc(C.c_void_p(k.data_ptr()), C.c_void_p(v.data_ptr()),
                                        C.c_void_p(ok.data_ptr()), C.c_void_p(ov.data_ptr()), k.numel(), max_key,
                                        None)
    assert st == 0, st
    return ok, ov


def test_noalloc_sort_matches_sort_pairs_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import libnt_b200 as L
    rng = np.random.default_rng(2024)
    # calls in a row, different sizes and key widths: an even number of digit
    # passes (36 and 63-bit keys), an odd number (24-bit keys: the first pass
    # writes the caller's output), and max_key 1 (nothing to sort: a copy)
    cases = [(MAX_PAIRS, 2 ** 36), (100003, 2 ** 63), (MAX_PAIRS - 5, 2 ** 24), (4097, 1)]
    for n, max_key in cases:
        keys = rng.integers(0, max_key, n, dtype=np.uint64) if max_key > 1 else np.zeros(n, np.uint64)
        keys[: n // 4] = keys[n // 2]  # duplicates: stability is part of the contract
        vals = rng.standard_normal(n)
        k = torch.from_numpy(keys.view(np.int64)).cuda()
        v = torch.from_numpy(vals).cuda()
        rk, rv = _sort_reference(L, torch, k, v, max_key)
        nk, nv = _sort_noalloc(L, torch, k, v, max_key)
        torch.cuda.synchronize()
        assert torch.equal(nk, rk)
        assert torch.equal(nv, rv)
    assert L.device_status() == 0


def test_noalloc_sort_limits():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import libnt_b200 as L
    buf = torch.zeros(64, dtype=torch.int64, device="cuda")
    at = lambda i: C.c_void_p(buf.data_ptr() + 8 * i)  # noqa: E731
    f = L.lib().lnt_sort_pairs_noalloc
    # too many pairs (separate, non-overlapping buffers): rejected before any device work
    big = [torch.zeros(MAX_PAIRS + 1, dtype=torch.int64, device="cuda") for _ in range(4)]
    assert f(*[C.c_void_p(t.data_ptr()) for t in big], MAX_PAIRS + 1, 2 ** 36, None) == 8
    # 8 pairs each at elements 0 (keys in), 8 (vals in), 16 (keys out), 24 (vals out): accepted
    assert f(at(0), at(8), at(16), at(24), 8, 2 ** 36, None) == 0
    # any output range sharing bytes with an input range or the other output: rejected
    assert f(at(0), at(8), at(0), at(24), 8, 2 ** 36, None) == 1    # keys out == keys in
    assert f(at(0), at(8), at(4), at(24), 8, 2 ** 36, None) == 1    # keys out overlaps keys in
    assert f(at(0), at(8), at(16), at(12), 8, 2 ** 36, None) == 1   # vals out overlaps vals in
    assert f(at(0), at(8), at(12), at(24), 8, 2 ** 36, None) == 1   # keys out overlaps vals in
    assert f(at(0), at(8), at(16), at(20), 8, 2 ** 36, None) == 1   # the outputs overlap
    assert f(at(0), at(8), None, at(24), 8, 2 ** 36, None) == 1     # null output
    torch.cuda.synchronize()
    assert L.device_status() == 0
