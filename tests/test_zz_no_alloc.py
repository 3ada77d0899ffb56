"""The allocation-free sort entry point (lnt_sort_pairs_noalloc), for callers
that cannot call cudaMalloc (graph capture, allocation-free loops, plugins
without an allocator).  Collected last on purpose.

Called straight through the C ABI: two calls in a row on different inputs,
each compared with lnt_sort_pairs on the same input (both sorts are stable,
so the results must be identical), plus the size and aliasing limits."""
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
    cases = [(MAX_PAIRS, 2 ** 36), (100003, 2 ** 63)]  # two calls in a row, different sizes and key widths
    for n, max_key in cases:
        keys = rng.integers(0, max_key, n, dtype=np.uint64)
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
    k = torch.zeros(8, dtype=torch.int64, device="cuda")
    v = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(k.data_ptr())
    q = C.c_void_p(v.data_ptr())
    # too many pairs: rejected before any device work
    assert L.lib().lnt_sort_pairs_noalloc(p, q, p, q, MAX_PAIRS + 1, 2 ** 36, None) == 8
    # output aliasing the input: rejected
    assert L.lib().lnt_sort_pairs_noalloc(p, q, p, q, 8, 2 ** 36, None) == 1
