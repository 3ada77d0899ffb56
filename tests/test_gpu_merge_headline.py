"""GPU parity of the sparse merge under permutation at the benchmarked size,
and of the stream-ordered merge captured in a CUDA graph.

c(i,j,k,l) = a(i,j,k,l) + b(l,k,j,i) with both operands unsorted is the
reference's SparseMIA::sortMerge (SparseMIA.h:833-887): A (the operand that
is not larger) is re-keyed into B's order {3,2,1,0}, both are concatenated,
sorted, and equal keys are folded by collect_duplicates (SparseMIA.h:636-665,
with its rule that a key whose addends are all exactly zero is dropped unless
it sits at position 0).  At 2 x 2^26 pairs over 512^4 the library takes its
bucketed path with 2^15 buckets (a 7-bit first digit pass), a geometry that
smaller cases do not reach.
"""
import numpy as np
import pytest

import oracle
from conftest import rel_ok
from test_gpu_sort import to_dev, to_host

pytestmark = pytest.mark.gpu

DIMS = [512] * 4
MAX_KEY = 512 ** 4


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def _operands(rng, n, zero_frac):
    ak = rng.integers(0, MAX_KEY, n, dtype=np.uint64)
    bk = rng.integers(0, MAX_KEY, n, dtype=np.uint64)
    av = rng.uniform(-1, 1, n)
    bv = rng.uniform(-1, 1, n)
    av[rng.random(n) < zero_frac] = 0.0
    bv[rng.random(n) < zero_frac] = 0.0
    return ak, av, bk, bv


def _expected(ak, av, bk, bv):
    """sortMerge on the host: the reference's own re-key and MSD radix sort when
    they were compiled (oracle/_ref), else the restatement; then the restated
    collect_duplicates with the per-key sum of |addends| (the value tolerance)."""
    if oracle.ref_available():
        ka = oracle.ref_rekey(ak, DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
        sk, sv = oracle.ref_radix_sort(np.concatenate([ka, bk]), np.concatenate([av, bv]), MAX_KEY)
    else:
        ka = oracle.rekey(ak, DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
        sk, sv = oracle.sort_pairs(np.concatenate([ka, bk]), np.concatenate([av, bv]))
    return oracle.collect_duplicates(sk, sv, with_abs=True)


def test_sort_merge_full_size_matches_oracle(cuda, torch):
    """2 x 2^26 pairs, 512^4, 5% exact zeros, the smallest key present only with
    zero addends (kept: position 0) and one more all-zero key (dropped).
    Keys bit-exact; values within 1e-12 of the sum of |addends| per key (the
    reference's sort is unstable, so its summation order within a key is not
    defined)."""
    import libnt_b200 as L
    rng = np.random.default_rng(2026)
    n = 1 << 26
    ak, av, bk, bv = _operands(rng, n, 0.05)
    # Key 0 (the origin under every mode order) and key 12345 of B's order get
    # zero addends only, from both operands.  With equal extents, reversing the
    # mode order is its own inverse, so A's key for a B-order key k is rekey(k).
    k_zero = 12345
    a_k_zero = oracle.rekey(np.array([k_zero], np.uint64), DIMS, [0, 1, 2, 3], [3, 2, 1, 0])[0]
    ka_now = oracle.rekey(ak, DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
    ak[(ka_now == 0) | (ka_now == k_zero)] = 7  # random draws of these keys move elsewhere
    bk[(bk == 0) | (bk == k_zero)] = 7
    ak[:3], av[:3] = 0, 0.0
    bk[:2], bv[:2] = 0, 0.0
    ak[3:6], av[3:6] = a_k_zero, 0.0
    bk[2:4], bv[2:4] = k_zero, 0.0
    spec = L.RekeySpec.make(DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
    k, v = cuda.sort_reduce(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch),
                            max_key=MAX_KEY, a_rekey=spec)
    assert cuda.device_status() == 0
    gk, gv = to_host(k, np.uint64), to_host(v)
    del k, v
    torch.cuda.empty_cache()
    ek, ev, ea = _expected(ak, av, bk, bv)
    assert ek[0] == 0 and ev[0] == 0.0  # position 0 kept although all its addends are zero
    assert not np.any(ek == k_zero)    # an all-zero key elsewhere is dropped
    np.testing.assert_array_equal(gk, ek)
    assert rel_ok(gv, ev, ea)


def _graph_case(rng, skewed):
    n = 1 << 21
    ak, av, bk, bv = _operands(rng, n, 0.05)
    if skewed:  # 1/8 of A on one key: its bucket exceeds a CTA, so the LSD path runs
        ak[: n // 8] = ak[0]
    return ak, av, bk, bv


@pytest.mark.parametrize("skewed", [False, True])
def test_sort_merge_graph_capture_matches_oracle(cuda, torch, skewed):
    """One lnt_sort_reduce captured into a CUDA graph and replayed twice on new
    inputs: the bucket-size decision is taken on the device, so the call has
    no host synchronisation and captures whole, for uniform keys (bucketed
    path) and for a bucket that overflows (the gated LSD path)."""
    import libnt_b200 as L
    rng = np.random.default_rng(77 + int(skewed))
    ak, av, bk, bv = _graph_case(rng, skewed)
    dk = [to_dev(x, torch) for x in (ak, av, bk, bv)]
    n = ak.size + bk.size
    spec = L.RekeySpec.make(DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
    ok = torch.empty(n, dtype=torch.int64, device="cuda")
    ov = torch.empty(n, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = L.workspace(L.sort_reduce_workspace(ak.size, bk.size, MAX_KEY))

    def call():
        L.sort_reduce(dk[0], dk[1], dk[2], dk[3], max_key=MAX_KEY, a_rekey=spec, out_keys=ok, out_vals=ov,
                      count=cnt, ws=ws, sync=False)

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        call()  # warm-up outside the capture (function attributes, occupancy queries)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        call()
    for rep in range(2):
        if rep:  # new inputs in the captured buffers
            ak, av, bk, bv = _graph_case(rng, skewed)
            for d, h in zip(dk, (ak, av, bk, bv)):
                d.copy_(to_dev(h, torch))
        ok.fill_(-1)
        g.replay()
        torch.cuda.synchronize()
        m = int(cnt.item())
        ek, ev, ea = _expected(ak, av, bk, bv)
        np.testing.assert_array_equal(to_host(ok[:m], np.uint64), ek)
        assert rel_ok(to_host(ov[:m]), ev, ea)
    assert cuda.device_status() == 0
    del g


def test_sort_merge_non_power_of_two_full_buckets(cuda, torch):
    """2 x 3 x 2^24 pairs (a size that is not a power of two): 2^15 buckets of
    3072 pairs on average, so the bucketed path (7-bit first pass) completes
    instead of handing the call to the LSD path; the bucket kernel does the
    work (its time dwarfs the gated fallback's), and the result matches the
    oracle."""
    import libnt_b200 as L
    rng = np.random.default_rng(77)
    n = 3 << 24
    ak, av, bk, bv = _operands(rng, n, 0.05)
    spec = L.RekeySpec.make(DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
    L.profile_reset()
    L.profile_enable(True)
    k, v = cuda.sort_reduce(to_dev(ak, torch), to_dev(av, torch), to_dev(bk, torch), to_dev(bv, torch),
                            max_key=MAX_KEY, a_rekey=spec)
    torch.cuda.synchronize()
    L.profile_enable(False)
    bucket_ms = L.profile_query("bucket_sort_collect")[0]
    fallback_ms = L.profile_query("collect_fallback")[0]
    L.profile_reset()
    assert cuda.device_status() == 0
    assert bucket_ms > 10 * fallback_ms, (bucket_ms, fallback_ms)
    gk, gv = to_host(k, np.uint64), to_host(v)
    del k, v
    torch.cuda.empty_cache()
    ek, ev, ea = _expected(ak, av, bk, bv)
    np.testing.assert_array_equal(gk, ek)
    assert rel_ok(gv, ev, ea)
