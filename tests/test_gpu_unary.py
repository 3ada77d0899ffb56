"""GPU parity of the unary contraction / attraction (contract_attract, the
reference's SparseMIABase.h:1913-2053) through the C ABI against the oracle:
output keys, their order and the sorted flag bit-exact, values within
1e-12 * sum|terms| per output key."""
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


def run_case(cuda, torch, rng, labels, dims, n, vals=None, keys=None):
    total = int(np.prod(dims))
    if keys is None:
        keys = rng.choice(total, size=min(n, total), replace=False).astype(np.uint64)
    if vals is None:
        vals = rng.uniform(-1, 1, keys.size)
    m = oracle.SparseMIA(list(dims), keys, vals, sorted=False)
    o = oracle.unary_orders(labels)
    ref = m.copy()
    c = oracle.contract_attract(ref, o["contract"], o["contract_part"], o["attract"], o["attract_part"])
    mabs = m.copy()
    mabs.vals = np.abs(mabs.vals)
    cabs = oracle.contract_attract(mabs, o["contract"], o["contract_part"], o["attract"], o["attract_part"])
    # the device call takes the operand already sorted under [contract, attract, other]
    sdims = [dims[q] for q in ref.seq]
    k, v, flag = cuda.contract_attract(to_dev(ref.keys, torch), to_dev(ref.vals, torch), sdims, o["contract_part"],
                                       o["attract_part"])
    np.testing.assert_array_equal(to_host(k, np.uint64), c.keys)
    assert flag == c.sorted
    abs_sum = dict(zip(cabs.keys.tolist(), cabs.vals.tolist()))
    assert rel_ok(to_host(v), c.vals, np.array([abs_sum.get(x, 0.0) for x in c.keys.tolist()]))
    assert cuda.device_status() == 0
    return c


@pytest.mark.parametrize("labels,dims,n", [
    (["i", "j", "i", "j", "k"], [4, 3, 4, 3, 5], 500),         # double trace
    (["!i", "j", "!i", "k", "j"], [6, 5, 6, 7, 5], 3000),      # attraction of i, contraction of j
    (["!i", "k", "!i"], [4, 5, 4], 60),                        # attraction only: unsorted emission
    (["i", "k", "i", "!m", "!m"], [30, 20, 30, 9, 9], 40000),
    (["j", "i", "i", "j"], [8, 9, 9, 8], 2000),                # full contraction to one entry
])
def test_contract_attract_matches_oracle(cuda, torch, rng, labels, dims, n):
    run_case(cuda, torch, rng, labels, dims, n)


def test_contract_attract_large(cuda, torch, rng):
    """300 000 entries, so the fold and the scan span many tiles."""
    run_case(cuda, torch, rng, ["i", "i", "k"], [600, 600, 50], 300_000)


def test_contract_attract_zero_sums_dropped(cuda, torch, rng):
    keys = np.array([0, 3, 10, 16, 21], np.uint64)    # (0,0,0) (1,1,0) (0,1,2) (0,0,4) (1,0,5) in 2x2x6
    vals = np.array([1.0, -1.0, 5.0, 0.0, 2.0])
    c = run_case(cuda, torch, rng, ["i", "i", "k"], [2, 2, 6], 0, vals=vals, keys=keys)
    assert c.keys.size == 0   # k=0 cancels, k=4 sums to zero, the rest are off the diagonal


def test_contract_attract_bad_args(cuda, torch):
    import ctypes as C

    import libnt_b200 as L
    z = to_dev(np.zeros(1, np.uint64), torch)
    zv = to_dev(np.zeros(1), torch)
    sd = np.array([3, 4, 5], np.int64)   # a contraction set over different extents
    cp = np.array([2], np.int32)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = L.workspace(1 << 20)
    st = L.lib().lnt_contract_attract(C.c_void_p(z.data_ptr()), C.c_void_p(zv.data_ptr()), 1, 3, sd.ctypes.data, 1,
                                      cp.ctypes.data, 0, None, C.c_void_p(z.data_ptr()), C.c_void_p(zv.data_ptr()),
                                      C.c_void_p(cnt.data_ptr()), None, C.c_void_p(ws.data_ptr()), ws.numel(), None)
    assert st == 2
