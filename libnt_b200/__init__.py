"""libnt_b200 — B200 (sm_100a) implementation of the LibNT / LibMIA sparse and
dense multi-index-array hot path.

The product is the CUDA library ``liblnt_cuda.so`` (C ABI in ``include/lnt.h``)
and the header-only C++ front end under ``libnt_b200/include/lnt/``.  This
Python module is plumbing: it loads the library with ctypes and calls it on
torch-allocated device buffers and torch's current CUDA stream.  There is no
CPU fallback: if the library is missing, importing raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "liblnt_cuda.so"
MAX_ORDER = 16

STATUS = {
    0: "ok", 1: "bad argument", 2: "dimension mismatch", 3: "sequence is not a permutation",
    4: "dimensionality does not fit in 63 bits", 5: "workspace too small", 6: "device-side wait expired",
    7: "CUDA error", 8: "unsupported request",
}


class LntError(RuntimeError):
    """A non-zero lnt_status returned by the CUDA library."""

    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: lnt status {status} ({STATUS.get(status, 'unknown')})")


class Lattice(C.Structure):
    """lnt_lattice (include/lnt.h)."""
    _fields_ = [("keys", C.c_void_p), ("vals", C.c_void_p), ("nnz", C.c_uint64), ("rows", C.c_int64),
                ("cols", C.c_int64), ("tabs", C.c_int64)]

    @classmethod
    def of(cls, keys, vals, rows, cols, tabs=1) -> "Lattice":
        return cls(keys.data_ptr() if keys.numel() else None, vals.data_ptr() if vals.numel() else None,
                   keys.numel(), rows, cols, tabs)


class RekeySpec(C.Structure):
    """lnt_rekey_spec (include/lnt.h)."""
    _fields_ = [("order", C.c_int32), ("cur_seq", C.c_int32 * MAX_ORDER), ("new_seq", C.c_int32 * MAX_ORDER),
                ("dims", C.c_int64 * MAX_ORDER)]

    @classmethod
    def make(cls, dims, cur_seq, new_seq) -> "RekeySpec":
        s = cls()
        s.order = len(dims)
        for i, (d, c, n) in enumerate(zip(dims, cur_seq, new_seq)):
            s.dims[i], s.cur_seq[i], s.new_seq[i] = int(d), int(c), int(n)
        return s


_vp = C.c_void_p
_sz = C.c_size_t
# lnt_host_alloc (include/lnt_mex.h): void* (*)(size_t); HostAlloc() is the NULL
# pointer (the gateway then uses malloc)
HostAlloc = C.CFUNCTYPE(C.c_void_p, C.c_size_t)
_pvp = C.POINTER(C.c_void_p)
_psz = C.POINTER(C.c_size_t)
_MEX_OUT = [HostAlloc, _pvp, _pvp, _psz]
_SIGS = {
    "lnt_mex_sparse_sort": ([_vp, _vp, _sz], C.c_int),
    "lnt_mex_sparse_change_linidx": ([_vp, _sz, C.c_int, _vp, _vp, _vp], C.c_int),
    "lnt_mex_sparse_permute": ([_vp, _vp, _sz, C.c_int, _vp, _vp, _vp], C.c_int),
    "lnt_mex_sparse_merge": ([_vp, _vp, _sz, _vp, _vp, _sz, C.c_int] + _MEX_OUT, C.c_int),
    "lnt_mex_sparselattice_mult": ([_vp, _vp, _sz, _vp, _vp, _vp, _sz, _vp, C.c_int] + _MEX_OUT, C.c_int),
    "lnt_mex_sparse_denselattice_mult": ([_vp, _vp, _sz, _vp, _vp, _vp, C.c_int] + _MEX_OUT, C.c_int),
    "lnt_status_string": ([C.c_int], C.c_char_p),
    "lnt_version": ([], C.c_int),
    "lnt_launch_count": ([], C.c_uint64),
    "lnt_device_status": ([C.c_int, _vp, C.POINTER(C.c_uint32)], C.c_int),
    "lnt_set_spin_limit": ([C.c_uint32], C.c_int),
    "lnt_diag_expired_wait": ([_vp], C.c_int),
    "lnt_profile_enable": ([C.c_int], C.c_int),
    "lnt_profile_reset": ([], C.c_int),
    "lnt_profile_query": ([C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64)], C.c_int),
    "lnt_rekey": ([_vp, _vp, _sz, C.c_int, _vp, _vp, _vp, _vp], C.c_int),
    "lnt_sort_variant_count": ([], C.c_int),
    "lnt_sort_variant": ([C.c_int] + [C.POINTER(C.c_int)] * 4, C.c_int),
    "lnt_sort_pairs_workspace": ([_sz, C.c_uint64, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_sort_pairs_noalloc": ([_vp, _vp, _vp, _vp, _sz, C.c_uint64, _vp], C.c_int),
    "lnt_sort_pairs": ([_vp, _vp, _vp, _vp, _sz, C.c_uint64, _vp, _sz, _vp], C.c_int),
    "lnt_collect_duplicates_workspace": ([_sz, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_collect_duplicates": ([_vp, _vp, _sz, C.c_int, _vp, _vp, _vp, _vp, _sz, _vp], C.c_int),
    "lnt_sort_reduce_workspace": ([_sz, _sz, C.c_uint64, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_sort_reduce": ([_vp, _vp, _sz, C.POINTER(RekeySpec), _vp, _vp, _sz, C.POINTER(RekeySpec), C.c_double,
                         C.c_uint64, C.c_int, _vp, _vp, _vp, _vp, _sz, _vp], C.c_int),
    "lnt_merge_sorted_workspace": ([_sz, _sz, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_merge_sorted": ([_vp, _vp, _sz, _vp, _vp, _sz, C.c_int, _vp, _vp, _vp, _vp, _sz, _vp], C.c_int),
    "lnt_permute_sort_workspace": ([_sz, C.c_uint64, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_permute_sort": ([_vp, _vp, _sz, C.POINTER(RekeySpec), _vp, _vp, C.c_uint64, _vp, _sz, _vp], C.c_int),
    "lnt_lattice_mult_plan_workspace": ([C.POINTER(Lattice), C.POINTER(Lattice), C.POINTER(C.c_size_t)], C.c_int),
    "lnt_lattice_mult_plan": ([C.POINTER(Lattice), C.POINTER(Lattice), _vp, _sz, _vp, _vp], C.c_int),
    "lnt_lattice_mult_workspace": ([C.POINTER(Lattice), C.POINTER(Lattice), C.c_uint64, C.POINTER(C.c_size_t)],
                                   C.c_int),
    "lnt_lattice_mult": ([C.POINTER(Lattice), C.POINTER(Lattice), _vp, C.c_uint64, _vp, _sz, _vp, _vp, _vp, _vp],
                         C.c_int),
    "lnt_contract_attract_workspace": ([_sz, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_contract_attract": ([_vp, _vp, _sz, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _sz,
                              _vp], C.c_int),
    "lnt_nolattice_mult_workspace": ([C.POINTER(Lattice), C.POINTER(Lattice), C.POINTER(C.c_size_t)], C.c_int),
    "lnt_nolattice_mult_count": ([C.POINTER(Lattice), C.POINTER(Lattice), _vp, _sz, _vp, _vp], C.c_int),
    "lnt_nolattice_mult": ([C.POINTER(Lattice), C.POINTER(Lattice), C.c_uint64, _vp, _sz, _vp, _vp, _vp], C.c_int),
    "lnt_dense_permute": ([_vp, _vp, C.c_int, _vp, _vp, _vp], C.c_int),
    "lnt_sparse_dense_mult_workspace": ([C.POINTER(Lattice), C.c_int64, C.c_int, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_sparse_dense_mult_count": ([C.POINTER(Lattice), C.c_int64, C.c_int, _vp, _sz, _vp, _vp], C.c_int),
    "lnt_sparse_dense_mult": ([_vp, C.POINTER(Lattice), C.c_int64, C.c_int, _vp, _sz, _vp, _vp, _vp], C.c_int),
    "lnt_batched_workspace": ([C.c_int, _vp, _vp, _vp, C.POINTER(C.c_size_t), C.POINTER(C.c_uint64)], C.c_int),
    "lnt_batched_prepare": ([C.c_int, _vp, _vp, _vp, _vp, _sz, _vp], C.c_int),
    "lnt_batched_lattice_mult": ([C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp, _vp], C.c_int),
    "lnt_batched_contract_workspace": ([C.c_int, _vp, _vp, _vp, C.POINTER(C.c_size_t), C.POINTER(C.c_uint64)],
                                       C.c_int),
    "lnt_batched_contract_prepare": ([C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp], C.c_int),
    "lnt_batched_contract": ([C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp, _vp], C.c_int),
    "lnt_dense_fp64_workspace": ([C.POINTER(C.c_size_t)], C.c_int),
    "lnt_dense_lattice_mult_fp64": ([_vp, _vp, _vp, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _vp, _sz, _vp],
                                    C.c_int),
    "lnt_dense_split_workspace": ([C.c_int64, C.c_int64, C.c_int64, C.c_int, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_dense_lattice_mult_split": ([_vp, _vp, _vp, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, _vp,
                                      _sz, _vp], C.c_int),
    "lnt_dense_crt_workspace": ([C.c_int64, C.c_int64, C.c_int64, C.c_int, C.POINTER(C.c_size_t)], C.c_int),
    "lnt_dense_crt_moduli": ([_vp, _vp, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_double, _vp, _sz,
                              C.POINTER(C.c_int), _vp], C.c_int),
    "lnt_dense_lattice_mult_crt": ([_vp, _vp, _vp, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, _vp,
                                    _sz, _vp], C.c_int),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m libnt_b200.build` "
                              "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
        env = os.environ.get("LNT_SPIN_LIMIT")
        if env:
            set_spin_limit(int(env))
    return _lib


def declared_symbols() -> list[str]:
    return list(_SIGS)


def _check(st: int, what: str):
    if st != 0:
        raise LntError(st, what)


# ---------------------------------------------------------------------------
# torch plumbing
# ---------------------------------------------------------------------------

def _torch():
    import torch
    return torch


def _stream():
    return _vp(_torch().cuda.current_stream().cuda_stream)


def _ptr(t):
    return _vp(t.data_ptr()) if t is not None else None


def _dev(t):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t


def workspace(nbytes: int, device=None):
    torch = _torch()
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device or "cuda")


def _arr(vals, dtype):
    return (dtype * len(vals))(*[int(v) for v in vals])


def launch_count() -> int:
    return int(lib().lnt_launch_count())


def device_status(clear: bool = True) -> int:
    word = C.c_uint32(0)
    st = lib().lnt_device_status(int(clear), _stream(), C.byref(word))
    if st not in (0, 6):
        _check(st, "lnt_device_status")
    return int(word.value)


def set_spin_limit(polls: int = 0):
    """Poll budget of every bounded device wait on the current device (0 = default)."""
    _check(lib().lnt_set_spin_limit(int(polls)), "lnt_set_spin_limit")


def diag_expired_wait():
    """Runs one look-back wait on a state nothing publishes (lnt_diag_expired_wait)."""
    _check(lib().lnt_diag_expired_wait(_stream()), "lnt_diag_expired_wait")


def profile_enable(on: bool = True):
    _check(lib().lnt_profile_enable(int(bool(on))), "lnt_profile_enable")


def profile_reset():
    _check(lib().lnt_profile_reset(), "lnt_profile_reset")


def profile_query(kernel: str):
    """(total device ms, launches) of a kernel since the last reset."""
    t = C.c_double(0)
    n = C.c_uint64(0)
    _check(lib().lnt_profile_query(kernel.encode(), C.byref(t), C.byref(n)), "lnt_profile_query")
    return t.value, int(n.value)


def rekey(keys, dims, cur_seq, new_seq, out=None):
    """Re-linearise int64/uint64 keys (device tensor) from cur_seq to new_seq."""
    torch = _torch()
    _dev(keys)
    out = torch.empty_like(keys) if out is None else _dev(out)
    n = len(dims)
    st = lib().lnt_rekey(_ptr(keys), _ptr(out), keys.numel(), n, _arr(dims, C.c_int64), _arr(cur_seq, C.c_int32),
                         _arr(new_seq, C.c_int32), _stream())
    _check(st, "lnt_rekey")
    return out


def sort_pairs_workspace(n: int, max_key: int) -> int:
    nb = C.c_size_t(0)
    _check(lib().lnt_sort_pairs_workspace(n, int(max_key), C.byref(nb)), "lnt_sort_pairs_workspace")
    return nb.value


def sort_pairs(keys, vals, max_key: int, out_keys=None, out_vals=None, ws=None):
    """Stable ascending sort by key; returns (keys, vals) (new tensors unless given)."""
    torch = _torch()
    _dev(keys), _dev(vals)
    n = keys.numel()
    ok = torch.empty_like(keys) if out_keys is None else out_keys
    ov = torch.empty_like(vals) if out_vals is None else out_vals
    need = sort_pairs_workspace(n, max_key)
    if ws is None or ws.numel() < need:
        ws = workspace(need, keys.device)
    st = lib().lnt_sort_pairs(_ptr(keys), _ptr(vals), _ptr(ok), _ptr(ov), n, int(max_key), _ptr(ws), ws.numel(),
                              _stream())
    _check(st, "lnt_sort_pairs")
    return ok, ov


def collect_duplicates(keys, vals, skip_zero_heads: bool = True):
    """Fold equal-key runs of key-sorted pairs; returns trimmed (keys, vals)."""
    torch = _torch()
    _dev(keys), _dev(vals)
    n = keys.numel()
    ok = torch.empty_like(keys)
    ov = torch.empty_like(vals)
    cnt = torch.zeros(1, dtype=torch.int64, device=keys.device)
    nb = C.c_size_t(0)
    _check(lib().lnt_collect_duplicates_workspace(n, C.byref(nb)), "lnt_collect_duplicates_workspace")
    ws = workspace(nb.value, keys.device)
    st = lib().lnt_collect_duplicates(_ptr(keys), _ptr(vals), n, int(bool(skip_zero_heads)), _ptr(ok), _ptr(ov),
                                      _ptr(cnt), _ptr(ws), nb.value, _stream())
    _check(st, "lnt_collect_duplicates")
    m = int(cnt.item())
    return ok[:m], ov[:m]


def sort_reduce_workspace(na: int, nb: int, max_key: int) -> int:
    b = C.c_size_t(0)
    _check(lib().lnt_sort_reduce_workspace(na, nb, int(max_key), C.byref(b)), "lnt_sort_reduce_workspace")
    return b.value


def sort_reduce(a_keys, a_vals, b_keys=None, b_vals=None, *, max_key: int, a_rekey: RekeySpec | None = None,
                b_rekey: RekeySpec | None = None, b_scale: float = 1.0, skip_zero_heads: bool = True,
                out_keys=None, out_vals=None, count=None, ws=None, sync: bool = True):
    """Concatenate A and B (each optionally re-keyed, B scaled), sort and
    collect duplicates.  With sync=True returns trimmed (keys, vals); else
    returns (keys, vals, count_tensor) without synchronising."""
    torch = _torch()
    _dev(a_keys), _dev(a_vals)
    na = a_keys.numel()
    nb = b_keys.numel() if b_keys is not None else 0
    n = na + nb
    ok = torch.empty(n, dtype=a_keys.dtype, device=a_keys.device) if out_keys is None else out_keys
    ov = torch.empty(n, dtype=a_vals.dtype, device=a_vals.device) if out_vals is None else out_vals
    cnt = torch.zeros(1, dtype=torch.int64, device=a_keys.device) if count is None else count
    need = sort_reduce_workspace(na, nb, max_key)
    if ws is None or ws.numel() < need:
        ws = workspace(need, a_keys.device)
    st = lib().lnt_sort_reduce(_ptr(a_keys), _ptr(a_vals), na, C.byref(a_rekey) if a_rekey else None,
                               _ptr(b_keys), _ptr(b_vals), nb, C.byref(b_rekey) if b_rekey else None,
                               float(b_scale), int(max_key), int(bool(skip_zero_heads)), _ptr(ok), _ptr(ov),
                               _ptr(cnt), _ptr(ws), ws.numel(), _stream())
    _check(st, "lnt_sort_reduce")
    if not sync:
        return ok, ov, cnt
    m = int(cnt.item())
    return ok[:m], ov[:m]


def merge_sorted(a_keys, a_vals, b_keys, b_vals, op: int = 0, out_keys=None, out_vals=None, count=None,
                 ws=None, sync: bool = True):
    """Scan merge of two key-sorted operands (op 0 = +, 1 = -)."""
    torch = _torch()
    na, nb = a_keys.numel(), b_keys.numel()
    dev = a_keys.device
    ok = torch.empty(na + nb, dtype=torch.int64, device=dev) if out_keys is None else out_keys
    ov = torch.empty(na + nb, dtype=torch.float64, device=dev) if out_vals is None else out_vals
    cnt = torch.zeros(1, dtype=torch.int64, device=dev) if count is None else count
    b = C.c_size_t(0)
    _check(lib().lnt_merge_sorted_workspace(na, nb, C.byref(b)), "lnt_merge_sorted_workspace")
    if ws is None or ws.numel() < b.value:
        ws = workspace(b.value, dev)
    st = lib().lnt_merge_sorted(_ptr(a_keys), _ptr(a_vals), na, _ptr(b_keys), _ptr(b_vals), nb, int(op), _ptr(ok),
                                _ptr(ov), _ptr(cnt), _ptr(ws), ws.numel(), _stream())
    _check(st, "lnt_merge_sorted")
    if not sync:
        return ok, ov, cnt
    m = int(cnt.item())
    return ok[:m], ov[:m]


def permute_sort_workspace(n: int, max_key: int) -> int:
    b = C.c_size_t(0)
    _check(lib().lnt_permute_sort_workspace(n, int(max_key), C.byref(b)), "lnt_permute_sort_workspace")
    return b.value


def permute_sort(keys, vals, *, max_key: int, rekey: RekeySpec | None = None, out_keys=None, out_vals=None,
                 ws=None):
    """Re-key (optional) and stable sort, out of place."""
    torch = _torch()
    n = keys.numel()
    ok = torch.empty_like(keys) if out_keys is None else out_keys
    ov = torch.empty_like(vals) if out_vals is None else out_vals
    need = permute_sort_workspace(n, max_key)
    if ws is None or ws.numel() < need:
        ws = workspace(need, keys.device)
    st = lib().lnt_permute_sort(_ptr(keys), _ptr(vals), n, C.byref(rekey) if rekey else None, _ptr(ok), _ptr(ov),
                                int(max_key), _ptr(ws), ws.numel(), _stream())
    _check(st, "lnt_permute_sort")
    return ok, ov


def lattice_mult(a_keys, a_vals, b_keys, b_vals, h: int, w: int, wB: int, d: int = 1):
    """Sparse lattice product (column-major keys, both key-sorted); returns
    trimmed (keys, vals) of C (h x wB x d) and the product count."""
    torch = _torch()
    A = Lattice.of(a_keys, a_vals, h, w, d)
    B = Lattice.of(b_keys, b_vals, w, wB, d)
    dev = a_keys.device
    b = C.c_size_t(0)
    _check(lib().lnt_lattice_mult_plan_workspace(C.byref(A), C.byref(B), C.byref(b)), "lnt_lattice_mult_plan_workspace")
    plan = workspace(b.value, dev)
    counts = torch.zeros(2, dtype=torch.int64, device=dev)
    _check(lib().lnt_lattice_mult_plan(C.byref(A), C.byref(B), _ptr(plan), plan.numel(), _ptr(counts), _stream()),
           "lnt_lattice_mult_plan")
    products, cap = (int(x) for x in counts.tolist())
    _check(lib().lnt_lattice_mult_workspace(C.byref(A), C.byref(B), products, C.byref(b)),
           "lnt_lattice_mult_workspace")
    ws = workspace(b.value, dev)
    ck = torch.empty(max(cap, 1), dtype=torch.int64, device=dev)
    cv = torch.empty(max(cap, 1), dtype=torch.float64, device=dev)
    nc = torch.zeros(1, dtype=torch.int64, device=dev)
    _check(lib().lnt_lattice_mult(C.byref(A), C.byref(B), _ptr(plan), products, _ptr(ws), ws.numel(), _ptr(ck),
                                  _ptr(cv), _ptr(nc), _stream()), "lnt_lattice_mult")
    m = int(nc.item())
    return ck[:m], cv[:m], products


def nolattice_mult(a_keys, a_vals, b_keys, b_vals, h: int, wB: int, d: int = 1):
    """Product with no contracted index (noLatticeMult): A key-sorted as an
    h x 1 x d lattice, B as 1 x wB x d; returns (keys, vals) of C (h x wB x d),
    ascending, equal keys not folded."""
    torch = _torch()
    A = Lattice.of(a_keys, a_vals, h, 1, d)
    B = Lattice.of(b_keys, b_vals, 1, wB, d)
    dev = a_keys.device
    b = C.c_size_t(0)
    _check(lib().lnt_nolattice_mult_workspace(C.byref(A), C.byref(B), C.byref(b)), "lnt_nolattice_mult_workspace")
    ws = workspace(b.value, dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    _check(lib().lnt_nolattice_mult_count(C.byref(A), C.byref(B), _ptr(ws), ws.numel(), _ptr(cnt), _stream()),
           "lnt_nolattice_mult_count")
    n = int(cnt.item())
    ck = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    cv = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    _check(lib().lnt_nolattice_mult(C.byref(A), C.byref(B), n, _ptr(ws), ws.numel(), _ptr(ck), _ptr(cv), _stream()),
           "lnt_nolattice_mult")
    return ck[:n], cv[:n]


def sparse_dense_mult(dense, s_keys, s_vals, rows: int, cols: int, tabs: int, other: int, dense_first: bool):
    """Mixed lattice product (SparseDenseLatticeMultMex).  dense_first: C = A * S
    with A (other x rows x tabs) and S column-major key-sorted; else C = S * B
    with S row-major key-sorted (col + cols (row + rows tab)) and B (cols x
    other x tabs).  dense: float64 column-major device tensor.  Returns (keys,
    vals) of C, ascending (column-major keys for dense_first, row-major
    lattice keys otherwise)."""
    torch = _torch()
    _dev(dense)
    S = Lattice.of(s_keys, s_vals, rows, cols, tabs)
    dev = s_keys.device
    df = 1 if dense_first else 0
    b = C.c_size_t(0)
    _check(lib().lnt_sparse_dense_mult_workspace(C.byref(S), other, df, C.byref(b)),
           "lnt_sparse_dense_mult_workspace")
    ws = workspace(b.value, dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    _check(lib().lnt_sparse_dense_mult_count(C.byref(S), other, df, _ptr(ws), ws.numel(), _ptr(cnt), _stream()),
           "lnt_sparse_dense_mult_count")
    n = int(cnt.item())
    ck = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    cv = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    _check(lib().lnt_sparse_dense_mult(_ptr(dense), C.byref(S), other, df, _ptr(ws), ws.numel(), _ptr(ck), _ptr(cv),
                                       _stream()), "lnt_sparse_dense_mult")
    return ck[:n], cv[:n]


def contract_attract(keys, vals, sdims, con_part, att_part):
    """Unary contraction / attraction of a tensor sorted under [contraction
    modes, attraction modes, other modes] (extents sdims in that order);
    returns (keys, vals, sorted_flag)."""
    torch = _torch()
    _dev(keys), _dev(vals)
    n = keys.numel()
    dev = keys.device
    b = C.c_size_t(0)
    _check(lib().lnt_contract_attract_workspace(n, C.byref(b)), "lnt_contract_attract_workspace")
    ws = workspace(b.value, dev)
    ok = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    ov = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    flag = torch.zeros(1, dtype=torch.int32, device=dev)
    sd = np.ascontiguousarray(sdims, np.int64)
    cp = np.ascontiguousarray(con_part, np.int32)
    ap = np.ascontiguousarray(att_part, np.int32)
    _check(lib().lnt_contract_attract(_ptr(keys), _ptr(vals), n, len(sd), sd.ctypes.data, len(cp), cp.ctypes.data,
                                      len(ap), ap.ctypes.data, _ptr(ok), _ptr(ov), _ptr(cnt), _ptr(flag), _ptr(ws),
                                      ws.numel(), _stream()), "lnt_contract_attract")
    m = int(cnt.item())
    return ok[:m], ov[:m], bool(flag.item())


class Batch:
    """A batch of lattice products on one device (see lnt_batched_* in include/lnt.h).

    dims: int64 array (count, 4) of (h, w, wB, d); a_off / b_off: uint64 (count+1)
    offsets into the concatenated device tensors a_keys/a_vals, b_keys/b_vals.
    Without re-key specs the operands are key-sorted lattices
    (lnt_batched_lattice_mult); with a_rekey / b_rekey (a sequence of count
    RekeySpec, or None for "already in lattice order") they are unsorted tensors
    that the call re-keys and sorts (lnt_batched_contract)."""

    def __init__(self, dims, a_off, b_off, a_keys, a_vals, b_keys, b_vals, a_rekey=None, b_rekey=None):
        torch = _torch()
        self.count = int(len(dims))
        self.dims = np.ascontiguousarray(dims, np.int64)
        self.a_off = np.ascontiguousarray(a_off, np.uint64)
        self.b_off = np.ascontiguousarray(b_off, np.uint64)
        self.tensors = (a_keys, a_vals, b_keys, b_vals)
        self.contract = a_rekey is not None or b_rekey is not None
        pre = "lnt_batched_contract" if self.contract else "lnt_batched"
        dev = a_keys.device
        nb = C.c_size_t(0)
        cap = C.c_uint64(0)
        _check(getattr(lib(), pre + "_workspace")(self.count, self.dims.ctypes.data, self.a_off.ctypes.data,
                                                  self.b_off.ctypes.data, C.byref(nb), C.byref(cap)),
               pre + "_workspace")
        self.ws = workspace(nb.value, dev)
        self.capacity = int(cap.value)
        self.c_keys = torch.empty(max(self.capacity, 1), dtype=torch.int64, device=dev)
        self.c_vals = torch.empty(max(self.capacity, 1), dtype=torch.float64, device=dev)
        self.c_off = torch.zeros(self.count + 1, dtype=torch.int64, device=dev)
        if self.contract:
            specs = []
            for seq in (a_rekey, b_rekey):
                arr = (RekeySpec * self.count)()
                if seq is not None:
                    for p, sp in enumerate(seq):
                        if sp is not None:
                            arr[p] = sp
                specs.append(arr)
            self._specs = specs
            _check(lib().lnt_batched_contract_prepare(self.count, self.dims.ctypes.data, self.a_off.ctypes.data,
                                                      self.b_off.ctypes.data, C.cast(specs[0], _vp),
                                                      C.cast(specs[1], _vp), _ptr(self.ws), self.ws.numel(),
                                                      _stream()), "lnt_batched_contract_prepare")
        else:
            _check(lib().lnt_batched_prepare(self.count, self.dims.ctypes.data, self.a_off.ctypes.data,
                                             self.b_off.ctypes.data, _ptr(self.ws), self.ws.numel(), _stream()),
                   "lnt_batched_prepare")

    def run(self):
        """Enqueue the batched product on the current stream (capturable)."""
        ak, av, bk, bv = self.tensors
        f = lib().lnt_batched_contract if self.contract else lib().lnt_batched_lattice_mult
        _check(f(self.count, self.dims.ctypes.data, self.a_off.ctypes.data, self.b_off.ctypes.data, _ptr(ak),
                 _ptr(av), _ptr(bk), _ptr(bv), _ptr(self.ws), self.ws.numel(), _ptr(self.c_keys),
                 _ptr(self.c_vals), _ptr(self.c_off), _stream()),
               "lnt_batched_contract" if self.contract else "lnt_batched_lattice_mult")

    def result(self, p):
        off = self.c_off.tolist()
        return self.c_keys[off[p]:off[p + 1]], self.c_vals[off[p]:off[p + 1]]


def dense_split_workspace(h: int, w: int, wB: int, slices: int = 7) -> int:
    b = C.c_size_t(0)
    _check(lib().lnt_dense_split_workspace(h, w, wB, slices, C.byref(b)), "lnt_dense_split_workspace")
    return b.value


def dense_mult_split(A, B, h: int, w: int, wB: int, d: int = 1, slices: int = 7, out=None, ws=None):
    """Split-precision dense lattice product of column-major float64 A (h*w*d)
    and B (w*wB*d); returns C (h*wB*d, column-major)."""
    torch = _torch()
    Cm = torch.empty(h * wB * d, dtype=torch.float64, device=A.device) if out is None else out
    need = dense_split_workspace(h, w, wB, slices)
    if ws is None or ws.numel() < need:
        ws = workspace(need, A.device)
    _check(lib().lnt_dense_lattice_mult_split(_ptr(A), _ptr(B), _ptr(Cm), h, w, wB, d, slices, _ptr(ws), ws.numel(),
                                              _stream()), "lnt_dense_lattice_mult_split")
    return Cm


def dense_mult_fp64(A, B, h: int, w: int, wB: int, d: int = 1, out=None, ws=None):
    torch = _torch()
    Cm = torch.empty(h * wB * d, dtype=torch.float64, device=A.device) if out is None else out
    if ws is None:
        ws = workspace(64 << 20, A.device)
    _check(lib().lnt_dense_lattice_mult_fp64(_ptr(A), _ptr(B), _ptr(Cm), h, w, wB, d, _ptr(ws), ws.numel(),
                                             _stream()), "lnt_dense_lattice_mult_fp64")
    return Cm


def dense_crt_workspace(h: int, w: int, wB: int, moduli: int = 13) -> int:
    b = C.c_size_t(0)
    _check(lib().lnt_dense_crt_workspace(h, w, wB, moduli, C.byref(b)), "lnt_dense_crt_workspace")
    return b.value


def dense_crt_moduli(A, B, h: int, w: int, wB: int, d: int = 1, tol: float = 1e-12) -> int:
    """Moduli count for dense_mult_crt within tol * |A||B| per entry (lnt_dense_crt_moduli)."""
    ws = workspace(16 * h + 768, A.device)
    m = C.c_int(0)
    _check(lib().lnt_dense_crt_moduli(_ptr(A), _ptr(B), h, w, wB, d, float(tol), _ptr(ws), ws.numel(), C.byref(m),
                                      _stream()), "lnt_dense_crt_moduli")
    return int(m.value)


def dense_permute(x, dims, perm):
    """Dense mode permutation (column-major): mode k of the result is mode
    perm[k] of x.  Returns a new float64 device tensor."""
    torch = _torch()
    _dev(x)
    d = np.ascontiguousarray(dims, np.int64)
    pm = np.ascontiguousarray(perm, np.int32)
    out = torch.empty_like(x)
    _check(lib().lnt_dense_permute(_ptr(x), _ptr(out), len(d), d.ctypes.data, pm.ctypes.data, _stream()),
           "lnt_dense_permute")
    return out


def dense_mult_crt(A, B, h: int, w: int, wB: int, d: int = 1, moduli: int = 13, out=None, ws=None):
    """Dense lattice product by integer moduli + Chinese remaindering (scheme II)."""
    torch = _torch()
    Cm = torch.empty(h * wB * d, dtype=torch.float64, device=A.device) if out is None else out
    need = dense_crt_workspace(h, w, wB, moduli)
    if ws is None or ws.numel() < need:
        ws = workspace(need, A.device)
    _check(lib().lnt_dense_lattice_mult_crt(_ptr(A), _ptr(B), _ptr(Cm), h, w, wB, d, moduli, _ptr(ws), ws.numel(),
                                            _stream()), "lnt_dense_lattice_mult_crt")
    return Cm
