"""Oracle for the LNT hot path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import this package; it is the checker, never the product.

Two layers:

* ``liblnt_oracle.so`` (``lnt_oracle.cpp``): a C++ restatement of the reference
  kernels (re-key, sort, collect_duplicates, merge, csc_no_accum, dense
  per-tab GEMM), each citing the reference lines it follows.
* ``_ref/liblnt_ref.so`` (``ref_driver.cpp``): the reference's own compiled
  Boost-free kernels (re-key with libdivide, MSD radix sort, introsort), built
  in place from the reference tree when it is present.  Optional at run time.

On top, :class:`SparseMIA` restates the tensor-level semantics the hot path
has in the reference: ``linIdxSequence`` bookkeeping, the sorted flag and its
side effects, the merge decision table (``perform_outside_merge``,
``sortMerge``, ``outside_scanMerge``) and the lattice product of the
index-label expression layer (``MIA_Atom::operator*``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB_PATH = HERE / "liblnt_oracle.so"
_REF_PATH = HERE / "_ref" / "liblnt_ref.so"

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build(reference: bool = True) -> None:
    """Compile the restatement (and, if the reference tree is present, _ref)."""
    target = "all" if reference else "liblnt_oracle.so"
    subprocess.run(["make", "-s", "-C", str(HERE), target], check=True)


def _load():
    if not _LIB_PATH.exists():
        build(reference=False)
    lib = C.CDLL(str(_LIB_PATH))
    lib.lnto_rekey.argtypes = [_u64p, _u64p, C.c_size_t, C.c_int, _i64p, _i32p, _i32p]
    lib.lnto_rekey.restype = None
    lib.lnto_sort_pairs.argtypes = [_u64p, _f64p, C.c_size_t]
    lib.lnto_sort_pairs.restype = None
    lib.lnto_collect_duplicates.argtypes = [_u64p, _f64p, C.c_size_t, C.c_int, C.c_void_p]
    lib.lnto_collect_duplicates.restype = C.c_size_t
    lib.lnto_merge_sorted.argtypes = [_u64p, _f64p, C.c_size_t, _u64p, _f64p, C.c_size_t, C.c_int, _u64p, _f64p]
    lib.lnto_merge_sorted.restype = C.c_size_t
    lib.lnto_lattice_mult.argtypes = [_u64p, _f64p, C.c_size_t, C.c_int64, C.c_int64, C.c_int64,
                                      _u64p, _f64p, C.c_size_t, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.lnto_lattice_mult.restype = C.c_size_t
    lib.lnto_dense_lattice_mult.argtypes = [_f64p, _f64p, _f64p, C.c_int64, C.c_int64, C.c_int64, C.c_int64]
    lib.lnto_dense_lattice_mult.restype = None
    lib.lnto_dense_entries.argtypes = [_f64p, _f64p, C.c_int64, C.c_int64, _i64p, _i64p, C.c_size_t, _f64p, _f64p]
    lib.lnto_dense_entries.restype = None
    return lib


_lib = _load()
_ref = None


def ref_available() -> bool:
    """True when the reference's own kernels were compiled into _ref/."""
    global _ref
    if _ref is None and _REF_PATH.exists():
        r = C.CDLL(str(_REF_PATH))
        r.lntr_rekey.argtypes = [_i64p, C.c_size_t, C.c_int, _i64p, _i32p, _i32p]
        r.lntr_rekey.restype = C.c_int
        r.lntr_radix_sort.argtypes = [_i64p, _f64p, C.c_size_t, C.c_size_t]
        r.lntr_radix_sort.restype = None
        r.lntr_introsort.argtypes = [_i64p, _f64p, C.c_size_t]
        r.lntr_introsort.restype = None
        _ref = r
    return _ref is not None


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------------------
# kernel-level restatements
# ---------------------------------------------------------------------------

def rekey(keys, dims, cur_seq, new_seq) -> np.ndarray:
    k = _u64(keys)
    out = np.empty_like(k)
    _lib.lnto_rekey(k, out, k.size, len(dims), np.asarray(dims, np.int64), np.asarray(cur_seq, np.int32),
                    np.asarray(new_seq, np.int32))
    return out


def sort_pairs(keys, vals):
    k, v = _u64(keys).copy(), _f64(vals).copy()
    _lib.lnto_sort_pairs(k, v, k.size)
    return k, v


def collect_duplicates(keys, vals, skip_zero_heads=True, with_abs=False):
    """Fold equal-key runs of a key-sorted array (see lnt_oracle.cpp)."""
    k, v = _u64(keys).copy(), _f64(vals).copy()
    a = np.empty(k.size, np.float64) if with_abs else None
    n = _lib.lnto_collect_duplicates(k, v, k.size, int(bool(skip_zero_heads)),
                                     a.ctypes.data if a is not None else None)
    if with_abs:
        return k[:n], v[:n], a[:n]
    return k[:n], v[:n]


def merge_sorted(ak, av, bk, bv, op=0):
    ak, av, bk, bv = _u64(ak), _f64(av), _u64(bk), _f64(bv)
    ck = np.empty(ak.size + bk.size, np.uint64)
    cv = np.empty(ak.size + bk.size, np.float64)
    n = _lib.lnto_merge_sorted(ak, av, ak.size, bk, bv, bk.size, int(op), ck, cv)
    return ck[:n], cv[:n]


def lattice_mult(ak, av, h, w, d, bk, bv, wB, with_abs=False):
    """csc_no_accum restatement; A, B key-sorted column-major lattices."""
    ak, av, bk, bv = _u64(ak), _f64(av), _u64(bk), _f64(bv)
    n = _lib.lnto_lattice_mult(ak, av, ak.size, h, w, d, bk, bv, bk.size, wB, None, None, None)
    ck = np.empty(n, np.uint64)
    cv = np.empty(n, np.float64)
    ca = np.empty(n, np.float64)
    _lib.lnto_lattice_mult(ak, av, ak.size, h, w, d, bk, bv, bk.size, wB, ck.ctypes.data, cv.ctypes.data,
                           ca.ctypes.data)
    if with_abs:
        return ck, cv, ca
    return ck, cv


def csc_times(ak, av, h, w, d, bk, bv, wB):
    """Second oracle for the lattice product: SparseLatticeBase::csc_times
    (SparseLatticeBase.h:2226-2351), Gustavson's column-by-column product with
    a dense accumulator per tab.  For each column of B, its entries in row
    order scatter A's column into the accumulator (first touch sets, later
    ones add); every touched row is emitted, in row order.  Same pattern as
    csc_no_accum (exact zero sums kept), different summation order."""
    ak, bk = _u64(ak), _u64(bk)
    av, bv = _f64(av), _f64(bv)
    keys, vals = [], []
    at, bt = ak // np.uint64(h * w), bk // np.uint64(w * wB)
    for t in np.intersect1d(np.unique(at), np.unique(bt)):
        sa, sb = at == t, bt == t
        a_loc, a_val = ak[sa] % np.uint64(h * w), av[sa]
        a_row, a_col = (a_loc % np.uint64(h)).astype(np.int64), (a_loc // np.uint64(h)).astype(np.int64)
        b_loc, b_val = bk[sb] % np.uint64(w * wB), bv[sb]
        b_row, b_col = (b_loc % np.uint64(w)).astype(np.int64), (b_loc // np.uint64(w)).astype(np.int64)
        for c in np.unique(b_col):
            acc, touched = {}, []
            for k, bvv in zip(b_row[b_col == c], b_val[b_col == c]):
                for r, avv in zip(a_row[a_col == k], a_val[a_col == k]):
                    if r in acc:
                        acc[r] += avv * bvv
                    else:
                        acc[r] = avv * bvv
                        touched.append(r)
            for r in sorted(touched):
                keys.append(r + h * (c + wB * int(t)))
                vals.append(acc[r])
    return np.array(keys, np.uint64), np.array(vals, np.float64)


def outer_times(ak, av, h, w, d, bk, bv, wB):
    """Second oracle for the lattice product: SparseLatticeBase::outer_times
    (SparseLatticeBase.h:2036-2183).  Per tab, for every inner index k present
    in both, all products A(:,k) x B(k,:) are listed, then sorted by output key
    and folded with collect_duplicates_function (+, zeros kept)."""
    ak, bk = _u64(ak), _u64(bk)
    av, bv = _f64(av), _f64(bv)
    keys, vals = [], []
    at, bt = ak // np.uint64(h * w), bk // np.uint64(w * wB)
    for t in np.intersect1d(np.unique(at), np.unique(bt)):
        sa, sb = at == t, bt == t
        a_loc, a_val = ak[sa] % np.uint64(h * w), av[sa]
        a_row, a_col = (a_loc % np.uint64(h)).astype(np.int64), (a_loc // np.uint64(h)).astype(np.int64)
        b_loc, b_val = bk[sb] % np.uint64(w * wB), bv[sb]
        b_row, b_col = (b_loc % np.uint64(w)).astype(np.int64), (b_loc // np.uint64(w)).astype(np.int64)
        pk, pv = [], []
        for k in np.intersect1d(a_col, b_row):
            ia, ib = a_col == k, b_row == k
            pk.append((a_row[ia][:, None] + h * b_col[ib][None, :]).ravel())
            pv.append((a_val[ia][:, None] * b_val[ib][None, :]).ravel())
        if not pk:
            continue
        lk, lv = sort_pairs(np.concatenate(pk).astype(np.uint64), np.concatenate(pv))
        ck, cv = collect_duplicates(lk, lv, skip_zero_heads=False)
        keys.append(ck + np.uint64(h * wB) * np.uint64(t))
        vals.append(cv)
    if not keys:
        return np.zeros(0, np.uint64), np.zeros(0, np.float64)
    return np.concatenate(keys), np.concatenate(vals)


def dense_lattice_mult(A, B, h, w, wB, d) -> np.ndarray:
    """Column-major per-tab product; A (h*w*d), B (w*wB*d) flat arrays."""
    A, B = _f64(A).ravel(), _f64(B).ravel()
    Cm = np.empty(h * wB * d, np.float64)
    _lib.lnto_dense_lattice_mult(A, B, Cm, h, w, wB, d)
    return Cm


def dense_entries(A, B, h, w, rows, cols):
    """Compensated FP64 entries C[r, c] of a single-tab product, and sum |a b|."""
    A, B = _f64(A).ravel(), _f64(B).ravel()
    rows = np.ascontiguousarray(rows, np.int64)
    cols = np.ascontiguousarray(cols, np.int64)
    out = np.empty(rows.size, np.float64)
    mag = np.empty(rows.size, np.float64)
    _lib.lnto_dense_entries(A, B, h, w, rows, cols, rows.size, out, mag)
    return out, mag


# ---- the reference's own kernels (if compiled) -----------------------------

def ref_rekey(keys, dims, cur_seq, new_seq) -> np.ndarray:
    assert ref_available()
    k = np.ascontiguousarray(keys, np.int64).copy()
    rc = _ref.lntr_rekey(k, k.size, len(dims), np.asarray(dims, np.int64), np.asarray(cur_seq, np.int32),
                         np.asarray(new_seq, np.int32))
    assert rc == 0
    return k.view(np.uint64)


def ref_radix_sort(keys, vals, max_size):
    assert ref_available()
    k = np.ascontiguousarray(keys, np.int64).copy()
    v = _f64(vals).copy()
    _ref.lntr_radix_sort(k, v, k.size, int(max_size))
    return k.view(np.uint64), v


def ref_introsort(keys, vals):
    assert ref_available()
    k = np.ascontiguousarray(keys, np.int64).copy()
    v = _f64(vals).copy()
    _ref.lntr_introsort(k, v, k.size)
    return k.view(np.uint64), v


# ---------------------------------------------------------------------------
# index-label classification (restates ExprUtil.h / MIA_Expr.h)
# ---------------------------------------------------------------------------

def _base(label: str) -> str:
    return label.lstrip("!")


def _is_elem(label: str) -> bool:
    return label.startswith("!")


def decrement(labels, inter: int):
    """MIA_Atom::operator~ (MIA_Expr.h:1376-1379; decrement_back_indices,
    ExprUtil.h:740-766): the last `inter` labels lose one '!'."""
    labels = list(labels)
    for q in range(len(labels) - inter, len(labels)):
        if labels[q].startswith("!"):
            labels[q] = labels[q][1:]
    return labels


def product_orders(l_labels, r_labels) -> dict:
    """Mode classification of a product l(...) * r(...).

    Restates solve_product_expr_helper (MIA_Expr.h:449-529) built on
    pull_left_operand_index_sequence (ExprUtil.h:311-393) and
    pull_right_index_order (ExprUtil.h:564-645): a left label found once in
    the right operand is inner (contracted) unless marked element-wise ('!'),
    then it is inter (a tab); a left label not found is outer.  Right inner /
    inter orders follow the left's inner / inter order.
    """
    l_outer, l_inner, l_inter = [], [], []
    for i, lab in enumerate(l_labels):
        n = sum(1 for r in r_labels if r == lab)
        if n == 0:
            if any(_base(r) == _base(lab) for r in r_labels):
                raise ValueError("same index with different element-wise marks")
            l_outer.append(i)
        elif n == 1:
            (l_inter if _is_elem(lab) else l_inner).append(i)
        else:
            raise ValueError("index repeated in right operand")
    r_outer = [j for j, lab in enumerate(r_labels) if lab not in l_labels]
    r_inner = [r_labels.index(l_labels[i]) for i in l_inner]
    r_inter = [r_labels.index(l_labels[i]) for i in l_inter]
    return dict(l_outer=l_outer, l_inner=l_inner, l_inter=l_inter, r_outer=r_outer, r_inner=r_inner,
                r_inter=r_inter)


def merge_index_order(l_labels, r_labels) -> list:
    """For each left label its position in the right operand
    (pull_match_order, ExprUtil.h:511-562), labels matched by index identity
    whatever their element-wise marks (same_product_index_id, Index.h:174-184)."""
    lb, rb = [_base(x) for x in l_labels], [_base(x) for x in r_labels]
    if sorted(lb) != sorted(rb):
        raise ValueError("merge operands must carry the same labels")
    return [rb.index(lab) for lab in lb]


def reverse_order(order):
    """internal::reverseOrder (IndexUtil.h:893-914)."""
    out = [len(order)] * len(order)
    for i in range(len(order)):
        for j, o in enumerate(order):
            if o == i:
                out[i] = j
                break
    return out


def reorder_from(from_array, seq):
    """internal::reorder_from (IndexUtil.h:231-252): [from_array[s] for s in seq]."""
    return [from_array[s] for s in seq]


# ---------------------------------------------------------------------------
# tensor-level restatement
# ---------------------------------------------------------------------------

@dataclass
class SparseMIA:
    """SparseMIA<double, N> state: dims, LCO keys/values, linIdxSequence and
    the sorted flag (SparseMIA.h:167-206; SparseMIABase.h:98-153)."""
    dims: list
    keys: np.ndarray
    vals: np.ndarray
    seq: list = field(default=None)
    sorted: bool = True  # ctor default (SparseMIABase.h:220, 234)

    def __post_init__(self):
        self.dims = [int(d) for d in self.dims]
        if self.seq is None:
            self.seq = list(range(len(self.dims)))
        self.keys = _u64(self.keys)
        self.vals = _f64(self.vals)

    @property
    def order(self):
        return len(self.dims)

    @property
    def dimensionality(self):
        return int(np.prod(self.dims, dtype=object))

    def copy(self) -> "SparseMIA":
        return SparseMIA(list(self.dims), self.keys.copy(), self.vals.copy(), list(self.seq), self.sorted)

    @property
    def size(self):
        return int(self.keys.size)

    # SparseMIABase::change_linIdx_sequence (SparseMIABase.h:768-814)
    def change_linIdx_sequence(self, seq):
        seq = list(seq)
        if seq == self.seq or self.order == 1:
            return
        self.keys = rekey(self.keys, self.dims, self.seq, seq)
        self.seq = seq
        self.sorted = False

    # SparseMIABase::sort() (SparseMIABase.h:701-734)
    def sort(self, seq=None):
        if seq is None:
            if not self.sorted:
                self.keys, self.vals = sort_pairs(self.keys, self.vals)
            self.sorted = True
            return
        # SparseMIABase::sort(seq) (SparseMIABase.h:590-645)
        seq = list(seq)
        if not self.sorted:
            self.change_linIdx_sequence(seq)
            self.sort()
        elif self.order != 1 and seq != self.seq:
            self.change_linIdx_sequence(seq)
            self.keys, self.vals = sort_pairs(self.keys, self.vals)
            if self.size < 3000:
                # introsort branch returns before setSorted(true) (:615-618)
                self.sorted = False
                return
            self.sorted = True
        else:
            self.sorted = True

    # SparseMIA::collect_duplicates(std::plus) (SparseMIA.h:636-665)
    def collect_duplicates(self):
        self.sort()
        self.keys, self.vals = collect_duplicates(self.keys, self.vals, skip_zero_heads=True)
        self.sorted = True

    def to_dense(self) -> np.ndarray:
        """Dense array indexed [i0, i1, ...] (duplicates summed)."""
        out = np.zeros(self.dims, np.float64)
        k = self.keys.astype(object)
        strides = []
        s = 1
        for m in self.seq:
            strides.append(s)
            s *= self.dims[m]
        for key, v in zip(self.keys.tolist(), self.vals.tolist()):
            idx = [0] * self.order
            for pos in range(self.order - 1, -1, -1):
                q, key = divmod(key, strides[pos])
                idx[self.seq[pos]] = q
            out[tuple(idx)] += v
        return out


def merge(a: SparseMIA, b: SparseMIA, index_order, op=0) -> SparseMIA:
    """C = a (op) b with b's modes matched by index_order.

    Restates SparseMIABase::perform_outside_merge (SparseMIABase.h:1377-1402):
    scan merge if either operand is sorted, else C = copy(a), C.sortMerge(b).
    Operands are mutated as in the reference (re-keyed / re-sorted)."""
    if a.dims != [b.dims[i] for i in index_order]:
        raise ValueError("merge dimension mismatch")
    if a.sorted or b.sorted:
        return _scan_merge(a, b, index_order, op)
    c = a.copy()
    _sort_merge(c, b, index_order, op)
    return c


def _sort_merge(c: SparseMIA, b: SparseMIA, index_order, op):
    """SparseMIA::sortMerge (SparseMIA.h:833-887)."""
    if c.size > b.size:
        b.change_linIdx_sequence(reorder_from(index_order, c.seq))
    else:
        lhs = reverse_order(index_order)
        c.change_linIdx_sequence(reorder_from(lhs, b.seq))
    bv = -b.vals if op == 1 else b.vals
    c.keys = np.concatenate([c.keys, b.keys])
    c.vals = np.concatenate([c.vals, bv])
    c.sorted = False
    c.collect_duplicates()


def _scan_merge(a: SparseMIA, b: SparseMIA, index_order, op) -> SparseMIA:
    """SparseMIABase::outside_scanMerge (SparseMIABase.h:1404-1455)."""
    if b.sorted and not a.sorted:
        a.sort(reorder_from(reverse_order(index_order), b.seq))
    elif a.sorted and not b.sorted:
        b.sort(reorder_from(index_order, a.seq))
    else:
        if b.size < a.size:
            b.sort(reorder_from(index_order, a.seq))
        else:
            a.sort(reorder_from(reverse_order(index_order), b.seq))
    ck, cv = merge_sorted(a.keys, a.vals, b.keys, b.vals, op)
    # C(dims) is sorted by construction; change_linIdx_sequence on an empty MIA
    # sets the sequence and clears the flag (SparseMIABase.h:811-812).
    c = SparseMIA(list(a.dims), ck, cv, list(a.seq), sorted=(a.seq == list(range(a.order))))
    return c


def to_lattice(m: SparseMIA, rows, cols, tabs):
    """toStraightLattice / toLatticeSort (SparseMIABase.h:1457-1586), column
    major: sort under seq = rows+cols+tabs (default sequence when that is
    0..N-1), return (keys, vals, h, w, d) and clear the sorted flag."""
    seq = list(rows) + list(cols) + list(tabs)
    m.sort(seq)
    h = int(np.prod([m.dims[i] for i in rows], dtype=np.int64)) if rows else 1
    w = int(np.prod([m.dims[i] for i in cols], dtype=np.int64)) if cols else 1
    d = int(np.prod([m.dims[i] for i in tabs], dtype=np.int64)) if tabs else 1
    m.sorted = False
    return m.keys, m.vals, h, w, d


def nolattice_mult(ak, av, h, d, bk, bv, wB):
    """Core of SparseMIABase::perform_noLatticeMult (SparseMIABase.h:1749-1820):
    A key-sorted as outer + h * inter, B as outer + wB * inter; for each inter
    index present in both, every (B entry, A entry) pair, B major: key
    a_outer + b_outer * h + inter * h * wB, value a * b.  No fold of equal keys;
    the result is ascending."""
    ak = np.asarray(ak, np.uint64)
    bk = np.asarray(bk, np.uint64)
    av = np.asarray(av, np.float64)
    bv = np.asarray(bv, np.float64)
    ga, gb = ak // np.uint64(h), bk // np.uint64(wB)
    common = np.intersect1d(np.unique(ga), np.unique(gb))
    keys, vals = [], []
    for g in common:
        a0, a1 = np.searchsorted(ga, g, "left"), np.searchsorted(ga, g, "right")
        b0, b1 = np.searchsorted(gb, g, "left"), np.searchsorted(gb, g, "right")
        ao = (ak[a0:a1] % np.uint64(h)).astype(np.uint64)
        bo = (bk[b0:b1] % np.uint64(wB)).astype(np.uint64)
        k = ao[None, :] + np.uint64(h) * bo[:, None] + np.uint64(g) * np.uint64(h) * np.uint64(wB)
        keys.append(k.ravel())
        vals.append((av[a0:a1][None, :] * bv[b0:b1][:, None]).ravel())
    if not keys:
        return np.zeros(0, np.uint64), np.zeros(0, np.float64)
    return np.concatenate(keys), np.concatenate(vals)


def _lines(sk, W):
    """Start offsets and values g = key // W of the runs of equal g in sorted keys."""
    g = sk // np.uint64(W)
    if g.size == 0:
        return np.zeros(1, np.int64), g
    heads = np.flatnonzero(np.concatenate([[True], g[1:] != g[:-1]]))
    return np.append(heads, g.size), g[heads]


def dense_sparse_mult(A, sk, sv, h, w, wB, d):
    """DenseLatticeBase::operator*(SparseLatticeBase) (DenseLatticeBase.h:
    436-500): A dense h x w x d (column-major, flat), S w x wB x d key-sorted
    column-major.  For every (tab, col) of S with entries, in key order, h
    outputs with keys i + h (col + wB tab): c = 0, then c = c + v * A(i, row,
    tab) for the column's entries in order (zeros kept).  Ascending keys."""
    A = np.asarray(A, np.float64).reshape(-1)
    sk = np.asarray(sk, np.uint64)
    sv = np.asarray(sv, np.float64)
    starts, gs = _lines(sk, w)
    keys, vals = [], []
    for q, g in enumerate(gs):
        t = int(g) // wB
        c = np.zeros(h)
        for k in range(starts[q], starts[q + 1]):
            r = int(sk[k]) % w
            c = c + sv[k] * A[h * (r + w * t): h * (r + w * t) + h]
        keys.append(np.arange(h, dtype=np.uint64) + np.uint64(h) * g)
        vals.append(c)
    if not keys:
        return np.zeros(0, np.uint64), np.zeros(0, np.float64)
    return np.concatenate(keys), np.concatenate(vals)


def sparse_dense_mult(sk, sv, B, h, w, wB, d):
    """SparseLatticeBase::operator*(DenseLatticeBase) (SparseLatticeBase.h:
    1148-1162), which the reference evaluates as (B^T S^T)^T through the dense
    x sparse product: S h x w x d key-sorted ROW-major (col + w (row + h
    tab)), B dense w x wB x d (column-major, flat).  For every (tab, row) of S
    with entries, in key order, wB outputs with the row-major lattice keys
    j + wB (row + h tab): c = 0, then c = c + v * B(col, j, tab) for the row's
    entries in order.  Ascending keys."""
    B = np.asarray(B, np.float64).reshape(-1)
    sk = np.asarray(sk, np.uint64)
    sv = np.asarray(sv, np.float64)
    starts, gs = _lines(sk, w)
    js = np.arange(wB, dtype=np.int64)
    keys, vals = [], []
    for q, g in enumerate(gs):
        t = int(g) // h
        c = np.zeros(wB)
        for k in range(starts[q], starts[q + 1]):
            col = int(sk[k]) % w
            c = c + sv[k] * B[col + w * (js + wB * t)]
        keys.append(np.arange(wB, dtype=np.uint64) + np.uint64(wB) * g)
        vals.append(c)
    if not keys:
        return np.zeros(0, np.uint64), np.zeros(0, np.float64)
    return np.concatenate(keys), np.concatenate(vals)


def product(a: SparseMIA, a_labels, b: SparseMIA, b_labels):
    """Product a(a_labels) * b(b_labels) (MIA_Atom::operator*, MIA_Expr.h:
    864-925 with inner indices: a lattice product; 1012-1057 without: noLatticeMult).
    Returns (C, c_labels); C has dims [a outer, b outer, inter], the default
    linIdxSequence and sorted = True (SparseMIA.h:362-372)."""
    o = product_orders(a_labels, b_labels)
    if a is b:
        b = b.copy()  # MIA_Atom::check_if_copy_needed (MIA_Expr.h:767-802)
    dims = [a.dims[i] for i in o["l_outer"]] + [b.dims[j] for j in o["r_outer"]] + \
           [a.dims[i] for i in o["l_inter"]]
    labels = [a_labels[i] for i in o["l_outer"]] + [b_labels[j] for j in o["r_outer"]] + \
             [a_labels[i] for i in o["l_inter"]]
    if not o["l_inner"]:
        # pure outer / element-wise product: noLatticeMult (MIA_Expr.h:1012-1057,
        # SparseMIABase.h:1701-1826): both operands sorted (in place) under
        # [outer, inter], no lattice, C sorted by construction
        if [a.dims[i] for i in o["l_inter"]] != [b.dims[j] for j in o["r_inter"]]:
            raise ValueError("Element-wise dimensions must match during MIA multiplication")
        a.sort(list(o["l_outer"]) + list(o["l_inter"]))
        b.sort(list(o["r_outer"]) + list(o["r_inter"]))
        h = int(np.prod([a.dims[i] for i in o["l_outer"]], dtype=np.int64)) if o["l_outer"] else 1
        wB = int(np.prod([b.dims[j] for j in o["r_outer"]], dtype=np.int64)) if o["r_outer"] else 1
        d = int(np.prod([a.dims[i] for i in o["l_inter"]], dtype=np.int64)) if o["l_inter"] else 1
        ck, cv = nolattice_mult(a.keys, a.vals, h, d, b.keys, b.vals, wB)
        return SparseMIA(dims, ck, cv, list(range(len(dims))), True), labels
    ak, av, h, w, d = to_lattice(a, o["l_outer"], o["l_inner"], o["l_inter"])
    bk, bv, hb, wB, db = to_lattice(b, o["r_inner"], o["r_outer"], o["r_inter"])
    if hb != w or db != d:
        raise ValueError("lattice dimension mismatch")
    ck, cv = lattice_mult(ak, av, h, w, d, bk, bv, wB)
    return SparseMIA(dims, ck, cv, list(range(len(dims))), True), labels


def mixed_product(s: SparseMIA, s_labels, D, d_dims, d_labels, dense_first: bool):
    """MIA_Atom::operator* with one sparse and one dense operand (MIA_Expr.h:
    864-925): the dense operand's modes are already in lattice order (zero-copy
    DenseMIA::toStraightLattice, DenseMIA.h:1240-1255); the sparse operand is
    sorted into its lattice and flagged unsorted.  dense_first: D * s through
    dense_sparse_mult, result sorted in the default sequence.  Otherwise s * D
    through sparse_dense_mult (s sorted under [inner, outer, inter], the
    row-major lattice), result re-keyed from the row-major lattice to the
    default sequence and flagged unsorted (SparseMIA.h:362-372).  Returns
    (C, c_labels) with C dims [left outer, right outer, inter]."""
    def pd(dims, modes):
        return int(np.prod([dims[i] for i in modes], dtype=np.int64)) if modes else 1
    if dense_first:
        o = product_orders(d_labels, s_labels)
        h, w, d = pd(d_dims, o["l_outer"]), pd(d_dims, o["l_inner"]), pd(d_dims, o["l_inter"])
        wB = pd(s.dims, o["r_outer"])
        bk, bv, _, _, _ = to_lattice(s, o["r_inner"], o["r_outer"], o["r_inter"])
        ck, cv = dense_sparse_mult(D, bk, bv, h, w, wB, d)
        dims = [d_dims[i] for i in o["l_outer"]] + [s.dims[j] for j in o["r_outer"]] + [d_dims[i] for i in o["l_inter"]]
        labels = [d_labels[i] for i in o["l_outer"]] + [s_labels[j] for j in o["r_outer"]] + \
                 [d_labels[i] for i in o["l_inter"]]
        return SparseMIA(dims, ck, cv, list(range(len(dims))), True), labels
    o = product_orders(s_labels, d_labels)
    h, w, d = pd(s.dims, o["l_outer"]), pd(s.dims, o["l_inner"]), pd(s.dims, o["l_inter"])
    wB = pd(d_dims, o["r_outer"])
    ak, av, _, _, _ = to_lattice(s, o["l_inner"], o["l_outer"], o["l_inter"])
    ck, cv = sparse_dense_mult(ak, av, D, h, w, wB, d)
    dims = [s.dims[i] for i in o["l_outer"]] + [d_dims[j] for j in o["r_outer"]] + [s.dims[i] for i in o["l_inter"]]
    labels = [s_labels[i] for i in o["l_outer"]] + [d_labels[j] for j in o["r_outer"]] + \
             [s_labels[i] for i in o["l_inter"]]
    nl, nr, ni = len(o["l_outer"]), len(o["r_outer"]), len(o["l_inter"])
    rowmajor = list(range(nl, nl + nr)) + list(range(nl)) + list(range(nl + nr, nl + nr + ni))
    c = SparseMIA(dims, ck, cv, rowmajor, True)
    c.change_linIdx_sequence(list(range(len(dims))))
    c.sorted = False
    return c, labels


def unary_orders(labels) -> dict:
    """Contraction / attraction classification of one operand's labels, a
    restatement of unary_helper (MIA_Expr.h:632-662) with pull_contract_indices,
    pull_attract_indices (ExprUtil.h:80-248) and pull_sequence_from_list
    (ExprUtil.h:250-300): a plain label repeated in the operand is contracted,
    an element-wise ('!') label repeated among the rest is attracted; sets are
    listed in the order of their labels' last occurrences, each with its
    positions ascending.  Result labels: the others, then one per attraction."""
    labels = list(labels)

    def pull(seq, elem):
        found = []
        for q in range(len(seq) - 1, -1, -1):
            lab = seq[q]
            if seq.count(lab) > 1 and _is_elem(lab) == elem and lab not in found:
                found.insert(0, lab)
        rest = [lab for lab in seq if not (seq.count(lab) > 1 and _is_elem(lab) == elem)]
        return found, rest

    con, rest1 = pull(labels, False)
    att, rest2 = pull(rest1, True)

    def positions(sub):
        pos, part = [], []
        for lab in sub:
            ps = [q for q, x in enumerate(labels) if x == lab]
            pos += ps
            part.append(len(ps))
        return pos, part

    cpos, cpart = positions(con)
    apos, apart = positions(att)
    other = sorted(set(range(len(labels))) - set(cpos) - set(apos))
    return dict(contract=cpos, contract_part=cpart, attract=apos, attract_part=apart, other=other,
                labels=rest2 + att)


def contract_attract(m: SparseMIA, cpos, cpart, apos, apart) -> SparseMIA:
    """SparseMIABase::contract_attract (SparseMIABase.h:1913-2053), loop kept as
    in the reference: sort m (in place) under [contract, attract, other]; walk
    the entries; an entry whose attraction sets disagree is skipped; otherwise
    the run of entries with equal key / contract_dimensionality (equal attract
    and other indices) is summed over the entries whose contraction sets agree,
    and a non-zero sum is pushed at key/(contract_dim * attract_dim) +
    attract_idx * other_dim.  Result dims [other, attraction ranges]; sorted
    flag as push_back leaves it (SparseMIA.h:570-578)."""
    order = m.order
    other = sorted(set(range(order)) - set(cpos) - set(apos))
    sort_order = list(cpos) + list(apos) + other
    m.sort(sort_order)
    sdims = [m.dims[q] for q in sort_order]
    contract_dim, cur = 1, 0
    for part in cpart:
        contract_dim *= m.dims[cpos[cur]] ** part
        cur += part
    ranges, attract_dim, cur = [], 1, 0
    for part in apart:
        ranges.append(m.dims[apos[cur]])
        attract_dim *= ranges[-1] ** part
        cur += part
    other_dim = int(np.prod([m.dims[q] for q in other], dtype=np.int64)) if other else 1

    def ind2sub(k):
        out = []
        for dd in sdims:
            out.append(k % dd)
            k //= dd
        return out

    keys = [int(x) for x in m.keys]
    vals = m.vals
    out_k, out_v = [], []
    ncon = len(cpos)
    e = 0
    while e < len(keys):
        idx = ind2sub(keys[e])
        ok, start, cur_att = True, ncon, []
        for part in apart:
            if any(idx[q] != idx[start] for q in range(start + 1, start + part)):
                ok = False
                break
            cur_att.append(idx[start])
            start += part
        if not ok:
            e += 1
            continue
        att_idx, stride = 0, 1
        for v_, r_ in zip(cur_att, ranges):
            att_idx += v_ * stride
            stride *= r_
        head = keys[e]
        total = 0.0
        while e < len(keys) and head // contract_dim == keys[e] // contract_dim:
            idx = ind2sub(keys[e])
            add, start = True, 0
            for part in cpart:
                if any(idx[q] != idx[start] for q in range(start + 1, start + part)):
                    add = False
                    break
                start += part
            if add:
                total += float(vals[e])
            e += 1
        if total:
            out_k.append(head // (contract_dim * attract_dim) + att_idx * other_dim)
            out_v.append(total)
    ok_ = np.array(out_k, np.uint64)
    sorted_ = bool(np.all(ok_[1:] >= ok_[:-1])) if ok_.size > 1 else True
    dims = [m.dims[q] for q in other] + ranges
    return SparseMIA(dims, ok_, np.array(out_v, np.float64), list(range(len(dims))), sorted_)


def unary(m: SparseMIA, labels):
    """m(labels) with repeated labels (perform_unary, MIA_Expr.h:690-735):
    returns (result, result labels); m itself when no label repeats."""
    o = unary_orders(labels)
    if not o["contract"] and not o["attract"]:
        return m, list(labels)
    return contract_attract(m, o["contract"], o["contract_part"], o["attract"], o["attract_part"]), o["labels"]


def assign(dest_labels, src: SparseMIA, src_labels) -> SparseMIA:
    """c(dest_labels) = <expression result with src_labels>: when the label
    orders differ only linIdxSequence and dims are rewritten, no sort
    (SparseMIA::assign, SparseMIA.h:891-928)."""
    db, sb = [_base(x) for x in dest_labels], [_base(x) for x in src_labels]  # matched by index identity
    if db == sb:
        return src
    index_order = [sb.index(l) for l in db]
    new_dims = [src.dims[i] for i in index_order]
    lhs = reverse_order(index_order)
    new_seq = [lhs[s] for s in src.seq]
    return SparseMIA(new_dims, src.keys.copy(), src.vals.copy(), new_seq, src.sorted)
