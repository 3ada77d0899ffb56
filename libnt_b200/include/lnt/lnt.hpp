// lnt.hpp - header-only C++17 front end of the LibNT B200 hot path.
//
// Mirrors the reference's index-label operator API (MIA.h:222-238,
// MIA_Expr.h, Index.h): sparse and dense multi-index arrays addressed with
// index labels,
//
//     lnt::Index i, j, k, l;
//     c(i, l) = a(i, j, k) * b(k, l, j);        // lattice contraction
//     c4(i, j, k, l) = a4(i, j, k, l) + b4(l, k, j, i);   // merge under permutation
//     d(i, l, !n) = a(i, j, !n) * b(j, l, !n);  // element-wise index (a tab)
//
// with the same results and the same side effects on the operands as the
// reference: operands are re-keyed / re-sorted in place exactly where the
// reference does it (sortMerge, outside_scanMerge, toStraightLattice,
// toLatticeSort), linIdxSequence() and is_sorted() follow the reference's
// rules, and assignment to a differently ordered target only relabels.
//
// All arithmetic runs on the current CUDA device through the C ABI of
// include/lnt.h; tensors own device buffers.  Labels are run-time objects
// (the reference resolves them at compile time with Boost.MPL); the
// classification into outer / inner / element-wise modes follows
// solve_product_expr_helper (MIA_Expr.h:449-529).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "lnt.h"

namespace lnt {

// ---- errors (the reference's exception names, LibMIAException.h:25-92) ----
struct LibMIAException : std::runtime_error {
  explicit LibMIAException(const std::string& m) : std::runtime_error(m) {}
};
struct DimensionMismatchException : LibMIAException {
  using LibMIAException::LibMIAException;
};
struct MIAParameterException : LibMIAException {
  using LibMIAException::LibMIAException;
};
struct LatticeParameterException : LibMIAException {
  using LibMIAException::LibMIAException;
};
struct DeviceException : LibMIAException {
  using LibMIAException::LibMIAException;
};

inline void check(int st, const char* what) {
  if (st == LNT_OK) return;
  std::string m = std::string(what) + ": " + lnt_status_string(st);
  if (st == LNT_BAD_DIMS) throw DimensionMismatchException(m);
  if (st == LNT_BAD_ARG || st == LNT_BAD_SEQ || st == LNT_OVERFLOW_KEYBITS) throw MIAParameterException(m);
  throw DeviceException(m);
}

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw DeviceException(std::string(what) + ": " + cudaGetErrorString(e));
}

// ---- device memory ----------------------------------------------------------
template <class T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t n) { resize(n); }
  DeviceBuffer(const DeviceBuffer& o) { *this = o; }
  DeviceBuffer& operator=(const DeviceBuffer& o) {
    if (this != &o) {
      resize(o.n_);
      if (o.n_) cuda_check(cudaMemcpy(p_, o.p_, o.n_ * sizeof(T), cudaMemcpyDeviceToDevice), "copy");
    }
    return *this;
  }
  DeviceBuffer(DeviceBuffer&& o) noexcept : p_(o.p_), n_(o.n_), cap_(o.cap_) { o.p_ = nullptr, o.n_ = o.cap_ = 0; }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    std::swap(p_, o.p_), std::swap(n_, o.n_), std::swap(cap_, o.cap_);
    return *this;
  }
  ~DeviceBuffer() {
    if (p_) cudaFree(p_);
  }
  void resize(size_t n) {  // contents are not preserved when growing
    if (n > cap_) {
      if (p_) cudaFree(p_);
      p_ = nullptr;
      cuda_check(cudaMalloc(&p_, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
      cap_ = n;
    }
    n_ = n;
  }
  void shrink(size_t n) { n_ = std::min(n, n_); }  // keep contents, drop the tail
  T* data() { return p_; }
  const T* data() const { return p_; }
  size_t size() const { return n_; }

 private:
  T* p_ = nullptr;
  size_t n_ = 0, cap_ = 0;
};

// Grow-only scratch shared by operations on this thread.
inline void* scratch(size_t bytes) {
  thread_local DeviceBuffer<unsigned char> buf;
  if (buf.size() < bytes) buf.resize(bytes);
  return buf.data();
}

inline uint64_t read_u64(const uint64_t* d) {
  uint64_t h = 0;
  cuda_check(cudaMemcpy(&h, d, 8, cudaMemcpyDeviceToHost), "read count");
  return h;
}

// ---- index labels -------------------------------------------------------------
// An index label (MIAINDEX / NTINDEX, Index.h:28-30); each ! raises its
// element-wise level by one (!i, !!i: Index.h:54-57, ProdInd's counter).  Each
// label object has its own identity; products match labels by identity and
// level, merges and assignments by identity alone (same_product_index_id,
// Index.h:174-184).
class Index {
 public:
  Index() : id_(next_id()), level_(0) {}
  Index operator!() const { return Index(id_, level_ + 1); }
  Index decremented() const { return Index(id_, level_ > 0 ? level_ - 1 : 0); }
  int id() const { return id_; }
  int level() const { return level_; }
  bool elementwise() const { return level_ > 0; }
  bool operator==(const Index& o) const { return id_ == o.id_ && level_ == o.level_; }
  bool same_id(const Index& o) const { return id_ == o.id_; }

 private:
  Index(int id, int level) : id_(id), level_(level) {}
  static int next_id() {
    static std::atomic<int> n{0};
    return n++;
  }
  int id_;
  int level_;
};
using Labels = std::vector<Index>;

// ---- sparse tensors ------------------------------------------------------------
// Run-time-order sparse multi-index array (SparseMIA<double, N> with N known
// at run time): LCO storage on the device, linIdxSequence, sorted flag.
class SparseTensor {
 public:
  SparseTensor() = default;
  explicit SparseTensor(std::vector<int64_t> dims) : dims_(std::move(dims)), seq_(dims_.size()) {
    std::iota(seq_.begin(), seq_.end(), 0);
    for (auto d : dims_)
      if (d <= 0) throw MIAParameterException("dimensions must be positive");
  }

  // Host upload: keys linearised under `seq` (default sequence if empty).
  void assign_host(const std::vector<uint64_t>& keys, const std::vector<double>& vals, bool is_sorted,
                   std::vector<int> seq = {}) {
    if (keys.size() != vals.size()) throw MIAParameterException("keys and values differ in length");
    pk_.clear();
    pv_.clear();
    keys_.resize(keys.size());
    vals_.resize(vals.size());
    if (!keys.empty()) {
      cuda_check(cudaMemcpy(keys_.data(), keys.data(), keys.size() * 8, cudaMemcpyHostToDevice), "upload");
      cuda_check(cudaMemcpy(vals_.data(), vals.data(), vals.size() * 8, cudaMemcpyHostToDevice), "upload");
    }
    if (!seq.empty()) seq_ = std::move(seq);
    sorted_ = is_sorted;
  }
  void download(std::vector<uint64_t>& keys, std::vector<double>& vals) const {
    sync_();
    keys.resize(size());
    vals.resize(size());
    if (size()) {
      cuda_check(cudaMemcpy(keys.data(), keys_.data(), size() * 8, cudaMemcpyDeviceToHost), "download");
      cuda_check(cudaMemcpy(vals.data(), vals_.data(), size() * 8, cudaMemcpyDeviceToHost), "download");
    }
  }

  size_t order() const { return dims_.size(); }
  const std::vector<int64_t>& dims() const { return dims_; }
  int64_t dim(size_t i) const { return dims_[i]; }
  const std::vector<int>& linIdxSequence() const { return seq_; }
  bool is_sorted() const { return sorted_; }
  void setSorted(bool s) { sorted_ = s; }
  size_t size() const { return keys_.size() + pk_.size(); }
  uint64_t dimensionality() const {
    uint64_t d = 1;
    for (auto x : dims_) d *= (uint64_t)x;
    return d;
  }
  uint64_t* keys() { return sync_(), keys_.data(); }
  double* vals() { return sync_(), vals_.data(); }
  const uint64_t* keys() const { return sync_(), keys_.data(); }
  const double* vals() const { return sync_(), vals_.data(); }

  // SparseMIA::push_back (SparseMIA.h:570-578): appends one entry whose key is
  // in this tensor's linIdxSequence; the sorted flag drops when the key is
  // below the previous last key.  Entries wait on the host and go to the
  // device in one copy at the next operation that reads the storage.
  void push_back(double value, uint64_t key) {
    if (sorted_ && size() > 0 && key < last_key_()) sorted_ = false;
    pk_.push_back(key);
    pv_.push_back(value);
  }

  // SparseMIABase::change_linIdx_sequence (SparseMIABase.h:768-814)
  void change_linIdx_sequence(const std::vector<int>& seq) {
    if (seq == seq_ || order() == 1) return;
    if (size()) {
      check(lnt_rekey(keys(), keys(), size(), (int)order(), dims_.data(), seq_.data(), seq.data(), nullptr),
            "change_linIdx_sequence");
    }
    seq_ = seq;
    sorted_ = false;
  }

  // SparseMIABase::sort() (SparseMIABase.h:701-734)
  void sort() {
    if (!sorted_ && size()) sort_keys_();
    sorted_ = true;
  }

  // SparseMIABase::sort(seq) (SparseMIABase.h:590-645)
  void sort(const std::vector<int>& seq) {
    if (!sorted_) {
      change_linIdx_sequence(seq);
      sort();
    } else if (order() != 1 && seq != seq_) {
      change_linIdx_sequence(seq);
      if (size()) sort_keys_();
      if (size() < 3000) {  // the introsort branch returns before setSorted(true)
        sorted_ = false;
        return;
      }
      sorted_ = true;
    } else {
      sorted_ = true;
    }
  }

  // SparseMIA::collect_duplicates(std::plus) (SparseMIA.h:636-665)
  void collect_duplicates() {
    if (!size()) {
      sorted_ = true;
      return;
    }
    const size_t n = size();
    DeviceBuffer<uint64_t> k(n);
    DeviceBuffer<double> v(n);
    DeviceBuffer<uint64_t> cnt(1);
    size_t need = 0;
    check(lnt_sort_reduce_workspace(n, 0, dimensionality(), &need), "collect_duplicates");
    if (sorted_) {
      check(lnt_collect_duplicates_workspace(n, &need), "collect_duplicates");
      check(lnt_collect_duplicates(keys(), vals(), n, 1, k.data(), v.data(), cnt.data(), scratch(need), need,
                                   nullptr),
            "collect_duplicates");
    } else {
      check(lnt_sort_reduce(keys(), vals(), n, nullptr, nullptr, nullptr, 0, nullptr, 1.0, dimensionality(), 1,
                            k.data(), v.data(), cnt.data(), scratch(need), need, nullptr),
            "collect_duplicates");
    }
    const uint64_t m = read_u64(cnt.data());
    k.shrink(m);
    v.shrink(m);
    keys_ = std::move(k);
    vals_ = std::move(v);
    sorted_ = true;
  }

  // internal: replace storage
  void take(DeviceBuffer<uint64_t>&& k, DeviceBuffer<double>&& v) {
    pk_.clear();
    pv_.clear();
    keys_ = std::move(k);
    vals_ = std::move(v);
  }
  void set_seq(std::vector<int> s) { seq_ = std::move(s); }
  void set_dims(std::vector<int64_t> d) { dims_ = std::move(d); }

 private:
  void sort_keys_() {
    const size_t n = size();
    DeviceBuffer<uint64_t> k(n);
    DeviceBuffer<double> v(n);
    size_t need = 0;
    check(lnt_permute_sort_workspace(n, dimensionality(), &need), "sort");
    check(lnt_permute_sort(keys(), vals(), n, nullptr, k.data(), v.data(), dimensionality(), scratch(need), need,
                           nullptr),
          "sort");
    keys_ = std::move(k);
    vals_ = std::move(v);
  }

  // appends the entries staged by push_back to the device storage
  void sync_() const {
    if (pk_.empty()) return;
    const size_t n = keys_.size(), m = pk_.size();
    DeviceBuffer<uint64_t> k(n + m);
    DeviceBuffer<double> v(n + m);
    if (n) {
      cuda_check(cudaMemcpy(k.data(), keys_.data(), n * 8, cudaMemcpyDeviceToDevice), "push_back");
      cuda_check(cudaMemcpy(v.data(), vals_.data(), n * 8, cudaMemcpyDeviceToDevice), "push_back");
    }
    cuda_check(cudaMemcpy(k.data() + n, pk_.data(), m * 8, cudaMemcpyHostToDevice), "push_back");
    cuda_check(cudaMemcpy(v.data() + n, pv_.data(), m * 8, cudaMemcpyHostToDevice), "push_back");
    keys_ = std::move(k);
    vals_ = std::move(v);
    pk_.clear();
    pv_.clear();
  }
  uint64_t last_key_() const {
    if (!pk_.empty()) return pk_.back();
    uint64_t h = 0;
    cuda_check(cudaMemcpy(&h, keys_.data() + keys_.size() - 1, 8, cudaMemcpyDeviceToHost), "push_back");
    return h;
  }

  std::vector<int64_t> dims_;
  std::vector<int> seq_;
  bool sorted_ = true;  // the dims-only constructor's default (SparseMIABase.h:220)
  mutable DeviceBuffer<uint64_t> keys_;  // mutable: staged push_back entries are appended on first read
  mutable DeviceBuffer<double> vals_;
  mutable std::vector<uint64_t> pk_;     // push_back entries not yet on the device
  mutable std::vector<double> pv_;
};

// ---- expression layer ---------------------------------------------------------
namespace detail {

inline std::vector<int> reverse_order(const std::vector<int>& o) {  // IndexUtil.h:893-914
  std::vector<int> r(o.size(), (int)o.size());
  for (size_t i = 0; i < o.size(); ++i)
    for (size_t j = 0; j < o.size(); ++j)
      if (o[j] == (int)i) {
        r[i] = (int)j;
        break;
      }
  return r;
}

inline std::vector<int> reorder_from(const std::vector<int>& from, const std::vector<int>& seq) {  // IndexUtil.h:231-252
  std::vector<int> r(seq.size());
  for (size_t i = 0; i < seq.size(); ++i) r[i] = from[seq[i]];
  return r;
}

// pull_match_order (ExprUtil.h:511-562): position of every left label in the right operand
inline std::vector<int> match_order(const Labels& l, const Labels& r) {
  if (l.size() != r.size()) throw MIAParameterException("operands of a merge must have the same order");
  std::vector<int> o(l.size());
  for (size_t i = 0; i < l.size(); ++i) {
    int pos = -1;
    for (size_t j = 0; j < r.size(); ++j)
      if (r[j].same_id(l[i])) pos = (int)j;
    if (pos < 0) throw MIAParameterException("merge operands must carry the same index labels");
    o[i] = pos;
  }
  return o;
}

struct ProductOrders {
  std::vector<int> l_outer, l_inner, l_inter, r_outer, r_inner, r_inter;
};

// solve_product_expr_helper (MIA_Expr.h:449-529) over pull_left_operand_index_sequence
// (ExprUtil.h:311-393) and pull_right_index_order (ExprUtil.h:564-645)
inline ProductOrders product_orders(const Labels& l, const Labels& r) {
  ProductOrders o;
  for (size_t i = 0; i < l.size(); ++i) {
    int n = 0, same_id = 0;
    for (const auto& x : r) {
      n += (x == l[i]);
      same_id += x.same_id(l[i]);
    }
    if (n > 1) throw MIAParameterException("index repeated in an operand");
    if (n == 0 && same_id) throw MIAParameterException("an index appears with different element-wise marks");
    if (n == 0)
      o.l_outer.push_back((int)i);
    else if (l[i].elementwise())
      o.l_inter.push_back((int)i);
    else
      o.l_inner.push_back((int)i);
  }
  auto find = [&](const Index& x) {
    for (size_t j = 0; j < r.size(); ++j)
      if (r[j] == x) return (int)j;
    return -1;
  };
  for (size_t j = 0; j < r.size(); ++j) {
    bool in_l = false;
    for (const auto& x : l) in_l = in_l || x == r[j];
    if (!in_l) o.r_outer.push_back((int)j);
  }
  for (int i : o.l_inner) o.r_inner.push_back(find(l[i]));
  for (int i : o.l_inter) o.r_inter.push_back(find(l[i]));
  return o;
}

inline uint64_t prod_dims(const SparseTensor& m, const std::vector<int>& modes) {
  uint64_t p = 1;
  for (int i : modes) p *= (uint64_t)m.dim(i);
  return p;
}

// toStraightLattice / toLatticeSort (SparseMIABase.h:1457-1586), column major:
// sort under rows+cols+tabs and clear the sorted flag.
inline void to_lattice(SparseTensor& m, const std::vector<int>& rows, const std::vector<int>& cols,
                       const std::vector<int>& tabs) {
  std::vector<int> seq = rows;
  seq.insert(seq.end(), cols.begin(), cols.end());
  seq.insert(seq.end(), tabs.begin(), tabs.end());
  m.sort(seq);
  m.setSorted(false);
}

}  // namespace detail

struct SparseAtom;

// The result of an expression: an owned tensor and its labels.
struct SparseExpr {
  SparseTensor t;
  Labels labels;
  size_t inter = 0;  // trailing element-wise (inter) labels of a product result
};

// a(i, j, k): a tensor viewed with labels (MIA_Atom, MIA_Expr.h:738-1400).
struct SparseAtom {
  SparseTensor* m;
  Labels labels;
  std::shared_ptr<SparseTensor> owned;  // set when the atom holds a contraction / attraction result

  // c(...) = expression: relabel only (SparseMIA::assign, SparseMIA.h:891-928)
  SparseAtom& operator=(SparseExpr&& e) {
    if (e.labels.size() != labels.size()) throw MIAParameterException("assignment between different orders");
    bool same = true;  // labels match by identity, whatever their element-wise marks
    for (size_t q = 0; q < labels.size(); ++q) same = same && labels[q].same_id(e.labels[q]);
    if (same) {
      *m = std::move(e.t);
      return *this;
    }
    const std::vector<int> index_order = detail::match_order(labels, e.labels);
    std::vector<int64_t> nd(labels.size());
    for (size_t i = 0; i < labels.size(); ++i) nd[i] = e.t.dim(index_order[i]);
    const std::vector<int> lhs = detail::reverse_order(index_order);
    std::vector<int> nseq(labels.size());
    for (size_t i = 0; i < labels.size(); ++i) nseq[i] = lhs[e.t.linIdxSequence()[i]];
    e.t.set_dims(nd);
    e.t.set_seq(nseq);
    *m = std::move(e.t);
    return *this;
  }
  SparseAtom& operator=(const SparseAtom& o) {
    SparseExpr e{*o.m, o.labels};
    return *this = std::move(e);
  }
  SparseAtom& operator+=(const SparseAtom& o);
  SparseAtom& operator-=(const SparseAtom& o);
};

namespace detail {

// SparseMIA::sortMerge (SparseMIA.h:833-887): C is a copy of A; both unsorted.
inline void sort_merge(SparseTensor& c, SparseTensor& b, const std::vector<int>& index_order, int op) {
  lnt_rekey_spec spec{};
  const lnt_rekey_spec* a_spec = nullptr;
  const lnt_rekey_spec* b_spec = nullptr;
  std::vector<int> new_seq;
  const SparseTensor* rekeyed = nullptr;
  if (c.size() > b.size()) {
    new_seq = reorder_from(index_order, c.linIdxSequence());  // b into c's order; b itself is re-keyed
    b.change_linIdx_sequence(new_seq);
  } else {
    new_seq = reorder_from(reverse_order(index_order), b.linIdxSequence());
    rekeyed = &c;
  }
  if (rekeyed) {  // fused: c re-keyed inside the sort's first pass
    spec.order = (int32_t)c.order();
    for (size_t i = 0; i < c.order(); ++i) {
      spec.cur_seq[i] = c.linIdxSequence()[i];
      spec.new_seq[i] = new_seq[i];
      spec.dims[i] = c.dim(i);
    }
    a_spec = &spec;
  }
  const size_t na = c.size(), nb = b.size(), n = na + nb;
  DeviceBuffer<uint64_t> k(std::max<size_t>(n, 1));
  DeviceBuffer<double> v(std::max<size_t>(n, 1));
  DeviceBuffer<uint64_t> cnt(1);
  size_t need = 0;
  check(lnt_sort_reduce_workspace(na, nb, c.dimensionality(), &need), "merge");
  check(lnt_sort_reduce(c.keys(), c.vals(), na, a_spec, b.keys(), b.vals(), nb, b_spec, op == 1 ? -1.0 : 1.0,
                        c.dimensionality(), 1, k.data(), v.data(), cnt.data(), scratch(need), need, nullptr),
        "merge");
  const uint64_t m = read_u64(cnt.data());
  k.shrink(m);
  v.shrink(m);
  if (rekeyed) c.set_seq(new_seq);
  c.take(std::move(k), std::move(v));
  c.setSorted(true);
}

// SparseMIABase::outside_scanMerge (SparseMIABase.h:1404-1455)
inline SparseTensor scan_merge(SparseTensor& a, SparseTensor& b, const std::vector<int>& index_order, int op) {
  if (b.is_sorted() && !a.is_sorted()) {
    a.sort(reorder_from(reverse_order(index_order), b.linIdxSequence()));
  } else if (a.is_sorted() && !b.is_sorted()) {
    b.sort(reorder_from(index_order, a.linIdxSequence()));
  } else if (b.size() < a.size()) {
    b.sort(reorder_from(index_order, a.linIdxSequence()));
  } else {
    a.sort(reorder_from(reverse_order(index_order), b.linIdxSequence()));
  }
  SparseTensor c(a.dims());
  c.change_linIdx_sequence(a.linIdxSequence());  // empty: sets the sequence, clears the flag if it differs
  const size_t n = a.size() + b.size();
  DeviceBuffer<uint64_t> k(std::max<size_t>(n, 1));
  DeviceBuffer<double> v(std::max<size_t>(n, 1));
  DeviceBuffer<uint64_t> cnt(1);
  size_t need = 0;
  check(lnt_merge_sorted_workspace(a.size(), b.size(), &need), "merge");
  check(lnt_merge_sorted(a.keys(), a.vals(), a.size(), b.keys(), b.vals(), b.size(), op, k.data(), v.data(),
                         cnt.data(), scratch(need), need, nullptr),
        "merge");
  const uint64_t m = read_u64(cnt.data());
  k.shrink(m);
  v.shrink(m);
  c.take(std::move(k), std::move(v));
  return c;
}

// perform_outside_merge (SparseMIABase.h:1377-1402)
inline SparseExpr merge(SparseAtom& a, SparseAtom& b, int op) {
  const std::vector<int> order = match_order(a.labels, b.labels);
  for (size_t i = 0; i < order.size(); ++i)
    if (a.m->dim(i) != b.m->dim(order[i])) throw DimensionMismatchException("merge dimension mismatch");
  SparseTensor bcopy;
  SparseTensor* bp = b.m;
  if (a.m == b.m) {  // self-merge: merge with a copy (SparseMIABase.h:1368-1372)
    bcopy = *b.m;
    bp = &bcopy;
  }
  if (a.m->is_sorted() || bp->is_sorted()) return {scan_merge(*a.m, *bp, order, op), a.labels};
  SparseTensor c = *a.m;
  sort_merge(c, *bp, order, op);
  return {std::move(c), a.labels};
}

// MIA_Atom::operator* for pure outer / element-wise products (MIA_Expr.h:
// 1012-1057) -> SparseMIABase::noLatticeMult (SparseMIABase.h:1701-1826): both
// operands are sorted in place under [outer, inter] (and stay flagged sorted),
// C = [a outer, b outer, inter] comes out sorted, equal keys are not folded.
inline SparseExpr nolattice_product(SparseAtom& a, SparseAtom& b, const ProductOrders& o) {
  SparseTensor bcopy;
  SparseTensor* bp = b.m;
  if (a.m == b.m) {  // the product sorts both operands: multiply by a copy (SparseMIABase.h:1706-1710)
    bcopy = *b.m;
    bp = &bcopy;
  }
  for (size_t q = 0; q < o.l_inter.size(); ++q)
    if (a.m->dim(o.l_inter[q]) != bp->dim(o.r_inter[q]))
      throw DimensionMismatchException("Element-wise dimensions must match during MIA multiplication");
  std::vector<int> sa = o.l_outer, sb = o.r_outer;
  sa.insert(sa.end(), o.l_inter.begin(), o.l_inter.end());
  sb.insert(sb.end(), o.r_inter.begin(), o.r_inter.end());
  a.m->sort(sa);
  bp->sort(sb);
  const int64_t d = (int64_t)prod_dims(*a.m, o.l_inter);
  lnt_lattice A{a.m->keys(), a.m->vals(), a.m->size(), (int64_t)prod_dims(*a.m, o.l_outer), 1, d};
  lnt_lattice B{bp->keys(), bp->vals(), bp->size(), 1, (int64_t)prod_dims(*bp, o.r_outer), d};
  size_t need = 0;
  check(lnt_nolattice_mult_workspace(&A, &B, &need), "product");
  void* ws = scratch(need);
  DeviceBuffer<uint64_t> cnt(1);
  check(lnt_nolattice_mult_count(&A, &B, ws, need, cnt.data(), nullptr), "product");
  const uint64_t n = read_u64(cnt.data());
  DeviceBuffer<uint64_t> k(std::max<uint64_t>(n, 1));
  DeviceBuffer<double> v(std::max<uint64_t>(n, 1));
  check(lnt_nolattice_mult(&A, &B, n, ws, need, k.data(), v.data(), nullptr), "product");
  k.shrink(n);
  v.shrink(n);
  std::vector<int64_t> dims;
  Labels labels;
  for (int i : o.l_outer) dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  for (int j : o.r_outer) dims.push_back(bp->dim(j)), labels.push_back(b.labels[j]);
  for (int i : o.l_inter) dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  SparseTensor c(dims);
  c.take(std::move(k), std::move(v));
  c.setSorted(true);  // C.setSorted(true) (SparseMIABase.h:1822)
  return {std::move(c), std::move(labels), o.l_inter.size()};
}

// MIA_Atom::operator* for the lattice case (MIA_Expr.h:864-925) -> csc_no_accum.
inline SparseExpr product(SparseAtom& a, SparseAtom& b) {
  const ProductOrders o = product_orders(a.labels, b.labels);
  if (o.l_inner.empty()) return nolattice_product(a, b, o);
  SparseTensor bcopy;
  SparseTensor* bp = b.m;
  if (a.m == b.m) {  // check_if_copy_needed (MIA_Expr.h:767-802)
    bcopy = *b.m;
    bp = &bcopy;
  }
  for (size_t q = 0; q < o.l_inner.size(); ++q)
    if (a.m->dim(o.l_inner[q]) != bp->dim(o.r_inner[q])) throw DimensionMismatchException("inner dimensions differ");
  for (size_t q = 0; q < o.l_inter.size(); ++q)
    if (a.m->dim(o.l_inter[q]) != bp->dim(o.r_inter[q]))
      throw DimensionMismatchException("element-wise dimensions differ");
  to_lattice(*a.m, o.l_outer, o.l_inner, o.l_inter);
  to_lattice(*bp, o.r_inner, o.r_outer, o.r_inter);
  lnt_lattice A{a.m->keys(), a.m->vals(), a.m->size(), (int64_t)prod_dims(*a.m, o.l_outer),
                (int64_t)prod_dims(*a.m, o.l_inner), (int64_t)prod_dims(*a.m, o.l_inter)};
  lnt_lattice B{bp->keys(), bp->vals(), bp->size(), (int64_t)prod_dims(*bp, o.r_inner),
                (int64_t)prod_dims(*bp, o.r_outer), (int64_t)prod_dims(*bp, o.r_inter)};
  size_t plan_bytes = 0;
  check(lnt_lattice_mult_plan_workspace(&A, &B, &plan_bytes), "product");
  DeviceBuffer<unsigned char> plan(plan_bytes);
  DeviceBuffer<uint64_t> counts(2);
  check(lnt_lattice_mult_plan(&A, &B, plan.data(), plan_bytes, counts.data(), nullptr), "product");
  uint64_t hc[2];
  cuda_check(cudaMemcpy(hc, counts.data(), 16, cudaMemcpyDeviceToHost), "product counts");
  size_t need = 0;
  check(lnt_lattice_mult_workspace(&A, &B, hc[0], &need), "product");
  DeviceBuffer<uint64_t> k(std::max<uint64_t>(hc[1], 1));
  DeviceBuffer<double> v(std::max<uint64_t>(hc[1], 1));
  DeviceBuffer<uint64_t> nc(1);
  check(lnt_lattice_mult(&A, &B, plan.data(), hc[0], scratch(need), need, k.data(), v.data(), nc.data(), nullptr),
        "product");
  const uint64_t m = read_u64(nc.data());
  k.shrink(m);
  v.shrink(m);
  std::vector<int64_t> dims;
  Labels labels;
  for (int i : o.l_outer) dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  for (int j : o.r_outer) dims.push_back(bp->dim(j)), labels.push_back(b.labels[j]);
  for (int i : o.l_inter) dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  SparseTensor c(dims);  // default sequence, sorted (SparseMIA.h:362-372)
  c.take(std::move(k), std::move(v));
  c.setSorted(true);
  return {std::move(c), std::move(labels), o.l_inter.size()};
}

}  // namespace detail

inline SparseExpr operator+(SparseAtom a, SparseAtom b) { return detail::merge(a, b, 0); }
inline SparseExpr operator-(SparseAtom a, SparseAtom b) { return detail::merge(a, b, 1); }
inline SparseExpr operator*(SparseAtom a, SparseAtom b) { return detail::product(a, b); }

// Expressions as operands (a product or merge result feeding a further one,
// as MIA_Atom temporaries with ownership do in the reference): the result is
// held by an atom that owns it.
namespace detail {
inline SparseAtom hold(SparseExpr&& e) {
  auto p = std::make_shared<SparseTensor>(std::move(e.t));
  SparseAtom a{p.get(), std::move(e.labels), {}};
  a.owned = std::move(p);
  return a;
}
}  // namespace detail
inline SparseExpr operator*(SparseExpr a, SparseAtom b) { return detail::hold(std::move(a)) * b; }
inline SparseExpr operator*(SparseAtom a, SparseExpr b) { return a * detail::hold(std::move(b)); }
inline SparseExpr operator*(SparseExpr a, SparseExpr b) { return detail::hold(std::move(a)) * detail::hold(std::move(b)); }
inline SparseExpr operator+(SparseExpr a, SparseAtom b) { return detail::hold(std::move(a)) + b; }
inline SparseExpr operator+(SparseAtom a, SparseExpr b) { return a + detail::hold(std::move(b)); }
inline SparseExpr operator+(SparseExpr a, SparseExpr b) { return detail::hold(std::move(a)) + detail::hold(std::move(b)); }
inline SparseExpr operator-(SparseExpr a, SparseAtom b) { return detail::hold(std::move(a)) - b; }
inline SparseExpr operator-(SparseAtom a, SparseExpr b) { return a - detail::hold(std::move(b)); }
inline SparseExpr operator-(SparseExpr a, SparseExpr b) { return detail::hold(std::move(a)) - detail::hold(std::move(b)); }

// Destructive merges (perform_destructive_merge -> SparseMIA::merge, SparseMIA.h:1030-1060):
// the result replaces the left operand.
inline SparseAtom& SparseAtom::operator+=(const SparseAtom& o) {
  SparseAtom b = o;
  SparseExpr e = detail::merge(*this, b, 0);
  *m = std::move(e.t);
  return *this;
}
inline SparseAtom& SparseAtom::operator-=(const SparseAtom& o) {
  SparseAtom b = o;
  SparseExpr e = detail::merge(*this, b, 1);
  *m = std::move(e.t);
  return *this;
}

namespace detail {

// Repeated labels inside one operand (perform_unary, MIA_Expr.h:690-735):
// classification as unary_helper (MIA_Expr.h:632-662) with
// pull_contract_indices / pull_attract_indices / pull_sequence_from_list
// (ExprUtil.h:80-300) - a plain label repeated is contracted, an element-wise
// label repeated among the rest is attracted, sets in the order of their
// labels' last occurrences, positions ascending - then
// SparseMIABase::contract_attract (SparseMIABase.h:1913-2053): the operand is
// sorted in place under [contract, attract, other]; the result has modes
// [other..., one per attraction] and its sorted flag as push_back leaves it.
inline SparseAtom unary(SparseTensor& t, Labels labels) {
  auto count = [](const Labels& seq, const Index& x) {
    return (int)std::count(seq.begin(), seq.end(), x);
  };
  auto pull = [&](const Labels& seq, bool elem, Labels& found, Labels& rest) {
    for (size_t q = seq.size(); q-- > 0;)
      if (count(seq, seq[q]) > 1 && seq[q].elementwise() == elem && !count(found, seq[q]))
        found.insert(found.begin(), seq[q]);
    for (const Index& x : seq)
      if (!(count(seq, x) > 1 && x.elementwise() == elem)) rest.push_back(x);
  };
  Labels con, rest1, att, rest2;
  pull(labels, false, con, rest1);
  pull(rest1, true, att, rest2);
  if (con.empty() && att.empty()) return SparseAtom{&t, std::move(labels), nullptr};
  std::vector<int> seq, cpart, apart;
  auto positions = [&](const Labels& sub, std::vector<int>& part) {
    for (const Index& x : sub) {
      int c = 0;
      for (size_t q = 0; q < labels.size(); ++q)
        if (labels[q] == x) seq.push_back((int)q), ++c;
      part.push_back(c);
    }
  };
  positions(con, cpart);
  positions(att, apart);
  std::vector<int> other;
  for (int q = 0; q < (int)labels.size(); ++q)
    if (std::find(seq.begin(), seq.end(), q) == seq.end()) other.push_back(q);
  seq.insert(seq.end(), other.begin(), other.end());
  t.sort(seq);
  std::vector<int64_t> sdims, rdims;
  for (int q : seq) sdims.push_back(t.dim(q));
  for (int q : other) rdims.push_back(t.dim(q));
  size_t at = 0;
  for (int q = 0; q < (int)cpart.size(); ++q) at += (size_t)cpart[q];
  for (int c : apart) {
    rdims.push_back(sdims[at]);
    at += (size_t)c;
  }
  size_t need = 0;
  check(lnt_contract_attract_workspace(t.size(), &need), "contract_attract");
  const size_t n = t.size();
  DeviceBuffer<uint64_t> k(std::max<size_t>(n, 1));
  DeviceBuffer<double> v(std::max<size_t>(n, 1));
  DeviceBuffer<uint64_t> cnt(1);
  DeviceBuffer<uint32_t> flag(1);
  check(lnt_contract_attract(t.keys(), t.vals(), n, (int)sdims.size(), sdims.data(), (int)cpart.size(), cpart.data(),
                             (int)apart.size(), apart.data(), k.data(), v.data(), cnt.data(), flag.data(),
                             scratch(need), need, nullptr),
        "contract_attract");
  const uint64_t m = read_u64(cnt.data());
  uint32_t sorted = 0;
  cuda_check(cudaMemcpy(&sorted, flag.data(), 4, cudaMemcpyDeviceToHost), "contract_attract flag");
  k.shrink(m);
  v.shrink(m);
  auto r = std::make_shared<SparseTensor>(rdims);
  r->take(std::move(k), std::move(v));
  r->setSorted(sorted != 0);
  Labels rl = rest2;
  rl.insert(rl.end(), att.begin(), att.end());
  return SparseAtom{r.get(), std::move(rl), r};
}

}  // namespace detail

// SparseNT<N> / SparseMIA<double, N>: a SparseTensor of fixed order N.
template <size_t N>
class SparseNT : public SparseTensor {
 public:
  SparseNT() : SparseTensor(std::vector<int64_t>(N, 1)) {}
  template <class... D, typename = std::enable_if_t<sizeof...(D) == N>>
  explicit SparseNT(D... dims) : SparseTensor(std::vector<int64_t>{(int64_t)dims...}) {}
  template <class... I, typename = std::enable_if_t<sizeof...(I) == N>>
  SparseAtom operator()(const I&... idx) {
    return detail::unary(*this, Labels{idx...});
  }
  SparseNT& operator=(SparseTensor&& t) {
    if (t.order() != N) throw MIAParameterException("order mismatch");
    SparseTensor::operator=(std::move(t));
    return *this;
  }
};
template <class T, size_t N>
using SparseMIA = SparseNT<N>;

// ---- dense tensors -------------------------------------------------------------
// Column-major dense multi-index array (DenseMIA<double, N>); products run as
// lattice products (DenseLatticeBase::operator*).  By default they are
// float64-class products emulated on the INT8 tensor cores (Ozaki scheme II,
// lnt_dense_lattice_mult_crt): every entry of C is within 1e-12 of
// (|A||B|)_ij -- the error metric is relative to the product of magnitudes,
// not to |C_ij|, which cancellation can make arbitrarily small -- with the
// number of moduli chosen from the operands (lnt_dense_crt_moduli).
// precision() = Precision::Float64 selects the plain float64 GEMM, slices() > 0
// the scheme I slices (error about 2^(1-7s) |A||B|).
class DenseTensor {
 public:
  DenseTensor() = default;
  explicit DenseTensor(std::vector<int64_t> dims) : dims_(std::move(dims)) { data_.resize(numel()); }
  size_t order() const { return dims_.size(); }
  const std::vector<int64_t>& dims() const { return dims_; }
  int64_t dim(size_t i) const { return dims_[i]; }
  size_t numel() const {
    size_t n = 1;
    for (auto d : dims_) n *= (size_t)d;
    return n;
  }
  double* data() { return data_.data(); }
  const double* data() const { return data_.data(); }
  void upload(const std::vector<double>& h) {
    if (h.size() != numel()) throw MIAParameterException("size mismatch");
    cuda_check(cudaMemcpy(data(), h.data(), h.size() * 8, cudaMemcpyHostToDevice), "upload");
  }
  void download(std::vector<double>& h) const {
    h.resize(numel());
    cuda_check(cudaMemcpy(h.data(), data(), h.size() * 8, cudaMemcpyDeviceToHost), "download");
  }
  enum class Precision { Emulated, Float64 };
  static Precision& precision() {  // Emulated (default): scheme II within 1e-12 of |A||B|
    thread_local Precision p = Precision::Emulated;
    return p;
  }
  static int& slices() {  // > 0 (5..8): scheme I with that many slices, overriding precision()
    thread_local int s = 0;
    return s;
  }

 private:
  std::vector<int64_t> dims_;
  DeviceBuffer<double> data_;
};

struct DenseExpr {
  DenseTensor t;
  Labels labels;
  size_t inter = 0;  // trailing element-wise (inter) labels of a product result
};

struct DenseAtom {
  DenseTensor* m;
  Labels labels;
  // DenseMIA assignment (MIA_Atom::operator=, MIA_Expr.h:1114-1182): labels
  // match by identity; a different label order permutes the result's modes
  // into the target's (inplace_permute, DenseMIA.h:700-780).
  DenseAtom& operator=(DenseExpr&& e) {
    if (e.labels.size() != labels.size()) throw MIAParameterException("assignment between different orders");
    std::vector<int32_t> perm(labels.size());
    bool identity = true;
    for (size_t q = 0; q < labels.size(); ++q) {
      int pos = -1;
      for (size_t r = 0; r < e.labels.size(); ++r)
        if (e.labels[r].same_id(labels[q])) pos = (int)r;
      if (pos < 0) throw MIAParameterException("assignment with different index labels");
      perm[q] = pos;
      identity = identity && pos == (int)q;
    }
    if (identity) {
      *m = std::move(e.t);
      return *this;
    }
    std::vector<int64_t> nd;
    for (int32_t q : perm) nd.push_back(e.t.dim(q));
    DenseTensor out(nd);
    check(lnt_dense_permute(e.t.data(), out.data(), (int)e.t.order(), e.t.dims().data(), perm.data(), nullptr),
          "dense assignment");
    *m = std::move(out);
    return *this;
  }
};

namespace detail {

// A dense operand's data in the lattice order [x, y, z] (mode indices): its own
// buffer when the modes are already in that order (toStraightLattice,
// DenseMIA.h:1240-1255), else a permuted copy held in `copy` (latticeCopy,
// FunctionUtil.h:195; the operand itself is left as it is).
inline const double* lattice_data(const DenseTensor& t, const std::vector<int>& x, const std::vector<int>& y,
                                  const std::vector<int>& z, DenseTensor& copy) {
  std::vector<int> s = x;
  s.insert(s.end(), y.begin(), y.end());
  s.insert(s.end(), z.begin(), z.end());
  bool ordered = true;
  for (size_t i = 0; i < s.size(); ++i) ordered = ordered && s[i] == (int)i;
  if (ordered) return t.data();
  std::vector<int64_t> nd;
  for (int m : s) nd.push_back(t.dim(m));
  copy = DenseTensor(nd);
  const std::vector<int32_t> perm(s.begin(), s.end());
  check(lnt_dense_permute(t.data(), copy.data(), (int)t.order(), t.dims().data(), perm.data(), nullptr),
        "dense permute");
  return copy.data();
}

}  // namespace detail

inline DenseExpr operator*(DenseAtom a, DenseAtom b) {
  const detail::ProductOrders o = detail::product_orders(a.labels, b.labels);
  DenseTensor acopy, bcopy;
  const double* ad = detail::lattice_data(*a.m, o.l_outer, o.l_inner, o.l_inter, acopy);
  const double* bd = detail::lattice_data(*b.m, o.r_inner, o.r_outer, o.r_inter, bcopy);
  auto pd = [](const DenseTensor& t, const std::vector<int>& m) {
    int64_t p = 1;
    for (int i : m) p *= t.dim(i);
    return p;
  };
  const int64_t h = pd(*a.m, o.l_outer), w = pd(*a.m, o.l_inner), d = pd(*a.m, o.l_inter);
  const int64_t wB = pd(*b.m, o.r_outer);
  if (pd(*b.m, o.r_inner) != w || pd(*b.m, o.r_inter) != d) throw DimensionMismatchException("dense product dims");
  std::vector<int64_t> dims;
  Labels labels;
  for (int i : o.l_outer) dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  for (int j : o.r_outer) dims.push_back(b.m->dim(j)), labels.push_back(b.labels[j]);
  for (int i : o.l_inter) dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  DenseTensor c(dims);
  const int s = DenseTensor::slices();
  if (s > 0) {
    size_t need = 0;
    check(lnt_dense_split_workspace(h, w, wB, s, &need), "dense product");
    check(lnt_dense_lattice_mult_split(ad, bd, c.data(), h, w, wB, d, s, scratch(need), need, nullptr),
          "dense product");
  } else if (DenseTensor::precision() == DenseTensor::Precision::Float64 || w >= (int64_t{1} << 17)) {
    size_t need = 0;  // (scheme II needs w < 2^17: INT32 exactness of the residue products)
    check(lnt_dense_fp64_workspace(&need), "dense product");
    check(lnt_dense_lattice_mult_fp64(ad, bd, c.data(), h, w, wB, d, scratch(need), need, nullptr),
          "dense product");
  } else {
    int moduli = 0;
    const size_t qneed = (size_t)h * 16 + 768;
    check(lnt_dense_crt_moduli(ad, bd, h, w, wB, d, 1e-12, scratch(qneed), qneed, &moduli, nullptr),
          "dense product");
    size_t need = 0;
    check(lnt_dense_crt_workspace(h, w, wB, moduli, &need), "dense product");
    check(lnt_dense_lattice_mult_crt(ad, bd, c.data(), h, w, wB, d, moduli, scratch(need), need, nullptr),
          "dense product");
  }
  return {std::move(c), std::move(labels), o.l_inter.size()};
}

// ---- mixed sparse / dense products ---------------------------------------------
// MIA_Atom::operator* with one sparse and one dense operand (MIA_Expr.h:
// 864-925): the sparse operand becomes a sorted lattice, the dense one a
// zero-copy lattice or a permuted copy (detail::lattice_data), and the lattice
// product is the mixed one
// (SparseDenseLatticeMultMex).  The result is sparse with dims [left outer,
// right outer, inter]: every non-empty line of the sparse operand gives a full
// line of it.
namespace detail {

inline int64_t dense_prod(const DenseTensor& t, const std::vector<int>& m) {
  int64_t p = 1;
  for (int i : m) p *= t.dim(i);
  return p;
}

// S keyed as a lattice (column-major for dense_first, row-major otherwise)
inline void mixed_mult(const double* D, const lnt_lattice& S, int64_t other, int dense_first,
                       DeviceBuffer<uint64_t>& k, DeviceBuffer<double>& v) {
  size_t need = 0;
  check(lnt_sparse_dense_mult_workspace(&S, other, dense_first, &need), "mixed product");
  void* ws = scratch(need);
  DeviceBuffer<uint64_t> cnt(1);
  check(lnt_sparse_dense_mult_count(&S, other, dense_first, ws, need, cnt.data(), nullptr), "mixed product");
  const uint64_t n = read_u64(cnt.data());
  k = DeviceBuffer<uint64_t>(std::max<uint64_t>(n, 1));
  v = DeviceBuffer<double>(std::max<uint64_t>(n, 1));
  check(lnt_sparse_dense_mult(D, &S, other, dense_first, ws, need, k.data(), v.data(), nullptr), "mixed product");
  k.shrink(n);
  v.shrink(n);
}

}  // namespace detail

// SparseMIA * DenseMIA: SparseLatticeBase::operator*(DenseLatticeBase)
// (SparseLatticeBase.h:1148-1162).  The sparse operand is left sorted under
// [inner, outer, inter] (the row-major lattice order that product sorts it
// into), flagged unsorted; the result is re-keyed from the row-major lattice
// to the default sequence and flagged unsorted, as SparseMIA(dims,
// SparseLattice&&) does with a row-major lattice (SparseMIA.h:362-372).
inline SparseExpr operator*(SparseAtom a, DenseAtom b) {
  const detail::ProductOrders o = detail::product_orders(a.labels, b.labels);
  if (o.l_inner.empty()) throw MIAParameterException("a sparse x dense product needs a contracted index");
  const int64_t h = (int64_t)detail::prod_dims(*a.m, o.l_outer), w = (int64_t)detail::prod_dims(*a.m, o.l_inner);
  const int64_t d = (int64_t)detail::prod_dims(*a.m, o.l_inter), wB = detail::dense_prod(*b.m, o.r_outer);
  if (detail::dense_prod(*b.m, o.r_inner) != w || detail::dense_prod(*b.m, o.r_inter) != d)
    throw DimensionMismatchException("mixed product dims");
  detail::to_lattice(*a.m, o.l_inner, o.l_outer, o.l_inter);
  const lnt_lattice S{a.m->keys(), a.m->vals(), a.m->size(), h, w, d};
  DeviceBuffer<uint64_t> k;
  DeviceBuffer<double> v;
  DenseTensor bcopy;
  detail::mixed_mult(detail::lattice_data(*b.m, o.r_inner, o.r_outer, o.r_inter, bcopy), S, wB, 0, k, v);
  std::vector<int64_t> dims;
  Labels labels;
  std::vector<int> lo, ro, in;
  for (int i : o.l_outer) lo.push_back((int)dims.size()), dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  for (int j : o.r_outer) ro.push_back((int)dims.size()), dims.push_back(b.m->dim(j)), labels.push_back(b.labels[j]);
  for (int i : o.l_inter) in.push_back((int)dims.size()), dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  SparseTensor c(dims);
  c.take(std::move(k), std::move(v));
  std::vector<int> rowmajor = ro;  // keys j + wB (row + h tab)
  rowmajor.insert(rowmajor.end(), lo.begin(), lo.end());
  rowmajor.insert(rowmajor.end(), in.begin(), in.end());
  c.set_seq(rowmajor);
  std::vector<int> def(dims.size());
  std::iota(def.begin(), def.end(), 0);
  c.change_linIdx_sequence(def);
  c.setSorted(false);
  return {std::move(c), std::move(labels), o.l_inter.size()};
}

// DenseMIA * SparseMIA: DenseLatticeBase::operator*(SparseLatticeBase)
// (DenseLatticeBase.h:436-500).  The sparse operand is sorted column-major
// (under [inner, outer, inter]) and flagged unsorted; the result's keys are in
// the default sequence, ascending, flagged sorted.
inline SparseExpr operator*(DenseAtom a, SparseAtom b) {
  const detail::ProductOrders o = detail::product_orders(a.labels, b.labels);
  if (o.l_inner.empty()) throw MIAParameterException("a dense x sparse product needs a contracted index");
  const int64_t h = detail::dense_prod(*a.m, o.l_outer), w = detail::dense_prod(*a.m, o.l_inner);
  const int64_t d = detail::dense_prod(*a.m, o.l_inter), wB = (int64_t)detail::prod_dims(*b.m, o.r_outer);
  if ((int64_t)detail::prod_dims(*b.m, o.r_inner) != w || (int64_t)detail::prod_dims(*b.m, o.r_inter) != d)
    throw DimensionMismatchException("mixed product dims");
  detail::to_lattice(*b.m, o.r_inner, o.r_outer, o.r_inter);
  const lnt_lattice S{b.m->keys(), b.m->vals(), b.m->size(), w, wB, d};
  DeviceBuffer<uint64_t> k;
  DeviceBuffer<double> v;
  DenseTensor acopy;
  detail::mixed_mult(detail::lattice_data(*a.m, o.l_outer, o.l_inner, o.l_inter, acopy), S, h, 1, k, v);
  std::vector<int64_t> dims;
  Labels labels;
  for (int i : o.l_outer) dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  for (int j : o.r_outer) dims.push_back(b.m->dim(j)), labels.push_back(b.labels[j]);
  for (int i : o.l_inter) dims.push_back(a.m->dim(i)), labels.push_back(a.labels[i]);
  SparseTensor c(dims);
  c.take(std::move(k), std::move(v));
  c.setSorted(true);
  return {std::move(c), std::move(labels), o.l_inter.size()};
}

// MIA_Atom::operator~ (MIA_Expr.h:1376-1379, decrement_back_indices,
// ExprUtil.h:740-766): the trailing element-wise (inter) labels of a product
// result lose one '!' each, so the result can take part in a further product
// with those indices at the lower level:
//   c(i,k,m,n) = ~(a(i,!j,k,!l) * b(!j,!l,m,n)) * d(j,l).
inline SparseExpr operator~(SparseExpr e) {
  for (size_t q = e.labels.size() - e.inter; q < e.labels.size(); ++q) e.labels[q] = e.labels[q].decremented();
  e.inter = 0;
  return e;
}
inline DenseExpr operator~(DenseExpr e) {
  for (size_t q = e.labels.size() - e.inter; q < e.labels.size(); ++q) e.labels[q] = e.labels[q].decremented();
  e.inter = 0;
  return e;
}

template <size_t N>
class DenseNT : public DenseTensor {
 public:
  template <class... D, typename = std::enable_if_t<sizeof...(D) == N>>
  explicit DenseNT(D... dims) : DenseTensor(std::vector<int64_t>{(int64_t)dims...}) {}
  template <class... I, typename = std::enable_if_t<sizeof...(I) == N>>
  DenseAtom operator()(const I&... idx) {
    return DenseAtom{this, Labels{idx...}};
  }
};
template <class T, size_t N>
using DenseMIA = DenseNT<N>;

}  // namespace lnt
