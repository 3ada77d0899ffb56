// Host-buffer gateways with the reference's mex wire formats (include/lnt_mex.h):
// copy in, run the device entry points of lnt.h, copy out.  Host code only.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/lnt_mex.h"
#include "lnt_common.cuh"

namespace {

typedef uint64_t u64;  // the ABI's key type

// Device buffer owned for the duration of one gateway call.
struct DevBuf {
  void* p = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t bytes) {
    return cudaMalloc(&p, std::max<size_t>(bytes, 256)) == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

int upload(DevBuf& d, const void* host, size_t bytes) {
  int st = d.alloc(bytes);
  if (st != LNT_OK) return st;
  if (bytes && cudaMemcpy(d.p, host, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return LNT_DEVICE_ERROR;
  return LNT_OK;
}

int download(void* host, const void* dev, size_t bytes) {
  if (bytes && cudaMemcpy(host, dev, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return LNT_DEVICE_ERROR;
  return LNT_OK;
}

int finish(int st) {
  if (st != LNT_OK) return st;
  return cudaDeviceSynchronize() == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
}

// non-negative keys; *max_key = largest key + 1
int check_keys(const int64_t* k, size_t n, u64* max_key) {
  if (n && !k) return LNT_BAD_ARG;
  u64 m = 0;
  for (size_t i = 0; i < n; ++i) {
    if (k[i] < 0) return LNT_BAD_ARG;
    m = std::max(m, (u64)k[i] + 1);
  }
  if (max_key) *max_key = std::max<u64>(m, 1);
  return LNT_OK;
}

// 1-based uint8 order -> 0-based int32 permutation of 0..order-1
int seq0(const uint8_t* s1, int order, std::vector<int32_t>& out) {
  if (!s1) return LNT_BAD_ARG;
  out.assign(order, 0);
  std::vector<char> seen(order, 0);
  for (int i = 0; i < order; ++i) {
    const int v = (int)s1[i] - 1;
    if (v < 0 || v >= order || seen[v]) return LNT_BAD_SEQ;
    seen[v] = 1;
    out[i] = v;
  }
  return LNT_OK;
}

int host_outputs(lnt_host_alloc alloc, size_t n, double** v, int64_t** k) {
  if (!v || !k) return LNT_BAD_ARG;
  const size_t bytes = std::max<size_t>(n, 1) * 8;
  *v = static_cast<double*>(alloc ? alloc(bytes) : std::malloc(bytes));
  *k = static_cast<int64_t*>(alloc ? alloc(bytes) : std::malloc(bytes));
  return (*v && *k) ? LNT_OK : LNT_BAD_ARG;
}

int read_count(const u64* d, u64* h) { return download(h, d, 8); }

// Sort (device keys, device vals) of n pairs in place, keys < max_key.
int sort_in_place(u64* k, double* v, size_t n, u64 max_key) {
  size_t wsb = 0;
  int st = lnt_sort_pairs_workspace(n, max_key, &wsb);
  if (st != LNT_OK) return st;
  DevBuf ws;
  if ((st = ws.alloc(wsb)) != LNT_OK) return st;
  return lnt_sort_pairs(k, v, k, v, n, max_key, ws.p, wsb, nullptr);
}

// Copies a device result of *nc pairs into caller-allocated host arrays.
int emit(lnt_host_alloc alloc, const u64* dk, const double* dv, u64 count, double** c_vals, int64_t** c_keys,
         size_t* nc) {
  int st = host_outputs(alloc, count, c_vals, c_keys);
  if (st != LNT_OK) return st;
  if ((st = download(*c_vals, dv, count * 8)) != LNT_OK) return st;
  if ((st = download(*c_keys, dk, count * 8)) != LNT_OK) return st;
  *nc = count;
  return LNT_OK;
}

}  // namespace

extern "C" {

int lnt_mex_sparse_sort(double* vals, int64_t* keys, size_t n) {
  if (n == 0) return LNT_OK;
  if (!vals) return LNT_BAD_ARG;
  u64 max_key = 0;
  int st = check_keys(keys, n, &max_key);
  if (st != LNT_OK) return st;
  DevBuf k, v;
  if ((st = upload(k, keys, n * 8)) != LNT_OK || (st = upload(v, vals, n * 8)) != LNT_OK) return st;
  if ((st = finish(sort_in_place(k.as<u64>(), v.as<double>(), n, max_key))) != LNT_OK) return st;
  if ((st = download(keys, k.p, n * 8)) != LNT_OK) return st;
  return download(vals, v.p, n * 8);
}

int lnt_mex_sparse_change_linidx(int64_t* keys, size_t n, int order, const uint8_t* cur, const uint8_t* desired,
                                 const int64_t* dims) {
  if (order < 1 || order > LNT_MAX_ORDER || !dims) return LNT_BAD_ARG;
  std::vector<int32_t> c, d;
  int st = seq0(cur, order, c);
  if (st != LNT_OK) return st;
  if ((st = seq0(desired, order, d)) != LNT_OK) return st;
  if (n == 0 || c == d) return LNT_OK;
  if ((st = check_keys(keys, n, nullptr)) != LNT_OK) return st;
  DevBuf k;
  if ((st = upload(k, keys, n * 8)) != LNT_OK) return st;
  st = lnt_rekey(k.as<u64>(), k.as<u64>(), n, order, dims, c.data(), d.data(), nullptr);
  if ((st = finish(st)) != LNT_OK) return st;
  return download(keys, k.p, n * 8);
}

int lnt_mex_sparse_permute(double* vals, int64_t* keys, size_t n, int order, const uint8_t* cur,
                           const uint8_t* desired, const int64_t* dims) {
  if (order < 1 || order > LNT_MAX_ORDER || !dims) return LNT_BAD_ARG;
  std::vector<int32_t> c, d;
  int st = seq0(cur, order, c);
  if (st != LNT_OK) return st;
  if ((st = seq0(desired, order, d)) != LNT_OK) return st;
  if (n == 0 || c == d) return LNT_OK;
  if (!vals) return LNT_BAD_ARG;
  unsigned __int128 total = 1;
  for (int i = 0; i < order; ++i) {
    if (dims[i] <= 0) return LNT_BAD_DIMS;
    total *= (u64)dims[i];
  }
  if (total >> 63) return LNT_OVERFLOW_KEYBITS;
  u64 max_key = 0;
  if ((st = check_keys(keys, n, &max_key)) != LNT_OK) return st;
  if (max_key > (u64)total) return LNT_BAD_ARG;
  DevBuf k, v;
  if ((st = upload(k, keys, n * 8)) != LNT_OK || (st = upload(v, vals, n * 8)) != LNT_OK) return st;
  if ((st = finish(sort_in_place(k.as<u64>(), v.as<double>(), n, (u64)total))) != LNT_OK) return st;
  if ((st = download(keys, k.p, n * 8)) != LNT_OK) return st;
  return download(vals, v.p, n * 8);
}

int lnt_mex_sparse_merge(const double* a_vals, const int64_t* a_keys, size_t na, const double* b_vals,
                         const int64_t* b_keys, size_t nb, int op, lnt_host_alloc alloc, double** c_vals,
                         int64_t** c_keys, size_t* nc) {
  if (!nc || (na && !a_vals) || (nb && !b_vals)) return LNT_BAD_ARG;
  int st = check_keys(a_keys, na, nullptr);
  if (st != LNT_OK || (st = check_keys(b_keys, nb, nullptr)) != LNT_OK) return st;
  DevBuf ak, av, bk, bv, ck, cv, cnt, ws;
  if ((st = upload(ak, a_keys, na * 8)) != LNT_OK || (st = upload(av, a_vals, na * 8)) != LNT_OK ||
      (st = upload(bk, b_keys, nb * 8)) != LNT_OK || (st = upload(bv, b_vals, nb * 8)) != LNT_OK ||
      (st = ck.alloc((na + nb) * 8)) != LNT_OK || (st = cv.alloc((na + nb) * 8)) != LNT_OK ||
      (st = cnt.alloc(8)) != LNT_OK)
    return st;
  size_t wsb = 0;
  if ((st = lnt_merge_sorted_workspace(na, nb, &wsb)) != LNT_OK || (st = ws.alloc(wsb)) != LNT_OK) return st;
  st = lnt_merge_sorted(ak.as<u64>(), av.as<double>(), na, bk.as<u64>(), bv.as<double>(), nb, op ? 1 : 0,
                        ck.as<u64>(), cv.as<double>(), cnt.as<u64>(), ws.p, wsb, nullptr);
  if ((st = finish(st)) != LNT_OK) return st;
  u64 m = 0;
  if ((st = read_count(cnt.as<u64>(), &m)) != LNT_OK) return st;
  return emit(alloc, ck.as<u64>(), cv.as<double>(), m, c_vals, c_keys, nc);
}

int lnt_mex_sparselattice_mult(const double* a_vals, const int64_t* a_keys, size_t na, const int64_t* a_dims,
                               const double* b_vals, const int64_t* b_keys, size_t nb, const int64_t* b_dims,
                               int alg, lnt_host_alloc alloc, double** c_vals, int64_t** c_keys, size_t* nc) {
  if (!nc || !a_dims || !b_dims || (na && !a_vals) || (nb && !b_vals)) return LNT_BAD_ARG;
  // 0 operator*, 1 csc_times<false>, 2 csc_times<true> (DCSC), 3 csc_no_accum: the
  // same product with the same pattern (zero sums kept) in column-major order.
  // 4 and 5 reach mtt_times (4 falls through into 5, sparselattice_mul.cpp:52-62),
  // whose body ends after its declarations without computing or returning a
  // result (SparseLatticeBase.h:1582-1640): nothing to reproduce.
  if (alg < 0 || alg > 3) return LNT_UNSUPPORTED;
  if (a_dims[1] != b_dims[0] || a_dims[2] != b_dims[2]) return LNT_BAD_DIMS;
  int st = check_keys(a_keys, na, nullptr);
  if (st != LNT_OK || (st = check_keys(b_keys, nb, nullptr)) != LNT_OK) return st;
  DevBuf ak, av, bk, bv, counts, plan;
  if ((st = upload(ak, a_keys, na * 8)) != LNT_OK || (st = upload(av, a_vals, na * 8)) != LNT_OK ||
      (st = upload(bk, b_keys, nb * 8)) != LNT_OK || (st = upload(bv, b_vals, nb * 8)) != LNT_OK ||
      (st = counts.alloc(16)) != LNT_OK)
    return st;
  const lnt_lattice A{ak.as<u64>(), av.as<double>(), na, a_dims[0], a_dims[1], a_dims[2]};
  const lnt_lattice B{bk.as<u64>(), bv.as<double>(), nb, b_dims[0], b_dims[1], b_dims[2]};
  size_t pb = 0;
  if ((st = lnt_lattice_mult_plan_workspace(&A, &B, &pb)) != LNT_OK || (st = plan.alloc(pb)) != LNT_OK) return st;
  if ((st = finish(lnt_lattice_mult_plan(&A, &B, plan.p, pb, counts.as<u64>(), nullptr))) != LNT_OK) return st;
  u64 hc[2];
  if ((st = download(hc, counts.p, 16)) != LNT_OK) return st;
  size_t wsb = 0;
  DevBuf ws, ck, cv;
  if ((st = lnt_lattice_mult_workspace(&A, &B, hc[0], &wsb)) != LNT_OK || (st = ws.alloc(wsb)) != LNT_OK ||
      (st = ck.alloc(hc[1] * 8)) != LNT_OK || (st = cv.alloc(hc[1] * 8)) != LNT_OK)
    return st;
  st = lnt_lattice_mult(&A, &B, plan.p, hc[0], ws.p, wsb, ck.as<u64>(), cv.as<double>(), counts.as<u64>(), nullptr);
  if ((st = finish(st)) != LNT_OK) return st;
  u64 m = 0;
  if ((st = read_count(counts.as<u64>(), &m)) != LNT_OK) return st;
  return emit(alloc, ck.as<u64>(), cv.as<double>(), m, c_vals, c_keys, nc);
}

int lnt_mex_sparse_denselattice_mult(const double* a_vals, const int64_t* a_keys, size_t na, const int64_t* a_dims,
                                     const double* B, const int64_t* b_dims, int dense_first, lnt_host_alloc alloc,
                                     double** c_vals, int64_t** c_keys, size_t* nc) {
  if (!nc || !a_dims || !b_dims || !B || (na && !a_vals)) return LNT_BAD_ARG;
  for (int i = 0; i < 3; ++i)
    if (a_dims[i] <= 0 || b_dims[i] <= 0) return LNT_BAD_DIMS;
  if (a_dims[2] != b_dims[2]) return LNT_BAD_DIMS;
  if (dense_first ? b_dims[1] != a_dims[0] : a_dims[1] != b_dims[0]) return LNT_BAD_DIMS;
  const unsigned __int128 dense_n = (unsigned __int128)(u64)b_dims[0] * (u64)b_dims[1] * (u64)b_dims[2];
  const unsigned __int128 sparse_n = (unsigned __int128)(u64)a_dims[0] * (u64)a_dims[1] * (u64)a_dims[2];
  if ((dense_n >> 60) || (sparse_n >> 63)) return LNT_OVERFLOW_KEYBITS;
  u64 max_key = 0;
  int st = check_keys(a_keys, na, &max_key);
  if (st != LNT_OK) return st;
  if (max_key > (u64)sparse_n) return LNT_BAD_ARG;
  DevBuf ak, av, db, cnt;
  if ((st = upload(ak, a_keys, na * 8)) != LNT_OK || (st = upload(av, a_vals, na * 8)) != LNT_OK ||
      (st = upload(db, B, (size_t)dense_n * 8)) != LNT_OK || (st = cnt.alloc(8)) != LNT_OK)
    return st;
  if (!dense_first && na) {  // the row-major lattice order the product sorts A into
    const int32_t cm[3] = {0, 1, 2}, rm[3] = {1, 0, 2};
    if ((st = lnt_rekey(ak.as<u64>(), ak.as<u64>(), na, 3, a_dims, cm, rm, nullptr)) != LNT_OK) return st;
  }
  if (na && (st = sort_in_place(ak.as<u64>(), av.as<double>(), na, (u64)sparse_n)) != LNT_OK) return st;
  const lnt_lattice S{ak.as<u64>(), av.as<double>(), na, a_dims[0], a_dims[1], a_dims[2]};
  const int64_t other = dense_first ? b_dims[0] : b_dims[1];
  size_t wsb = 0;
  DevBuf ws;
  if ((st = lnt_sparse_dense_mult_workspace(&S, other, dense_first ? 1 : 0, &wsb)) != LNT_OK ||
      (st = ws.alloc(wsb)) != LNT_OK)
    return st;
  st = lnt_sparse_dense_mult_count(&S, other, dense_first ? 1 : 0, ws.p, wsb, cnt.as<u64>(), nullptr);
  if ((st = finish(st)) != LNT_OK) return st;
  u64 m = 0;
  if ((st = read_count(cnt.as<u64>(), &m)) != LNT_OK) return st;
  DevBuf ck, cv;
  if ((st = ck.alloc(m * 8)) != LNT_OK || (st = cv.alloc(m * 8)) != LNT_OK) return st;
  st = lnt_sparse_dense_mult(db.as<double>(), &S, other, dense_first ? 1 : 0, ws.p, wsb, ck.as<u64>(),
                             cv.as<double>(), nullptr);
  if ((st = finish(st)) != LNT_OK) return st;
  return emit(alloc, ck.as<u64>(), cv.as<double>(), m, c_vals, c_keys, nc);
}

}  // extern "C"
