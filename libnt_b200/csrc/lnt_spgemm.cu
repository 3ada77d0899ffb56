// Sparse lattice product C_t = A_t * B_t for every tab t (the reference's
// SparseLatticeBase::operator* -> csc_no_accum<true>, SparseLatticeBase.h:
// 1572-1576, 1854-1990).  Lattices are column-major LCO: A key =
// row + h*(col + w*tab), B key = row + w*(col + wB*tab), both ascending; C key
// = row + h*(col + wB*tab), ascending, duplicates summed, exact zeros kept.
//
// Plan phase (both engines): A column pointers (dense over w*d columns when
// that fits, else binary search on A's keys), product count per B entry and
// its prefix sum (total = products P).
//
// SPA engine (h <= 1024, and A's w*d and B's w_B*d columns fit dense pointer
// arrays): one warp per output column (tab, col).  Lanes take B
// entries of the column, walk the matching A columns and add a*b into a
// dense h-row accumulator in shared memory while setting a row bitmap; the
// column's rows are then emitted in ascending order.  A symbolic pass counts
// rows per column first, so output offsets come from a prefix sum and the
// numeric pass writes C directly, already sorted.  This is Gustavson's
// column-by-column product; the reference does the same per column with a
// scatter + radix sort + duplicate fold.
//
// ESC engine (any shape): expand all P products (key, a*b) load-balanced by
// product index, radix-sort them by key, fold duplicates (no zero skipping).
//
// Tile engine (lnt_tile.cu): products whose output is dense or nearly so.
//
// Engine choice (lnt_lattice_mult_workspace and lnt_lattice_mult, from the
// shape and the product count P): SPA when h <= 1024; else the tile engine
// when its bitmaps fit and P >= 2^30 or P >= (nnz(A) + h*d) * ceil(wB/64)
// (the tile engine's work per 64-column tile is one pass over A's entries);
// else ESC.  LNT_SPGEMM_ENGINE=tile|esc in the environment forces an engine
// (tile only where its bitmaps fit).
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "lnt_scan.cuh"
#include "lnt_sort.cuh"

namespace lnt {

int run_collect(const u64* keys, const double* vals, size_t n, int skip_zero_heads, u64* out_k, double* out_v,
                u64* d_nout, void* ws, cudaStream_t s);
size_t collect_workspace_bytes(size_t n);
bool tile_shape_ok(u64 h, u64 w, u64 wB, u64 d, u64 na, u64 nb);
size_t tile_workspace_bytes(u64 h, u64 w, u64 wB, u64 d, u64 na, u64 nb);
int run_tile_mult(const u64* akeys, const double* avals, u64 na, const u64* bkeys, const double* bvals, u64 nb,
                  u64 h, u64 w, u64 wB, u64 d, void* ws, size_t ws_bytes, u64* ck, double* cv, u64* d_nc,
                  cudaStream_t s);

namespace {

constexpr u64 kMaxDenseAColumns = 1ull << 27;
constexpr u64 kMaxDenseBColumns = 1ull << 24;
constexpr int kSpaMaxRows = 1024;
constexpr int kSpaWarps = 4;  // 4 x (8 KB accumulator + 128 B bitmap) of static shared memory

struct Lat {
  const u64* keys;
  const double* vals;
  u64 nnz;
  u64 rows, cols, tabs;
};

// ptr[c] = first index whose column id (key / div) is >= c, for c in [0, ncol].
__global__ void colptr_kernel(const u64* __restrict__ keys, u64 n, Divider div, u64 ncol,
                              u64* __restrict__ ptr) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) {
    const long long prev = i == 0 ? -1ll : (long long)min(divide(keys[i - 1], div), ncol);
    const u64 cur = i == n ? ncol : min(divide(keys[i], div), ncol);
    for (long long c = prev + 1; c <= (long long)cur; ++c) ptr[c] = i;
  }
}

// [lo, hi) of A entries in A column `acol` (acol = col + w*tab).
struct AColumns {
  const u64* ptr;  // dense pointers, or null
  const u64* keys;
  u64 n, h;
  __device__ __forceinline__ void range(u64 acol, u64& lo, u64& hi) const {
    if (ptr) {
      lo = ptr[acol];
      hi = ptr[acol + 1];
      return;
    }
    const u64 k0 = acol * h, k1 = k0 + h;
    u64 a = 0, b = n;
    while (a < b) {
      const u64 m = (a + b) >> 1;
      if (keys[m] < k0) a = m + 1; else b = m;
    }
    lo = a;
    b = n;
    while (a < b) {
      const u64 m = (a + b) >> 1;
      if (keys[m] < k1) a = m + 1; else b = m;
    }
    hi = a;
  }
};

// Products contributed by B entry e: size of the A column its row selects.
struct ProductCount {
  AColumns ac;
  const u64* bkeys;
  Divider div_w, div_wB;
  u64 w;
  __device__ __forceinline__ u64 operator()(size_t e) const {
    const u64 k = bkeys[e];
    const u64 bcol = divide(k, div_w);  // col + wB*tab
    const u64 t = divide(bcol, div_wB);
    const u64 brow = k - bcol * w;
    u64 lo, hi;
    ac.range(brow + w * t, lo, hi);
    return hi - lo;
  }
};

struct Identity64 {
  const u64* v;
  __device__ __forceinline__ u64 operator()(size_t i) const { return v[i]; }
};

// ---- ESC engine ----------------------------------------------------------
__global__ void expand_kernel(Lat A, Lat B, AColumns ac, const u64* __restrict__ boff, u64 P, Divider div_w,
                              Divider div_wB, u64* __restrict__ pk, double* __restrict__ pv) {
  const u64 h = A.rows, w = A.cols;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 p = (u64)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += stride) {
    // B entry e with boff[e] <= p < boff[e+1]
    u64 a = 0, b = B.nnz;
    while (a < b) {
      const u64 m = (a + b + 1) >> 1;
      if (boff[m] <= p) a = m; else b = m - 1;
    }
    const u64 e = a;
    const u64 k = B.keys[e];
    const u64 bcol = divide(k, div_w);
    const u64 t = divide(bcol, div_wB);
    const u64 brow = k - bcol * w;
    const u64 acol = brow + w * t;
    u64 lo, hi;
    ac.range(acol, lo, hi);
    const u64 x = lo + (p - boff[e]);
    const u64 arow = A.keys[x] - acol * h;
    pk[p] = arow + h * bcol;  // row + h*(col + wB*tab): bcol already is col + wB*tab
    pv[p] = A.vals[x] * B.vals[e];
  }
}

// ---- SPA engine ----------------------------------------------------------
template <bool NUMERIC>
__global__ void __launch_bounds__(kSpaWarps * 32) spa_kernel(Lat A, Lat B, AColumns ac, const u64* __restrict__ bptr,
                                                              u64 units, u64* __restrict__ ucount,
                                                              const u64* __restrict__ uoff, u64* __restrict__ ck,
                                                              double* __restrict__ cv) {
  __shared__ u32 s_bits[kSpaWarps][kSpaMaxRows / 32];
  __shared__ double s_acc[NUMERIC ? kSpaWarps : 1][NUMERIC ? kSpaMaxRows : 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const u64 h = A.rows, w = A.cols, wB = B.cols;
  const int hw = (int)((h + 31) / 32);
  u32* bits = s_bits[warp];
  double* acc = s_acc[NUMERIC ? warp : 0];
  const u64 nwarps = (u64)gridDim.x * kSpaWarps;
  for (u64 u = (u64)blockIdx.x * kSpaWarps + warp; u < units; u += nwarps) {
    const u64 e0 = bptr[u], e1 = bptr[u + 1];
    if (e0 == e1) {  // empty B column: no output rows
      if (!NUMERIC && lane == 0) ucount[u] = 0;
      continue;
    }
    for (int i = lane; i < hw; i += 32) bits[i] = 0u;
    if (NUMERIC)
      for (int i = lane; i < (int)h; i += 32) acc[i] = 0.0;
    __syncwarp();
    const u64 t = u / wB;
    for (u64 e = e0 + lane; e < e1; e += 32) {
      const u64 brow = B.keys[e] - w * u;  // B col id of this unit is u
      const u64 acol = brow + w * t;
      u64 lo, hi;
      ac.range(acol, lo, hi);
      const double beta = NUMERIC ? B.vals[e] : 0.0;
      for (u64 x = lo; x < hi; ++x) {
        const u32 r = (u32)(A.keys[x] - acol * h);
        atomicOr(&bits[r >> 5], 1u << (r & 31));
        if (NUMERIC) atomicAdd(&acc[r], A.vals[x] * beta);
      }
    }
    __syncwarp();
    if (!NUMERIC) {
      u32 c = 0;
      for (int i = lane; i < hw; i += 32) c += __popc(bits[i]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == 0) ucount[u] = c;
    } else {
      u64 out = uoff[u];
      const u64 colkey = h * u;  // h*(col + wB*tab)
      for (int g = 0; g < hw; ++g) {
        const u32 word = bits[g];
        if (word & (1u << lane)) {
          const u32 r = (u32)g * 32 + lane;
          const u64 o = out + __popc(word & ((1u << lane) - 1u));
          ck[o] = colkey + r;
          cv[o] = acc[r];
        }
        out += __popc(word);
      }
    }
    __syncwarp();
  }
}

// ---- host side ------------------------------------------------------------
struct Shape {
  Lat A, B;
  u64 h, w, wB, d;
  bool dense_a, dense_b;
};

int check_shape(const lnt_lattice* a, const lnt_lattice* b, Shape* s) {
  if (!a || !b) return LNT_BAD_ARG;
  if (a->rows <= 0 || a->cols <= 0 || a->tabs <= 0 || b->rows <= 0 || b->cols <= 0 || b->tabs <= 0)
    return LNT_BAD_DIMS;
  if (a->cols != b->rows || a->tabs != b->tabs) return LNT_BAD_DIMS;  // check_mult_dims
  if ((a->nnz && (!a->keys || !a->vals)) || (b->nnz && (!b->keys || !b->vals))) return LNT_BAD_ARG;
  unsigned __int128 ka = (unsigned __int128)a->rows * a->cols * a->tabs;
  unsigned __int128 kb = (unsigned __int128)b->rows * b->cols * b->tabs;
  unsigned __int128 kc = (unsigned __int128)a->rows * b->cols * a->tabs;
  if ((ka >> 63) || (kb >> 63) || (kc >> 63)) return LNT_OVERFLOW_KEYBITS;
  s->A = {(const u64*)a->keys, a->vals, a->nnz, (u64)a->rows, (u64)a->cols, (u64)a->tabs};
  s->B = {(const u64*)b->keys, b->vals, b->nnz, (u64)b->rows, (u64)b->cols, (u64)b->tabs};
  s->h = (u64)a->rows;
  s->w = (u64)a->cols;
  s->wB = (u64)b->cols;
  s->d = (u64)a->tabs;
  s->dense_a = s->w * s->d <= kMaxDenseAColumns;
  s->dense_b = s->wB * s->d <= kMaxDenseBColumns;
  return LNT_OK;
}

// Plan workspace layout.
struct PlanLayout {
  size_t off_aptr, off_bptr, off_boff, off_ucount, off_uoff, off_scan, total;
  u64 units;
};

PlanLayout plan_layout(const Shape& s) {
  PlanLayout L;
  size_t off = 0;
  L.units = s.dense_b ? s.wB * s.d : 0;
  L.off_aptr = off;
  off += align_up(s.dense_a ? (s.w * s.d + 1) * 8 : 8, 256);
  L.off_bptr = off;
  off += align_up(s.dense_b ? (L.units + 1) * 8 : 8, 256);
  L.off_boff = off;
  off += align_up((s.B.nnz + 1) * 8, 256);
  L.off_ucount = off;
  off += align_up((L.units + 1) * 8, 256);
  L.off_uoff = off;
  off += align_up((L.units + 1) * 8, 256);
  L.off_scan = off;
  off += align_up(std::max(scan::workspace_bytes(s.B.nnz), scan::workspace_bytes(L.units)), 256);
  L.total = off;
  return L;
}

bool spa_eligible(const Shape& s) { return s.h <= (u64)kSpaMaxRows && s.dense_a && s.dense_b; }

enum class Engine { Spa, Esc, Tile };

Engine choose_engine(const Shape& s, u64 products) {
  const bool tile_ok = tile_shape_ok(s.h, s.w, s.wB, s.d, s.A.nnz, s.B.nnz);
  if (const char* e = std::getenv("LNT_SPGEMM_ENGINE")) {
    if (!std::strcmp(e, "tile") && tile_ok) return Engine::Tile;
    if (!std::strcmp(e, "esc")) return Engine::Esc;
  }
  if (spa_eligible(s)) return Engine::Spa;
  const u64 nt = (s.wB + 63) / 64;
  if (tile_ok && (products >= (1ull << 30) || products >= (s.A.nnz + s.h * s.d) * nt)) return Engine::Tile;
  return Engine::Esc;
}

// counts[1] = min(counts[0], dense): the output holds at most one entry per
// (row, col, tab) and at most one per product.
__global__ void capacity_kernel(u64* counts, u64 dense) { counts[1] = min(counts[0], dense); }

int grid_for(u64 work, int threads, int per_sm = 8) {
  const u64 want = (work + threads - 1) / threads;
  const u64 cap = (u64)sm_count() * per_sm;
  return (int)std::max<u64>(1, std::min(want, cap));
}

}  // namespace
}  // namespace lnt

using namespace lnt;

extern "C" {

int lnt_lattice_mult_plan_workspace(const lnt_lattice* a, const lnt_lattice* b, size_t* bytes) {
  Shape s;
  int st = check_shape(a, b, &s);
  if (st != LNT_OK) return st;
  if (!bytes) return LNT_BAD_ARG;
  *bytes = plan_layout(s).total;
  return LNT_OK;
}

int lnt_lattice_mult_plan(const lnt_lattice* a, const lnt_lattice* b, void* plan, size_t plan_bytes,
                          uint64_t* d_counts, void* stream) {
  Shape s;
  int st = check_shape(a, b, &s);
  if (st != LNT_OK) return st;
  if (!d_counts) return LNT_BAD_ARG;
  PlanLayout L = plan_layout(s);
  if (!plan || plan_bytes < L.total || (uintptr_t)plan % 256) return LNT_WORKSPACE;
  cudaStream_t cs = as_stream(stream);
  unsigned char* p = static_cast<unsigned char*>(plan);
  u64* aptr = reinterpret_cast<u64*>(p + L.off_aptr);
  u64* bptr = reinterpret_cast<u64*>(p + L.off_bptr);
  u64* boff = reinterpret_cast<u64*>(p + L.off_boff);
  u64* ucount = reinterpret_cast<u64*>(p + L.off_ucount);
  u64* uoff = reinterpret_cast<u64*>(p + L.off_uoff);
  if (s.dense_a) {
    ProfScope prof("spgemm_colptr", cs);
    colptr_kernel<<<grid_for(s.A.nnz + 1, 256), 256, 0, cs>>>(s.A.keys, s.A.nnz, make_divider(s.h), s.w * s.d, aptr);
    count_launch();
  }
  AColumns ac{s.dense_a ? aptr : nullptr, s.A.keys, s.A.nnz, s.h};
  ProductCount pc{ac, s.B.keys, make_divider(s.w), make_divider(s.wB), s.w};
  // products per B entry -> prefix -> total products into d_counts[0]
  st = scan::run(pc, s.B.nnz, (unsigned long long*)boff, (unsigned long long*)d_counts, p + L.off_scan, cs,
                 "spgemm_count");
  if (st != LNT_OK) return st;
  if (spa_eligible(s)) {
    {
      ProfScope prof("spgemm_colptr", cs);
      colptr_kernel<<<grid_for(s.B.nnz + 1, 256), 256, 0, cs>>>(s.B.keys, s.B.nnz, make_divider(s.w), L.units,
                                                                 bptr);
      count_launch();
    }
    {
      ProfScope prof("spgemm_spa_symbolic", cs);
      spa_kernel<false><<<grid_for(L.units * 32, kSpaWarps * 32), kSpaWarps * 32, 0, cs>>>(
          s.A, s.B, ac, bptr, L.units, ucount, nullptr, nullptr, nullptr);
      count_launch();
    }
    // output rows per column -> prefix -> exact output count into d_counts[1]
    st = scan::run(Identity64{ucount}, L.units, (unsigned long long*)uoff, (unsigned long long*)(d_counts + 1),
                   p + L.off_scan, cs, "spgemm_scan");
    if (st != LNT_OK) return st;
  } else {
    capacity_kernel<<<1, 1, 0, cs>>>((u64*)d_counts, s.h * s.wB * s.d);
    count_launch();
  }
  return launch_status();
}

int lnt_lattice_mult_workspace(const lnt_lattice* a, const lnt_lattice* b, uint64_t products, size_t* bytes) {
  Shape s;
  int st = check_shape(a, b, &s);
  if (st != LNT_OK) return st;
  if (!bytes) return LNT_BAD_ARG;
  const Engine eng = choose_engine(s, products);
  if (eng == Engine::Spa) {
    *bytes = 256;
    return LNT_OK;
  }
  if (eng == Engine::Tile) {
    *bytes = tile_workspace_bytes(s.h, s.w, s.wB, s.d, s.A.nnz, s.B.nnz);
    return LNT_OK;
  }
  if (products >= (1ull << 30)) return LNT_UNSUPPORTED;
  const u64 maxc = s.h * s.wB * s.d;
  SortPlan sp = make_sort_plan(products, maxc);
  size_t off = 0;
  off += align_up(sp.ctrl_bytes, 256);
  off += 4 * align_up(products * 8, 256);  // products (k, v) + sort ping-pong (k, v)
  off += align_up(collect_workspace_bytes(products), 256);
  *bytes = off;
  return LNT_OK;
}

int lnt_lattice_mult(const lnt_lattice* a, const lnt_lattice* b, const void* plan, uint64_t products,
                     void* workspace, size_t workspace_bytes, uint64_t* c_keys, double* c_vals, uint64_t* d_nc,
                     void* stream) {
  Shape s;
  int st = check_shape(a, b, &s);
  if (st != LNT_OK) return st;
  if (!plan || !d_nc) return LNT_BAD_ARG;
  PlanLayout L = plan_layout(s);
  cudaStream_t cs = as_stream(stream);
  const unsigned char* p = static_cast<const unsigned char*>(plan);
  const u64* aptr = reinterpret_cast<const u64*>(p + L.off_aptr);
  const u64* bptr = reinterpret_cast<const u64*>(p + L.off_bptr);
  const u64* boff = reinterpret_cast<const u64*>(p + L.off_boff);
  const u64* uoff = reinterpret_cast<const u64*>(p + L.off_uoff);
  AColumns ac{s.dense_a ? aptr : nullptr, s.A.keys, s.A.nnz, s.h};
  size_t need = 0;
  st = lnt_lattice_mult_workspace(a, b, products, &need);
  if (st != LNT_OK) return st;
  if (workspace_bytes < need || (need > 256 && !workspace)) return LNT_WORKSPACE;
  if (products && (!c_keys || !c_vals)) return LNT_BAD_ARG;
  const Engine eng = choose_engine(s, products);
  if (eng == Engine::Tile)
    return run_tile_mult(s.A.keys, s.A.vals, s.A.nnz, s.B.keys, s.B.vals, s.B.nnz, s.h, s.w, s.wB, s.d, workspace,
                         workspace_bytes, (u64*)c_keys, c_vals, (u64*)d_nc, cs);
  if (eng == Engine::Spa) {
    {
      ProfScope prof("spgemm_spa_numeric", cs);
      spa_kernel<true><<<grid_for(L.units * 32, kSpaWarps * 32), kSpaWarps * 32, 0, cs>>>(
          s.A, s.B, ac, bptr, L.units, nullptr, uoff, (u64*)c_keys, c_vals);
      count_launch();
    }
    if (cudaMemcpyAsync(d_nc, uoff + L.units, 8, cudaMemcpyDeviceToDevice, cs) != cudaSuccess)
      return LNT_DEVICE_ERROR;
    return launch_status();
  }
  // ESC
  if (products == 0) return cudaMemsetAsync(d_nc, 0, 8, cs) == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
  const u64 maxc = s.h * s.wB * s.d;
  SortPlan sp = make_sort_plan(products, maxc);
  unsigned char* w = static_cast<unsigned char*>(workspace);
  size_t off = 0;
  void* ctrl = w + off;
  off += align_up(sp.ctrl_bytes, 256);
  u64* pk = reinterpret_cast<u64*>(w + off);
  off += align_up(products * 8, 256);
  double* pv = reinterpret_cast<double*>(w + off);
  off += align_up(products * 8, 256);
  u64* k0 = reinterpret_cast<u64*>(w + off);
  off += align_up(products * 8, 256);
  double* v0 = reinterpret_cast<double*>(w + off);
  off += align_up(products * 8, 256);
  void* coll = w + off;
  // Pass p of the sort writes buffer (passes-1-p)&1 (0 = (k0,v0), the final one);
  // expand into the buffer pass 0 does not write.
  const bool even = sp.passes % 2 == 0;
  u64* ek = even ? k0 : pk;
  double* ev = even ? v0 : pv;
  {
    ProfScope prof("spgemm_expand", cs);
    expand_kernel<<<grid_for(products, 256), 256, 0, cs>>>(s.A, s.B, ac, boff, products, make_divider(s.w),
                                                          make_divider(s.wB), ek, ev);
    count_launch();
  }
  // sort products by output key: the sorted run lands in (k0, v0)
  st = run_sort(sp, plain_source(ek, ev, products), k0, v0, pk, pv, ctrl, cs);
  if (st != LNT_OK) return st;
  return run_collect(k0, v0, products, 0, (u64*)c_keys, c_vals, (u64*)d_nc, coll, cs);
}

}  // extern "C"

// ---- noLatticeMult ----------------------------------------------------------
// Products with no contracted index (SparseMIABase::perform_noLatticeMult,
// SparseMIABase.h:1716-1826): A as a lattice (h = its outer size) x 1 x d and B
// as 1 x wB x d (d = the inter size), both key-sorted.  Expanding every B
// entry's products against the A entries of its tab (a warp per B entry, at
// the entry's prefix-summed offset) yields them in the reference's emission
// order - B entries major, A entries minor, tab by tab - which is ascending
// key order, so C needs neither a sort nor a fold (equal keys from operands
// with duplicate keys stay separate, as in the reference).
namespace lnt {
namespace {
// One warp per B entry e (grid-stride): its products are the A entries of its
// tab, written contiguously at boff[e] with coalesced reads of A and writes.
__global__ void nolattice_expand_kernel(Lat A, Lat B, AColumns ac, const u64* __restrict__ boff, Divider div_wB,
                                        u64* __restrict__ ck, double* __restrict__ cv) {
  const int lane = threadIdx.x & 31;
  const u64 nw = ((u64)gridDim.x * blockDim.x) >> 5;
  const u64 h = A.rows;
  for (u64 e = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < B.nnz; e += nw) {
    const u64 bk = B.keys[e];          // col + wB * tab (B has one row)
    const u64 t = divide(bk, div_wB);
    u64 lo, hi;
    ac.range(t, lo, hi);
    const double bv = B.vals[e];
    const u64 o = boff[e];
    const u64 shift = h * bk - t * h;  // output key = A key - t*h + h*bk
    for (u64 x0 = lo + lane; x0 < hi; x0 += 128) {  // four products per lane: loads first, then stores
      u64 k[4];
      double v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const u64 x = x0 + 32 * q;
        k[q] = x < hi ? A.keys[x] : 0;
        v[q] = x < hi ? A.vals[x] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const u64 x = x0 + 32 * q;
        if (x < hi) {
          ck[o + (x - lo)] = k[q] + shift;
          cv[o + (x - lo)] = v[q] * bv;
        }
      }
    }
  }
}

struct NoLatLayout {
  size_t off_aptr, off_boff, off_scan, total;
};
NoLatLayout nolat_layout(const Shape& s) {
  NoLatLayout L;
  size_t off = 0;
  L.off_aptr = off;
  off += align_up(s.dense_a ? (s.w * s.d + 1) * 8 : 8, 256);
  L.off_boff = off;
  off += align_up((s.B.nnz + 1) * 8, 256);
  L.off_scan = off;
  off += align_up(scan::workspace_bytes(s.B.nnz), 256);
  L.total = off;
  return L;
}
int nolat_shape(const lnt_lattice* a, const lnt_lattice* b, Shape* s) {
  int st = check_shape(a, b, s);
  if (st != LNT_OK) return st;
  if (s->w != 1) return LNT_BAD_DIMS;  // A: h x 1 x d, B: 1 x wB x d
  return LNT_OK;
}
}  // namespace
}  // namespace lnt

extern "C" {

int lnt_nolattice_mult_workspace(const lnt_lattice* a, const lnt_lattice* b, size_t* bytes) {
  Shape s;
  int st = nolat_shape(a, b, &s);
  if (st != LNT_OK) return st;
  if (!bytes) return LNT_BAD_ARG;
  *bytes = nolat_layout(s).total;
  return LNT_OK;
}

int lnt_nolattice_mult_count(const lnt_lattice* a, const lnt_lattice* b, void* workspace, size_t workspace_bytes,
                             uint64_t* d_products, void* stream) {
  Shape s;
  int st = nolat_shape(a, b, &s);
  if (st != LNT_OK) return st;
  if (!d_products) return LNT_BAD_ARG;
  const NoLatLayout L = nolat_layout(s);
  if (!workspace || workspace_bytes < L.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  cudaStream_t cs = as_stream(stream);
  unsigned char* p = static_cast<unsigned char*>(workspace);
  u64* aptr = reinterpret_cast<u64*>(p + L.off_aptr);
  if (s.dense_a) {
    ProfScope prof("spgemm_colptr", cs);
    colptr_kernel<<<grid_for(s.A.nnz + 1, 256), 256, 0, cs>>>(s.A.keys, s.A.nnz, make_divider(s.h), s.w * s.d, aptr);
    count_launch();
  }
  AColumns ac{s.dense_a ? aptr : nullptr, s.A.keys, s.A.nnz, s.h};
  ProductCount pc{ac, s.B.keys, make_divider(s.w), make_divider(s.wB), s.w};
  st = scan::run(pc, s.B.nnz, (unsigned long long*)(p + L.off_boff), (unsigned long long*)d_products,
                 p + L.off_scan, cs, "spgemm_count");
  if (st != LNT_OK) return st;
  return launch_status();
}

int lnt_nolattice_mult(const lnt_lattice* a, const lnt_lattice* b, uint64_t products, void* workspace,
                       size_t workspace_bytes, uint64_t* c_keys, double* c_vals, void* stream) {
  Shape s;
  int st = nolat_shape(a, b, &s);
  if (st != LNT_OK) return st;
  const NoLatLayout L = nolat_layout(s);
  if (!workspace || workspace_bytes < L.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  if (products == 0) return LNT_OK;
  if (!c_keys || !c_vals) return LNT_BAD_ARG;
  cudaStream_t cs = as_stream(stream);
  unsigned char* p = static_cast<unsigned char*>(workspace);
  AColumns ac{s.dense_a ? reinterpret_cast<const u64*>(p + L.off_aptr) : nullptr, s.A.keys, s.A.nnz, s.h};
  {
    ProfScope prof("nolattice_expand", cs);
    nolattice_expand_kernel<<<grid_for(s.B.nnz * 32, 256), 256, 0, cs>>>(
        s.A, s.B, ac, reinterpret_cast<const u64*>(p + L.off_boff), make_divider(s.wB), (u64*)c_keys, c_vals);
    count_launch();
  }
  return launch_status();
}

}  // extern "C"
