// Tile engine of the sparse lattice product, for products whose output is
// dense or nearly so (the skewed contraction c(i,j,m) = a(i,j,k,l) * b(k,l,m)
// with Zipf-distributed contracted modes: 2^20 x 4096 output, about 9e10
// products).  Same result as csc_no_accum<true> (SparseLatticeBase.h:
// 1854-1990): C keys = row + h*(col + wB*tab) ascending, products of equal
// keys summed, exact zeros kept.
//
// Layout built in the workspace:
//   A row-major: A re-keyed to c + w*(r + h*t) and radix-sorted, with row
//     pointers (h*d + 1);
//   B row-major: B re-keyed to j + wB*(c + w*t), sorted, duplicate keys
//     summed, with row pointers (w*d + 1); a row holding at least an eighth of
//     its columns is also expanded into a dense row of Bd (one slot per such
//     row, zero-filled, padded to whole 256-column tiles); for every row
//     tp[row][q] = position in B of the row's first entry at or right of
//     column 256q (q = 0..nt);
//   A records: per A entry its B row (c + w*t), that row's dense slot and the
//     value, 16 bytes, so one load per entry serves every tile;
//   bitmaps, one bit per (row, column), 64-column words: Bbits (B rows) and
//     Cbits (C rows, = OR of the Bbits rows that A row selects) — the output
//     pattern, computed before any arithmetic.
// Output positions: per (tab, column, panel of 32 rows) the number of
// pattern bits, exclusive-scanned in (tab, column, panel) order, so each
// panel's rows of one column land at a known contiguous offset.
// Numeric pass: one CTA per (panel, 256-column tile) unit; warps take rows
// from a shared counter, eight columns per lane in registers.  Each 32-entry
// chunk of the row's A records is split by ballot into per-warp shared lists
// of dense-row items (Bd position, value) and sparse-row items (segment,
// value), so the inner loops read one broadcast shared-memory item per entry:
// a dense item adds four coalesced 512-byte loads and eight FMAs, a sparse
// item's segment is scattered by the lanes into the row's staging row in
// shared memory (distinct columns within a segment).  The 32 x 256 tile is
// staged in shared memory and written column by column (contiguous runs),
// at offsets fetched before the unit's arithmetic.
#include <algorithm>
#include <cstdlib>

#include "lnt_scan.cuh"
#include "lnt_sort.cuh"
#include "lnt_tuned.h"

namespace lnt {

int run_collect(const u64* keys, const double* vals, size_t n, int skip_zero_heads, u64* out_k, double* out_v,
                u64* d_nout, void* ws, cudaStream_t s);
size_t collect_workspace_bytes(size_t n);

namespace {

constexpr u32 FULL = 0xffffffffu;
constexpr int kWordCols = 64;      // columns per bitmap word
constexpr int kTileCols = 256;     // output columns per numeric tile (eight per lane)
constexpr int kPanelRows = 32;     // output rows per unit
constexpr int kTileThreads = 512;  // 16 warps
constexpr int kTileWarps = kTileThreads / 32;
constexpr int kTileGroup = 4;      // tiles of one panel processed by consecutive units
constexpr int kStageStride = 257;  // doubles per staged row
constexpr int kSparseBatch = 4;    // sparse segments whose first 32 entries are loaded together

struct ARec {
  u32 br;    // B row c + w*t
  int slot;  // its dense slot, or -1
  double v;
};
struct DenseItem {
  u64 pos;   // double2 index of the item's tile in Bd
  double v;
};
struct SparseItem {
  u64 s0;    // first entry of the segment in row-major B
  double v;
  u64 kb;    // key of the tile's column 0 in that B row
  u32 len;
  u32 pad;
};
constexpr size_t kStageBytes = (size_t)kPanelRows * kStageStride * 8;
constexpr size_t kNumericSmem = kStageBytes + (size_t)kTileWarps * 32 * (sizeof(DenseItem) + sizeof(SparseItem));
constexpr size_t kMaxBitmapBytes = 16ull << 30;

// A B row is expanded into a dense row when div * len >= max(wB, kTileCols):
// div = LNT_TILE_DENSE_DIV from the environment (1..64), else the tuned value
// (on the full skewed contraction: 4 -> 70.0 ms, 8 -> 67.7 ms, 16 -> 68.8 ms).
int dense_div() {
  const char* e = std::getenv("LNT_TILE_DENSE_DIV");
  const int v = e ? std::atoi(e) : kTunedTileDenseDiv;
  return v >= 1 && v <= 64 ? v : kTunedTileDenseDiv;
}

struct TileDims {
  u64 h, w, wB, d;
  u64 div;     // dense-row threshold divisor
  u32 nt, nw, np;  // 256-column tiles per row, 64-column bitmap words per row, 32-row panels per tab
  u64 smax;    // dense-row slots
};

TileDims tile_dims(u64 h, u64 w, u64 wB, u64 d, u64 nb) {
  TileDims t;
  t.h = h;
  t.w = w;
  t.wB = wB;
  t.d = d;
  t.nt = (u32)((wB + kTileCols - 1) / kTileCols);
  t.nw = (u32)((wB + kWordCols - 1) / kWordCols);
  t.np = (u32)((h + kPanelRows - 1) / kPanelRows);
  t.div = (u64)dense_div();
  const u64 thr = std::max<u64>(wB, kTileCols);  // dense: div * len >= thr
  t.smax = std::min<u64>(w * d, t.div * nb / thr);
  return t;
}

struct TileLayout {
  size_t ctrl, ak, av, tk, tv, bk, bv, arow, brow, dslot, tp, bbits, bd, cbits, cnt, base, scan, coll, arec, misc,
      total;
  SortPlan pa, pb;
};

TileLayout tile_layout(const TileDims& t, u64 na, u64 nb) {
  TileLayout L;
  L.pa = make_sort_plan(na, t.h * t.w * t.d);
  L.pb = make_sort_plan(nb, t.w * t.wB * t.d);
  const u64 ncnt = t.d * t.wB * t.np;
  const u64 nmax = std::max(na, nb);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align_up(std::max<size_t>(bytes, 8), 256);
    return o;
  };
  L.ctrl = take(std::max(L.pa.ctrl_bytes, L.pb.ctrl_bytes));
  L.ak = take(na * 8);
  L.av = take(na * 8);
  L.tk = take(nmax * 8);
  L.tv = take(nmax * 8);
  L.bk = take(nb * 8);
  L.bv = take(nb * 8);
  L.arow = take((t.h * t.d + 1) * 8);
  L.brow = take((t.w * t.d + 1) * 8);
  L.dslot = take(t.w * t.d * 4);
  L.tp = take(t.w * t.d * (u64)(t.nt + 1) * 8);
  L.bbits = take(t.w * t.d * (u64)t.nw * 8);
  L.bd = take(t.smax * (u64)t.nt * kTileCols * 8);
  L.cbits = take(t.h * t.d * (u64)t.nw * 8);
  L.cnt = take(ncnt * 4);
  L.base = take((ncnt + 1) * 8);
  L.scan = take(scan::workspace_bytes(ncnt));
  L.coll = take(collect_workspace_bytes(nb));
  L.arec = take(na * sizeof(ARec));
  L.misc = take(256);  // [0] unique B count, [1] slot counter
  L.total = off;
  return L;
}

// ptr[r] = first index whose row id (key / div) is >= r, r in [0, nrows];
// the entry count is *d_n when d_n is given, else n.
__global__ void tile_rowptr_kernel(const u64* __restrict__ keys, u64 n, const u64* __restrict__ d_n, Divider div,
                                   u64 nrows, u64* __restrict__ ptr) {
  if (d_n) n = *d_n;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) {
    const long long prev = i == 0 ? -1ll : (long long)min(divide(keys[i - 1], div), nrows);
    const u64 cur = i == n ? nrows : min(divide(keys[i], div), nrows);
    for (long long r = prev + 1; r <= (long long)cur; ++r) ptr[r] = i;
  }
}

// dslot[row] = dense slot of B row `row`, or -1.
__global__ void tile_slot_kernel(const u64* __restrict__ brow, u64 nrows, u64 thr, u64 div, u64 smax, int* __restrict__ dslot,
                                 u32* __restrict__ counter) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += stride) {
    const u64 len = brow[r + 1] - brow[r];
    int slot = -1;
    if (len * div >= thr) {
      const u32 s = atomicAdd(counter, 1u);
      if (s < smax) slot = (int)s;
    }
    dslot[r] = slot;
  }
}

// tp[row][*] = brow[row] for rows without entries (their segments are empty).
__global__ void tile_tp_empty_kernel(const u64* __restrict__ brow, u64 nrows, u32 nt, u64* __restrict__ tp) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += stride) {
    const u64 rs = brow[r];
    if (brow[r + 1] != rs) continue;
    for (u32 q = 0; q <= nt; ++q) tp[r * (u64)(nt + 1) + q] = rs;
  }
}

// A record per A entry (row-major order).
__global__ void tile_arec_kernel(const u64* __restrict__ ak, const double* __restrict__ av, u64 na, u64 w,
                                 Divider div_w, Divider div_h, const int* __restrict__ dslot, ARec* __restrict__ rec) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < na; e += stride) {
    const u64 k = ak[e];
    const u64 row = divide(k, div_w);  // r + h*t
    const u64 br = k - row * w + w * divide(row, div_h);
    ARec r;
    r.br = (u32)br;
    r.slot = dslot[br];
    r.v = av[e];
    rec[e] = r;
  }
}

// Per unique B entry: its bit in Bbits, its value in Bd (dense rows), and the
// tile pointers of its row.
__global__ void tile_bentry_kernel(const u64* __restrict__ bk, const double* __restrict__ bv,
                                   const u64* __restrict__ d_n, const u64* __restrict__ brow, Divider div_wB, u64 wB,
                                   u32 nt, u32 nw, const int* __restrict__ dslot, u64* __restrict__ bbits,
                                   u64* __restrict__ tp, double* __restrict__ bd) {
  const u64 n = *d_n;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const u64 k = bk[e];
    const u64 row = divide(k, div_wB);
    const u64 j = k - row * wB;
    const u32 q = (u32)(j / kTileCols);
    atomicOr(reinterpret_cast<unsigned long long*>(bbits + row * nw + j / kWordCols), 1ull << (j % kWordCols));
    const int slot = dslot[row];
    if (slot >= 0) bd[(u64)slot * nt * kTileCols + j] = bv[e];
    const u64 rs = brow[row], re = brow[row + 1];
    u64* t = tp + row * (u64)(nt + 1);
    long long qprev = -1;
    if (e > rs) qprev = (long long)((bk[e - 1] - row * wB) / kTileCols);
    for (long long qq = qprev + 1; qq <= (long long)q; ++qq) t[qq] = e;
    if (e + 1 == re)
      for (u32 qq = q + 1; qq <= nt; ++qq) t[qq] = e + 1;
  }
}

// Cbits[row] = OR of Bbits[c + w*t] over the A entries (row, c); warp per row.
// A warp stops reading B rows once every lane's word is full (all wB columns
// of its 64 set): further rows cannot change it, and rows of the hottest B
// entries are full under skewed inputs.
__global__ void tile_cbits_kernel(const u64* __restrict__ ak, const u64* __restrict__ arow,
                                  const u64* __restrict__ bbits, u64 h, u64 w, u64 d, u32 nw, u64 wB, Divider div_h,
                                  u64* __restrict__ cbits) {
  const int lane = threadIdx.x & 31;
  const u64 nrows = h * d;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 row = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrows; row += nwarps) {
    const u64 t = divide(row, div_h);
    const u64 e0 = arow[row], e1 = arow[row + 1];
    const u64 cbase = w * t - w * row;  // B row = A key + cbase
    for (u32 w0 = 0; w0 < nw; w0 += 32) {
      const u32 word = w0 + lane;
      const u64 rest = wB - (u64)word * kWordCols;  // columns of this word
      const u64 full = word >= nw ? 0ull : rest >= 64 ? ~0ull : (1ull << rest) - 1ull;
      u64 acc = 0;
      bool done = word >= nw;
      for (u64 eb = e0; eb < e1 && !__all_sync(FULL, done); eb += 32) {
        const u64 e = eb + lane;
        const u64 br = e < e1 ? ak[e] + cbase : 0;
        const int n = (int)(e1 - eb < 32 ? e1 - eb : 32);
        for (int k = 0; k < n; ++k) {
          const u64 b = __shfl_sync(FULL, br, k);
          if (!done) {
            acc |= bbits[b * nw + word];
            done = acc == full;
          }
          if (__all_sync(FULL, done)) break;
        }
      }
      if (word < nw) cbits[row * nw + word] = acc;
    }
  }
}

__device__ __forceinline__ u64 shfl_xor64(u64 v, int o) {
  const u32 lo = __shfl_xor_sync(FULL, (u32)v, o), hi = __shfl_xor_sync(FULL, (u32)(v >> 32), o);
  return ((u64)hi << 32) | lo;
}

// The warp's 32 x 64 bit matrix (one 64-bit word per lane) as six bit
// slices of its 64 column counts (each <= 32), held by every lane.  Bit-sliced
// butterfly: s[i] holds bit i of the counts; the step with offset o adds the
// partner lane's counts with a ripple carry over the slices, so after five
// steps every lane holds the counts of all 32 lanes (30 shuffles and about 75
// logic operations instead of 128 ballots and population counts).
__device__ __forceinline__ void column_count_slices(u64 word, u64 (&s)[6]) {
  s[0] = word;
#pragma unroll
  for (int step = 0; step < 5; ++step) {
    const int o = 1 << step;
    u64 c = 0;
#pragma unroll
    for (int i = 0; i <= step; ++i) {  // step + 1 slices before this step
      const u64 a = s[i], b = shfl_xor64(a, o);
      s[i] = a ^ b ^ c;
      c = (a & b) | (c & (a ^ b));
    }
    s[step + 1] = c;
  }
}

// cnt[(t*wB + col)*np + p] = pattern bits of column col among panel p's rows.
// Warp per (t, group of 32 panels, bitmap word q): for each panel of the
// group the lanes (one row each) form the column counts of its 64 columns,
// and lane i keeps panel i's slices (12 registers); then, column by column,
// the 32 lanes write the group's 32 consecutive counts as one 128-byte store.
// (One warp per panel wrote 64 counts 4 bytes at a time, np words apart.)
static_assert(kPanelRows == 32, "tile_count_kernel takes a panel as one row per lane");
__global__ void tile_count_kernel(const u64* __restrict__ cbits, u64 h, u64 wB, u64 d, u32 nt, u32 np,
                                  u32* __restrict__ cnt) {
  // here nt counts bitmap words per row
  const int lane = threadIdx.x & 31;
  const u32 ng = (np + 31) / 32;
  const u64 units = d * (u64)ng * nt;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 u = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < units; u += nwarps) {
    const u64 t = u / ((u64)ng * nt);
    const u64 rem = u - t * ng * nt;
    const u32 g = (u32)(rem / nt);
    const u32 q = (u32)(rem - (u64)g * nt);
    u64 keep[6] = {0, 0, 0, 0, 0, 0};
    for (int pp = 0; pp < 32; ++pp) {
      const u32 p = g * 32 + pp;
      if (p >= np) break;  // uniform across the warp
      const u64 r = (u64)p * kPanelRows + lane;  // a panel is one row per lane
      const u64 word = r < h ? cbits[(r + h * t) * nt + q] : 0ull;
      u64 sl[6];
      column_count_slices(word, sl);
      if (lane == pp) {
#pragma unroll
        for (int i = 0; i < 6; ++i) keep[i] = sl[i];
      }
    }
    const u32 p = g * 32 + lane;
    for (int c = 0; c < kWordCols; ++c) {
      const u64 col = (u64)q * kWordCols + c;
      if (col >= wB) break;
      u32 v = 0;
#pragma unroll
      for (int i = 0; i < 6; ++i) v |= (u32)((keep[i] >> c) & 1ull) << i;
      if (p < np) cnt[(t * wB + col) * np + p] = v;
    }
  }
}

struct CountGet {
  const u32* c;
  __device__ __forceinline__ u64 operator()(size_t i) const { return c[i]; }
};

struct NumArgs {
  const ARec* rec;
  const u64* arow;
  const u64* bk;
  const double* bv;
  const u64* tp;
  const double* bd;
  const u64* cbits;
  const unsigned long long* base;
  u64 h, w, wB, d;
  u32 nt, nw, np;
  u64 units;
  u64* ck;
  double* cv;
};

__global__ void __launch_bounds__(kTileThreads, 2) tile_numeric_kernel(NumArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* stage = reinterpret_cast<double*>(smem);  // [kPanelRows][kStageStride]
  DenseItem* dlist = reinterpret_cast<DenseItem*>(smem + kStageBytes);
  SparseItem* slist = reinterpret_cast<SparseItem*>(dlist + kTileWarps * 32);
  constexpr int kWords = kTileCols / kWordCols;
  __shared__ u64 s_bits[kPanelRows][kWords];
  __shared__ unsigned long long s_base[kTileCols];
  __shared__ u32 s_next;
  __shared__ u64 s_unit[4];  // first C row (row0 + h*t), first column + wB*t, tile q, row0
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  DenseItem* dl = dlist + warp * 32;
  SparseItem* sl = slist + warp * 32;
  const u32 lt = (1u << lane) - 1u;
  const double2* bd2 = reinterpret_cast<const double2*>(a.bd);
  const u64 per_tab = (u64)a.np * a.nt;
  for (u64 u = blockIdx.x; u < a.units; u += gridDim.x) {
    const u64 t = u / per_tab;
    const u64 idx = u - t * per_tab;
    const u64 qg = idx / ((u64)a.np * kTileGroup);
    const u64 within = idx - qg * a.np * kTileGroup;
    const u32 gs = min((u32)kTileGroup, a.nt - (u32)qg * kTileGroup);
    const u32 p = (u32)(within / gs);
    const u32 q = (u32)(qg * kTileGroup + (within - (u64)p * gs));
    const u64 row0 = (u64)p * kPanelRows;
    if (threadIdx.x < kPanelRows * kWords) {
      const int i = threadIdx.x / kWords, wd = threadIdx.x % kWords;
      const u64 r = row0 + i;
      const u32 word = kWords * q + wd;
      s_bits[i][wd] = r < a.h && word < a.nw ? a.cbits[(r + a.h * t) * a.nw + word] : 0ull;
    }
    if (threadIdx.x < kTileCols) {
      const u64 col = (u64)q * kTileCols + threadIdx.x;
      s_base[threadIdx.x] = col < a.wB ? a.base[(t * a.wB + col) * a.np + p] : 0ull;
    }
    if (threadIdx.x == 0) {
      s_next = 0;
      s_unit[0] = row0 + a.h * t;
      s_unit[1] = (u64)q * kTileCols + a.wB * t;
      s_unit[2] = q;
      s_unit[3] = row0;
    }
    __syncthreads();
    for (;;) {
      u32 i = 0;
      if (lane == 0) i = atomicAdd(&s_next, 1u);
      i = __shfl_sync(FULL, i, 0);
      if (i >= (u32)kPanelRows) break;
      u64 any = 0;
#pragma unroll
      for (int wd = 0; wd < kWords; ++wd) any |= s_bits[i][wd];
      if (any == 0ull) continue;
      const u64 row = s_unit[0] + i;
      const u32 q = (u32)s_unit[2];
      const u64 e0 = a.arow[row], e1 = a.arow[row + 1];
      double* st = stage + i * kStageStride;
      double acc[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[c] = 0.0;
      bool had_sparse = false;
      for (u64 eb = e0; eb < e1; eb += 32) {
        const u64 e = eb + lane;
        ARec rc;
        rc.br = 0;
        rc.slot = -1;
        rc.v = 0.0;
        if (e < e1) rc = a.rec[e];
        u64 s0 = 0;
        u32 len = 0;
        if (e < e1 && rc.slot < 0) {
          const u64* tpr = a.tp + (u64)rc.br * (a.nt + 1) + q;
          s0 = tpr[0];
          len = (u32)(tpr[1] - s0);
        }
        const bool dense = e < e1 && rc.slot >= 0;
        const u32 dm = __ballot_sync(FULL, dense);
        const u32 sm = __ballot_sync(FULL, len != 0);
        if (dense) {
          DenseItem it;
          it.pos = ((u64)rc.slot * a.nt + q) * (kTileCols / 2);
          it.v = rc.v;
          dl[__popc(dm & lt)] = it;
        }
        if (len != 0) {
          SparseItem it;
          it.s0 = s0;
          it.v = rc.v;
          it.kb = a.wB * rc.br + (u64)q * kTileCols;
          it.len = len;
          it.pad = 0;
          sl[__popc(sm & lt)] = it;
        }
        if (sm != 0u && !had_sparse) {  // the staging row accumulates the sparse products
          for (int c = lane; c < kTileCols; c += 32) st[c] = 0.0;
          had_sparse = true;
        }
        __syncwarp();
        const int nd = __popc(dm), ns = __popc(sm);
        for (int k = 0; k < nd; ++k) {
          const DenseItem it = dl[k];
          double2 b[4];
#pragma unroll
          for (int x = 0; x < 4; ++x) b[x] = bd2[it.pos + 32 * x + lane];
#pragma unroll
          for (int x = 0; x < 4; ++x) {
            acc[2 * x] = fma(it.v, b[x].x, acc[2 * x]);
            acc[2 * x + 1] = fma(it.v, b[x].y, acc[2 * x + 1]);
          }
        }
        for (int k = 0; k < ns; k += kSparseBatch) {
          // first 32 entries of kSparseBatch segments loaded together, then scattered one segment at a time
          u32 jj[kSparseBatch];
          double ww[kSparseBatch];
#pragma unroll
          for (int x = 0; x < kSparseBatch; ++x) {
            jj[x] = kTileCols;
            ww[x] = 0.0;
            if (k + x < ns) {
              const SparseItem it = sl[k + x];
              if ((u32)lane < it.len) {
                jj[x] = (u32)(a.bk[it.s0 + lane] - it.kb);
                ww[x] = a.bv[it.s0 + lane];
              }
            }
          }
#pragma unroll
          for (int x = 0; x < kSparseBatch; ++x) {
            if (k + x < ns) {
              const SparseItem it = sl[k + x];
              if (jj[x] < (u32)kTileCols) st[jj[x]] = fma(it.v, ww[x], st[jj[x]]);
              for (u32 y = lane + 32; y < it.len; y += 32) {
                const u32 j = (u32)(a.bk[it.s0 + y] - it.kb);
                st[j] = fma(it.v, a.bv[it.s0 + y], st[j]);
              }
              __syncwarp();
            }
          }
        }
        __syncwarp();
      }
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const int c = 64 * x + 2 * lane;
        if (had_sparse) {
          st[c] += acc[2 * x];
          st[c + 1] += acc[2 * x + 1];
        } else {
          st[c] = acc[2 * x];
          st[c + 1] = acc[2 * x + 1];
        }
      }
    }
    __syncthreads();
    for (int jj = warp; jj < kTileCols; jj += kTileWarps) {
      if ((u64)s_unit[2] * kTileCols + jj >= a.wB) continue;
      const bool bit = (s_bits[lane][jj >> 6] >> (jj & 63)) & 1ull;
      const u32 m = __ballot_sync(FULL, bit);
      if (bit) {
        const u64 o = s_base[jj] + __popc(m & lt);
        a.ck[o] = a.h * (s_unit[1] + jj) + s_unit[3] + lane;
        a.cv[o] = stage[lane * kStageStride + jj];
      }
    }
    __syncthreads();
  }
}

int grid_cap(u64 work, int threads, int per_sm = 8) {
  const u64 want = (work + threads - 1) / threads;
  const u64 cap = (u64)sm_count() * per_sm;
  return (int)std::max<u64>(1, std::min(want, cap));
}

}  // namespace

bool tile_shape_ok(u64 h, u64 w, u64 wB, u64 d, u64 na, u64 nb) {
  if (na >= (1ull << 32) || nb >= (1ull << 32) || w * d >= (1ull << 31)) return false;
  const TileDims t = tile_dims(h, w, wB, d, nb);
  const unsigned __int128 cb = (unsigned __int128)h * d * t.nw * 8;
  const unsigned __int128 bb = (unsigned __int128)w * d * (t.nt + 1 + t.nw) * 8;
  const unsigned __int128 cn = (unsigned __int128)d * wB * t.np * 12;
  return cb <= kMaxBitmapBytes && bb <= kMaxBitmapBytes && cn <= kMaxBitmapBytes;
}

size_t tile_workspace_bytes(u64 h, u64 w, u64 wB, u64 d, u64 na, u64 nb) {
  return tile_layout(tile_dims(h, w, wB, d, nb), na, nb).total;
}

int run_tile_mult(const u64* akeys, const double* avals, u64 na, const u64* bkeys, const double* bvals, u64 nb,
                  u64 h, u64 w, u64 wB, u64 d, void* ws, size_t ws_bytes, u64* ck, double* cv, u64* d_nc,
                  cudaStream_t s) {
  const TileDims t = tile_dims(h, w, wB, d, nb);
  const TileLayout L = tile_layout(t, na, nb);
  if (!ws || ws_bytes < L.total || (uintptr_t)ws % 256) return LNT_WORKSPACE;
  unsigned char* W = static_cast<unsigned char*>(ws);
  auto at = [&](size_t off) { return static_cast<void*>(W + off); };
  u64* ak = (u64*)at(L.ak);
  double* av = (double*)at(L.av);
  u64* tk = (u64*)at(L.tk);
  double* tv = (double*)at(L.tv);
  u64* bk = (u64*)at(L.bk);
  double* bv = (double*)at(L.bv);
  u64* arow = (u64*)at(L.arow);
  u64* brow = (u64*)at(L.brow);
  int* dslot = (int*)at(L.dslot);
  u64* tp = (u64*)at(L.tp);
  ARec* rec = (ARec*)at(L.arec);
  u64* bbits = (u64*)at(L.bbits);
  double* bd = (double*)at(L.bd);
  u64* cbits = (u64*)at(L.cbits);
  u32* cnt = (u32*)at(L.cnt);
  unsigned long long* base = (unsigned long long*)at(L.base);
  u64* misc = (u64*)at(L.misc);
  u64* d_nb = misc;
  u32* slot_counter = reinterpret_cast<u32*>(misc + 1);
  const u64 ncnt = d * wB * t.np;
  const u64 brows = w * d, crows = h * d;
  int st;

  if (cudaMemsetAsync(misc, 0, 256, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  // B row-major: (c, j, t) with dims (w, wB, d), sequence {0,1,2} -> {1,0,2}; sort; sum duplicate keys.
  {
    const int64_t dims[3] = {(int64_t)w, (int64_t)wB, (int64_t)d};
    const int32_t cur[3] = {0, 1, 2}, nxt[3] = {1, 0, 2};
    PairSource src = plain_source(bkeys, bvals, nb);
    if ((st = make_rekey_params(3, dims, cur, nxt, &src.ra)) != LNT_OK) return st;
    if (nb) {
      if ((st = run_sort(L.pb, src, tk, tv, bk, bv, at(L.ctrl), s)) != LNT_OK) return st;
      if ((st = run_collect(tk, tv, nb, 0, bk, bv, d_nb, at(L.coll), s)) != LNT_OK) return st;
    }
  }
  // A row-major: (r, c, t) with dims (h, w, d), sequence {0,1,2} -> {1,0,2}; sort.
  {
    const int64_t dims[3] = {(int64_t)h, (int64_t)w, (int64_t)d};
    const int32_t cur[3] = {0, 1, 2}, nxt[3] = {1, 0, 2};
    PairSource src = plain_source(akeys, avals, na);
    if ((st = make_rekey_params(3, dims, cur, nxt, &src.ra)) != LNT_OK) return st;
    if (na && (st = run_sort(L.pa, src, ak, av, tk, tv, at(L.ctrl), s)) != LNT_OK) return st;
  }
  {
    ProfScope prof("tile_rowptr", s);
    tile_rowptr_kernel<<<grid_cap(na + 1, 256), 256, 0, s>>>(ak, na, nullptr, make_divider(w), crows, arow);
    tile_rowptr_kernel<<<grid_cap(nb + 1, 256), 256, 0, s>>>(bk, nb, d_nb, make_divider(wB), brows, brow);
    count_launch(2);
  }
  if (cudaMemsetAsync(bbits, 0, brows * (u64)t.nw * 8, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  if (t.smax && cudaMemsetAsync(bd, 0, t.smax * (u64)t.nt * kTileCols * 8, s) != cudaSuccess)
    return LNT_DEVICE_ERROR;
  {
    ProfScope prof("tile_bprep", s);
    tile_slot_kernel<<<grid_cap(brows, 256), 256, 0, s>>>(brow, brows, std::max<u64>(wB, kTileCols), t.div, t.smax, dslot,
                                                         slot_counter);
    tile_bentry_kernel<<<grid_cap(nb, 256), 256, 0, s>>>(bk, bv, d_nb, brow, make_divider(wB), wB, t.nt, t.nw,
                                                        dslot, bbits, tp, bd);
    tile_tp_empty_kernel<<<grid_cap(brows, 256), 256, 0, s>>>(brow, brows, t.nt, tp);
    tile_arec_kernel<<<grid_cap(na, 256), 256, 0, s>>>(ak, av, na, w, make_divider(w), make_divider(h), dslot, rec);
    count_launch(4);
  }
  {
    ProfScope prof("tile_cbits", s);
    tile_cbits_kernel<<<grid_cap(crows * 32, 256), 256, 0, s>>>(ak, arow, bbits, h, w, d, t.nw, wB,
                                                               make_divider(h), cbits);
    count_launch();
  }
  {
    ProfScope prof("tile_count", s);
    tile_count_kernel<<<grid_cap(d * ((t.np + 31) / 32) * (u64)t.nw * 32, 256), 256, 0, s>>>(cbits, h, wB, d, t.nw,
                                                                                              t.np, cnt);
    count_launch();
  }
  if ((st = scan::run(CountGet{cnt}, ncnt, base, (unsigned long long*)d_nc, at(L.scan), s, "tile_scan")) != LNT_OK)
    return st;
  NumArgs a{rec, arow, bk, bv, tp, bd, cbits, base, h, w, wB, d, t.nt, t.nw, t.np, d * (u64)t.np * t.nt, ck, cv};
  {
    ProfScope prof("tile_numeric", s);
    auto kern = tile_numeric_kernel;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kNumericSmem) != cudaSuccess)
      return LNT_DEVICE_ERROR;
    const u64 grid = std::min<u64>(a.units, (u64)sm_count() * 2);
    kern<<<(unsigned)std::max<u64>(grid, 1), kTileThreads, kNumericSmem, s>>>(a);
    count_launch();
  }
  return launch_status();
}

}  // namespace lnt
