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
//     summed, with row pointers (w*d + 1); a row holding at least a quarter of
//     its columns is also expanded into a dense row of Bd (one slot per such
//     row, zero-filled, padded to whole 64-column tiles); for every row
//     tp[row][q] = entries of the row left of column 64q (q = 0..nt);
//   bitmaps, one bit per (row, column), 64-column words: Bbits (B rows) and
//     Cbits (C rows, = OR of the Bbits rows that A row selects) — the output
//     pattern, computed before any arithmetic.
// Output positions: per (tab, column, panel of 128 rows) the number of
// pattern bits, exclusive-scanned in (tab, column, panel) order, so each
// panel's rows of one column land at a known contiguous offset.
// Numeric pass: one CTA per (panel, 64-column tile) unit, one warp per row,
// two columns per lane in registers; per A entry of the row a dense B row
// adds one coalesced 512-byte load, a sparse one its tile segment (OR-reduced
// column mask, lanes pick their entries by shuffle).  The 128 x 64 tile is
// staged in shared memory and written column by column (contiguous runs).
#include <algorithm>

#include "lnt_scan.cuh"
#include "lnt_sort.cuh"

namespace lnt {

int run_collect(const u64* keys, const double* vals, size_t n, int skip_zero_heads, u64* out_k, double* out_v,
                u64* d_nout, void* ws, cudaStream_t s);
size_t collect_workspace_bytes(size_t n);

namespace {

constexpr u32 FULL = 0xffffffffu;
constexpr int kTileCols = 64;      // output columns per tile (two per lane)
constexpr int kPanelRows = 128;    // output rows per unit
constexpr int kTileThreads = 512;  // 16 warps, 8 rows each
constexpr int kTileGroup = 8;      // tiles of one panel processed by consecutive units
constexpr int kStageStride = 65;   // doubles per staged row
constexpr size_t kStageBytes = (size_t)kPanelRows * kStageStride * 8;
constexpr size_t kMaxBitmapBytes = 16ull << 30;

struct TileDims {
  u64 h, w, wB, d;
  u32 nt, np;  // 64-column tiles per row, 128-row panels per tab
  u64 smax;    // dense-row slots
};

TileDims tile_dims(u64 h, u64 w, u64 wB, u64 d, u64 nb) {
  TileDims t;
  t.h = h;
  t.w = w;
  t.wB = wB;
  t.d = d;
  t.nt = (u32)((wB + kTileCols - 1) / kTileCols);
  t.np = (u32)((h + kPanelRows - 1) / kPanelRows);
  const u64 thr = std::max<u64>(wB, kTileCols);  // dense: 4 * len >= thr
  t.smax = std::min<u64>(w * d, 4 * nb / thr);
  return t;
}

struct TileLayout {
  size_t ctrl, ak, av, tk, tv, bk, bv, arow, brow, dslot, tp, bbits, bd, cbits, cnt, base, scan, coll, misc, total;
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
  L.tp = take(t.w * t.d * (u64)(t.nt + 1) * 4);
  L.bbits = take(t.w * t.d * (u64)t.nt * 8);
  L.bd = take(t.smax * (u64)t.nt * kTileCols * 8);
  L.cbits = take(t.h * t.d * (u64)t.nt * 8);
  L.cnt = take(ncnt * 4);
  L.base = take((ncnt + 1) * 8);
  L.scan = take(scan::workspace_bytes(ncnt));
  L.coll = take(collect_workspace_bytes(nb));
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
__global__ void tile_slot_kernel(const u64* __restrict__ brow, u64 nrows, u64 thr, u64 smax, int* __restrict__ dslot,
                                 u32* __restrict__ counter) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 r = (u64)blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += stride) {
    const u64 len = brow[r + 1] - brow[r];
    int slot = -1;
    if (len * 4 >= thr) {
      const u32 s = atomicAdd(counter, 1u);
      if (s < smax) slot = (int)s;
    }
    dslot[r] = slot;
  }
}

// Per unique B entry: its bit in Bbits, its value in Bd (dense rows), and the
// tile pointers of its row.
__global__ void tile_bentry_kernel(const u64* __restrict__ bk, const double* __restrict__ bv,
                                   const u64* __restrict__ d_n, const u64* __restrict__ brow, Divider div_wB, u64 wB,
                                   u32 nt, const int* __restrict__ dslot, u64* __restrict__ bbits,
                                   u32* __restrict__ tp, double* __restrict__ bd) {
  const u64 n = *d_n;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const u64 k = bk[e];
    const u64 row = divide(k, div_wB);
    const u64 j = k - row * wB;
    const u32 q = (u32)(j >> 6);
    atomicOr(reinterpret_cast<unsigned long long*>(bbits + row * nt + q), 1ull << (j & 63));
    const int slot = dslot[row];
    if (slot >= 0) bd[(u64)slot * nt * kTileCols + j] = bv[e];
    const u64 rs = brow[row], re = brow[row + 1];
    u32* t = tp + row * (u64)(nt + 1);
    long long qprev = -1;
    if (e > rs) qprev = (long long)((bk[e - 1] - row * wB) >> 6);
    for (long long qq = qprev + 1; qq <= (long long)q; ++qq) t[qq] = (u32)(e - rs);
    if (e + 1 == re)
      for (u32 qq = q + 1; qq <= nt; ++qq) t[qq] = (u32)(e + 1 - rs);
  }
}

// Cbits[row] = OR of Bbits[c + w*t] over the A entries (row, c); warp per row.
__global__ void tile_cbits_kernel(const u64* __restrict__ ak, const u64* __restrict__ arow,
                                  const u64* __restrict__ bbits, u64 h, u64 w, u64 d, u32 nt, Divider div_h,
                                  u64* __restrict__ cbits) {
  const int lane = threadIdx.x & 31;
  const u64 nrows = h * d;
  const u64 nw = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 row = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrows; row += nw) {
    const u64 t = divide(row, div_h);
    const u64 e0 = arow[row], e1 = arow[row + 1];
    const u64 cbase = w * t - w * row;  // B row = A key + cbase
    for (u32 w0 = 0; w0 < nt; w0 += 32) {
      const u32 word = w0 + lane;
      u64 acc = 0;
      for (u64 eb = e0; eb < e1; eb += 32) {
        const u64 e = eb + lane;
        const u64 br = e < e1 ? ak[e] + cbase : 0;
        const int n = (int)(e1 - eb < 32 ? e1 - eb : 32);
        for (int k = 0; k < n; ++k) {
          const u64 b = __shfl_sync(FULL, br, k);
          if (word < nt) acc |= bbits[b * nt + word];
        }
      }
      if (word < nt) cbits[row * nt + word] = acc;
    }
  }
}

// cnt[(t*wB + col)*np + p] = pattern bits of column col among panel p's rows;
// warp per (t, p, q).
__global__ void tile_count_kernel(const u64* __restrict__ cbits, u64 h, u64 wB, u64 d, u32 nt, u32 np,
                                  u32* __restrict__ cnt) {
  const int lane = threadIdx.x & 31;
  const u64 units = d * np * (u64)nt;
  const u64 nw = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 u = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < units; u += nw) {
    const u64 t = u / ((u64)np * nt);
    const u64 rem = u - t * np * nt;
    const u32 p = (u32)(rem / nt);
    const u32 q = (u32)(rem - (u64)p * nt);
    u32 clo = 0, chi = 0;
    for (int g = 0; g < kPanelRows / 32; ++g) {
      const u64 r = (u64)p * kPanelRows + g * 32 + lane;
      const u64 word = r < h ? cbits[(r + h * t) * nt + q] : 0ull;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const u32 lo = __popc(__ballot_sync(FULL, (word >> j) & 1ull));
        const u32 hi = __popc(__ballot_sync(FULL, (word >> (32 + j)) & 1ull));
        if (lane == j) {
          clo += lo;
          chi += hi;
        }
      }
    }
    const u64 c0 = (u64)q * kTileCols + lane, c1 = c0 + 32;
    if (c0 < wB) cnt[(t * wB + c0) * np + p] = clo;
    if (c1 < wB) cnt[(t * wB + c1) * np + p] = chi;
  }
}

struct CountGet {
  const u32* c;
  __device__ __forceinline__ u64 operator()(size_t i) const { return c[i]; }
};

struct NumArgs {
  const u64* ak;
  const double* av;
  const u64* arow;
  const u64* bk;
  const double* bv;
  const u64* brow;
  const int* dslot;
  const u32* tp;
  const double* bd;
  const u64* cbits;
  const unsigned long long* base;
  u64 h, w, wB, d;
  u32 nt, np;
  u64 units;
  u64* ck;
  double* cv;
};

__global__ void __launch_bounds__(kTileThreads, 2) tile_numeric_kernel(NumArgs a) {
  extern __shared__ double stage[];  // [kPanelRows][kStageStride]
  __shared__ u64 s_bits[kPanelRows];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
    if (threadIdx.x < kPanelRows) {
      const u64 r = row0 + threadIdx.x;
      s_bits[threadIdx.x] = r < a.h ? a.cbits[(r + a.h * t) * a.nt + q] : 0ull;
    }
    __syncthreads();
    const double2* bd2 = reinterpret_cast<const double2*>(a.bd);
    for (int i = warp; i < kPanelRows; i += kTileThreads / 32) {
      if (s_bits[i] == 0ull) continue;
      const u64 row = row0 + i + a.h * t;
      const u64 e0 = a.arow[row], e1 = a.arow[row + 1];
      const u64 cbase = a.w * t - a.w * row;  // B row = A key + cbase
      double acc0 = 0.0, acc1 = 0.0;
      for (u64 eb = e0; eb < e1; eb += 32) {
        const u64 e = eb + lane;
        u64 br = 0, s0 = 0;
        double v = 0.0;
        int slot = -1;
        u32 len = 0;
        if (e < e1) {
          br = a.ak[e] + cbase;
          v = a.av[e];
          slot = a.dslot[br];
          if (slot < 0) {
            const u32* tpr = a.tp + br * (u64)(a.nt + 1);
            const u32 lo = tpr[q];
            len = tpr[q + 1] - lo;
            s0 = a.brow[br] + lo;
          }
        }
        const int n = (int)(e1 - eb < 32 ? e1 - eb : 32);
        for (int k = 0; k < n; ++k) {
          const double vk = __shfl_sync(FULL, v, k);
          const int sk = __shfl_sync(FULL, slot, k);
          if (sk >= 0) {
            const double2 b = bd2[((u64)sk * a.nt + q) * 32 + lane];
            acc0 = fma(vk, b.x, acc0);
            acc1 = fma(vk, b.y, acc1);
            continue;
          }
          const u32 lk = __shfl_sync(FULL, len, k);
          if (lk == 0) continue;
          const u64 sk0 = __shfl_sync(FULL, s0, k);
          const u64 kb = a.wB * __shfl_sync(FULL, br, k) + (u64)q * kTileCols;  // key of the tile's column 0
          u32 jl = 64, jh = 64;
          double wl = 0.0, wh = 0.0;
          if ((u32)lane < lk) {
            jl = (u32)(a.bk[sk0 + lane] - kb);
            wl = a.bv[sk0 + lane];
          }
          if ((u32)lane + 32 < lk) {
            jh = (u32)(a.bk[sk0 + 32 + lane] - kb);
            wh = a.bv[sk0 + 32 + lane];
          }
          const u32 mlo = __reduce_or_sync(FULL, (jl < 32 ? 1u << jl : 0u) | (jh < 32 ? 1u << jh : 0u));
          const u32 mhi = __reduce_or_sync(FULL, (jl >= 32 && jl < 64 ? 1u << (jl - 32) : 0u) |
                                                     (jh >= 32 && jh < 64 ? 1u << (jh - 32) : 0u));
          const u64 m = ((u64)mhi << 32) | mlo;
          const int c0 = 2 * lane;
          const bool has0 = (m >> c0) & 1ull, has1 = (m >> (c0 + 1)) & 1ull;
          const int i0 = __popcll(m & ((1ull << c0) - 1ull));  // entry index of column c0 (if present)
          const int i1 = i0 + (int)has0;                        // entry index of column c0 + 1
          const double x0l = __shfl_sync(FULL, wl, i0 & 31), x0h = __shfl_sync(FULL, wh, i0 & 31);
          const double x1l = __shfl_sync(FULL, wl, i1 & 31), x1h = __shfl_sync(FULL, wh, i1 & 31);
          if (has0) acc0 = fma(vk, i0 < 32 ? x0l : x0h, acc0);
          if (has1) acc1 = fma(vk, i1 < 32 ? x1l : x1h, acc1);
        }
      }
      stage[i * kStageStride + 2 * lane] = acc0;
      stage[i * kStageStride + 2 * lane + 1] = acc1;
    }
    __syncthreads();
    for (int jj = warp; jj < kTileCols; jj += kTileThreads / 32) {
      const u64 col = (u64)q * kTileCols + jj;
      if (col >= a.wB) continue;
      unsigned long long pos = a.base[(t * a.wB + col) * a.np + p];
      const u64 keybase = a.h * (col + a.wB * t) + row0;
#pragma unroll
      for (int g = 0; g < kPanelRows / 32; ++g) {
        const int i = g * 32 + lane;
        const bool bit = (s_bits[i] >> jj) & 1ull;
        const u32 m = __ballot_sync(FULL, bit);
        if (bit) {
          const u64 o = pos + __popc(m & ((1u << lane) - 1u));
          a.ck[o] = keybase + i;
          a.cv[o] = stage[i * kStageStride + jj];
        }
        pos += __popc(m);
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
  if (na >= (1ull << 32) || nb >= (1ull << 32)) return false;
  const TileDims t = tile_dims(h, w, wB, d, nb);
  const unsigned __int128 cb = (unsigned __int128)h * d * t.nt * 8;
  const unsigned __int128 bb = (unsigned __int128)w * d * (t.nt + 1) * 12;
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
  u32* tp = (u32*)at(L.tp);
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
  if (cudaMemsetAsync(tp, 0, brows * (u64)(t.nt + 1) * 4, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  if (cudaMemsetAsync(bbits, 0, brows * (u64)t.nt * 8, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  if (t.smax && cudaMemsetAsync(bd, 0, t.smax * (u64)t.nt * kTileCols * 8, s) != cudaSuccess)
    return LNT_DEVICE_ERROR;
  {
    ProfScope prof("tile_bprep", s);
    tile_slot_kernel<<<grid_cap(brows, 256), 256, 0, s>>>(brow, brows, std::max<u64>(wB, kTileCols), t.smax, dslot,
                                                         slot_counter);
    tile_bentry_kernel<<<grid_cap(nb, 256), 256, 0, s>>>(bk, bv, d_nb, brow, make_divider(wB), wB, t.nt, dslot,
                                                        bbits, tp, bd);
    count_launch(2);
  }
  {
    ProfScope prof("tile_cbits", s);
    tile_cbits_kernel<<<grid_cap(crows * 32, 256), 256, 0, s>>>(ak, arow, bbits, h, w, d, t.nt, make_divider(h),
                                                               cbits);
    count_launch();
  }
  {
    ProfScope prof("tile_count", s);
    tile_count_kernel<<<grid_cap(d * t.np * (u64)t.nt * 32, 256), 256, 0, s>>>(cbits, h, wB, d, t.nt, t.np, cnt);
    count_launch();
  }
  if ((st = scan::run(CountGet{cnt}, ncnt, base, (unsigned long long*)d_nc, at(L.scan), s, "tile_scan")) != LNT_OK)
    return st;
  NumArgs a{ak, av, arow, bk, bv, brow, dslot, tp, bd, cbits, base, h, w, wB, d, t.nt, t.np,
            d * (u64)t.np * t.nt, ck, cv};
  {
    ProfScope prof("tile_numeric", s);
    if (cudaFuncSetAttribute(tile_numeric_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageBytes) !=
        cudaSuccess)
      return LNT_DEVICE_ERROR;
    const u64 grid = std::min<u64>(a.units, (u64)sm_count() * 2);
    tile_numeric_kernel<<<(unsigned)std::max<u64>(grid, 1), kTileThreads, kStageBytes, s>>>(a);
    count_launch();
  }
  return launch_status();
}

}  // namespace lnt
