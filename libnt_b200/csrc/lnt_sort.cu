// One-sweep LSD radix sort of (u64 key, f64 value) pairs and the
// lnt_sort_pairs entry point.  Replaces the reference's in-place MSD radix
// sort RadixSortInPlace_PowerOf2Radix_Unsigned (LibMIARadix.h:444-484,
// 119-180): same ordering of keys; equal keys keep input order here (the
// reference's sort is unstable, so no order among equal keys is promised
// there).
#include <algorithm>
#include <cstring>

#include "lnt_sort.cuh"

namespace lnt {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr u32 kFlagAgg = 1u << 30;
constexpr u32 kFlagPre = 2u << 30;
constexpr u32 kFlagMask = 3u << 30;
constexpr u32 kValMask = (1u << 30) - 1u;

__device__ __forceinline__ u32 ld_volatile(const u32* p) {
  return *reinterpret_cast<const volatile u32*>(p);
}
__device__ __forceinline__ void st_volatile(u32* p, u32 v) {
  *reinterpret_cast<volatile u32*>(p) = v;
}

template <bool FIRST>
__device__ __forceinline__ u64 load_key(const PairSource& s, size_t i) {
  if (!FIRST) return __ldcs(s.ak + i);
  if (i < s.na) return rekey(__ldcs(s.ak + i), s.ra);
  return rekey(__ldcs(s.bk + (i - s.na)), s.rb);
}

template <bool FIRST>
__device__ __forceinline__ double load_val(const PairSource& s, size_t i) {
  if (!FIRST) return __ldcs(s.av + i);
  if (i < s.na) return __ldcs(s.av + i);
  return s.bscale * __ldcs(s.bv + (i - s.na));
}

// ---------------------------------------------------------------------------
// Histogram of every pass's digits in one read of the keys.
// ---------------------------------------------------------------------------
template <int BITS>
__global__ void __launch_bounds__(kThreads) hist_kernel(const PairSource src, u32 n, int passes,
                                                        int key_bits, u32* __restrict__ ghist,
                                                        u32* __restrict__ bstart,
                                                        u32* __restrict__ done) {
  constexpr int RADIX = 1 << BITS;
  extern __shared__ u32 sh_hist[];  // passes * RADIX
  __shared__ bool s_last;
  for (int i = threadIdx.x; i < passes * RADIX; i += kThreads) sh_hist[i] = 0;
  __syncthreads();
  const u32 stride = gridDim.x * kThreads;
  for (u32 i = blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
    u64 k = load_key<true>(src, i);
    for (int p = 0; p < passes; ++p) {
      int shift = p * BITS;
      int w = min(BITS, key_bits - shift);
      u32 d = (u32)(k >> shift) & ((1u << w) - 1u);
      atomicAdd(&sh_hist[p * RADIX + d], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * RADIX; i += kThreads) {
    u32 c = sh_hist[i];
    if (c) atomicAdd(&ghist[i], c);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(done, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // Last block: exclusive scan of each pass's histogram into bin starts.
  __shared__ u32 s_warp[kWarps];
  constexpr int DPT = (RADIX + kThreads - 1) / kThreads;
  for (int p = 0; p < passes; ++p) {
    u32 c[DPT];
    u32 local = 0;
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      int d = threadIdx.x * DPT + j;
      c[j] = d < RADIX ? __ldcg(&ghist[p * RADIX + d]) : 0u;
      local += c[j];
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32 inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      u32 t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    u32 wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += s_warp[w];
    u32 run = wpre + inc - local;
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      int d = threadIdx.x * DPT + j;
      if (d < RADIX) bstart[p * RADIX + d] = run;
      run += c[j];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// One digit pass.
// ---------------------------------------------------------------------------
template <int BITS, int ITEMS>
struct OnesweepSmem {
  static constexpr int RADIX = 1 << BITS;
  static constexpr int TILE = kThreads * ITEMS;
  static constexpr size_t bytes = (size_t)TILE * 8 + (size_t)kWarps * RADIX * 4 + (size_t)RADIX * 8 + 64;
};

template <int BITS, int ITEMS, bool FIRST>
__global__ void __launch_bounds__(kThreads) onesweep_kernel(const PairSource src, u64* __restrict__ out_k,
                                                            double* __restrict__ out_v, u32 n, u32 shift,
                                                            u32 mask, const u32* __restrict__ bstart,
                                                            u32* __restrict__ status,
                                                            u32* __restrict__ tile_counter) {
  constexpr int RADIX = 1 << BITS;
  constexpr int TILE = kThreads * ITEMS;
  constexpr int DPT = (RADIX + kThreads - 1) / kThreads;  // digits per thread
  extern __shared__ __align__(16) unsigned char smem[];
  u64* s_x = reinterpret_cast<u64*>(smem);                         // TILE
  u32* s_whist = reinterpret_cast<u32*>(s_x + TILE);               // kWarps * RADIX
  u32* s_tstart = s_whist + kWarps * RADIX;                        // RADIX
  u32* s_glob = s_tstart + RADIX;                                  // RADIX
  u32* s_misc = s_glob + RADIX;                                    // 16

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_misc[0] = atomicAdd(tile_counter, 1u);
  for (int i = tid; i < kWarps * RADIX; i += kThreads) s_whist[i] = 0;
  __syncthreads();
  const u32 tile = s_misc[0];
  const size_t tile_base = (size_t)tile * TILE;
  const u32 tile_n = (u32)min((size_t)TILE, (size_t)n - tile_base);
  const u32 warp_base = warp * ITEMS * 32;

  // ---- load keys (warp-striped: coalesced 256 B per warp per item) -------
  u64 key[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    u32 off = warp_base + i * 32 + lane;
    key[i] = off < tile_n ? load_key<FIRST>(src, tile_base + off) : ~0ull;
  }

  // ---- stable rank within (warp, digit) ----------------------------------
  u32 pos[ITEMS];
  const u32 lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    u32 off = warp_base + i * 32 + lane;
    u32 d = off < tile_n ? ((u32)(key[i] >> shift) & mask) : (u32)RADIX;
    u32 peers = __match_any_sync(0xffffffffu, d);
    int leader = __ffs(peers) - 1;
    u32 base = 0;
    if (lane == leader && d < (u32)RADIX) base = atomicAdd(&s_whist[warp * RADIX + d], (u32)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    pos[i] = base + __popc(peers & lt_mask);
  }
  __syncthreads();

  // ---- per digit: scan over warps, publish tile aggregate ----------------
  u32 cnt[DPT];
  u32 local = 0;
#pragma unroll
  for (int j = 0; j < DPT; ++j) {
    int d = tid * DPT + j;
    u32 sum = 0;
    if (d < RADIX) {
#pragma unroll
      for (int w = 0; w < kWarps; ++w) {
        u32 c = s_whist[w * RADIX + d];
        s_whist[w * RADIX + d] = sum;
        sum += c;
      }
      u32 word = tile == 0 ? (kFlagPre | (bstart[d] + sum)) : (kFlagAgg | sum);
      st_volatile(&status[(size_t)tile * RADIX + d], word);
    }
    cnt[j] = sum;
    local += sum;
  }
  // ---- block exclusive scan of digit counts -> tile-local digit starts ----
  {
    u32 inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      u32 t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) s_misc[4 + warp] = inc;
    __syncthreads();
    u32 run = inc - local;
    for (int w = 0; w < warp; ++w) run += s_misc[4 + w];
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      int d = tid * DPT + j;
      if (d < RADIX) s_tstart[d] = run;
      run += cnt[j];
    }
  }
  __syncthreads();

  // ---- tile positions; stage keys in digit order --------------------------
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    u32 off = warp_base + i * 32 + lane;
    if (off < tile_n) {
      u32 d = (u32)(key[i] >> shift) & mask;
      pos[i] += s_tstart[d] + s_whist[warp * RADIX + d];
      s_x[pos[i]] = key[i];
    }
  }
  // values are fetched now so their latency overlaps the look-back
  double val[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    u32 off = warp_base + i * 32 + lane;
    val[i] = off < tile_n ? load_val<FIRST>(src, tile_base + off) : 0.0;
  }

  // ---- decoupled look-back per digit ---------------------------------------
#pragma unroll
  for (int j = 0; j < DPT; ++j) {
    int d = tid * DPT + j;
    if (d >= RADIX) break;
    u32 excl;
    if (tile == 0) {
      excl = bstart[d];
    } else {
      excl = 0;
      int p = (int)tile - 1;
      u32 spins = 0;
      while (p >= 0) {
        u32 w = ld_volatile(&status[(size_t)p * RADIX + d]);
        u32 f = w & kFlagMask;
        if (f == 0) {
          if (++spins > kSpinLimit) {
            latch_error(kErrSortLookback);
            break;
          }
          continue;
        }
        excl += w & kValMask;
        if (f == kFlagPre) break;
        --p;
      }
      st_volatile(&status[(size_t)tile * RADIX + d], kFlagPre | (excl + cnt[j]));
    }
    s_glob[d] = excl - s_tstart[d];
  }
  __syncthreads();

  // ---- scatter keys (digit runs -> contiguous destination ranges) ---------
  u32 dst[ITEMS];
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    u32 idx = j * kThreads + tid;
    if (idx < tile_n) {
      u64 k = s_x[idx];
      u32 d = (u32)(k >> shift) & mask;
      dst[j] = s_glob[d] + idx;
      __stcs(out_k + dst[j], k);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    u32 off = warp_base + i * 32 + lane;
    if (off < tile_n) reinterpret_cast<double*>(s_x)[pos[i]] = val[i];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    u32 idx = j * kThreads + tid;
    if (idx < tile_n) __stcs(out_v + dst[j], reinterpret_cast<const double*>(s_x)[idx]);
  }
}

template <int BITS>
constexpr int items_for_bits() {
  return BITS <= 8 ? 16 : (BITS <= 10 ? 12 : 8);
}

template <int BITS>
int run_sort_bits(const SortPlan& plan, const PairSource& src, u64* buf0_k, double* buf0_v,
                  u64* buf1_k, double* buf1_v, void* ctrl, cudaStream_t s) {
  constexpr int RADIX = 1 << BITS;
  constexpr int ITEMS = items_for_bits<BITS>();
  constexpr int TILE = kThreads * ITEMS;
  if (plan.ntiles != (plan.n + TILE - 1) / TILE) return LNT_BAD_ARG;
  unsigned char* c = static_cast<unsigned char*>(ctrl);
  u32* ghist = reinterpret_cast<u32*>(c + plan.off_ghist);
  u32* bstart = reinterpret_cast<u32*>(c + plan.off_bstart);
  u32* status = reinterpret_cast<u32*>(c + plan.off_status);
  u32* counters = reinterpret_cast<u32*>(c + plan.off_counters);
  if (cudaMemsetAsync(ctrl, 0, plan.ctrl_bytes, s) != cudaSuccess) return LNT_DEVICE_ERROR;

  // histogram of all passes
  {
    size_t sh = (size_t)plan.passes * RADIX * 4;
    auto kern = hist_kernel<BITS>;
    if (sh > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    int blocks = std::max(1, std::min((int)((plan.n + kThreads * 16 - 1) / (kThreads * 16)), sm_count() * 4));
    ProfScope prof("sort_hist", s);
    kern<<<blocks, kThreads, sh, s>>>(src, plan.n, plan.passes, plan.key_bits, ghist, bstart,
                                      counters + plan.passes);
    count_launch();
  }
  constexpr size_t sh = OnesweepSmem<BITS, ITEMS>::bytes;
  // (function attributes are per device: set them on every call)
  cudaFuncSetAttribute(onesweep_kernel<BITS, ITEMS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  cudaFuncSetAttribute(onesweep_kernel<BITS, ITEMS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  const u64* in_k = nullptr;
  const double* in_v = nullptr;
  for (int p = 0; p < plan.passes; ++p) {
    int which = (plan.passes - 1 - p) & 1;
    u64* ok = which ? buf1_k : buf0_k;
    double* ov = which ? buf1_v : buf0_v;
    int shift = p * BITS;
    int w = std::min(BITS, plan.key_bits - shift);
    u32 mask = (1u << w) - 1u;
    u32* st = status + (size_t)p * plan.ntiles * RADIX;
    ProfScope prof("sort_onesweep", s);
    if (p == 0) {
      onesweep_kernel<BITS, ITEMS, true><<<plan.ntiles, kThreads, sh, s>>>(
          src, ok, ov, plan.n, (u32)shift, mask, bstart + p * RADIX, st, counters + p);
    } else {
      PairSource ps = plain_source(in_k, in_v, plan.n);
      onesweep_kernel<BITS, ITEMS, false><<<plan.ntiles, kThreads, sh, s>>>(
          ps, ok, ov, plan.n, (u32)shift, mask, bstart + p * RADIX, st, counters + p);
    }
    count_launch();
    in_k = ok;
    in_v = ov;
  }
  return launch_status();
}

// Copies the (possibly re-keyed / concatenated) source into buf0 unchanged;
// used when there is nothing to sort (all keys equal).
__global__ void copy_source_kernel(const PairSource src, u64* __restrict__ ok, double* __restrict__ ov, u32 n) {
  u32 stride = gridDim.x * blockDim.x;
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    ok[i] = load_key<true>(src, i);
    ov[i] = load_val<true>(src, i);
  }
}

}  // namespace

int choose_sort_bits(size_t n, int key_bits) {
  (void)n;
  if (key_bits <= 0) return 8;
  // Fewest passes at 8..10 bit digits, preferring narrower digits on ties.
  int best = 8, best_passes = (key_bits + 7) / 8;
  for (int b = 9; b <= 10; ++b) {
    int p = (key_bits + b - 1) / b;
    if (p < best_passes) {
      best = b;
      best_passes = p;
    }
  }
  return best;
}

SortPlan make_sort_plan(size_t n, u64 max_key, int bits) {
  SortPlan p;
  p.key_bits = key_bits_for(max_key);
  p.bits = bits;
  p.passes = p.key_bits == 0 ? 0 : (p.key_bits + bits - 1) / bits;
  p.n = (u32)n;
  int items = bits <= 8 ? 16 : (bits <= 10 ? 12 : 8);
  u32 tile = (u32)(kThreads * items);
  p.ntiles = (u32)((n + tile - 1) / tile);
  size_t radix = (size_t)1 << bits;
  size_t off = 0;
  p.off_ghist = off;
  off += align_up((size_t)std::max(p.passes, 1) * radix * 4, 256);
  p.off_bstart = off;
  off += align_up((size_t)std::max(p.passes, 1) * radix * 4, 256);
  p.off_status = off;
  off += align_up((size_t)p.passes * p.ntiles * radix * 4, 256);
  p.off_counters = off;
  off += 256;
  p.ctrl_bytes = off;
  return p;
}

int run_sort(const SortPlan& plan, const PairSource& src, u64* buf0_k, double* buf0_v, u64* buf1_k,
             double* buf1_v, void* ctrl, cudaStream_t s) {
  if (plan.n == 0) return LNT_OK;
  if (plan.passes == 0) {
    int blocks = std::max(1, std::min((int)((plan.n + 255) / 256), sm_count() * 8));
    ProfScope prof("sort_copy", s);
    copy_source_kernel<<<blocks, 256, 0, s>>>(src, buf0_k, buf0_v, plan.n);
    count_launch();
    return launch_status();
  }
  switch (plan.bits) {
    case 8: return run_sort_bits<8>(plan, src, buf0_k, buf0_v, buf1_k, buf1_v, ctrl, s);
    case 9: return run_sort_bits<9>(plan, src, buf0_k, buf0_v, buf1_k, buf1_v, ctrl, s);
    case 10: return run_sort_bits<10>(plan, src, buf0_k, buf0_v, buf1_k, buf1_v, ctrl, s);
    default: return LNT_UNSUPPORTED;
  }
}

}  // namespace lnt

using namespace lnt;

namespace {
// Workspace of lnt_sort_pairs: [ctrl | tmp keys | tmp vals | (tmp2 keys | tmp2 vals)].
struct SortPairsLayout {
  SortPlan plan;
  size_t off_tk, off_tv, off_t2k, off_t2v, total;
};

SortPairsLayout sort_pairs_layout(size_t n, u64 max_key) {
  SortPairsLayout L;
  int kb = key_bits_for(max_key);
  L.plan = make_sort_plan(n, max_key, choose_sort_bits(n, kb));
  size_t off = align_up(L.plan.ctrl_bytes, 256);
  L.off_tk = off;
  off += align_up(n * 8, 256);
  L.off_tv = off;
  off += align_up(n * 8, 256);
  L.off_t2k = off;
  off += align_up(n * 8, 256);
  L.off_t2v = off;
  off += align_up(n * 8, 256);
  L.total = off;
  return L;
}
}  // namespace

extern "C" {

int lnt_sort_pairs_workspace(size_t n, uint64_t max_key, size_t* bytes) {
  if (!bytes) return LNT_BAD_ARG;
  if (n >= (1u << 30)) return LNT_UNSUPPORTED;
  *bytes = sort_pairs_layout(n, max_key).total;
  return LNT_OK;
}

int lnt_sort_pairs(const uint64_t* keys_in, const double* vals_in, uint64_t* keys_out, double* vals_out,
                   size_t n, uint64_t max_key, void* workspace, size_t workspace_bytes, void* stream) {
  if (n == 0) return LNT_OK;
  if (!keys_in || !vals_in || !keys_out || !vals_out) return LNT_BAD_ARG;
  if (n >= (1u << 30)) return LNT_UNSUPPORTED;
  SortPairsLayout L = sort_pairs_layout(n, max_key);
  if (!workspace || workspace_bytes < L.total) return LNT_WORKSPACE;
  if ((uintptr_t)workspace % 256) return LNT_BAD_ARG;
  cudaStream_t s = as_stream(stream);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  u64* tk = reinterpret_cast<u64*>(ws + L.off_tk);
  double* tv = reinterpret_cast<double*>(ws + L.off_tv);
  PairSource src = plain_source((const u64*)keys_in, vals_in, n);
  const bool inplace = (const void*)keys_in == (const void*)keys_out || (const void*)vals_in == (const void*)vals_out;
  const int passes = L.plan.passes;
  if (!inplace || (passes % 2 == 0 && passes > 0)) {
    // pass 0 writes tmp when passes is even, so in-place is safe then.
    return run_sort(L.plan, src, (u64*)keys_out, vals_out, tk, tv, ws, s);
  }
  // In place with an odd pass count (or nothing to sort): sort into the
  // second scratch pair and copy back.
  u64* t2k = reinterpret_cast<u64*>(ws + L.off_t2k);
  double* t2v = reinterpret_cast<double*>(ws + L.off_t2v);
  if (passes == 0) return LNT_OK;  // all keys equal: input order is the stable order
  int st = run_sort(L.plan, src, t2k, t2v, tk, tv, ws, s);
  if (st != LNT_OK) return st;
  if (cudaMemcpyAsync(keys_out, t2k, n * 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  if (cudaMemcpyAsync(vals_out, t2v, n * 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  return LNT_OK;
}

}  // extern "C"
