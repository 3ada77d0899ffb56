// One-sweep LSD radix sort of (u64 key, f64 value) pairs and the
// lnt_sort_pairs entry point.  Replaces the reference's in-place MSD radix
// sort RadixSortInPlace_PowerOf2Radix_Unsigned (LibMIARadix.h:444-484,
// 119-180): same ordering of keys; equal keys keep input order here (the
// reference's sort is unstable, so no order among equal keys is promised
// there).
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "lnt_sort.cuh"

namespace lnt {
namespace {

constexpr int kThreads = 256;  // histogram kernel CTA size
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
  if (gated_off(src.gate, src.gate_run)) return;
  for (int i = threadIdx.x; i < passes * RADIX; i += kThreads) sh_hist[i] = 0;
  __syncthreads();
  const u32 stride = gridDim.x * kThreads;
  constexpr int U = 8;  // independent loads in flight per thread
  u32 i = blockIdx.x * kThreads + threadIdx.x;
  for (; i + (U - 1) * stride < n; i += U * stride) {
    u64 k[U];
#pragma unroll
    for (int u = 0; u < U; ++u) k[u] = load_key<true>(src, i + u * stride);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      for (int p = 0; p < passes; ++p) {
        const int shift = p * BITS;
        const int w = min(BITS, key_bits - shift);
        atomicAdd(&sh_hist[p * RADIX + ((u32)(k[u] >> shift) & ((1u << w) - 1u))], 1u);
      }
    }
  }
  for (; i < n; i += stride) {
    u64 k = load_key<true>(src, i);
    for (int p = 0; p < passes; ++p) {
      const int shift = p * BITS;
      const int w = min(BITS, key_bits - shift);
      atomicAdd(&sh_hist[p * RADIX + ((u32)(k >> shift) & ((1u << w) - 1u))], 1u);
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
template <int BITS, int THREADS, int ITEMS>
struct OnesweepShape {
  static constexpr int RADIX = 1 << BITS;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int TILE = THREADS * ITEMS;
  static constexpr int DPT = (RADIX + THREADS - 1) / THREADS;  // digits per thread
  static constexpr size_t smem = (size_t)TILE * 16 + (size_t)WARPS * RADIX * 4 + (size_t)RADIX * 8 + 64;
  // CTAs per SM that shared memory allows (228 KB per SM, 1 KB reserved per CTA), at most 4
  static constexpr int kFit = (int)((228u * 1024u) / (smem + 1024u));
  static constexpr int MINB = kFit < 1 ? 1 : (kFit > 4 ? 4 : kFit);
};

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <bool FIRST>
__device__ __forceinline__ const double* val_ptr(const PairSource& s, size_t i) {
  if (!FIRST || i < s.na) return s.av + i;
  return s.bv + (i - s.na);
}

// Lanes of the warp holding the same BITS-bit digit (one ballot per bit).
template <int BITS>
__device__ __forceinline__ u32 match_digit(u32 d) {
  u32 peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < BITS; ++b) {
    const u32 bit = (d >> b) & 1u;
    const u32 m = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? m : ~m;
  }
  return peers;
}

// PERSIST: a grid smaller than the tile count whose CTAs take tiles until
// none is left.  Tiles are taken in order and a CTA finishes its tile before
// taking another, so every predecessor a look-back waits on belongs to a
// running CTA.
template <int BITS, int THREADS, int ITEMS, int W, bool FIRST, bool PERSIST = false>
__global__ void __launch_bounds__(THREADS, (OnesweepShape<BITS, THREADS, ITEMS>::MINB))
    onesweep_kernel(const PairSource src, u64* __restrict__ out_k, double* __restrict__ out_v, u32 n, u32 shift,
                    u32 mask, const u32* __restrict__ bstart, u32* __restrict__ status,
                    u32* __restrict__ tile_counter) {
  if (gated_off(src.gate, src.gate_run)) return;
  using S = OnesweepShape<BITS, THREADS, ITEMS>;
  constexpr int RADIX = S::RADIX;
  constexpr int WARPS = S::WARPS;
  constexpr int TILE = S::TILE;
  constexpr int DPT = S::DPT;
  extern __shared__ __align__(16) unsigned char smem[];
  u64* s_x = reinterpret_cast<u64*>(smem);               // TILE: tile in digit order
  double* s_v = reinterpret_cast<double*>(s_x + TILE);   // TILE: values in input order
  u32* s_whist = reinterpret_cast<u32*>(s_v + TILE);     // WARPS * RADIX
  u32* s_tstart = s_whist + WARPS * RADIX;               // RADIX
  u32* s_glob = s_tstart + RADIX;                        // RADIX
  u32* s_misc = s_glob + RADIX;                          // 16

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32 ntiles = (n + TILE - 1) / TILE;
  for (;;) {
  if (tid == 0) s_misc[0] = atomicAdd(tile_counter, 1u);
  for (int i = tid; i < WARPS * RADIX; i += THREADS) s_whist[i] = 0;
  __syncthreads();
  const u32 tile = s_misc[0];
  if (PERSIST && tile >= ntiles) break;
  const size_t tile_base = (size_t)tile * TILE;
  const u32 tile_n = (u32)min((size_t)TILE, (size_t)n - tile_base);
  const u32 warp_base = warp * ITEMS * 32;

  // ---- load keys (warp-striped: coalesced 256 B per warp per item) -------
  u64 key[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const u32 off = warp_base + i * 32 + lane;
    key[i] = off < tile_n ? load_key<FIRST>(src, tile_base + off) : 0ull;
  }
  // values go straight to shared memory; the copy overlaps everything up to
  // the value scatter and holds no registers
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const u32 off = warp_base + i * 32 + lane;
    if (off < tile_n) cp_async8(&s_v[off], val_ptr<FIRST>(src, tile_base + off));
  }
  cp_async_commit();

  // ---- per-warp digit counts (no return values: fire-and-forget) ---------
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const u32 off = warp_base + i * 32 + lane;
    if (off < tile_n) atomicAdd(&s_whist[warp * RADIX + ((u32)(key[i] >> shift) & mask)], 1u);
  }
  __syncthreads();

  // ---- tile counts: publish at once so successors can look back ----------
  u32 cnt[DPT];
  u32 local = 0;
#pragma unroll
  for (int j = 0; j < DPT; ++j) {
    const int d = tid * DPT + j;
    u32 c = 0;
    if (d < RADIX) {
#pragma unroll
      for (int w = 0; w < WARPS; ++w) c += s_whist[w * RADIX + d];
      const u32 word = tile == 0 ? (kFlagPre | (bstart[d] + c)) : (kFlagAgg | c);
      st_volatile(&status[(size_t)tile * RADIX + d], word);
    }
    cnt[j] = c;
    local += c;
  }
  // ---- block exclusive scan of digit counts; per-(warp, digit) bases ------
  u32 tstart[DPT];
  {
    u32 inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) s_misc[4 + warp] = inc;
    __syncthreads();
    u32 run = inc - local;
    for (int w = 0; w < warp; ++w) run += s_misc[4 + w];
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      const int d = tid * DPT + j;
      tstart[j] = run;
      if (d < RADIX) {
        u32 b = run;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) {
          const u32 c = s_whist[w * RADIX + d];
          s_whist[w * RADIX + d] = b;
          b += c;
        }
      }
      run += cnt[j];
    }
  }

  __syncthreads();  // the per-(warp, digit) bases are complete
  // ---- stable rank: ballot match + per-(warp, digit) running base ---------
  u32 pos[ITEMS];
  const u32 lt_mask = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const u32 off = warp_base + i * 32 + lane;
    const bool valid = off < tile_n;
    const u32 vmask = __ballot_sync(0xffffffffu, valid);
    const u32 d = valid ? ((u32)(key[i] >> shift) & mask) : 0u;
    const u32 peers = match_digit<BITS>(d) & vmask;
    u32 base = 0;
    if (valid) base = s_whist[warp * RADIX + d];
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) s_whist[warp * RADIX + d] = base + __popc(peers);
    __syncwarp();
    pos[i] = base + __popc(peers & lt_mask);
  }
  // ---- stage keys in digit order ------------------------------------------
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const u32 off = warp_base + i * 32 + lane;
    if (off < tile_n) s_x[pos[i]] = key[i];
  }
  __syncthreads();

  // ---- decoupled look-back, W predecessors per round trip per digit -------
  // (after the local ranking: predecessors have had that long to publish
  // their inclusive prefixes, so the walk back is shorter)
  {
    u32 excl[DPT];
    int p[DPT];
    bool done[DPT];
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      const int d = tid * DPT + j;
      excl[j] = (tile == 0 && d < RADIX) ? bstart[d] : 0u;
      p[j] = (int)tile - 1;
      done[j] = (d >= RADIX) || tile == 0;
    }
    u32 spins = 0;
    while (true) {
      bool all_done = true;
#pragma unroll
      for (int j = 0; j < DPT; ++j) all_done = all_done && done[j];
      if (all_done) break;
      u32 w[DPT][W];
#pragma unroll
      for (int j = 0; j < DPT; ++j) {
        const int d = tid * DPT + j;
#pragma unroll
        for (int q = 0; q < W; ++q) {
          const int pp = p[j] - q;
          w[j][q] = (!done[j] && pp >= 0) ? ld_volatile(&status[(size_t)pp * RADIX + d]) : kFlagPre;
        }
      }
      bool stalled = false;
#pragma unroll
      for (int j = 0; j < DPT; ++j) {
        if (done[j]) continue;
        int q = 0;
#pragma unroll
        for (; q < W; ++q) {
          const u32 f = w[j][q] & kFlagMask;
          if (f == 0) break;
          excl[j] += w[j][q] & kValMask;
          if (f == kFlagPre) {
            done[j] = true;
            break;
          }
        }
        if (!done[j]) {
          p[j] -= q;
          if (q < W) stalled = true;
        }
      }
      if (stalled && ++spins > spin_limit()) {
        latch_error(kErrSortLookback);
        break;
      }
    }
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      const int d = tid * DPT + j;
      if (d >= RADIX) break;
      if (tile != 0) st_volatile(&status[(size_t)tile * RADIX + d], kFlagPre | (excl[j] + cnt[j]));
      s_glob[d] = excl[j] - tstart[j];
    }
  }
  __syncthreads();

  // ---- scatter keys (digit runs -> contiguous destination ranges) ---------
  // The clamp changes nothing in a correct run (every position is < n).  It
  // keeps writes inside the output after a look-back gave up: a pass that
  // reads a previous pass's partial output sees digit counts that no longer
  // match the histogram, so its offsets could otherwise pass n.
  u32 dst[ITEMS];
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const u32 idx = j * THREADS + tid;
    if (idx < tile_n) {
      const u64 k = s_x[idx];
      dst[j] = min(s_glob[(u32)(k >> shift) & mask] + idx, n - 1u);
      __stcs(out_k + dst[j], k);
    }
  }
  cp_async_wait_all();
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const u32 off = warp_base + i * 32 + lane;
    if (off < tile_n) {
      double v = s_v[off];
      if (FIRST && tile_base + off >= src.na) v *= src.bscale;
      reinterpret_cast<double*>(s_x)[pos[i]] = v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const u32 idx = j * THREADS + tid;
    if (idx < tile_n) __stcs(out_v + dst[j], reinterpret_cast<const double*>(s_x)[idx]);
  }
  if (!PERSIST) break;
  __syncthreads();  // shared memory is reused by the next tile
  }
}

// Copies the (possibly re-keyed / concatenated) source into buf0 unchanged;
// used when there is nothing to sort (all keys equal).
__global__ void copy_source_kernel(const PairSource src, u64* __restrict__ ok, double* __restrict__ ov, u32 n) {
  if (gated_off(src.gate, src.gate_run)) return;
  const u32 stride = gridDim.x * blockDim.x;
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    ok[i] = load_key<true>(src, i);
    ov[i] = load_val<true>(src, i);
  }
}

// Zeroes `words` 32-bit words (the gated form of the control block's memset).
__global__ void zero_words_kernel(u32* __restrict__ p, size_t words, const u32* gate, u32 want) {
  if (gated_off(gate, want)) return;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  uint4* p4 = reinterpret_cast<uint4*>(p);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words / 4; i += stride)
    p4[i] = make_uint4(0u, 0u, 0u, 0u);
  for (size_t i = (words / 4) * 4 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) p[i] = 0u;
}

#define LNT_SV_ENTRY(B, T, I, W) {B, T, I, W},
const SortVariant kVariants[] = {LNT_SORT_VARIANTS(LNT_SV_ENTRY)};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

template <int BITS, int THREADS, int ITEMS, int W>
int run_sort_variant(const SortPlan& plan, const PairSource& src, u64* buf0_k, double* buf0_v, u64* buf1_k,
                     double* buf1_v, void* ctrl, cudaStream_t s) {
  using Sh = OnesweepShape<BITS, THREADS, ITEMS>;
  constexpr int RADIX = Sh::RADIX;
  if (plan.tile != (u32)Sh::TILE || plan.bits != BITS) return LNT_BAD_ARG;
  unsigned char* c = static_cast<unsigned char*>(ctrl);
  u32* ghist = reinterpret_cast<u32*>(c + plan.off_ghist);
  u32* bstart = reinterpret_cast<u32*>(c + plan.off_bstart);
  u32* status = reinterpret_cast<u32*>(c + plan.off_status);
  u32* counters = reinterpret_cast<u32*>(c + plan.off_counters);
  const bool gated = src.gate != nullptr;
  if (gated) {  // skipped with the rest of the sort when the gate is closed
    const size_t words = plan.ctrl_bytes / 4;  // ctrl is 256-byte aligned, ctrl_bytes a multiple of 256
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((words / 4 + 255) / 256, (size_t)sm_count() * 4));
    zero_words_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<u32*>(ctrl), words, src.gate, src.gate_run);
    count_launch();
  } else if (cudaMemsetAsync(ctrl, 0, plan.ctrl_bytes, s) != cudaSuccess) {
    return LNT_DEVICE_ERROR;
  }

  // histogram of all passes
  {
    const size_t sh = (size_t)plan.passes * RADIX * 4;
    auto kern = hist_kernel<BITS>;
    if (sh > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    const int blocks =
        std::max(1, std::min((int)((plan.n + kThreads * 16 - 1) / (kThreads * 16)), sm_count() * 4));
    ProfScope prof(src.gate ? "sort_hist_fallback" : "sort_hist", s);
    kern<<<blocks, kThreads, sh, s>>>(src, plan.n, plan.passes, plan.key_bits, ghist, bstart,
                                      counters + plan.passes);
    count_launch();
  }
  constexpr size_t sh = Sh::smem;
  // (function attributes are per device: set them on every call)
  cudaFuncSetAttribute(onesweep_kernel<BITS, THREADS, ITEMS, W, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  cudaFuncSetAttribute(onesweep_kernel<BITS, THREADS, ITEMS, W, false>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
  u32 grid = plan.ntiles;
  if (gated) {  // persistent grid: a closed gate then costs one wave of empty CTAs
    cudaFuncSetAttribute(onesweep_kernel<BITS, THREADS, ITEMS, W, true, true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    cudaFuncSetAttribute(onesweep_kernel<BITS, THREADS, ITEMS, W, false, true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, onesweep_kernel<BITS, THREADS, ITEMS, W, false, true>,
                                                      THREADS, sh) != cudaSuccess)
      return LNT_DEVICE_ERROR;
    grid = std::min(grid, (u32)(std::max(per_sm, 1) * sm_count()));
  }
  const u64* in_k = nullptr;
  const double* in_v = nullptr;
  for (int p = 0; p < plan.passes; ++p) {
    const int which = (plan.passes - 1 - p) & 1;
    u64* ok = which ? buf1_k : buf0_k;
    double* ov = which ? buf1_v : buf0_v;
    const int shift = p * BITS;
    const int w = std::min(BITS, plan.key_bits - shift);
    const u32 mask = (1u << w) - 1u;
    u32* st = status + (size_t)p * plan.ntiles * RADIX;
    ProfScope prof(gated ? "sort_onesweep_fallback" : "sort_onesweep", s);
    if (p == 0) {
      if (gated)
        onesweep_kernel<BITS, THREADS, ITEMS, W, true, true><<<grid, THREADS, sh, s>>>(
            src, ok, ov, plan.n, (u32)shift, mask, bstart + p * RADIX, st, counters + p);
      else
        onesweep_kernel<BITS, THREADS, ITEMS, W, true><<<grid, THREADS, sh, s>>>(
            src, ok, ov, plan.n, (u32)shift, mask, bstart + p * RADIX, st, counters + p);
    } else {
      const PairSource ps = gated_source(plain_source(in_k, in_v, plan.n), src.gate, src.gate_run);
      if (gated)
        onesweep_kernel<BITS, THREADS, ITEMS, W, false, true><<<grid, THREADS, sh, s>>>(
            ps, ok, ov, plan.n, (u32)shift, mask, bstart + p * RADIX, st, counters + p);
      else
        onesweep_kernel<BITS, THREADS, ITEMS, W, false><<<grid, THREADS, sh, s>>>(
            ps, ok, ov, plan.n, (u32)shift, mask, bstart + p * RADIX, st, counters + p);
    }
    count_launch();
    in_k = ok;
    in_v = ov;
  }
  return launch_status();
}

}  // namespace

}  // namespace lnt

#include "lnt_tuned.h"

namespace lnt {

namespace {
template <int THREADS, int ITEMS, int W, int BITS = 8>
int launch_pass8(const PairSource& src, bool first, u64* out_k, double* out_v, u32 n, u32 shift, u32 mask,
                 const u32* bstart, u32* status, u32* tile_counter, cudaStream_t s) {
  using Sh = OnesweepShape<BITS, THREADS, ITEMS>;
  static_assert(Sh::TILE >= kOnesweepPassTile, "the look-back array is sized for kOnesweepPassTile-pair tiles");
  constexpr size_t sh = Sh::smem;
  auto k = first ? onesweep_kernel<BITS, THREADS, ITEMS, W, true> : onesweep_kernel<BITS, THREADS, ITEMS, W, false>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh) != cudaSuccess)
    return LNT_DEVICE_ERROR;
  const u32 ntiles = (n + Sh::TILE - 1) / Sh::TILE;
  ProfScope prof("sort_onesweep", s);
  k<<<ntiles, THREADS, sh, s>>>(src, out_k, out_v, n, shift, mask, bstart, status, tile_counter);
  count_launch();
  return launch_status();
}
}  // namespace

// Shape of the bucketed path's digit pass: 0 (256 threads x 16 keys, window 16), 1 (window 32),
// 2 (512 x 8), 3 (384 x 12); the tuned choice, or LNT_PASS8_VARIANT from the environment.
int run_onesweep_pass8(const PairSource& src, bool first, u64* out_k, double* out_v, u32 n, u32 shift, u32 mask,
                       const u32* bstart, u32* status, u32* tile_counter, cudaStream_t s) {
  int v = kTunedPass8Variant;
  if (const char* e = getenv("LNT_PASS8_VARIANT")) v = atoi(e);
  switch (v) {
    case 1:
      return launch_pass8<256, 16, 32>(src, first, out_k, out_v, n, shift, mask, bstart, status, tile_counter, s);
    case 2:
      return launch_pass8<512, 8, 16>(src, first, out_k, out_v, n, shift, mask, bstart, status, tile_counter, s);
    case 3:
      return launch_pass8<384, 12, 16>(src, first, out_k, out_v, n, shift, mask, bstart, status, tile_counter, s);
    default:
      // a 7-bit digit (the first pass of 2^15 buckets) on a 128-digit kernel:
      // seven ballots per key and half the counters, scans and look-back
      // (1.49 -> 1.42 ms for that pass over 2^27 pairs)
      if (mask == 0x7Fu)
        return launch_pass8<256, 16, 16, 7>(src, first, out_k, out_v, n, shift, mask, bstart, status, tile_counter,
                                            s);
      return launch_pass8<256, 16, 16>(src, first, out_k, out_v, n, shift, mask, bstart, status, tile_counter, s);
  }
}

int sort_variant_count() { return kNumVariants; }
const SortVariant& sort_variant(int i) { return kVariants[i]; }

int choose_sort_variant(size_t n, int key_bits) {
  if (const char* e = getenv("LNT_SORT_VARIANT")) {
    const int v = atoi(e);
    if (v >= 0 && v < kNumVariants) return v;
  }
  // tuned table: first entry whose key-width and size ranges contain the request
  for (const TunedSortEntry& t : kTunedSort) {
    if (key_bits <= t.key_bits_max && n <= t.n_max && t.variant >= 0 && t.variant < kNumVariants)
      return t.variant;
  }
  // untuned default: fewest passes, then the narrower digit
  int best = 0, best_passes = 1 << 20;
  for (int i = 0; i < kNumVariants; ++i) {
    const int p = key_bits <= 0 ? 0 : (key_bits + kVariants[i].bits - 1) / kVariants[i].bits;
    if (p < best_passes) {
      best = i;
      best_passes = p;
    }
  }
  return best;
}

SortPlan make_sort_plan(size_t n, u64 max_key, int variant) {
  SortPlan p;
  p.key_bits = key_bits_for(max_key);
  p.variant = variant >= 0 && variant < kNumVariants ? variant : choose_sort_variant(n, p.key_bits);
  const SortVariant& v = kVariants[p.variant];
  p.bits = v.bits;
  p.passes = p.key_bits == 0 ? 0 : (p.key_bits + v.bits - 1) / v.bits;
  p.n = (u32)n;
  p.tile = (u32)(v.threads * v.items);
  p.ntiles = (u32)((n + p.tile - 1) / p.tile);
  const size_t radix = (size_t)1 << v.bits;
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
    const int blocks = std::max(1, std::min((int)((plan.n + 255) / 256), sm_count() * 8));
    ProfScope prof("sort_copy", s);
    copy_source_kernel<<<blocks, 256, 0, s>>>(src, buf0_k, buf0_v, plan.n);
    count_launch();
    return launch_status();
  }
  int i = 0;
#define LNT_SV_CASE(B, T, I, W)                                                          \
  if (plan.variant == i) return run_sort_variant<B, T, I, W>(plan, src, buf0_k, buf0_v, \
                                                             buf1_k, buf1_v, ctrl, s);   \
  ++i;
  LNT_SORT_VARIANTS(LNT_SV_CASE)
#undef LNT_SV_CASE
  return LNT_UNSUPPORTED;
}

}  // namespace lnt

using namespace lnt;

namespace {
// Workspace of lnt_sort_pairs: [ctrl | tmp keys | tmp vals | tmp2 keys | tmp2 vals].
struct SortPairsLayout {
  SortPlan plan;
  size_t off_tk, off_tv, off_t2k, off_t2v, total;
};

SortPairsLayout sort_pairs_layout(size_t n, u64 max_key) {
  SortPairsLayout L;
  L.plan = make_sort_plan(n, max_key);
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

int lnt_sort_variant_count(void) { return sort_variant_count(); }

int lnt_sort_variant(int index, int* bits, int* threads, int* items, int* window) {
  if (index < 0 || index >= sort_variant_count() || !bits || !threads || !items || !window) return LNT_BAD_ARG;
  const SortVariant& v = sort_variant(index);
  *bits = v.bits;
  *threads = v.threads;
  *items = v.items;
  *window = v.window;
  return LNT_OK;
}

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
  const bool inplace =
      (const void*)keys_in == (const void*)keys_out || (const void*)vals_in == (const void*)vals_out;
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
