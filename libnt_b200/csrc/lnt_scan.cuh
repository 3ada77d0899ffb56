// Device-wide exclusive prefix sum of n 64-bit counts produced by a functor,
// single pass: tiles of 2048 values, block scan, warp-cooperative decoupled
// look-back (32 predecessor tiles per round trip).  out[i] = sum of get(j),
// j < i, for i in [0, n]; out[n] (the total) is also written to *d_total.
#pragma once

#include "lnt_common.cuh"

namespace lnt {
namespace scan {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagPre = 2ull << 62;
constexpr unsigned long long kFlagMask = 3ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1ull;

// Exclusive prefix of `tile` over status words (called by one full warp).
__device__ __forceinline__ unsigned long long warp_lookback(const unsigned long long* status, u32 tile, u32 err) {
  const int lane = threadIdx.x & 31;
  unsigned long long excl = 0;
  int base = (int)tile - 1;
  u32 spins = 0;
  while (base >= 0) {
    const int p = base - lane;
    const unsigned long long w =
        p >= 0 ? *reinterpret_cast<const volatile unsigned long long*>(status + p) : kFlagPre;
    const unsigned long long f = w & kFlagMask;
    const u32 notready = __ballot_sync(0xffffffffu, f == 0);
    const u32 pre = __ballot_sync(0xffffffffu, f == kFlagPre);
    const int first_nr = notready ? __ffs(notready) - 1 : 32;
    const int first_pre = pre ? __ffs(pre) - 1 : 32;
    const int take = first_pre < first_nr ? first_pre + 1 : first_nr;
    unsigned long long v = lane < take ? (w & kValMask) : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    excl += v;
    if (first_pre < first_nr) break;
    base -= first_nr;
    if (first_nr < 32 && ++spins > spin_limit()) {
      latch_error(err);
      break;
    }
  }
  return excl;
}

template <class Get>
__global__ void __launch_bounds__(kThreads) scan_kernel(Get get, size_t n, unsigned long long* __restrict__ out,
                                                        unsigned long long* __restrict__ d_total, u32 ntiles,
                                                        unsigned long long* __restrict__ status,
                                                        u32* __restrict__ counter) {
  __shared__ unsigned long long s_warp[kThreads / 32];
  __shared__ u32 s_tile;
  __shared__ unsigned long long s_off;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(counter, 1u);
  __syncthreads();
  const u32 tile = s_tile;
  const size_t base = (size_t)tile * kTile + (size_t)tid * kItems;  // blocked: 8 consecutive per thread
  unsigned long long v[kItems];
  unsigned long long local = 0;
#pragma unroll
  for (int q = 0; q < kItems; ++q) {
    v[q] = base + q < n ? (unsigned long long)get(base + q) : 0ull;
    local += v[q];
  }
  unsigned long long inc = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  unsigned long long excl = inc - local, tot = 0;
  for (int w = 0; w < kThreads / 32; ++w) {
    if (w < warp) excl += s_warp[w];
    tot += s_warp[w];
  }
  if (warp == 0) {
    if (lane == 0) *reinterpret_cast<volatile unsigned long long*>(&status[tile]) = (tile == 0 ? kFlagPre : kFlagAgg) | tot;
    unsigned long long off = tile == 0 ? 0ull : warp_lookback(status, tile, kErrSpgemmLookback);
    if (lane == 0) {
      if (tile != 0) *reinterpret_cast<volatile unsigned long long*>(&status[tile]) = kFlagPre | (off + tot);
      s_off = off;
      if (tile == ntiles - 1) {
        out[n] = off + tot;
        if (d_total) *d_total = off + tot;
      }
    }
  }
  __syncthreads();
  unsigned long long run = s_off + excl;
#pragma unroll
  for (int q = 0; q < kItems; ++q) {
    if (base + q < n) out[base + q] = run;
    run += v[q];
  }
}

inline size_t workspace_bytes(size_t n) {
  const size_t ntiles = (n + kTile - 1) / kTile;
  return align_up((ntiles ? ntiles : 1) * 8, 256) + 256;
}

// out must hold n + 1 values.  ws: workspace_bytes(n) bytes (zeroed here).
template <class Get>
int run(Get get, size_t n, unsigned long long* out, unsigned long long* d_total, void* ws, cudaStream_t s,
        const char* prof_name = "scan") {
  const u32 ntiles = (u32)((n + kTile - 1) / kTile);
  if (n == 0) {
    if (cudaMemsetAsync(out, 0, 8, s) != cudaSuccess) return LNT_DEVICE_ERROR;
    if (d_total && cudaMemsetAsync(d_total, 0, 8, s) != cudaSuccess) return LNT_DEVICE_ERROR;
    return LNT_OK;
  }
  if (cudaMemsetAsync(ws, 0, workspace_bytes(n), s) != cudaSuccess) return LNT_DEVICE_ERROR;
  unsigned char* w = static_cast<unsigned char*>(ws);
  unsigned long long* status = reinterpret_cast<unsigned long long*>(w);
  u32* counter = reinterpret_cast<u32*>(w + align_up((size_t)ntiles * 8, 256));
  {
    ProfScope prof(prof_name, s);
    scan_kernel<Get><<<ntiles, kThreads, 0, s>>>(get, n, out, d_total, ntiles, status, counter);
  }
  count_launch();
  return launch_status();
}

}  // namespace scan
}  // namespace lnt
