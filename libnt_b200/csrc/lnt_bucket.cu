// Bucketed sort + duplicate collection, the fast path of lnt_sort_reduce for
// wide keys and many pairs (the sparse merge under permutation):
//
//   1. bucket_hist_kernel: one read of all (re-keyed, concatenated) keys
//      counts the 2^T buckets given by the top T key bits (T <= 15; 16-bit
//      counts in shared memory, two CTAs per SM); the last CTA derives the
//      bucket starts, the maximum bucket size and the digit histograms of the
//      two passes below.
//   2. two stable one-sweep passes on the top T bits (T-8 bits, then 8 bits)
//      group the pairs by bucket; the first reads through the PairSource
//      (re-key + concatenation fused);
//   3. bucket_sort_collect_kernel: one CTA per bucket (at most 5120 pairs)
//      sorts the remaining low bits entirely in shared memory: packed (low
//      key << 13 | local index) words are counted into 4096 sub-buckets,
//      placed, and ranked within their sub-bucket (7-bit local LSD passes
//      instead when a sub-bucket holds more than 32 words); values stay put
//      and are gathered once.  It folds runs of equal keys (equal keys share
//      their bucket) with the collect_duplicates rule, takes its output offset
//      by decoupled look-back over buckets and writes the result once.
// DRAM traffic: 8 B (histogram) + 2 x 32 B (passes) + 16 B + 16 B per pair
// = 104 B/pair, against 8 + 5 x 32 + 32 = 200 B/pair for five LSD passes
// plus a separate collect over 36-bit keys.  The order within equal keys is
// the input order (every step is stable), as on the LSD path.
#include <algorithm>
#include <cstdlib>

#include "lnt_sort.cuh"
#include "lnt_tuned.h"

namespace lnt {
namespace {

constexpr int kHistThreads = 1024;
// Bucket geometries (the bucket kernel's CTA size, pairs per thread, bits of
// the local index field and of the counting pass).  Large: 2^(lg n - 12)
// buckets of about 4096 pairs (at most 5120), 512-thread CTAs.  Small:
// 2^(lg n - 11) buckets of about 2048 pairs (at most 2560), 256-thread CTAs,
// more of them resident per SM.
template <int BT, int ITEMS, int IDXB, int SUBB>
struct BucketGeom {
  static constexpr int kBT = BT;
  static constexpr int kBWarps = BT / 32;
  static constexpr int kBItems = ITEMS;
  static constexpr int kBCap = BT * ITEMS;
  static constexpr int kIdxBits = IDXB;  // kBCap <= 2^IDXB
  static constexpr int kSubBits = SUBB;
  static constexpr int kSlots = kBCap + kBCap / 32;
  static constexpr int kMinBlocks = BT >= 512 ? 2 : 4;
};
using GeomLarge = BucketGeom<512, 10, 13, 12>;
using GeomSmall = BucketGeom<256, 10, 12, 11>;
constexpr int kLBits = 7;                // bits per local pass
constexpr int kLRadix = 1 << kLBits;
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagPre = 2ull << 62;
constexpr unsigned long long kFlagMask = 3ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1ull;

struct BucketCtrl {
  u32* counts;       // 2^T
  u32* start;        // 2^T + 1
  u32* bstart_a;     // 256
  u32* bstart_b;     // 256
  u32* digits_a;     // 256: pass A digit counts
  u32* digits_b;     // 256: pass B digit counts
  u32* misc;         // [0] max bucket, [1] hist done, [2] pass A tiles, [3] pass B tiles, [4] bucket counter
  u32* status_a;     // ntiles x 256
  u32* status_b;     // ntiles x 256
  unsigned long long* bstatus;  // 2^T
  u32* gate;         // written by the histogram: 0 = every bucket fits a CTA, 1 = take the LSD path
};

// Bucket counts in shared memory as 16-bit fields (two per word, 2^T / 2
// words: 64 KB at T = 15, so two 1024-thread CTAs fit per SM).  A field keeps
// 15 bits; the increment that takes it to 2^15 moves 2^15 to the bucket's
// global count and clears bit 15 again, so no field carries into its
// neighbour (the other increments that can land in between are far fewer
// than 2^15).
__device__ __forceinline__ void count16(u32* sh, u32 b, const BucketCtrl& c, int TA) {
  const u32 sh_bits = 16u * (b & 1u);
  const u32 old = atomicAdd(&sh[b >> 1], 1u << sh_bits);
  if (((old >> sh_bits) & 0x7FFFu) == 0x7FFFu) {  // rare: once per 2^15 keys of one bucket in one CTA
    atomicSub(&sh[b >> 1], 0x8000u << sh_bits);
    atomicAdd(&c.counts[b], 0x8000u);
    atomicAdd(&c.digits_a[b & ((1u << TA) - 1u)], 0x8000u);
    atomicAdd(&c.digits_b[b >> TA], 0x8000u);
  }
}

__global__ void __launch_bounds__(kHistThreads, 2) bucket_hist_kernel(const PairSource src, u32 n, int T, int low_bits,
                                                                   u32 cap, BucketCtrl c) {
  extern __shared__ u32 sh[];  // 2^T 16-bit fields
  __shared__ u32 s_ha[256], s_hb[256];
  const int nb = 1 << T, nw = nb >> 1;
  const int TA = T - 8;
  for (int i = threadIdx.x; i < nw; i += kHistThreads) sh[i] = 0;
  if (threadIdx.x < 256) s_ha[threadIdx.x] = s_hb[threadIdx.x] = 0;
  __syncthreads();
  const u32 stride = gridDim.x * kHistThreads;
  const u32 bmask = (u32)(nb - 1);
  constexpr int U = 8;
  u32 i = blockIdx.x * kHistThreads + threadIdx.x;
  for (; i + (U - 1) * stride < n; i += U * stride) {
    u64 k[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const size_t x = i + u * stride;
      k[u] = x < src.na ? rekey(__ldcs(src.ak + x), src.ra) : rekey(__ldcs(src.bk + (x - src.na)), src.rb);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) count16(sh, (u32)(k[u] >> low_bits) & bmask, c, TA);
  }
  for (; i < n; i += stride) {
    const u64 k = i < src.na ? rekey(__ldcs(src.ak + i), src.ra) : rekey(__ldcs(src.bk + (i - src.na)), src.rb);
    count16(sh, (u32)(k >> low_bits) & bmask, c, TA);
  }
  __syncthreads();
  // flush: bucket counts, and this CTA's share of the two passes' digit counts
  // (pass A digit = bucket & (2^TA - 1), pass B digit = bucket >> TA)
  for (int b = threadIdx.x; b < nb; b += kHistThreads) {
    const u32 v = (sh[b >> 1] >> (16 * (b & 1))) & 0xFFFFu;
    if (v) {
      atomicAdd(&c.counts[b], v);
      atomicAdd(&s_ha[b & ((1 << TA) - 1)], v);
      atomicAdd(&s_hb[b >> TA], v);
    }
  }
  __syncthreads();
  if (threadIdx.x < 256) {
    if (s_ha[threadIdx.x]) atomicAdd(&c.digits_a[threadIdx.x], s_ha[threadIdx.x]);
    if (s_hb[threadIdx.x]) atomicAdd(&c.digits_b[threadIdx.x], s_hb[threadIdx.x]);
  }
  __threadfence();
  __syncthreads();
  __shared__ bool s_last;
  if (threadIdx.x == 0) s_last = atomicAdd(&c.misc[1], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // ---- last CTA: bucket starts, maximum, the two passes' digit starts ----
  __shared__ u32 s_w[kHistThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (nb + kHistThreads - 1) / kHistThreads;
  u32 local = 0, mx = 0;
  for (int j = 0; j < per; ++j) {
    const int b = tid * per + j;
    const u32 v = b < nb ? __ldcg(&c.counts[b]) : 0u;
    local += v;
    mx = max(mx, v);
  }
  u32 inc = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  u32 run = inc - local;
  for (int w = 0; w < warp; ++w) run += s_w[w];
  for (int j = 0; j < per; ++j) {
    const int b = tid * per + j;
    if (b < nb) {
      c.start[b] = run;
      run += __ldcg(&c.counts[b]);
    }
  }
  if (tid == kHistThreads - 1) c.start[nb] = run;  // total
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __syncthreads();
  if (lane == 0) s_w[warp] = mx;
  __syncthreads();
  if (tid == 0) {
    u32 m = 0;
    for (int w = 0; w < kHistThreads / 32; ++w) m = max(m, s_w[w]);
    c.misc[0] = m;
    *c.gate = m > cap ? 1u : 0u;
  }
  // digit counts of the two passes (flushed shares and overflow moves)
  if (tid < 256) {
    s_ha[tid] = __ldcg(&c.digits_a[tid]);
    s_hb[tid] = __ldcg(&c.digits_b[tid]);
  }
  __syncthreads();
  if (tid == 0) {
    u32 ra = 0, rb = 0;
    for (int d = 0; d < 256; ++d) {
      c.bstart_a[d] = ra;
      ra += d < (1 << TA) ? s_ha[d] : 0u;
      c.bstart_b[d] = rb;
      rb += s_hb[d];
    }
  }
}

// Lanes of the warp holding the same 7-bit digit: seven ballots, or the
// hardware match instruction.
template <bool HW_MATCH>
__device__ __forceinline__ u32 match7(u32 d) {
  if (HW_MATCH) return __match_any_sync(0xffffffffu, d);
  u32 peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < kLBits; ++b) {
    const u32 bit = (d >> b) & 1u;
    const u32 m = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? m : ~m;
  }
  return peers;
}

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

// Shared-memory slot of bucket position p: one spare word per 32 keeps
// blocked (stride-kBItems) accesses free of bank conflicts.
__device__ __forceinline__ u32 slot(u32 p) { return p + (p >> 5); }

constexpr int kSubMax = 32;               // largest sub-bucket ranked by counting

template <class G>
constexpr size_t bucket_smem_bytes() {
  return (size_t)G::kSlots * 8 * 2 + (size_t)G::kBWarps * kLRadix * 4 + ((size_t)1 << G::kSubBits) * 4 + 256;
}

template <class G, bool HW_MATCH>
__global__ void __launch_bounds__(G::kBT, G::kMinBlocks) bucket_sort_collect_kernel(
    const u64* __restrict__ keys, const double* __restrict__ vals, BucketCtrl c, int T, int low_bits,
    int local_passes, int skip_zero_heads, u64* __restrict__ out_k, double* __restrict__ out_v,
    u64* __restrict__ d_nout) {
  if (gated_off(c.gate, 0)) return;  // a bucket is too large: the LSD path runs instead
  constexpr int kBT = G::kBT, kBWarps = G::kBWarps, kBItems = G::kBItems, kIdxBits = G::kIdxBits;
  constexpr int kSubBits = G::kSubBits, kSlots = G::kSlots;
  extern __shared__ __align__(16) unsigned char smem[];
  u64* s_x = reinterpret_cast<u64*>(smem);                       // kSlots packed words
  double* s_v = reinterpret_cast<double*>(s_x + kSlots);         // kSlots values (input order)
  u32* s_whist = reinterpret_cast<u32*>(s_v + kSlots);           // kBWarps x kLRadix
  u32* s_sub = s_whist + kBWarps * kLRadix;                      // 2^kSubBits
  u32* s_misc = s_sub + (1 << kSubBits);                         // 32
  unsigned long long* s_off = reinterpret_cast<unsigned long long*>(s_misc + 32);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32 nb = 1u << T;
  const int sb_bits = min(low_bits, kSubBits);
  const int nsb = 1 << sb_bits;
  const int sb_shift = kIdxBits + low_bits - sb_bits;
  if (tid == 0) s_misc[0] = atomicAdd(&c.misc[4], 1u);
  for (int x = tid; x < kBWarps * kLRadix; x += kBT) s_whist[x] = 0;
  for (int x = tid; x < nsb; x += kBT) s_sub[x] = 0;  // counting pass below
  __syncthreads();
  const u32 b = s_misc[0];
  const u32 start = c.start[b];
  const u32 cnt = c.start[b + 1] - start;  // <= G::kBCap (the gate is open)
  const u64 lowmask = (1ull << low_bits) - 1ull;
  const u32 warp_base = warp * kBItems * 32;

  // ---- load: packed (low key << 13 | local index); the values go to shared
  // memory by asynchronous copies that complete while the keys are sorted ----
#pragma unroll
  for (int i = 0; i < kBItems; ++i) {
    const u32 p = warp_base + i * 32 + lane;
    if (p < cnt) cp_async8(&s_v[slot(p)], vals + start + p);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  u64 w[kBItems];
#pragma unroll
  for (int i = 0; i < kBItems; ++i) {
    const u32 p = warp_base + i * 32 + lane;
    w[i] = p < cnt ? ((__ldcs(keys + start + p) & lowmask) << kIdxBits) | p : 0ull;
  }

  // ---- counting pass over the top sub-bucket bits ----------------------------
  // Shared atomics hand out a slot inside each sub-bucket; a block scan of the
  // sub-bucket counts places every word; each word then finds its rank among
  // the (few) words of its sub-bucket by the whole packed word, i.e. by key
  // and then by input index, so the result is the stable order.
  u32 rnk[kBItems];
#pragma unroll
  for (int i = 0; i < kBItems; ++i) {
    const u32 p = warp_base + i * 32 + lane;
    rnk[i] = p < cnt ? atomicAdd(&s_sub[(u32)(w[i] >> sb_shift) & (u32)(nsb - 1)], 1u) : 0u;
  }
  __syncthreads();
  {  // exclusive scan of the sub-bucket counts in place; largest count to s_misc[1]
    const int per = (nsb + kBT - 1) / kBT;
    u32 loc[(1 << kSubBits) / kBT];
    u32 sum = 0, mx = 0;
#pragma unroll
    for (int j = 0; j < (1 << kSubBits) / kBT; ++j) {
      const int x = tid * per + j;
      loc[j] = (j < per && x < nsb) ? s_sub[x] : 0u;
      sum += loc[j];
      mx = max(mx, loc[j]);
    }
    u32 inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 31) s_misc[8 + warp] = inc;
    if (lane == 0) s_misc[40 + warp] = mx;
    __syncthreads();
    u32 run = inc - sum;
    for (int ww = 0; ww < warp; ++ww) run += s_misc[8 + ww];
#pragma unroll
    for (int j = 0; j < (1 << kSubBits) / kBT; ++j) {
      const int x = tid * per + j;
      if (j < per && x < nsb) {
        s_sub[x] = run;
        run += loc[j];
      }
    }
    if (tid == 0) {
      u32 m = 0;
      for (int ww = 0; ww < kBWarps; ++ww) m = max(m, s_misc[40 + ww]);
      s_misc[1] = m;
    }
    __syncthreads();
  }
  const bool small_subs = s_misc[1] <= (u32)kSubMax;
  if (small_subs) {
    // place each word in its sub-bucket, then rank it among the (few) words of
    // its sub-bucket: every thread ranks its own words, with no serial pass
#pragma unroll
    for (int i = 0; i < kBItems; ++i) {
      const u32 p = warp_base + i * 32 + lane;
      if (p < cnt) s_x[slot(s_sub[(u32)(w[i] >> sb_shift) & (u32)(nsb - 1)] + rnk[i])] = w[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kBItems; ++i) {  // rnk[i] becomes the final position, or ~0 if already there
      const u32 p = warp_base + i * 32 + lane;
      u32 fin = ~0u;
      if (p < cnt) {
        const u32 sb = (u32)(w[i] >> sb_shift) & (u32)(nsb - 1);
        const u32 lo = s_sub[sb], hi = sb + 1 < (u32)nsb ? s_sub[sb + 1] : cnt;
        if (hi - lo > 1) {
          u32 r = 0;
          for (u32 q = lo; q < hi; ++q) r += s_x[slot(q)] < w[i] ? 1u : 0u;
          fin = lo + r;
        }
      }
      rnk[i] = fin;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kBItems; ++i)
      if (rnk[i] != ~0u) s_x[slot(rnk[i])] = w[i];
    asm volatile("cp.async.wait_all;\n" ::: "memory");  // this thread's value copies have landed
    __syncthreads();                                    // ... and everyone's, for the fold
  } else {
  // ---- clustered keys: local LSD passes over the low bits -----------------------
  const u32 lt_mask = (1u << lane) - 1u;
  for (int q = 0; q < local_passes; ++q) {
    const int shift = kIdxBits + q * kLBits;
#pragma unroll
    for (int i = 0; i < kBItems; ++i) {
      const u32 p = warp_base + i * 32 + lane;
      if (p < cnt) atomicAdd(&s_whist[warp * kLRadix + ((u32)(w[i] >> shift) & (kLRadix - 1))], 1u);
    }
    __syncthreads();
    if (tid < kLRadix) {  // per digit: total, exclusive scan over digits (4 warps), per-warp bases
      u32 cc[kBWarps];
      u32 v = 0;
#pragma unroll
      for (int ww = 0; ww < kBWarps; ++ww) {
        cc[ww] = s_whist[ww * kLRadix + tid];
        v += cc[ww];
      }
      u32 inc = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
      }
      if (lane == 31) s_misc[8 + warp] = inc;
      asm volatile("bar.sync 1, 128;" ::: "memory");  // the 4 warps holding digits
      u32 base = inc - v;
      for (int ww = 0; ww < warp; ++ww) base += s_misc[8 + ww];
#pragma unroll
      for (int ww = 0; ww < kBWarps; ++ww) {
        s_whist[ww * kLRadix + tid] = base;
        base += cc[ww];
      }
    }
    __syncthreads();
    u32 pos[kBItems];
#pragma unroll
    for (int i = 0; i < kBItems; ++i) {
      const u32 p = warp_base + i * 32 + lane;
      const bool valid = p < cnt;
      const u32 vmask = __ballot_sync(0xffffffffu, valid);
      const u32 d = valid ? ((u32)(w[i] >> shift) & (kLRadix - 1)) : 0u;
      const u32 peers = match7<HW_MATCH>(d) & vmask;
      u32 base = 0;
      if (valid) base = s_whist[warp * kLRadix + d];
      __syncwarp();
      if (valid && lane == __ffs(peers) - 1) s_whist[warp * kLRadix + d] = base + __popc(peers);
      __syncwarp();
      pos[i] = base + __popc(peers & lt_mask);
    }
#pragma unroll
    for (int i = 0; i < kBItems; ++i) {
      const u32 p = warp_base + i * 32 + lane;
      if (p < cnt) s_x[slot(pos[i])] = w[i];
    }
    if (q + 1 == local_passes) asm volatile("cp.async.wait_all;\n" ::: "memory");  // values, for the fold
    __syncthreads();
    if (q + 1 < local_passes) {
#pragma unroll
      for (int i = 0; i < kBItems; ++i) {
        const u32 p = warp_base + i * 32 + lane;
        if (p < cnt) w[i] = s_x[slot(p)];
      }
      for (int x = tid; x < kBWarps * kLRadix; x += kBT) s_whist[x] = 0;
      __syncthreads();
    }
  }
  }  // clustered keys

  // ---- fold runs of equal keys (they all lie in this bucket) ------------------
  const u64 prefix = (u64)b << low_bits;
  u64 rk[kBItems];
  double rs[kBItems];
  u32 kept_mask = 0;
#pragma unroll
  for (int j = 0; j < kBItems; ++j) {
    const u32 p = tid * kBItems + j;
    rk[j] = 0;
    rs[j] = 0.0;
    if (p >= cnt) continue;
    const u64 word = s_x[slot(p)];
    const u64 low = word >> kIdxBits;
    if (p > 0 && (s_x[slot(p - 1)] >> kIdxBits) == low) continue;  // not the first of its run
    double sum = s_v[slot((u32)(word & ((1u << kIdxBits) - 1)))];
    bool anynz = sum != 0.0;
    for (u32 m = p + 1; m < cnt; ++m) {
      const u64 wm = s_x[slot(m)];
      if ((wm >> kIdxBits) != low) break;
      const double x = s_v[slot((u32)(wm & ((1u << kIdxBits) - 1)))];
      sum += x;
      anynz |= (x != 0.0);
    }
    const bool kept = !skip_zero_heads || anynz || (start == 0 && p == 0);
    if (kept) {
      kept_mask |= 1u << j;
      rk[j] = prefix | low;
      rs[j] = sum;
    }
  }
  const u32 local = __popc(kept_mask);
  u32 inc = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_misc[16 + warp] = inc;
  __syncthreads();
  u32 excl = inc - local, total = 0;
  for (int ww = 0; ww < kBWarps; ++ww) {
    if (ww < warp) excl += s_misc[16 + ww];
    total += s_misc[16 + ww];
  }
  // ---- output offset: decoupled look-back over buckets (warp 0) --------------
  if (warp == 0) {
    if (lane == 0)
      *reinterpret_cast<volatile unsigned long long*>(&c.bstatus[b]) = (b == 0 ? kFlagPre : kFlagAgg) | total;
    unsigned long long off = 0;
    if (b != 0) {
      int base = (int)b - 1;
      u32 spins = 0;
      while (base >= 0) {
        const int p = base - lane;
        const unsigned long long wv =
            p >= 0 ? *reinterpret_cast<const volatile unsigned long long*>(&c.bstatus[p]) : kFlagPre;
        const unsigned long long f = wv & kFlagMask;
        const u32 notready = __ballot_sync(0xffffffffu, f == 0);
        const u32 pre = __ballot_sync(0xffffffffu, f == kFlagPre);
        const int first_nr = notready ? __ffs(notready) - 1 : 32;
        const int first_pre = pre ? __ffs(pre) - 1 : 32;
        const int take = first_pre < first_nr ? first_pre + 1 : first_nr;
        unsigned long long v = lane < take ? (wv & kValMask) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        off += v;
        if (first_pre < first_nr) break;
        base -= first_nr;
        if (first_nr < 32 && ++spins > spin_limit()) {
          latch_error(kErrReduceLookback);
          break;
        }
      }
      if (lane == 0) *reinterpret_cast<volatile unsigned long long*>(&c.bstatus[b]) = kFlagPre | (off + total);
    }
    if (lane == 0) {
      *s_off = off;
      if (b == nb - 1) *d_nout = off + total;
    }
  }
  __syncthreads();  // all reads of s_x / s_v are done
  u32 r = excl;
#pragma unroll
  for (int j = 0; j < kBItems; ++j) {
    if (kept_mask & (1u << j)) {
      s_x[r] = rk[j];
      s_v[r] = rs[j];
      ++r;
    }
  }
  __syncthreads();
  const unsigned long long off = *s_off;
  for (u32 x = tid; x < total; x += kBT) {
    __stcs(out_k + off + x, s_x[x]);
    __stcs(out_v + off + x, s_v[x]);
  }
}

// Geometry of the bucketed path: the small one when LNT_BUCKET_SMALL=1 is set
// in the environment, else the tuned choice.
bool small_geometry() {
  if (const char* e = getenv("LNT_BUCKET_SMALL")) return atoi(e) != 0;
  return kTunedBucketSmall != 0;
}

// Bucket bits for n pairs: ceil(log2 n) - 12 (large geometry), so that the
// average bucket holds between 2048 and 4096 pairs, below the CTA capacity
// (5120); rounding log2 n down would put n = 3 x 2^25 at 6144 per bucket and
// send every such call to the LSD path.
int bucket_bits_for(u32 n, bool small) {
  int lg = 0;
  while (lg < 31 && (1u << lg) < n) ++lg;  // ceil(log2 n)
  return small ? std::max(9, std::min(16, lg - 11))   // 1024..2048 pairs per bucket
               : std::max(9, std::min(15, lg - 12));  // 2048..4096 pairs per bucket
}

struct BucketLayout {
  int T;
  u32 ntiles;
  size_t off_counts, off_start, off_ba, off_bb, off_da, off_db, off_misc, off_sa, off_sb, off_bstatus, total;
};

BucketLayout bucket_layout(u32 n, bool small) {
  BucketLayout L;
  L.T = bucket_bits_for(n, small);
  const size_t nb = (size_t)1 << L.T;
  L.ntiles = (n + kOnesweepPassTile - 1) / kOnesweepPassTile;
  size_t off = 0;
  L.off_counts = off;
  off += align_up(nb * 4, 256);
  L.off_start = off;
  off += align_up((nb + 1) * 4, 256);
  L.off_ba = off;
  off += 1024;
  L.off_bb = off;
  off += 1024;
  L.off_da = off;
  off += 1024;
  L.off_db = off;
  off += 1024;
  L.off_misc = off;
  off += 256;
  L.off_sa = off;
  off += align_up((size_t)L.ntiles * 256 * 4, 256);
  L.off_sb = off;
  off += align_up((size_t)L.ntiles * 256 * 4, 256);
  L.off_bstatus = off;
  off += align_up(nb * 8, 256);
  L.total = off;
  return L;
}

template <class G>
int launch_bucket_sort_collect(const u64* k0, const double* v0, const BucketCtrl& c, int T, int low,
                               int skip_zero_heads, u64* out_k, double* out_v, u64* d_nout, cudaStream_t s) {
  constexpr size_t sh = bucket_smem_bytes<G>();
  const int local_passes = (low + kLBits - 1) / kLBits;
  const bool hw = getenv("LNT_BUCKET_HWMATCH") != nullptr;
  auto kern = hw ? bucket_sort_collect_kernel<G, true> : bucket_sort_collect_kernel<G, false>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh) != cudaSuccess)
    return LNT_DEVICE_ERROR;
  ProfScope prof("bucket_sort_collect", s);
  kern<<<1u << T, G::kBT, sh, s>>>(k0, v0, c, T, low, local_passes, skip_zero_heads, out_k, out_v, d_nout);
  count_launch();
  return launch_status();
}

}  // namespace

// Scratch for either geometry (the choice can change between the workspace
// query and the call through the environment).
size_t bucket_ctrl_bytes(size_t n) {
  return std::max(bucket_layout((u32)n, false).total, bucket_layout((u32)n, true).total);
}

bool bucket_path_applies(size_t n, int key_bits) {
  if (n < (1u << 20) || n >= (1u << 30)) return false;
  const int T = bucket_bits_for((u32)n, small_geometry());
  const int low = key_bits - T;
  return low >= 0 && low <= 4 * kLBits && key_bits > T;  // at most four local passes (41-bit packed words)
}

// Buffers: (k1, v1) and (k0, v0), n pairs each.  The kernels after the
// histogram are gated on *gate == 0 (every bucket fits a CTA); the caller
// enqueues the LSD path gated on *gate == 1.
int run_bucketed_sort_reduce(const PairSource& src, u32 n, int key_bits, int skip_zero_heads, u64* k0, double* v0,
                             u64* k1, double* v1, void* ctrl, u64* out_k, double* out_v, u64* d_nout, u32* gate,
                             cudaStream_t s) {
  const bool small = small_geometry();
  const BucketLayout L = bucket_layout(n, small);
  const int T = L.T, TA = T - 8, low = key_bits - T;
  const u32 cap = small ? (u32)GeomSmall::kBCap : (u32)GeomLarge::kBCap;
  unsigned char* w = static_cast<unsigned char*>(ctrl);
  BucketCtrl c;
  c.counts = reinterpret_cast<u32*>(w + L.off_counts);
  c.start = reinterpret_cast<u32*>(w + L.off_start);
  c.bstart_a = reinterpret_cast<u32*>(w + L.off_ba);
  c.bstart_b = reinterpret_cast<u32*>(w + L.off_bb);
  c.digits_a = reinterpret_cast<u32*>(w + L.off_da);
  c.digits_b = reinterpret_cast<u32*>(w + L.off_db);
  c.misc = reinterpret_cast<u32*>(w + L.off_misc);
  c.status_a = reinterpret_cast<u32*>(w + L.off_sa);
  c.status_b = reinterpret_cast<u32*>(w + L.off_sb);
  c.bstatus = reinterpret_cast<unsigned long long*>(w + L.off_bstatus);
  c.gate = gate;
  if (cudaMemsetAsync(ctrl, 0, L.total, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  {
    const size_t sh = ((size_t)1 << T) * 2;  // 16-bit fields
    if (cudaFuncSetAttribute(bucket_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh) != cudaSuccess)
      return LNT_DEVICE_ERROR;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bucket_hist_kernel, kHistThreads, sh) != cudaSuccess)
      return LNT_DEVICE_ERROR;
    ProfScope prof("sort_hist", s);
    bucket_hist_kernel<<<std::max(per_sm, 1) * sm_count(), kHistThreads, sh, s>>>(src, n, T, low, cap, c);
    count_launch();
  }
  // the bucket-size decision stays on the device: the passes below return at
  // once when the histogram found a bucket above the CTA capacity (skewed keys)
  int st = run_onesweep_pass8(gated_source(src, gate, 0), true, k1, v1, n, (u32)low, (1u << TA) - 1u, c.bstart_a,
                              c.status_a, c.misc + 2, s);
  if (st != LNT_OK) return st;
  st = run_onesweep_pass8(gated_source(plain_source(k1, v1, n), gate, 0), false, k0, v0, n, (u32)(low + TA), 0xFFu,
                          c.bstart_b, c.status_b, c.misc + 3, s);
  if (st != LNT_OK) return st;
  return small ? launch_bucket_sort_collect<GeomSmall>(k0, v0, c, T, low, skip_zero_heads, out_k, out_v, d_nout, s)
               : launch_bucket_sort_collect<GeomLarge>(k0, v0, c, T, low, skip_zero_heads, out_k, out_v, d_nout, s);
}

}  // namespace lnt
