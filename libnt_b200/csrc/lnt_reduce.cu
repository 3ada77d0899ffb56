// Duplicate collection on key-sorted pairs (segmented sum + compaction) and
// the fused sort-merge entry point.
//
// collect: two kernels over tiles of 2048 pairs.
//   lead_kernel   - one warp per tile sums the tile's leading run (the
//                   elements before the tile's first new key; a warp tree
//                   reduction per 32 elements) so a run that crosses tiles is
//                   finished from per-tile summaries instead of element by
//                   element.  Sums start from -0.0, the additive identity that
//                   keeps the sign of an all-zero run.
//   collect_kernel- stages the tile in shared memory, sums the runs with a
//                   segmented reduction (per-thread sums of 8 consecutive
//                   items, then a reverse segmented scan over the threads),
//                   counts the runs kept, takes its output offset by decoupled
//                   look-back and writes (key, sum) pairs contiguously.
// Traffic: 16 B read per input pair + 16 B written per output pair.
#include <algorithm>
#include <cstdlib>

#include "lnt_sort.cuh"

namespace lnt {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;  // 2048
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagPre = 2ull << 62;
constexpr unsigned long long kFlagMask = 3ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1ull;

struct LeadSummary {
  double sum;     // sum of the tile's leading run
  u32 anynz;      // some value in the leading run is non-zero
  u32 full;       // the whole tile is one leading run (no new key inside)
};

// Summary of tile `tile`'s leading run (one warp).
__device__ __forceinline__ void lead_summary(const u64* __restrict__ keys, const double* __restrict__ vals, size_t n,
                                             u32 tile, int lane, LeadSummary* __restrict__ lead) {
  const size_t base = (size_t)tile * kTile;
  const size_t end = min(n, base + kTile);
  LeadSummary r{0.0, 0u, 0u};
  if (base == 0) {  // tile 0 has no leading run (position 0 starts a run)
    if (lane == 0) lead[tile] = r;
    return;
  }
  const u64 prev = keys[base - 1];
  double sum = -0.0;  // -0.0 is the additive identity that keeps the sign of zero sums
  bool anynz = false;
  bool stop = false;
  for (size_t c = base; c < end; c += 32) {
    const size_t i = c + lane;
    const bool brk = (i < end) && keys[i] != prev;
    const u32 m = __ballot_sync(0xffffffffu, brk);  // lanes where a new key starts
    const int nvalid = (int)min((size_t)32, end - c);
    const int upto = m ? (__ffs(m) - 1) : nvalid;  // warp-uniform
    double v = (lane < upto) ? vals[i] : -0.0;
    anynz |= __ballot_sync(0xffffffffu, lane < upto && v != 0.0) != 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);  // the chunk's sum, every lane
    sum += v;
    if (m) {
      stop = true;
      break;
    }
  }
  if (lane == 0) {
    r.sum = sum;
    r.anynz = anynz ? 1u : 0u;
    r.full = stop ? 0u : 1u;
    lead[tile] = r;
  }
}

__global__ void __launch_bounds__(128) lead_kernel(const u64* __restrict__ keys, const double* __restrict__ vals,
                                                   size_t n, u32 ntiles, LeadSummary* __restrict__ lead,
                                                   const u32* gate, u32 want) {
  if (gated_off(gate, want)) return;
  const int lane = threadIdx.x & 31;
  for (u32 tile = blockIdx.x * 4 + (threadIdx.x >> 5); tile < ntiles; tile += gridDim.x * 4)
    lead_summary(keys, vals, n, tile, lane, lead);
}

__device__ __forceinline__ void st_volatile64(unsigned long long* p, unsigned long long v) {
  *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

// Shared-memory slot of tile element i (+1 for the predecessor key at slot 0),
// padded by one word per 8 so blocked (stride-8) reads are conflict-free.
__device__ __forceinline__ u32 pk(u32 i) { return i + (i >> 3); }
constexpr u32 kPadded = kTile + 1 + (kTile + 1) / 8 + 1;

// Warp-cooperative decoupled look-back over single-value tile states:
// lane q reads the state of tile (base - q); one round trip covers 32
// predecessors.  Returns the exclusive prefix of `tile` (all lanes).
__device__ __forceinline__ unsigned long long warp_lookback(const unsigned long long* status, u32 tile, u32 err) {
  const int lane = threadIdx.x & 31;
  unsigned long long excl = 0;
  int base = (int)tile - 1;
  u32 spins = 0;
  while (base >= 0) {
    const int p = base - lane;
    const unsigned long long w = p >= 0 ? *reinterpret_cast<const volatile unsigned long long*>(status + p)
                                        : kFlagPre;
    const unsigned long long f = w & kFlagMask;
    const u32 notready = __ballot_sync(0xffffffffu, f == 0);
    const u32 pre = __ballot_sync(0xffffffffu, f == kFlagPre);
    const int first_nr = notready ? __ffs(notready) - 1 : 32;
    const int first_pre = pre ? __ffs(pre) - 1 : 32;
    const int take = first_pre < first_nr ? first_pre + 1 : first_nr;  // lanes [0, take) contribute
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

// PERSIST: a grid smaller than the tile count whose CTAs take tiles until
// none is left (tiles are taken in order, so every predecessor a look-back
// waits on belongs to a running CTA).
template <bool PERSIST>
__global__ void __launch_bounds__(kThreads) collect_kernel(const u64* __restrict__ keys,
                                                           const double* __restrict__ vals, size_t n,
                                                           u32 ntiles, int skip_zero_heads,
                                                           const LeadSummary* __restrict__ lead,
                                                           unsigned long long* __restrict__ status,
                                                           u32* __restrict__ tile_counter,
                                                           u64* __restrict__ out_k, double* __restrict__ out_v,
                                                           u64* __restrict__ d_nout, const u32* gate, u32 want) {
  if (gated_off(gate, want)) return;
  __shared__ u64 s_k[kPadded];
  __shared__ double s_v[kPadded];
  __shared__ u32 s_warp[kThreads / 32];
  __shared__ double s_wsum[kThreads / 32];
  __shared__ bool s_wnz[kThreads / 32], s_wf[kThreads / 32];
  __shared__ double s_rsum[kThreads];
  __shared__ bool s_rnz[kThreads], s_rf[kThreads];
  __shared__ u32 s_tile;
  __shared__ unsigned long long s_off;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (;;) {
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const u32 tile = s_tile;
  if (PERSIST && tile >= ntiles) break;
  const size_t base = (size_t)tile * kTile;
  const u32 tn = (u32)min((size_t)kTile, n - base);
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    u32 idx = j * kThreads + tid;
    if (idx < tn) {
      s_k[pk(idx + 1)] = __ldcs(keys + base + idx);
      s_v[pk(idx)] = __ldcs(vals + base + idx);
    }
  }
  if (tid == 0) s_k[0] = base ? keys[base - 1] : 0ull;
  __syncthreads();

  // ---- runs: segmented sum over the tile ----------------------------------
  // Each thread sums its kItems consecutive items: a run that ends inside the
  // thread is finished here; the part before the thread's first head (its
  // "lead", L) and whether it holds a head (H) feed a reverse segmented scan
  // over the threads, R_t = L_t + (H_t ? 0 : R_{t+1}), so the thread holding
  // a run's head adds R of the next thread to the run's open tail.  A run that
  // reaches the tile end continues through the next tiles' lead summaries.
  u64 rk[kItems];
  double rs[kItems];
  u32 kept_mask = 0;
  double lead_sum = -0.0, cur = -0.0;  // -0.0: the identity that keeps the sign of zero sums
  bool lead_nz = false, cur_nz = false, seen = false;
  int cur_j = -1;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    rk[j] = 0;
    rs[j] = 0.0;
    const u32 idx = tid * kItems + j;
    if (idx >= tn) continue;
    const size_t gi = base + idx;
    const u64 k = s_k[pk(idx + 1)];
    const bool head = (gi == 0) || (k != s_k[pk(idx)]);
    const double v = s_v[pk(idx)];
    if (head) {
      if (seen && (!skip_zero_heads || base + tid * kItems + cur_j == 0 || cur_nz)) {  // a run ends here
        kept_mask |= 1u << cur_j;
        const u64 hk = s_k[pk(tid * kItems + cur_j + 1)];
#pragma unroll
        for (int q = 0; q < kItems; ++q)  // static indices keep rk / rs in registers
          if (q == cur_j) {
            rk[q] = hk;
            rs[q] = cur;
          }
      }
      seen = true;
      cur_j = j;
      cur = v;
      cur_nz = v != 0.0;
    } else if (seen) {
      cur += v;
      cur_nz |= v != 0.0;
    } else {
      lead_sum += v;
      lead_nz |= v != 0.0;
    }
  }
  {  // reverse segmented scan of (L, any non-zero in L, H) over the threads
    double rsum = lead_sum;
    bool rnz = lead_nz, rf = seen;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double s2 = __shfl_down_sync(0xffffffffu, rsum, o);
      const bool n2 = __shfl_down_sync(0xffffffffu, (int)rnz, o) != 0;
      const bool f2 = __shfl_down_sync(0xffffffffu, (int)rf, o) != 0;
      if (lane + o < 32) {
        if (!rf) {
          rsum += s2;
          rnz = rnz || n2;
        }
        rf = rf || f2;
      }
    }
    if (lane == 0) {
      s_wsum[warp] = rsum;
      s_wnz[warp] = rnz;
      s_wf[warp] = rf;
    }
    __syncthreads();
    double tsum = -0.0;  // the threads of the later warps
    bool tnz = false, tf = false;
    for (int w = kThreads / 32 - 1; w > warp; --w) {
      tsum = s_wsum[w] + (s_wf[w] ? -0.0 : tsum);
      tnz = s_wnz[w] || (!s_wf[w] && tnz);
      tf = s_wf[w] || tf;
    }
    s_rsum[tid] = rsum + (rf ? -0.0 : tsum);
    s_rnz[tid] = rnz || (!rf && tnz);
    s_rf[tid] = rf || tf;
    __syncthreads();
  }
  if (seen) {  // the run opened by this thread's last head
    double sum = cur;
    bool anynz = cur_nz;
    bool to_end = true;
    if (tid + 1 < kThreads) {
      sum += s_rsum[tid + 1];
      anynz = anynz || s_rnz[tid + 1];
      to_end = !s_rf[tid + 1];
    }
    if (to_end) {  // the run may continue into later tiles
      for (u32 u = tile + 1; u < ntiles; ++u) {
        LeadSummary L = lead[u];
        sum += L.sum;
        anynz |= (L.anynz != 0u);
        if (!L.full) break;
      }
    }
    const size_t gi = base + tid * kItems + cur_j;
    if (!skip_zero_heads || gi == 0 || anynz) {
      kept_mask |= 1u << cur_j;
      const u64 hk = s_k[pk(tid * kItems + cur_j + 1)];
#pragma unroll
      for (int q = 0; q < kItems; ++q)
        if (q == cur_j) {
          rk[q] = hk;
          rs[q] = sum;
        }
    }
  }

  // ---- block scan of kept counts -----------------------------------------
  const u32 local = __popc(kept_mask);
  u32 inc = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    u32 t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  u32 excl = inc - local;
  u32 total = 0;
  for (int w = 0; w < kThreads / 32; ++w) {
    if (w < warp) excl += s_warp[w];
    total += s_warp[w];
  }

  // ---- look-back for the tile's output offset (warp 0) --------------------
  if (warp == 0) {
    if (lane == 0)
      st_volatile64(&status[tile], (tile == 0 ? kFlagPre : kFlagAgg) | total);
    unsigned long long off = tile == 0 ? 0ull : warp_lookback(status, tile, kErrReduceLookback);
    if (lane == 0) {
      if (tile != 0) st_volatile64(&status[tile], kFlagPre | (off + total));
      s_off = off;
      if (tile == ntiles - 1) *d_nout = off + total;
    }
  }
  __syncthreads();  // everyone is done reading s_k / s_v

  // ---- stage results contiguously, then write coalesced -------------------
  u32 r = excl;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    if (kept_mask & (1u << j)) {
      s_k[r] = rk[j];
      s_v[r] = rs[j];
      ++r;
    }
  }
  __syncthreads();
  const unsigned long long off = s_off;
  for (u32 i = tid; i < total; i += kThreads) {
    __stcs(out_k + off + i, s_k[i]);
    __stcs(out_v + off + i, s_v[i]);
  }
  if (!PERSIST) break;
  __syncthreads();  // s_k / s_v / s_tile are reused by the next tile
  }
}

// Look-back states of two tiles that no kernel ever publishes (zero-initialised
// with the module).
__device__ unsigned long long g_unpublished_status[2];

// One warp of "tile 1" looks back at "tile 0", which never publishes: the
// collect kernels' look-back spins through its poll budget, latches
// kErrReduceLookback and returns.
__global__ void expired_lookback_kernel() {
  const unsigned long long off = warp_lookback(g_unpublished_status, 1u, kErrReduceLookback);
  (void)off;
}

}  // namespace

struct CollectLayout {
  u32 ntiles;
  size_t off_lead, off_status, off_counter, total;
};

static CollectLayout collect_layout(size_t n) {
  CollectLayout L;
  L.ntiles = (u32)((n + kTile - 1) / kTile);
  size_t off = 0;
  L.off_lead = off;
  off += align_up((size_t)L.ntiles * sizeof(LeadSummary), 256);
  L.off_status = off;
  off += align_up((size_t)L.ntiles * 8, 256);
  L.off_counter = off;
  off += 256;
  L.total = off;
  return L;
}

size_t collect_workspace_bytes(size_t n) { return collect_layout(n).total; }

// gate/want: see gated_off.  A gated call runs the persistent collect (a grid
// of resident CTAs), so that skipping it costs a few hundred empty CTAs.
int run_collect_gated(const u64* keys, const double* vals, size_t n, int skip_zero_heads, u64* out_k,
                      double* out_v, u64* d_nout, void* ws, cudaStream_t s, const u32* gate, u32 want) {
  if (n == 0) {
    return cudaMemsetAsync(d_nout, 0, sizeof(u64), s) == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
  }
  CollectLayout L = collect_layout(n);
  unsigned char* w = static_cast<unsigned char*>(ws);
  // status + counter are contiguous: one memset
  if (cudaMemsetAsync(w + L.off_status, 0, L.total - L.off_status, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  LeadSummary* lead = reinterpret_cast<LeadSummary*>(w + L.off_lead);
  const u32 lead_blocks = (L.ntiles + 3) / 4;
  {
    ProfScope prof(gate ? "collect_lead_fallback" : "collect_lead", s);
    lead_kernel<<<gate ? std::min(lead_blocks, (u32)sm_count() * 8u) : lead_blocks, 128, 0, s>>>(
        keys, vals, n, L.ntiles, lead, gate, want);
  }
  unsigned long long* status = reinterpret_cast<unsigned long long*>(w + L.off_status);
  u32* counter = reinterpret_cast<u32*>(w + L.off_counter);
  ProfScope prof(gate ? "collect_fallback" : "collect", s);
  if (gate) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, collect_kernel<true>, kThreads, 0) != cudaSuccess)
      return LNT_DEVICE_ERROR;
    const u32 grid = std::min(L.ntiles, (u32)(std::max(per_sm, 1) * sm_count()));
    collect_kernel<true><<<grid, kThreads, 0, s>>>(keys, vals, n, L.ntiles, skip_zero_heads, lead, status, counter,
                                                   out_k, out_v, d_nout, gate, want);
  } else {
    collect_kernel<false><<<L.ntiles, kThreads, 0, s>>>(keys, vals, n, L.ntiles, skip_zero_heads, lead, status,
                                                        counter, out_k, out_v, d_nout, nullptr, 0);
  }
  count_launch(2);
  return launch_status();
}

int run_collect(const u64* keys, const double* vals, size_t n, int skip_zero_heads, u64* out_k,
                double* out_v, u64* d_nout, void* ws, cudaStream_t s) {
  return run_collect_gated(keys, vals, n, skip_zero_heads, out_k, out_v, d_nout, ws, s, nullptr, 0);
}

}  // namespace lnt

using namespace lnt;

namespace {
struct SortReduceLayout {
  SortPlan plan;
  size_t off_ctrl, off_k0, off_v0, off_k1, off_v1, off_coll, off_gate, total;
};

SortReduceLayout sort_reduce_layout(size_t n, u64 max_key) {
  SortReduceLayout L;
  L.plan = make_sort_plan(n, max_key);
  size_t off = 0;
  L.off_ctrl = off;
  off += align_up(std::max(L.plan.ctrl_bytes, bucket_ctrl_bytes(n)), 256);
  L.off_k0 = off;
  off += align_up(n * 8, 256);
  L.off_v0 = off;
  off += align_up(n * 8, 256);
  L.off_k1 = off;
  off += align_up(n * 8, 256);
  L.off_v1 = off;
  off += align_up(n * 8, 256);
  L.off_coll = off;
  off += align_up(collect_workspace_bytes(n), 256);
  L.off_gate = off;  // the bucketed path's decision word (outside every region a memset clears)
  off += 256;
  L.total = off;
  return L;
}
}  // namespace

extern "C" {

int lnt_diag_expired_wait(void* stream) {
  cudaStream_t s = as_stream(stream);
  expired_lookback_kernel<<<1, 32, 0, s>>>();
  count_launch();
  return launch_status();
}

int lnt_collect_duplicates_workspace(size_t n, size_t* bytes) {
  if (!bytes) return LNT_BAD_ARG;
  *bytes = collect_workspace_bytes(n);
  return LNT_OK;
}

int lnt_collect_duplicates(const uint64_t* keys, const double* vals, size_t n, int skip_zero_heads,
                           uint64_t* keys_out, double* vals_out, uint64_t* d_nout, void* workspace,
                           size_t workspace_bytes, void* stream) {
  if (!d_nout) return LNT_BAD_ARG;
  if (n && (!keys || !vals || !keys_out || !vals_out)) return LNT_BAD_ARG;
  if (n && (!workspace || workspace_bytes < collect_workspace_bytes(n))) return LNT_WORKSPACE;
  return run_collect((const u64*)keys, vals, n, skip_zero_heads, (u64*)keys_out, vals_out, (u64*)d_nout,
                     workspace, as_stream(stream));
}

int lnt_sort_reduce_workspace(size_t na, size_t nb, uint64_t max_key, size_t* bytes) {
  if (!bytes) return LNT_BAD_ARG;
  if (na + nb >= (1u << 30)) return LNT_UNSUPPORTED;
  *bytes = sort_reduce_layout(na + nb, max_key).total;
  return LNT_OK;
}

int lnt_sort_reduce(const uint64_t* a_keys, const double* a_vals, size_t na, const lnt_rekey_spec* a_rekey,
                    const uint64_t* b_keys, const double* b_vals, size_t nb, const lnt_rekey_spec* b_rekey,
                    double b_scale, uint64_t max_key, int skip_zero_heads, uint64_t* keys_out,
                    double* vals_out, uint64_t* d_nout, void* workspace, size_t workspace_bytes,
                    void* stream) {
  const size_t n = na + nb;
  if (!d_nout) return LNT_BAD_ARG;
  if ((na && (!a_keys || !a_vals)) || (nb && (!b_keys || !b_vals))) return LNT_BAD_ARG;
  if (n && (!keys_out || !vals_out)) return LNT_BAD_ARG;
  if (n >= (1u << 30)) return LNT_UNSUPPORTED;
  cudaStream_t s = as_stream(stream);
  if (n == 0) return run_collect(nullptr, nullptr, 0, skip_zero_heads, nullptr, nullptr, (u64*)d_nout, nullptr, s);
  SortReduceLayout L = sort_reduce_layout(n, max_key);
  if (!workspace || workspace_bytes < L.total) return LNT_WORKSPACE;
  if ((uintptr_t)workspace % 256) return LNT_BAD_ARG;
  PairSource src;
  src.ak = (const u64*)a_keys;
  src.av = a_vals;
  src.na = na;
  src.bk = (const u64*)b_keys;
  src.bv = b_vals;
  src.nb = nb;
  src.bscale = b_scale;
  src.pad = 0;
  src.gate = nullptr;
  src.gate_run = 0;
  src.pad2 = 0;
  int st = make_rekey_params(a_rekey, &src.ra);
  if (st != LNT_OK) return st;
  st = make_rekey_params(b_rekey, &src.rb);
  if (st != LNT_OK) return st;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  u64* k0 = reinterpret_cast<u64*>(w + L.off_k0);
  double* v0 = reinterpret_cast<double*>(w + L.off_v0);
  u64* k1 = reinterpret_cast<u64*>(w + L.off_k1);
  double* v1 = reinterpret_cast<double*>(w + L.off_v1);
  const int key_bits = key_bits_for(max_key);
  // Wide keys, many pairs: the bucketed path, whose histogram decides on the
  // device whether it can finish (every bucket fits a CTA); the LSD path is
  // enqueued behind it gated on the opposite answer.  Nothing waits on the host.
  const u32* gate = nullptr;
  if (bucket_path_applies(n, key_bits) && !getenv("LNT_NO_BUCKETS")) {
    u32* g = reinterpret_cast<u32*>(w + L.off_gate);
    st = run_bucketed_sort_reduce(src, (u32)n, key_bits, skip_zero_heads, k0, v0, k1, v1, w + L.off_ctrl,
                                  (u64*)keys_out, vals_out, (u64*)d_nout, g, s);
    if (st != LNT_OK) return st;
    gate = g;
  }
  st = run_sort(L.plan, gated_source(src, gate, 1), k0, v0, k1, v1, w + L.off_ctrl, s);
  if (st != LNT_OK) return st;
  return run_collect_gated(k0, v0, n, skip_zero_heads, (u64*)keys_out, vals_out, (u64*)d_nout, w + L.off_coll, s,
                           gate, 1);
}

}  // extern "C"
