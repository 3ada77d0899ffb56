// Merge of two key-sorted operands (the scan-merge path) and the fused
// re-key + sort entry point.
//
// lnt_merge_sorted reproduces outside_merge_sparse_storage_containers
// (FunctionUtil.h:373-419): walking both arrays, A-only keys are copied,
// B-only keys become op(0, b), and equal keys consume one A and one B into
// op(a, b).  Within a run of equal keys this pairs the j-th A with the j-th B;
// surplus A's are copied and surplus B's become op(0, b).
//
// GPU formulation: the stable merge of A and B (A first on ties) is split by
// merge-path diagonals into tiles of 2048 merged elements.  In that order the
// j-th A of a key run sits before every B of the run, so each element decides
// locally (from its merged position and at most two neighbour reads) whether
// it is emitted and with which partner:
//   A_i with key k: lbB = (merged position) - i is the first B with key k;
//     j = occurrence of k in A up to i; partner B[lbB + j] if it has key k.
//   B_i with key k: ubA = (merged position) - i is one past the last A with
//     key k; j = occurrence of k in B up to i; B_i is consumed iff
//     A[ubA - 1 - j] has key k.
// A partition kernel finds every tile's split first (one merge-path search per
// tile boundary, all in parallel); each tile then stages its A and B slices
// (keys and values) in shared memory with coalesced loads, and run indices and
// partners are read from there - global memory only when a run of equal keys
// crosses the slice boundary.  Emitted elements keep merged order; their output
// offsets come from a block scan plus a decoupled look-back over tiles.
// Traffic: 16 B read per input pair + 16 B written per output pair.
#include <algorithm>

#include "lnt_sort.cuh"

namespace lnt {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagPre = 2ull << 62;
constexpr unsigned long long kFlagMask = 3ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1ull;

// Number of A elements among the first d of the stable merge (A first on ties).
__device__ __forceinline__ size_t merge_path(const u64* __restrict__ a, size_t na, const u64* __restrict__ b,
                                             size_t nb, size_t d) {
  size_t lo = d > nb ? d - nb : 0;
  size_t hi = d < na ? d : na;
  while (lo < hi) {
    const size_t mid = (lo + hi) >> 1;
    if (a[mid] <= b[d - 1 - mid])
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Same search over shared-memory slices.
__device__ __forceinline__ int merge_path_smem(const u64* a, int na, const u64* b, int nb, int d) {
  int lo = d > nb ? d - nb : 0;
  int hi = d < na ? d : na;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= b[d - 1 - mid])
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Occurrence index of x[i] within its run of equal keys.
__device__ __forceinline__ size_t run_index(const u64* __restrict__ x, size_t i, u64 k) {
  size_t j = 0;
  while (i > j && x[i - 1 - j] == k) ++j;
  return j;
}

__device__ __forceinline__ double apply_op(int op, double a, double b) { return op == 0 ? a + b : a - b; }

// splits[t] = A elements among the first min(t * kTile, na + nb) of the merge.
__global__ void merge_partition_kernel(const u64* __restrict__ a, size_t na, const u64* __restrict__ b, size_t nb,
                                       u32 ntiles, u64* __restrict__ splits) {
  const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles) return;
  splits[t] = merge_path(a, na, b, nb, min(na + nb, (size_t)t * kTile));
}

__global__ void __launch_bounds__(kThreads) merge_kernel(const u64* __restrict__ ak, const double* __restrict__ av,
                                                         size_t na, const u64* __restrict__ bk,
                                                         const double* __restrict__ bv, size_t nb, int op,
                                                         u32 ntiles, const u64* __restrict__ splits,
                                                         unsigned long long* __restrict__ status,
                                                         u32* __restrict__ tile_counter, u64* __restrict__ ck,
                                                         double* __restrict__ cv, u64* __restrict__ d_nout) {
  __shared__ u64 s_k[kTile];
  __shared__ double s_v[kTile];
  __shared__ u32 s_warp[kThreads / 32];
  __shared__ u32 s_tile;
  __shared__ unsigned long long s_off;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const u32 tile = s_tile;
  const size_t total = na + nb;
  const size_t d0 = (size_t)tile * kTile;
  const size_t d1 = min(total, d0 + kTile);
  const size_t a0 = splits[tile], a1 = splits[tile + 1];
  const size_t b0 = d0 - a0, b1 = d1 - a1;
  const int la = (int)(a1 - a0), lb = (int)(b1 - b0);
  // stage the tile's A slice then its B slice, keys and values, in shared memory
  for (int i = tid; i < la + lb; i += kThreads) {
    if (i < la) {
      s_k[i] = __ldcs(ak + a0 + i);
      s_v[i] = __ldcs(av + a0 + i);
    } else {
      s_k[i] = __ldcs(bk + b0 + (i - la));
      s_v[i] = __ldcs(bv + b0 + (i - la));
    }
  }
  __syncthreads();
  // each thread merges kItems consecutive merged positions
  const int dt = min(tid * kItems, la + lb);
  int ia = merge_path_smem(s_k, la, s_k + la, lb, dt);
  int ib = dt - ia;
  bool emit[kItems];
  u64 ek[kItems];
  double evv[kItems];
  u32 nemit = 0;
#pragma unroll
  for (int q = 0; q < kItems; ++q) {
    emit[q] = false;
    ek[q] = 0;
    evv[q] = 0.0;
    const int m = dt + q;
    if (m >= la + lb) continue;
    const bool take_a = ib >= lb || (ia < la && s_k[ia] <= s_k[la + ib]);
    const size_t mg = d0 + (size_t)m;  // global merged position
    if (take_a) {
      const size_t i = a0 + ia;
      const u64 k = s_k[ia];
      const size_t lbB = mg - i;  // B elements before A_i: those with key < k
      size_t j = 0;               // occurrence of k in A before A_i
      while ((int)j < ia && s_k[ia - 1 - j] == k) ++j;
      if ((int)j == ia) j += run_index(ak, a0, k);
      double v = s_v[ia];
      const size_t pb = lbB + j;  // the partner B, if it has key k
      if (pb >= b0 && pb < b1) {
        if (s_k[la + (int)(pb - b0)] == k) v = apply_op(op, v, s_v[la + (int)(pb - b0)]);
      } else if (pb < nb && bk[pb] == k) {
        v = apply_op(op, v, bv[pb]);
      }
      emit[q] = true;
      ek[q] = k;
      evv[q] = v;
      ++ia;
    } else {
      const size_t i = b0 + ib;
      const u64 k = s_k[la + ib];
      const size_t ubA = mg - i;  // A elements before B_i: those with key <= k
      size_t j = 0;               // occurrence of k in B before B_i
      while ((int)j < ib && s_k[la + ib - 1 - j] == k) ++j;
      if ((int)j == ib) j += run_index(bk, b0, k);
      bool consumed = false;
      if (ubA >= j + 1) {
        const size_t pa = ubA - 1 - j;  // the A it would pair with
        consumed = (pa >= a0 && pa < a1) ? s_k[(int)(pa - a0)] == k : ak[pa] == k;
      }
      if (!consumed) {
        emit[q] = true;
        ek[q] = k;
        evv[q] = apply_op(op, 0.0, s_v[la + ib]);
      }
      ++ib;
    }
    nemit += emit[q] ? 1u : 0u;
  }
  // ---- block scan of emitted counts -------------------------------------
  u32 inc = nemit;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  u32 excl = inc - nemit, tot = 0;
  for (int w = 0; w < kThreads / 32; ++w) {
    if (w < warp) excl += s_warp[w];
    tot += s_warp[w];
  }
  // ---- look-back for the tile's output offset (warp 0) --------------------
  if (warp == 0) {
    if (lane == 0) *reinterpret_cast<volatile unsigned long long*>(&status[tile]) = (tile == 0 ? kFlagPre : kFlagAgg) | tot;
    unsigned long long off = 0;
    if (tile != 0) {
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
        off += v;
        if (first_pre < first_nr) break;
        base -= first_nr;
        if (first_nr < 32 && ++spins > spin_limit()) {
          latch_error(kErrMergeLookback);
          break;
        }
      }
      if (lane == 0) *reinterpret_cast<volatile unsigned long long*>(&status[tile]) = kFlagPre | (off + tot);
    }
    if (lane == 0) {
      s_off = off;
      if (tile == ntiles - 1) *d_nout = off + tot;
    }
  }
  __syncthreads();  // s_k reads done; s_off ready
  u32 r = excl;
#pragma unroll
  for (int q = 0; q < kItems; ++q) {
    if (emit[q]) {
      s_k[r] = ek[q];
      s_v[r] = evv[q];
      ++r;
    }
  }
  __syncthreads();
  const unsigned long long off = s_off;
  for (u32 i = tid; i < tot; i += kThreads) {
    __stcs(ck + off + i, s_k[i]);
    __stcs(cv + off + i, s_v[i]);
  }
}

}  // namespace

struct MergeLayout {
  u32 ntiles;
  size_t off_status, off_counter, off_splits, total;
};

static MergeLayout merge_layout(size_t n) {
  MergeLayout L;
  L.ntiles = (u32)((n + kTile - 1) / kTile);
  L.off_status = 0;
  L.off_counter = align_up((size_t)std::max<u32>(L.ntiles, 1) * 8, 256);
  L.off_splits = L.off_counter + 256;
  L.total = L.off_splits + align_up(((size_t)L.ntiles + 1) * 8, 256);
  return L;
}

}  // namespace lnt

using namespace lnt;

namespace {
struct PermuteSortLayout {
  SortPlan plan;
  size_t off_ctrl, off_tk, off_tv, total;
};
PermuteSortLayout permute_sort_layout(size_t n, u64 max_key) {
  PermuteSortLayout L;
  L.plan = make_sort_plan(n, max_key);
  size_t off = 0;
  L.off_ctrl = off;
  off += align_up(L.plan.ctrl_bytes, 256);
  L.off_tk = off;
  off += align_up(n * 8, 256);
  L.off_tv = off;
  off += align_up(n * 8, 256);
  L.total = off;
  return L;
}
}  // namespace

extern "C" {

int lnt_merge_sorted_workspace(size_t na, size_t nb, size_t* bytes) {
  if (!bytes) return LNT_BAD_ARG;
  *bytes = merge_layout(na + nb).total;
  return LNT_OK;
}

int lnt_merge_sorted(const uint64_t* a_keys, const double* a_vals, size_t na, const uint64_t* b_keys,
                     const double* b_vals, size_t nb, int op, uint64_t* c_keys, double* c_vals, uint64_t* d_nout,
                     void* workspace, size_t workspace_bytes, void* stream) {
  if (!d_nout || (op != 0 && op != 1)) return LNT_BAD_ARG;
  if ((na && (!a_keys || !a_vals)) || (nb && (!b_keys || !b_vals))) return LNT_BAD_ARG;
  const size_t n = na + nb;
  cudaStream_t s = as_stream(stream);
  if (n == 0) return cudaMemsetAsync(d_nout, 0, 8, s) == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
  if (!c_keys || !c_vals) return LNT_BAD_ARG;
  MergeLayout L = merge_layout(n);
  if (!workspace || workspace_bytes < L.total) return LNT_WORKSPACE;
  if (cudaMemsetAsync(workspace, 0, L.off_splits, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  u64* splits = reinterpret_cast<u64*>(w + L.off_splits);
  {
    ProfScope prof("merge", s);
    merge_partition_kernel<<<(L.ntiles + 1 + 255) / 256, 256, 0, s>>>((const u64*)a_keys, na, (const u64*)b_keys, nb,
                                                                       L.ntiles, splits);
    merge_kernel<<<L.ntiles, kThreads, 0, s>>>((const u64*)a_keys, a_vals, na, (const u64*)b_keys, b_vals, nb, op,
                                               L.ntiles, splits, reinterpret_cast<unsigned long long*>(w + L.off_status),
                                               reinterpret_cast<u32*>(w + L.off_counter), (u64*)c_keys, c_vals,
                                               (u64*)d_nout);
  }
  count_launch(2);
  return launch_status();
}

int lnt_permute_sort_workspace(size_t n, uint64_t max_key, size_t* bytes) {
  if (!bytes) return LNT_BAD_ARG;
  if (n >= (1u << 30)) return LNT_UNSUPPORTED;
  *bytes = permute_sort_layout(n, max_key).total;
  return LNT_OK;
}

int lnt_permute_sort(const uint64_t* keys_in, const double* vals_in, size_t n, const lnt_rekey_spec* rekey,
                     uint64_t* keys_out, double* vals_out, uint64_t max_key, void* workspace,
                     size_t workspace_bytes, void* stream) {
  if (n == 0) return LNT_OK;
  if (!keys_in || !vals_in || !keys_out || !vals_out) return LNT_BAD_ARG;
  if ((const void*)keys_in == (const void*)keys_out || (const void*)vals_in == (const void*)vals_out)
    return LNT_BAD_ARG;  // out of place only
  if (n >= (1u << 30)) return LNT_UNSUPPORTED;
  PermuteSortLayout L = permute_sort_layout(n, max_key);
  if (!workspace || workspace_bytes < L.total) return LNT_WORKSPACE;
  if ((uintptr_t)workspace % 256) return LNT_BAD_ARG;
  PairSource src = plain_source((const u64*)keys_in, vals_in, n);
  int st = make_rekey_params(rekey, &src.ra);
  if (st != LNT_OK) return st;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  return run_sort(L.plan, src, (u64*)keys_out, vals_out, reinterpret_cast<u64*>(w + L.off_tk),
                  reinterpret_cast<double*>(w + L.off_tv), w + L.off_ctrl, as_stream(stream));
}

}  // extern "C"
