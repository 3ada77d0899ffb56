// Batched sparse lattice products: thousands of independent, unevenly sized
// C_p = A_p * B_p (each as in lnt_lattice_mult) in a fixed number of launches,
// all stream-ordered and capturable in one CUDA graph.  The reference has no
// batching: its equivalent is a loop of csc_no_accum calls
// (SparseLatticeBase.h:1854-1990), one per contraction.
//
// Layout: operands are concatenated (A of problem p at a_off[p] .. a_off[p+1],
// likewise B); a descriptor per problem holds its dims, magic dividers and
// offsets into the scratch tables.  Output C is concatenated too; problem p's
// part starts at c_off[p].
//
// Pipeline (per call):
//   colptr (A and B): dense column pointers of every problem (u32 offsets);
//   spa<symbolic>: persistent warps pull chunks of output columns ("units") of
//     all problems from an atomic queue and count each column's output rows;
//   scan: global exclusive sum over units -> output position of every column;
//   spa<numeric>: persistent warps pull chunks again and write each column's
//     rows (dense accumulator in shared memory, ascending emission);
//   coff: per-problem output offsets.
// The queue chunk size (units per grab) is the segment-split knob the
// autotuner sets: small chunks balance uneven columns, large ones cut queue
// traffic.  Problems with more than 512 rows are accumulated in blocks of
// 512 rows (each A column's entries for the block found by binary search).
//
// lnt_batched_contract takes the operands as the tensors are stored (unsorted,
// keys in each tensor's own mode order) and does the per-problem work of
// toLatticeSort (SparseMIABase.h:1457-1586) inside the call: one kernel
// re-keys every pair into its problem's lattice order and prefixes the key
// with (problem, operand), one stable radix sort of all pairs orders every
// problem's A and B at once (their segments end up interleaved: A_0 B_0 A_1
// B_1 ..), and the product kernels read the sorted pairs with the prefix
// masked off.  The sort's digit width is the autotuned one for the pair count
// and composite key width.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "lnt_tuned.h"
#include "lnt_scan.cuh"
#include "lnt_sort.cuh"

namespace lnt {
namespace {

constexpr int kMaxRows = 512;  // accumulator rows per warp (4 KB of FP64 sums: eight 4-warp CTAs per SM)
constexpr int kWarps = 4;

struct ProbDesc {
  u64 a_off, a_n, b_off, b_n;
  u64 aptr_off, bptr_off;  // into the u32 pointer tables
  u64 unit_off, units;     // global unit range (units = wB * d)
  u64 h, w, wB, d;
  Divider div_h, div_w, div_wB;
};

struct BatchArgs {
  const u64* ak;
  const double* av;
  const u64* bk;
  const double* bv;
  const ProbDesc* prob;
  int count;
  u64 total_units;
  u32* aptr;
  u32* bptr;
  u64 kmask;  // lattice key bits of the stored keys (the rest is the sort prefix)
  const u32* uprob;  // the problem of every unit (output column), built at prepare time
};

// Column pointers of every problem's A (which == 0) or B (which == 1).
// Position q enumerates, problem by problem, the n_p + 1 boundaries; position
// i of problem p fills the pointer entries of the (possibly many empty)
// columns between entry i-1's column and entry i's.  A warp takes 256
// consecutive positions, lane-striped (w0 + 32 k + lane: coalesced key loads,
// adjacent lanes' short ranges adjacent), each lane one binary search for its
// problem, and each thread fills short ranges itself; a range longer than kLongRun columns (a run of empty columns,
// common in problems with far more columns than entries) is filled by the
// whole warp together in coalesced stores, so no thread writes a long run
// alone.
__global__ void batch_colptr_kernel(BatchArgs args, int which, const u64* __restrict__ pos_off, u64 total_pos) {
  constexpr u64 kPer = 8;
  constexpr long long kLongRun = 32;
  const int lane = threadIdx.x & 31;
  const u64 warps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u64 warp_id = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  for (u64 w0 = warp_id * 32 * kPer; w0 < total_pos; w0 += warps * 32 * kPer) {
    const u64 q0 = w0 + (u64)lane;  // lane-striped: positions w0 + 32 k + lane
    int p = 0;
    if (q0 < total_pos) {
      int lo = 0, hi = args.count - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pos_off[mid] <= q0) lo = mid; else hi = mid - 1;
      }
      p = lo;
    }
    for (u64 k = 0; k < kPer; ++k) {
      const u64 q = q0 + 32 * k;
      long long prev = 0, cur = -1;
      u32 idx = 0;
      u32* ptr = nullptr;
      if (q < total_pos) {
        while (p + 1 < args.count && pos_off[p + 1] <= q) ++p;
        const ProbDesc& P = args.prob[p];
        const u64 i = q - pos_off[p];
        const u64 n = which == 0 ? P.a_n : P.b_n;
        const u64* keys = which == 0 ? args.ak + P.a_off : args.bk + P.b_off;
        const Divider& dv = which == 0 ? P.div_h : P.div_w;
        const u64 ncol = which == 0 ? P.w * P.d : P.units;
        ptr = which == 0 ? args.aptr + P.aptr_off : args.bptr + P.bptr_off;
        prev = i == 0 ? -1ll : (long long)min(divide(keys[i - 1] & args.kmask, dv), ncol);
        cur = i == n ? (long long)ncol : (long long)min(divide(keys[i] & args.kmask, dv), ncol);
        idx = (u32)i;
        if (cur - prev <= kLongRun)
          for (long long c = prev + 1; c <= cur; ++c) ptr[c] = idx;
      }
      u32 longm = __ballot_sync(0xffffffffu, cur - prev > kLongRun);
      while (longm) {
        const int j = __ffs(longm) - 1;
        longm &= longm - 1u;
        const long long pj = __shfl_sync(0xffffffffu, prev, j);
        const long long cj = __shfl_sync(0xffffffffu, cur, j);
        const u32 ij = __shfl_sync(0xffffffffu, idx, j);
        u32* pp = reinterpret_cast<u32*>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(ptr), j));
        for (long long c = pj + 1 + lane; c <= cj; c += 32) pp[c] = ij;
      }
    }
  }
}

// First entry at or after position lo of A column acol (entries lo..hi-1,
// ascending rows) whose row is >= r0.
__device__ __forceinline__ u32 lower_row(const u64* __restrict__ ak, u64 kmask, u32 lo, u32 hi, u64 base, u64 r0) {
  while (lo < hi) {
    const u32 mid = (lo + hi) >> 1;
    if ((ak[mid] & kmask) - base < r0) lo = mid + 1; else hi = mid;
  }
  return lo;
}

template <bool NUMERIC>
__global__ void __launch_bounds__(kWarps * 32, 8) batch_spa_kernel(BatchArgs args, u32 chunk, u32* __restrict__ queue,
                                                                 u64* __restrict__ ucount,
                                                                 const u64* __restrict__ uoff,
                                                                 u64* __restrict__ ck, double* __restrict__ cv) {
  __shared__ u32 s_bits[kWarps][kMaxRows / 32];
  __shared__ double s_acc[NUMERIC ? kWarps : 1][NUMERIC ? kMaxRows : 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u32* bits = s_bits[warp];
  double* acc = s_acc[NUMERIC ? warp : 0];
  const u64 kmask = args.kmask;
  while (true) {
    u64 first = 0;
    if (lane == 0) first = (u64)atomicAdd(queue, chunk);
    first = __shfl_sync(0xffffffffu, first, 0);
    if (first >= args.total_units) break;
    const u64 last = min(first + chunk, args.total_units);
    for (u64 u = first; u < last; ++u) {
      const ProbDesc& P = args.prob[args.uprob[u]];  // chunks may span problems
      const u64 lu = u - P.unit_off;  // column id within the problem: col + wB*tab
      const u32* bptr = args.bptr + P.bptr_off;
      const u64 e0 = bptr[lu], e1 = bptr[lu + 1];
      if (e0 == e1) {
        if (!NUMERIC && lane == 0) ucount[u] = 0;
        continue;
      }
      const u64 h = P.h, w = P.w;
      const u64 t = divide(lu, P.div_wB);
      const u64* ak = args.ak + P.a_off;
      const double* av = args.av + P.a_off;
      const u64* bk = args.bk + P.b_off;
      const double* bv = args.bv + P.b_off;
      const u32* aptr = args.aptr + P.aptr_off;
      const bool blocked = h > (u64)kMaxRows;
      u64 out = NUMERIC ? uoff[u] : 0;
      u32 count = 0;
      const u64 colkey = h * lu;
      // rows in blocks of kMaxRows (one block unless h > kMaxRows), ascending
      for (u64 r0 = 0; r0 < h; r0 += kMaxRows) {
        const u64 hb = min((u64)kMaxRows, h - r0);
        const int hw = (int)((hb + 31) / 32);
        for (int i = lane; i < hw; i += 32) bits[i] = 0u;
        if (NUMERIC)
          for (int i = lane; i < (int)hb; i += 32) acc[i] = 0.0;
        __syncwarp();
        for (u64 e = e0 + lane; e < e1; e += 32) {
          const u64 acol = ((bk[e] & kmask) - w * lu) + w * t;
          const u64 abase = acol * h;
          u32 lo = aptr[acol];
          const u32 hi = aptr[acol + 1];
          if (blocked) lo = lower_row(ak, kmask, lo, hi, abase, r0);
          const double beta = NUMERIC ? bv[e] : 0.0;
          // four A entries loaded before their accumulations, so that their
          // loads overlap instead of each waiting behind the previous atomics
          bool stop = false;
          u32 x = lo;
          for (; x + 4 <= hi && !stop; x += 4) {
            u64 kk[4];
            double vv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              kk[j] = ak[x + j];
              vv[j] = NUMERIC ? av[x + j] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const u64 rr = (kk[j] & kmask) - abase;
              if (blocked && rr >= r0 + hb) {
                stop = true;
                break;
              }
              const u32 r = (u32)(rr - r0);
              atomicOr(&bits[r >> 5], 1u << (r & 31));
              if (NUMERIC) atomicAdd(&acc[r], vv[j] * beta);
            }
          }
          for (; x < hi && !stop; ++x) {
            const u64 rr = (ak[x] & kmask) - abase;
            if (blocked && rr >= r0 + hb) break;
            const u32 r = (u32)(rr - r0);
            atomicOr(&bits[r >> 5], 1u << (r & 31));
            if (NUMERIC) atomicAdd(&acc[r], av[x] * beta);
          }
        }
        __syncwarp();
        if (!NUMERIC) {
          u32 c = 0;
          for (int i = lane; i < hw; i += 32) c += __popc(bits[i]);
          count += c;
        } else {
          for (int g = 0; g < hw; ++g) {
            const u32 word = bits[g];
            if (word & (1u << lane)) {
              const u32 r = (u32)g * 32 + lane;
              const u64 o = out + __popc(word & ((1u << lane) - 1u));
              ck[o] = colkey + r0 + r;
              cv[o] = acc[r];
            }
            out += __popc(word);
          }
        }
        __syncwarp();
      }
      if (!NUMERIC) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
        if (lane == 0) ucount[u] = count;
      }
    }
  }
}

__global__ void batch_coff_kernel(const ProbDesc* __restrict__ prob, int count, const u64* __restrict__ uoff,
                                  u64 total_units, u64* __restrict__ c_off) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < count) c_off[p] = uoff[prob[p].unit_off];
  if (p == count) c_off[count] = uoff[total_units];
}

struct BatchLayout {
  u64 total_units, aptr_len, bptr_len, a_pos, b_pos, c_bound;
  size_t off_prob, off_apos, off_bpos, off_aptr, off_bptr, off_ucount, off_uoff, off_queue, off_scan, off_uprob,
      total;
};

// interleaved: the operands are read from one array holding A_0 B_0 A_1 B_1 ..
// (the output of the contract path's sort) instead of two concatenations.
int batch_layout(int count, const int64_t* dims, const uint64_t* a_off, const uint64_t* b_off, BatchLayout* L,
                 std::vector<ProbDesc>* descs, std::vector<u64>* apos, std::vector<u64>* bpos,
                 bool interleaved = false) {
  if (count <= 0 || !dims || !a_off || !b_off) return LNT_BAD_ARG;
  L->total_units = L->aptr_len = L->bptr_len = L->a_pos = L->b_pos = L->c_bound = 0;
  if (descs) descs->resize(count);
  if (apos) apos->resize(count);
  if (bpos) bpos->resize(count);
  for (int p = 0; p < count; ++p) {
    const int64_t h = dims[4 * p], w = dims[4 * p + 1], wB = dims[4 * p + 2], d = dims[4 * p + 3];
    if (h <= 0 || w <= 0 || wB <= 0 || d <= 0) return LNT_BAD_DIMS;
    if (a_off[p + 1] < a_off[p] || b_off[p + 1] < b_off[p]) return LNT_BAD_ARG;
    const u64 na = a_off[p + 1] - a_off[p], nb = b_off[p + 1] - b_off[p];
    if (na >= (1ull << 32) || nb >= (1ull << 32)) return LNT_UNSUPPORTED;
    unsigned __int128 ka = (unsigned __int128)h * w * d, kb = (unsigned __int128)w * wB * d;
    if ((ka >> 63) || (kb >> 63)) return LNT_OVERFLOW_KEYBITS;
    if (descs) {
      ProbDesc& P = (*descs)[p];
      P.a_off = interleaved ? a_off[p] + b_off[p] : a_off[p];
      P.a_n = na;
      P.b_off = interleaved ? P.a_off + na : b_off[p];
      P.b_n = nb;
      P.aptr_off = L->aptr_len;
      P.bptr_off = L->bptr_len;
      P.unit_off = L->total_units;
      P.units = (u64)wB * d;
      P.h = h;
      P.w = w;
      P.wB = wB;
      P.d = d;
      P.div_h = make_divider(h);
      P.div_w = make_divider(w);
      P.div_wB = make_divider(wB);
    }
    if (apos) (*apos)[p] = L->a_pos;
    if (bpos) (*bpos)[p] = L->b_pos;
    L->aptr_len += (u64)w * d + 1;
    L->bptr_len += (u64)wB * d + 1;
    L->total_units += (u64)wB * d;
    L->a_pos += na + 1;
    L->b_pos += nb + 1;
    L->c_bound += (u64)std::min<unsigned __int128>((unsigned __int128)h * wB * d, (unsigned __int128)nb * h);
  }
  size_t off = 0;
  L->off_prob = off;
  off += align_up((size_t)count * sizeof(ProbDesc), 256);
  L->off_apos = off;
  off += align_up((size_t)count * 8, 256);
  L->off_bpos = off;
  off += align_up((size_t)count * 8, 256);
  L->off_aptr = off;
  off += align_up(L->aptr_len * 4, 256);
  L->off_bptr = off;
  off += align_up(L->bptr_len * 4, 256);
  L->off_ucount = off;
  off += align_up((L->total_units + 1) * 8, 256);
  L->off_uoff = off;
  off += align_up((L->total_units + 1) * 8, 256);
  L->off_queue = off;
  off += 256;
  L->off_scan = off;
  off += align_up(scan::workspace_bytes(L->total_units), 256);
  L->off_uprob = off;
  off += align_up(std::max<u64>(L->total_units, 1) * 4, 256);
  L->total = off;
  return LNT_OK;
}

// The problem of every unit, from the descriptors (units are numbered problem
// by problem): the product kernels read it instead of searching the
// descriptors for each column they take.
std::vector<u32> unit_problems(const std::vector<ProbDesc>& descs, u64 total_units) {
  std::vector<u32> up(total_units);
  for (size_t p = 0; p < descs.size(); ++p)
    std::fill(up.begin() + descs[p].unit_off, up.begin() + descs[p].unit_off + descs[p].units, (u32)p);
  return up;
}

struct U64Of {
  const u64* v;
  __device__ __forceinline__ u64 operator()(size_t i) const { return v[i]; }
};

// Composite sort keys of the contract path: position q of the concatenated
// operand (A or B) belongs to the problem p with off[p] <= q < off[p+1]; its
// key is re-keyed into p's lattice order and prefixed with (p, which).  A warp
// takes 256 consecutive positions, lane-striped (position base + 32 j + lane),
// so loads and stores are coalesced; each lane finds its first position's
// problem by binary search and walks forward from there.  (A thread taking 8
// consecutive positions issued 8-byte stores 64 bytes apart: 0.86 ms for the
// 4096-problem batch.)
__global__ void batch_compose_kernel(const u64* __restrict__ keys, u64 n, const uint64_t* __restrict__ off,
                                     int count, const RekeyParams* __restrict__ rk, u64 which_bit, int S,
                                     u64* __restrict__ out) {
  constexpr u64 kSpan = 256;
  const int lane = threadIdx.x & 31;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 base = (((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kSpan; base < n; base += nwarps * kSpan) {
    const u64 q0 = base + lane;
    if (q0 >= n) continue;
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (off[mid] <= q0) lo = mid; else hi = mid - 1;
    }
    int p = lo;
    const u64 q1 = min(base + kSpan, n);
    for (u64 q = q0; q < q1; q += 32) {
      while (q >= off[p + 1]) ++p;
      out[q] = ((u64)p << (S + 1)) | which_bit | rekey(keys[q], rk[p]);
    }
  }
}

struct ContractLayout {
  BatchLayout B;
  u64 NA, NB;
  int S;  // lattice key bits of the widest operand
  SortPlan plan;
  size_t off_rk, off_aoff, off_boff, off_ck, off_k0, off_v0, off_k1, off_v1, off_ctrl, total;
};

int contract_layout(int count, const int64_t* dims, const uint64_t* a_off, const uint64_t* b_off,
                    ContractLayout* C) {
  int st = batch_layout(count, dims, a_off, b_off, &C->B, nullptr, nullptr, nullptr, true);
  if (st != LNT_OK) return st;
  if (a_off[0] != 0 || b_off[0] != 0) return LNT_BAD_ARG;
  C->NA = a_off[count];
  C->NB = b_off[count];
  const u64 N = C->NA + C->NB;
  if (N >= (1ull << 30)) return LNT_UNSUPPORTED;  // one radix sort of all pairs
  int S = 1;
  for (int p = 0; p < count; ++p) {
    const u64 h = dims[4 * p], w = dims[4 * p + 1], wB = dims[4 * p + 2], d = dims[4 * p + 3];
    S = std::max(S, std::max(key_bits_for(h * w * d), key_bits_for(w * wB * d)));
  }
  if (S + 1 + key_bits_for((u64)count) > 63) return LNT_OVERFLOW_KEYBITS;
  C->S = S;
  C->plan = make_sort_plan(N, (u64)count << (S + 1));
  size_t off = align_up(C->B.total, 256);
  C->off_rk = off;
  off += align_up((size_t)2 * count * sizeof(RekeyParams), 256);
  C->off_aoff = off;
  off += align_up((size_t)(count + 1) * 8, 256);
  C->off_boff = off;
  off += align_up((size_t)(count + 1) * 8, 256);
  C->off_ck = off;
  off += align_up(N * 8, 256);
  C->off_k0 = off;
  off += align_up(N * 8, 256);
  C->off_v0 = off;
  off += align_up(N * 8, 256);
  C->off_k1 = off;
  off += align_up(N * 8, 256);
  C->off_v1 = off;
  off += align_up(N * 8, 256);
  C->off_ctrl = off;
  off += align_up(C->plan.ctrl_bytes, 256);
  C->total = off;
  return LNT_OK;
}

u32 batch_chunk() {
  if (const char* e = getenv("LNT_BATCH_CHUNK")) {
    const int c = atoi(e);
    if (c >= 1 && c <= 4096) return (u32)c;
  }
  return kTunedBatchChunk;
}

int run_batch_product(const BatchArgs& args, const BatchLayout& L, unsigned char* w, int count, uint64_t* c_keys,
                      double* c_vals, uint64_t* d_c_off, cudaStream_t s) {
  int st = LNT_OK;
  u64* ucount = reinterpret_cast<u64*>(w + L.off_ucount);
  u64* uoff = reinterpret_cast<u64*>(w + L.off_uoff);
  u32* queue = reinterpret_cast<u32*>(w + L.off_queue);
  const int sms = sm_count();
  if (cudaMemsetAsync(queue, 0, 256, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  {
    ProfScope prof("batch_colptr", s);
    const int ga = (int)std::max<u64>(1, std::min<u64>((L.a_pos / 8 + 255) / 256, (u64)sms * 16));
    batch_colptr_kernel<<<ga, 256, 0, s>>>(args, 0, reinterpret_cast<const u64*>(w + L.off_apos), L.a_pos);
    const int gb = (int)std::max<u64>(1, std::min<u64>((L.b_pos / 8 + 255) / 256, (u64)sms * 16));
    batch_colptr_kernel<<<gb, 256, 0, s>>>(args, 1, reinterpret_cast<const u64*>(w + L.off_bpos), L.b_pos);
    count_launch(2);
  }
  const u32 chunk = batch_chunk();
  {
    ProfScope prof("batch_spa_symbolic", s);
    int per_sm = 0;  // persistent: as many CTAs as fit
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_spa_kernel<false>, kWarps * 32, 0) != cudaSuccess)
      return LNT_DEVICE_ERROR;
    batch_spa_kernel<false><<<sms * std::max(per_sm, 1), kWarps * 32, 0, s>>>(args, chunk, queue, ucount, nullptr,
                                                                              nullptr, nullptr);
    count_launch();
  }
  st = scan::run(U64Of{ucount}, L.total_units, (unsigned long long*)uoff, nullptr, w + L.off_scan, s, "batch_scan");
  if (st != LNT_OK) return st;
  {
    ProfScope prof("batch_spa_numeric", s);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_spa_kernel<true>, kWarps * 32, 0) != cudaSuccess)
      return LNT_DEVICE_ERROR;
    batch_spa_kernel<true><<<sms * std::max(per_sm, 1), kWarps * 32, 0, s>>>(args, chunk, queue + 1, nullptr, uoff,
                                                                             (u64*)c_keys, c_vals);
    count_launch();
  }
  {
    ProfScope prof("batch_coff", s);
    batch_coff_kernel<<<(count + 1 + 255) / 256, 256, 0, s>>>(args.prob, count, uoff, L.total_units,
                                                               (u64*)d_c_off);
    count_launch();
  }
  return launch_status();
}

}  // namespace
}  // namespace lnt

using namespace lnt;

extern "C" {

int lnt_batched_workspace(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                          const uint64_t* b_off_host, size_t* bytes, uint64_t* c_capacity) {
  if (!bytes) return LNT_BAD_ARG;
  BatchLayout L;
  int st = batch_layout(count, dims_host, a_off_host, b_off_host, &L, nullptr, nullptr, nullptr);
  if (st != LNT_OK) return st;
  *bytes = L.total;
  if (c_capacity) *c_capacity = L.c_bound;
  return LNT_OK;
}

int lnt_batched_prepare(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                        const uint64_t* b_off_host, void* workspace, size_t workspace_bytes, void* stream) {
  BatchLayout L;
  std::vector<ProbDesc> descs;
  std::vector<u64> apos, bpos;
  int st = batch_layout(count, dims_host, a_off_host, b_off_host, &L, &descs, &apos, &bpos);
  if (st != LNT_OK) return st;
  if (!workspace || workspace_bytes < L.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  cudaStream_t s = as_stream(stream);
  // synchronous copies: the host vectors die with this call
  if (cudaStreamSynchronize(s) != cudaSuccess) return LNT_DEVICE_ERROR;
  if (cudaMemcpy(w + L.off_prob, descs.data(), descs.size() * sizeof(ProbDesc), cudaMemcpyHostToDevice) != cudaSuccess)
    return LNT_DEVICE_ERROR;
  if (cudaMemcpy(w + L.off_apos, apos.data(), apos.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
    return LNT_DEVICE_ERROR;
  if (cudaMemcpy(w + L.off_bpos, bpos.data(), bpos.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
    return LNT_DEVICE_ERROR;
  const std::vector<u32> up = unit_problems(descs, L.total_units);
  if (!up.empty() && cudaMemcpy(w + L.off_uprob, up.data(), up.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return LNT_DEVICE_ERROR;
  return LNT_OK;
}

int lnt_batched_lattice_mult(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                             const uint64_t* b_off_host, const uint64_t* a_keys, const double* a_vals,
                             const uint64_t* b_keys, const double* b_vals, void* workspace, size_t workspace_bytes,
                             uint64_t* c_keys, double* c_vals, uint64_t* d_c_off, void* stream) {
  BatchLayout L;
  int st = batch_layout(count, dims_host, a_off_host, b_off_host, &L, nullptr, nullptr, nullptr);
  if (st != LNT_OK) return st;
  if (!workspace || workspace_bytes < L.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  if (!d_c_off) return LNT_BAD_ARG;
  if ((L.a_pos > (u64)count && (!a_keys || !a_vals)) || (L.b_pos > (u64)count && (!b_keys || !b_vals)))
    return LNT_BAD_ARG;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  cudaStream_t s = as_stream(stream);
  BatchArgs args;
  args.ak = (const u64*)a_keys;
  args.av = a_vals;
  args.bk = (const u64*)b_keys;
  args.bv = b_vals;
  args.prob = reinterpret_cast<const ProbDesc*>(w + L.off_prob);
  args.count = count;
  args.total_units = L.total_units;
  args.aptr = reinterpret_cast<u32*>(w + L.off_aptr);
  args.bptr = reinterpret_cast<u32*>(w + L.off_bptr);
  args.kmask = ~0ull;
  args.uprob = reinterpret_cast<const u32*>(w + L.off_uprob);
  return run_batch_product(args, L, w, count, c_keys, c_vals, d_c_off, s);
}

}  // extern "C"

extern "C" {

int lnt_batched_contract_workspace(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                                   const uint64_t* b_off_host, size_t* bytes, uint64_t* c_capacity) {
  if (!bytes) return LNT_BAD_ARG;
  ContractLayout C;
  int st = contract_layout(count, dims_host, a_off_host, b_off_host, &C);
  if (st != LNT_OK) return st;
  *bytes = C.total;
  if (c_capacity) *c_capacity = C.B.c_bound;
  return LNT_OK;
}

int lnt_batched_contract_prepare(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                                 const uint64_t* b_off_host, const lnt_rekey_spec* a_rekey_host,
                                 const lnt_rekey_spec* b_rekey_host, void* workspace, size_t workspace_bytes,
                                 void* stream) {
  ContractLayout C;
  int st = contract_layout(count, dims_host, a_off_host, b_off_host, &C);
  if (st != LNT_OK) return st;
  if (!workspace || workspace_bytes < C.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  BatchLayout L;
  std::vector<ProbDesc> descs;
  std::vector<u64> apos, bpos;
  st = batch_layout(count, dims_host, a_off_host, b_off_host, &L, &descs, &apos, &bpos, true);
  if (st != LNT_OK) return st;
  std::vector<RekeyParams> rk(2 * (size_t)count);
  for (int p = 0; p < count; ++p) {
    st = make_rekey_params(a_rekey_host ? &a_rekey_host[p] : nullptr, &rk[p]);
    if (st != LNT_OK) return st;
    st = make_rekey_params(b_rekey_host ? &b_rekey_host[p] : nullptr, &rk[count + p]);
    if (st != LNT_OK) return st;
  }
  const std::vector<u32> uprob = unit_problems(descs, L.total_units);
  unsigned char* w = static_cast<unsigned char*>(workspace);
  cudaStream_t s = as_stream(stream);
  // synchronous copies: the host vectors die with this call
  if (cudaStreamSynchronize(s) != cudaSuccess) return LNT_DEVICE_ERROR;
  const struct {
    size_t off;
    const void* src;
    size_t bytes;
  } copies[] = {{L.off_prob, descs.data(), descs.size() * sizeof(ProbDesc)},
                {L.off_apos, apos.data(), apos.size() * 8},
                {L.off_bpos, bpos.data(), bpos.size() * 8},
                {L.off_uprob, uprob.data(), uprob.size() * 4},
                {C.off_rk, rk.data(), rk.size() * sizeof(RekeyParams)},
                {C.off_aoff, a_off_host, (size_t)(count + 1) * 8},
                {C.off_boff, b_off_host, (size_t)(count + 1) * 8}};
  for (const auto& c : copies)
    if (c.bytes && cudaMemcpy(w + c.off, c.src, c.bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      return LNT_DEVICE_ERROR;
  return LNT_OK;
}

int lnt_batched_contract(int count, const int64_t* dims_host, const uint64_t* a_off_host, const uint64_t* b_off_host,
                         const uint64_t* a_keys, const double* a_vals, const uint64_t* b_keys, const double* b_vals,
                         void* workspace, size_t workspace_bytes, uint64_t* c_keys, double* c_vals,
                         uint64_t* d_c_off, void* stream) {
  ContractLayout C;
  int st = contract_layout(count, dims_host, a_off_host, b_off_host, &C);
  if (st != LNT_OK) return st;
  if (!workspace || workspace_bytes < C.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  if (!d_c_off) return LNT_BAD_ARG;
  if ((C.NA && (!a_keys || !a_vals)) || (C.NB && (!b_keys || !b_vals))) return LNT_BAD_ARG;
  unsigned char* w = static_cast<unsigned char*>(workspace);
  cudaStream_t s = as_stream(stream);
  const u64 N = C.NA + C.NB;
  u64* ck = reinterpret_cast<u64*>(w + C.off_ck);
  u64* k0 = reinterpret_cast<u64*>(w + C.off_k0);
  double* v0 = reinterpret_cast<double*>(w + C.off_v0);
  const RekeyParams* rk = reinterpret_cast<const RekeyParams*>(w + C.off_rk);
  const int sms = sm_count();
  {
    ProfScope prof("batch_compose", s);
    // one warp per 256 positions, at most 16 CTAs of 8 warps per SM
    const u64 ga = std::max<u64>(1, std::min<u64>((C.NA + 2047) / 2048, (u64)sms * 16));
    const u64 gb = std::max<u64>(1, std::min<u64>((C.NB + 2047) / 2048, (u64)sms * 16));
    if (C.NA)
      batch_compose_kernel<<<(unsigned)ga, 256, 0, s>>>((const u64*)a_keys, C.NA,
                                                        reinterpret_cast<const uint64_t*>(w + C.off_aoff), count, rk,
                                                        0ull, C.S, ck);
    if (C.NB)
      batch_compose_kernel<<<(unsigned)gb, 256, 0, s>>>((const u64*)b_keys, C.NB,
                                                        reinterpret_cast<const uint64_t*>(w + C.off_boff), count,
                                                        rk + count, 1ull << C.S, C.S, ck + C.NA);
    count_launch(2);
  }
  if (N) {
    PairSource src = plain_source(ck, a_vals, C.NA);
    src.bk = ck + C.NA;
    src.bv = b_vals;
    src.nb = C.NB;
    st = run_sort(C.plan, src, k0, v0, reinterpret_cast<u64*>(w + C.off_k1), reinterpret_cast<double*>(w + C.off_v1),
                  w + C.off_ctrl, s);
    if (st != LNT_OK) return st;
  }
  BatchArgs args;
  args.ak = k0;
  args.av = v0;
  args.bk = k0;
  args.bv = v0;
  args.prob = reinterpret_cast<const ProbDesc*>(w + C.B.off_prob);
  args.count = count;
  args.total_units = C.B.total_units;
  args.aptr = reinterpret_cast<u32*>(w + C.B.off_aptr);
  args.bptr = reinterpret_cast<u32*>(w + C.B.off_bptr);
  args.kmask = (1ull << C.S) - 1ull;
  args.uprob = reinterpret_cast<const u32*>(w + C.B.off_uprob);
  return run_batch_product(args, C.B, w, count, c_keys, c_vals, d_c_off, s);
}

}  // extern "C"
