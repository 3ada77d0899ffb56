// Mixed sparse / dense lattice products, the operations of the mex gateway
// SparseDenseLatticeMultMex (MATLAB/mex/sparse_denselattice_mul.cpp):
//   dense x sparse: DenseLatticeBase::operator*(SparseLatticeBase)
//                   (DenseLatticeBase.h:436-500);
//   sparse x dense: SparseLatticeBase::operator*(DenseLatticeBase)
//                   (SparseLatticeBase.h:1148-1162), which the reference
//                   evaluates as (B^T * A^T)^T through the former.
// Both emit one full dense line of C per non-empty line of the sparse
// operand.  The sparse operand's sorted keys split into segments of equal
// g = key / W (W = its contracted extent); segment g yields Q outputs
//   C[q + Q g] = sum over the segment's entries (key, v), in key order, of
//                v * M[q + Q (key mod W + W tab(g))],   q < Q,
// with M the dense operand laid out with the output dimension fastest:
//   dense x sparse: M = A (h x w x d, column-major), Q = h, tab(g) = g / wB;
//   sparse x dense: M = B^T per tab (B transposed into the workspace), Q = wB,
//                   tab(g) = g / h; the keys are the reference's row-major
//                   lattice keys j + wB (row + h tab).
// Pipeline: count (segment heads -> scan -> segment table), [transpose],
// product.  Product: one CTA job per (chunk of 512 output rows, segment),
// chunk-major, 256 threads x 2 outputs; the segment's entries are staged in
// shared memory 256 at a time and every output accumulates acc = acc + v * m
// with a separate multiply and add (the reference's c += b * a, not
// contracted) in key order, so results are bit-exact.  Bound by the gather of
// M: 8 B of M per (entry, output) from L2 (chunk-major jobs keep 512 rows of M
// resident), 16 B written per output.
#include <algorithm>

#include "lnt_scan.cuh"

namespace lnt {
namespace {

constexpr int kMT = 256;            // product CTA threads
constexpr int kMQ = 2;              // outputs per thread
constexpr int kMChunk = kMT * kMQ;  // outputs per CTA job
constexpr int kTT = 32;             // transpose tile

struct SegHead {
  const u64* keys;
  Divider wd;
  __device__ __forceinline__ u64 operator()(size_t i) const {
    return (i == 0 || divide(keys[i], wd) != divide(keys[i - 1], wd)) ? 1ull : 0ull;
  }
};

__global__ void seg_table_kernel(SegHead head, u64 n, const unsigned long long* __restrict__ pos, u64 q,
                                 u64* __restrict__ seg_start, u64* __restrict__ seg_g, u64* __restrict__ d_count) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    if (!head(i)) continue;
    seg_start[pos[i]] = i;
    seg_g[pos[i]] = divide(head.keys[i], head.wd);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    seg_start[pos[n]] = n;  // pos[n] = number of segments
    if (d_count) *d_count = pos[n] * q;
  }
}

// BT[j + wB (c + w t)] = B[c + w (j + wB t)]
__global__ void transpose_tabs_kernel(const double* __restrict__ B, double* __restrict__ BT, u64 w, u64 wB, u64 d) {
  __shared__ double tile[kTT][kTT + 1];
  const u64 tc = (w + kTT - 1) / kTT, tj = (wB + kTT - 1) / kTT;
  const u64 ntiles = tc * tj * d;
  for (u64 x = blockIdx.x; x < ntiles; x += gridDim.x) {
    const u64 t = x / (tc * tj), r = x - t * tc * tj;
    const u64 c0 = (r % tc) * kTT, j0 = (r / tc) * kTT;
    const double* Bt = B + w * wB * t;
    double* BTt = BT + w * wB * t;
    __syncthreads();
    for (int yy = threadIdx.y; yy < kTT; yy += blockDim.y) {  // read: c fastest
      const u64 c = c0 + threadIdx.x, j = j0 + yy;
      if (c < w && j < wB) tile[yy][threadIdx.x] = Bt[c + w * j];
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < kTT; yy += blockDim.y) {  // write: j fastest
      const u64 j = j0 + threadIdx.x, c = c0 + yy;
      if (c < w && j < wB) BTt[j + wB * c] = tile[threadIdx.x][yy];
    }
  }
}

__global__ void __launch_bounds__(kMT) mixed_product_kernel(const u64* __restrict__ keys,
                                                            const double* __restrict__ vals,
                                                            const u64* __restrict__ seg_start,
                                                            const u64* __restrict__ seg_g,
                                                            const unsigned long long* __restrict__ d_nseg, u64 chunks,
                                                            const double* __restrict__ M, u64 Q, Divider wd,
                                                            Divider td, u64 tabs, u64* __restrict__ ck,
                                                            double* __restrict__ cv) {
  __shared__ u64 s_inner[kMT];
  __shared__ double s_v[kMT];
  const int tid = threadIdx.x;
  // chunk-major: the CTAs in flight share one chunk of the output rows, so the
  // dense operand's working set is kMChunk rows of it, which stays in L2
  const u64 nseg = *d_nseg;
  const u64 jobs = nseg * chunks;
  for (u64 job = blockIdx.x; job < jobs; job += gridDim.x) {
    const u64 chunk = job / nseg;
    const u64 s = job - chunk * nseg;
    const u64 q0 = chunk * kMChunk;
    const u64 g = seg_g[s], t = divide(g, td);
    const u64 lo = seg_start[s], hi = t < tabs ? seg_start[s + 1] : lo;  // keys past the last tab add nothing
    const double* Mt = M + Q * wd.d * (t < tabs ? t : 0);
    double acc[kMQ];
#pragma unroll
    for (int r = 0; r < kMQ; ++r) acc[r] = 0.0;
    for (u64 base = lo; base < hi; base += kMT) {
      const u32 nb = (u32)min((u64)kMT, hi - base);
      __syncthreads();  // the previous batch is consumed
      if ((u32)tid < nb) {
        const u64 k = keys[base + tid];
        s_inner[tid] = k - divide(k, wd) * wd.d;
        s_v[tid] = vals[base + tid];
      }
      __syncthreads();
#pragma unroll 4
      for (u32 e = 0; e < nb; ++e) {
        const double v = s_v[e];
        const double* col = Mt + Q * s_inner[e];
#pragma unroll
        for (int r = 0; r < kMQ; ++r) {
          const u64 q = q0 + tid + r * kMT;
          if (q < Q) acc[r] = __dadd_rn(acc[r], __dmul_rn(v, col[q]));
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kMQ; ++r) {
      const u64 q = q0 + tid + r * kMT;
      if (q < Q) {
        ck[s * Q + q] = q + Q * g;
        cv[s * Q + q] = acc[r];
      }
    }
  }
}

struct MixedShape {
  u64 W, Q, segs_per_tab, tabs;
  bool dense_first;
};

int mixed_shape(const lnt_lattice* S, int64_t other, int dense_first, MixedShape* m) {
  if (!S || other <= 0 || S->rows <= 0 || S->cols <= 0 || S->tabs <= 0) return LNT_BAD_DIMS;
  if (S->nnz && (!S->keys || !S->vals)) return LNT_BAD_ARG;
  const unsigned __int128 in = (unsigned __int128)(u64)S->rows * (u64)S->cols * (u64)S->tabs;
  if (in >> 63) return LNT_OVERFLOW_KEYBITS;
  m->dense_first = dense_first != 0;
  m->tabs = (u64)S->tabs;
  if (m->dense_first) {  // A (other x rows x tabs) * S (rows x cols x tabs), S column-major
    m->W = (u64)S->rows;
    m->Q = (u64)other;
    m->segs_per_tab = (u64)S->cols;
  } else {  // S (rows x cols x tabs, row-major keys) * B (cols x other x tabs)
    m->W = (u64)S->cols;
    m->Q = (u64)other;
    m->segs_per_tab = (u64)S->rows;
  }
  const unsigned __int128 out = (unsigned __int128)m->Q * m->segs_per_tab * m->tabs;
  if (out >> 63) return LNT_OVERFLOW_KEYBITS;
  return LNT_OK;
}

struct MixedLayout {
  size_t pos, seg_start, seg_g, scan, bt, total;
};

MixedLayout mixed_layout(const MixedShape& m, size_t n) {
  MixedLayout L;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align_up(std::max<size_t>(bytes, 8), 256);
    return o;
  };
  L.pos = take((n + 1) * 8);
  L.seg_start = take((n + 1) * 8);
  L.seg_g = take(n * 8);
  L.scan = take(scan::workspace_bytes(n));
  L.bt = m.dense_first ? take(0) : take(m.W * m.Q * m.tabs * 8);
  L.total = off;
  return L;
}

int grid_for(u64 work, int per_sm) {
  const u64 want = std::max<u64>(1, work);
  return (int)std::min<u64>(want, (u64)sm_count() * per_sm);
}

}  // namespace
}  // namespace lnt

using namespace lnt;

extern "C" {

int lnt_sparse_dense_mult_workspace(const lnt_lattice* S, int64_t other, int dense_first, size_t* bytes) {
  if (!bytes) return LNT_BAD_ARG;
  MixedShape m;
  const int st = mixed_shape(S, other, dense_first, &m);
  if (st != LNT_OK) return st;
  *bytes = mixed_layout(m, S->nnz).total;
  return LNT_OK;
}

int lnt_sparse_dense_mult_count(const lnt_lattice* S, int64_t other, int dense_first, void* workspace,
                                size_t workspace_bytes, uint64_t* d_count, void* stream) {
  MixedShape m;
  int st = mixed_shape(S, other, dense_first, &m);
  if (st != LNT_OK) return st;
  if (!d_count) return LNT_BAD_ARG;
  const size_t n = S->nnz;
  const MixedLayout L = mixed_layout(m, n);
  if (!workspace || workspace_bytes < L.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  cudaStream_t s = as_stream(stream);
  unsigned char* W = static_cast<unsigned char*>(workspace);
  unsigned long long* pos = reinterpret_cast<unsigned long long*>(W + L.pos);
  SegHead head{(const u64*)S->keys, make_divider(m.W)};
  st = scan::run(head, n, pos, nullptr, W + L.scan, s, "mixed_count");
  if (st != LNT_OK) return st;
  {
    ProfScope prof("mixed_count", s);
    seg_table_kernel<<<grid_for((n + 255) / 256, 8), 256, 0, s>>>(head, n, pos, m.Q,
                                                                   reinterpret_cast<u64*>(W + L.seg_start),
                                                                   reinterpret_cast<u64*>(W + L.seg_g),
                                                                   (u64*)d_count);
    count_launch();
  }
  return launch_status();
}

int lnt_sparse_dense_mult(const double* D, const lnt_lattice* S, int64_t other, int dense_first, void* workspace,
                          size_t workspace_bytes, uint64_t* c_keys, double* c_vals, void* stream) {
  MixedShape m;
  int st = mixed_shape(S, other, dense_first, &m);
  if (st != LNT_OK) return st;
  const size_t n = S->nnz;
  if (n == 0) return LNT_OK;
  if (!D || !c_keys || !c_vals) return LNT_BAD_ARG;
  const MixedLayout L = mixed_layout(m, n);
  if (!workspace || workspace_bytes < L.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  cudaStream_t s = as_stream(stream);
  unsigned char* W = static_cast<unsigned char*>(workspace);
  const double* M = D;
  if (!m.dense_first) {  // B (W x Q x tabs) -> B^T (Q x W x tabs)
    double* bt = reinterpret_cast<double*>(W + L.bt);
    const u64 tiles = ((m.W + kTT - 1) / kTT) * ((m.Q + kTT - 1) / kTT) * m.tabs;
    ProfScope prof("mixed_transpose", s);
    transpose_tabs_kernel<<<grid_for(tiles, 16), dim3(kTT, 8), 0, s>>>(D, bt, m.W, m.Q, m.tabs);
    count_launch();
    M = bt;
  }
  {
    const u64 chunks = (m.Q + kMChunk - 1) / kMChunk;
    ProfScope prof("mixed_product", s);
    mixed_product_kernel<<<grid_for(n * chunks, 8), kMT, 0, s>>>(
        (const u64*)S->keys, S->vals, reinterpret_cast<const u64*>(W + L.seg_start),
        reinterpret_cast<const u64*>(W + L.seg_g), reinterpret_cast<const unsigned long long*>(W + L.pos) + n, chunks,
        M, m.Q, make_divider(m.W), make_divider(m.segs_per_tab), m.tabs, (u64*)c_keys, c_vals);
    count_launch();
  }
  return launch_status();
}

}  // extern "C"
