// Dense mode permutation: the copy that puts a dense operand's modes in
// lattice order before a product (latticeCopy, FunctionUtil.h:195, and
// DenseMIA::inplace_permute, DenseMIA.h:700-780: output mode k is input mode
// perm[k], both column-major).
//
// Two kernels, both one read and one write per element (HBM-bound):
//   permute_rows_kernel  perm[0] == 0: the fastest mode stays fastest, so
//                        every run along it is copied contiguously;
//   permute_tile_kernel  otherwise: 32 x 32 tiles over input mode 0 (fastest
//                        in the input) and input mode perm[0] (fastest in the
//                        output) are transposed through shared memory, so
//                        reads and writes are both coalesced; the other modes
//                        index the tiles.
#include <algorithm>

#include "lnt_common.cuh"

namespace lnt {
namespace {

constexpr int kPT = 32;  // tile edge

struct PermParams {
  int nb;                        // batch modes: every mode but input mode 0 and input mode perm[0]
  u64 d0, db;                    // extents of input mode 0 and of input mode b = perm[0]
  u64 in_sb, out_s0;             // input stride of mode b; output stride of input mode 0
  Divider bdim[LNT_MAX_ORDER];   // batch mode extents, input order
  u64 bin[LNT_MAX_ORDER];        // their input strides
  u64 bout[LNT_MAX_ORDER];       // their output strides
};

__device__ __forceinline__ void batch_offsets(u64 batch, const PermParams& P, u64& in_off, u64& out_off) {
  in_off = 0;
  out_off = 0;
  for (int m = 0; m < P.nb; ++m) {
    const u64 q = divide(batch, P.bdim[m]);
    const u64 c = batch - q * P.bdim[m].d;
    in_off += c * P.bin[m];
    out_off += c * P.bout[m];
    batch = q;
  }
}

__global__ void permute_rows_kernel(const double* __restrict__ in, double* __restrict__ out, PermParams P,
                                    u64 nbatch) {
  const u64 chunks = (P.d0 + 1023) / 1024;
  for (u64 job = blockIdx.x; job < nbatch * chunks; job += gridDim.x) {
    const u64 batch = job / chunks;
    const u64 x0 = (job - batch * chunks) * 1024;
    u64 io, oo;
    batch_offsets(batch, P, io, oo);
    for (u64 x = x0 + threadIdx.x; x < min(P.d0, x0 + 1024); x += blockDim.x) out[oo + x] = __ldcs(in + io + x);
  }
}

__global__ void permute_tile_kernel(const double* __restrict__ in, double* __restrict__ out, PermParams P,
                                    u64 nbatch) {
  __shared__ double tile[kPT][kPT + 1];
  const u64 tx = (P.d0 + kPT - 1) / kPT, ty = (P.db + kPT - 1) / kPT;
  const u64 per_batch = tx * ty;
  for (u64 job = blockIdx.x; job < nbatch * per_batch; job += gridDim.x) {
    const u64 batch = job / per_batch;
    const u64 r = job - batch * per_batch;
    const u64 x0 = (r % tx) * kPT, y0 = (r / tx) * kPT;
    u64 io, oo;
    batch_offsets(batch, P, io, oo);
    __syncthreads();  // the previous tile is written out
    for (int yy = threadIdx.y; yy < kPT; yy += blockDim.y) {  // read along input mode 0
      const u64 x = x0 + threadIdx.x, y = y0 + yy;
      if (x < P.d0 && y < P.db) tile[yy][threadIdx.x] = __ldcs(in + io + x + y * P.in_sb);
    }
    __syncthreads();
    for (int xx = threadIdx.y; xx < kPT; xx += blockDim.y) {  // write along output mode 0 (input mode b)
      const u64 y = y0 + threadIdx.x, x = x0 + xx;
      if (x < P.d0 && y < P.db) out[oo + y + x * P.out_s0] = tile[threadIdx.x][xx];
    }
  }
}

int grid_for(u64 jobs) { return (int)std::max<u64>(1, std::min<u64>(jobs, (u64)sm_count() * 16)); }

}  // namespace
}  // namespace lnt

using namespace lnt;

extern "C" {

int lnt_dense_permute(const double* in, double* out, int order, const int64_t* dims, const int32_t* perm,
                      void* stream) {
  if (order < 1 || order > LNT_MAX_ORDER || !dims || !perm) return LNT_BAD_ARG;
  bool seen[LNT_MAX_ORDER] = {false};
  int inv[LNT_MAX_ORDER];
  for (int k = 0; k < order; ++k) {
    if (perm[k] < 0 || perm[k] >= order || seen[perm[k]]) return LNT_BAD_SEQ;
    seen[perm[k]] = true;
    inv[perm[k]] = k;
  }
  unsigned __int128 total = 1;
  u64 s_in[LNT_MAX_ORDER], s_out[LNT_MAX_ORDER];
  for (int k = 0; k < order; ++k) {
    if (dims[k] <= 0) return LNT_BAD_DIMS;
    s_in[k] = (u64)total;
    total *= (u64)dims[k];
    if (total >> 63) return LNT_OVERFLOW_KEYBITS;
  }
  {
    u64 s = 1;
    for (int k = 0; k < order; ++k) {
      s_out[k] = s;
      s *= (u64)dims[perm[k]];
    }
  }
  if (!in || !out) return LNT_BAD_ARG;
  const u64 n = (u64)total;
  if ((in < out + n) && (out < in + n)) return LNT_BAD_ARG;  // must not overlap
  cudaStream_t st = as_stream(stream);
  bool identity = true;
  for (int k = 0; k < order; ++k) identity = identity && perm[k] == k;
  if (identity)
    return cudaMemcpyAsync(out, in, n * 8, cudaMemcpyDeviceToDevice, st) == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
  PermParams P{};
  const int b = perm[0];
  P.d0 = (u64)dims[0];
  P.db = (u64)dims[b];
  P.in_sb = s_in[b];
  P.out_s0 = s_out[inv[0]];
  u64 nbatch = 1;
  for (int m = 0; m < order; ++m) {
    if (m == 0 || m == b) continue;
    P.bdim[P.nb] = make_divider((u64)dims[m]);
    P.bin[P.nb] = s_in[m];
    P.bout[P.nb] = s_out[inv[m]];
    ++P.nb;
    nbatch *= (u64)dims[m];
  }
  ProfScope prof("dense_permute", st);
  if (b == 0) {  // mode 0 stays fastest: the batch is every other mode
    permute_rows_kernel<<<grid_for(nbatch * ((P.d0 + 1023) / 1024)), 256, 0, st>>>(in, out, P, nbatch);
  } else {
    const u64 tiles = ((P.d0 + kPT - 1) / kPT) * ((P.db + kPT - 1) / kPT);
    permute_tile_kernel<<<grid_for(nbatch * tiles), dim3(kPT, 8), 0, st>>>(in, out, P, nbatch);
  }
  count_launch();
  return launch_status();
}

}  // extern "C"
