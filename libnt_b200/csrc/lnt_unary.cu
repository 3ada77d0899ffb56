// Unary contraction / attraction of a sparse tensor: the reference's
// SparseMIABase::contract_attract (SparseMIABase.h:1913-2053), reached from
// index labels that repeat inside one operand (perform_unary, MIA_Expr.h:
// 690-735), e.g. b(k) = a(i,j,i,j,k) (a double trace) or b(k,!i) =
// a(!i,j,!i,k,j).
//
// Input: keys sorted under [contraction modes, attraction modes, other modes]
// with those modes' extents sdims.  Pipeline:
//   1. map: decode each key's digits (multiply-high division by the extents);
//      a value whose contraction sets disagree becomes 0 (it is not summed);
//      group key g = key / |contraction modes| (equal attraction + other
//      indices);
//   2. fold runs of equal g (the duplicate-collecting kernel, no zero
//      skipping): the reference's inner summation loop;
//   3. keep a group when its attraction sets agree and its sum is not zero
//      (the reference's "if (sum)"), one scan for the output positions, and
//      write key other + |other| * attraction index in the groups' order (the
//      reference's emission order); flag whether those keys never decrease
//      (the result's sorted flag, as push_back maintains it).
#include <algorithm>

#include "lnt_scan.cuh"

namespace lnt {

int run_collect(const u64* keys, const double* vals, size_t n, int skip_zero_heads, u64* out_k, double* out_v,
                u64* d_nout, void* ws, cudaStream_t s);
size_t collect_workspace_bytes(size_t n);

namespace {

struct UnaryParams {
  int order;      // modes in the sorted sequence
  int ncon_sets;  // contraction sets, over the first ncon modes
  int natt_sets;  // attraction sets, over the next natt modes
  int ncon, natt;
  int con_part[LNT_MAX_ORDER];
  int att_part[LNT_MAX_ORDER];
  Divider sd[LNT_MAX_ORDER];  // extents in sorted order
  Divider cdim;               // product of the contraction extents
  Divider afull;              // product of the attraction extents
  u64 other_dim;              // product of the other extents
};

__device__ __forceinline__ void digits_of(u64 k, const Divider* sd, int first, int count, u64* out) {
  for (int q = 0; q < count; ++q) {
    const u64 nk = divide(k, sd[first + q]);
    out[q] = k - nk * sd[first + q].d;
    k = nk;
  }
}

// true when every set of `part` consecutive digits agrees
__device__ __forceinline__ bool sets_agree(const u64* dg, const int* part, int nsets) {
  int s = 0;
  for (int p = 0; p < nsets; ++p) {
    for (int q = s + 1; q < s + part[p]; ++q)
      if (dg[q] != dg[s]) return false;
    s += part[p];
  }
  return true;
}

__global__ void unary_map_kernel(const u64* __restrict__ keys, const double* __restrict__ vals, u64 n,
                                 UnaryParams P, u64* __restrict__ gk, double* __restrict__ gv) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const u64 k = keys[e];
    u64 dg[LNT_MAX_ORDER];
    digits_of(k, P.sd, 0, P.ncon, dg);
    const bool ok = sets_agree(dg, P.con_part, P.ncon_sets);
    gk[e] = divide(k, P.cdim);
    gv[e] = ok ? vals[e] : 0.0;
  }
}

// Output key of folded group i, or ~0 when the group is not kept.
struct KeepKey {
  const u64* ck;
  const double* cv;
  const u64* d_nc;
  UnaryParams P;
  __device__ __forceinline__ u64 key(size_t i) const {
    if (i >= *d_nc || cv[i] == 0.0) return ~0ull;
    const u64 g = ck[i];
    u64 dg[LNT_MAX_ORDER];
    digits_of(g, P.sd, P.ncon, P.natt, dg);
    if (!sets_agree(dg, P.att_part, P.natt_sets)) return ~0ull;
    u64 att = 0, stride = 1;
    int s = 0;
    for (int p = 0; p < P.natt_sets; ++p) {  // sub2ind over the attraction ranges
      att += dg[s] * stride;
      stride *= P.sd[P.ncon + s].d;
      s += P.att_part[p];
    }
    return divide(g, P.afull) + P.other_dim * att;
  }
  __device__ __forceinline__ u64 operator()(size_t i) const { return key(i) != ~0ull ? 1ull : 0ull; }
};

__global__ void unary_write_kernel(KeepKey kk, u64 n, const unsigned long long* __restrict__ pos,
                                   u64* __restrict__ out_k, double* __restrict__ out_v) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const u64 k = kk.key(i);
    if (k == ~0ull) continue;
    out_k[pos[i]] = k;
    out_v[pos[i]] = kk.cv[i];
  }
}

__global__ void unary_sorted_kernel(const u64* __restrict__ out_k, const u64* __restrict__ d_nout,
                                    u32* __restrict__ d_sorted) {
  const u64 m = *d_nout;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x + 1; i < m; i += stride)
    if (out_k[i] < out_k[i - 1]) *d_sorted = 0u;
}

struct UnaryLayout {
  size_t gk, gv, ck, cv, pos, coll, scan, misc, total;
};

UnaryLayout unary_layout(size_t n) {
  UnaryLayout L;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align_up(std::max<size_t>(bytes, 8), 256);
    return o;
  };
  L.gk = take(n * 8);
  L.gv = take(n * 8);
  L.ck = take(n * 8);
  L.cv = take(n * 8);
  L.pos = take((n + 1) * 8);
  L.coll = take(collect_workspace_bytes(n));
  L.scan = take(scan::workspace_bytes(n));
  L.misc = take(256);
  L.total = off;
  return L;
}

int grid_n(u64 work) {
  const u64 want = (work + 255) / 256;
  const u64 cap = (u64)sm_count() * 8;
  return (int)std::max<u64>(1, std::min(want, cap));
}

}  // namespace
}  // namespace lnt

using namespace lnt;

extern "C" {

int lnt_contract_attract_workspace(size_t n, size_t* bytes) {
  if (!bytes) return LNT_BAD_ARG;
  *bytes = unary_layout(n).total;
  return LNT_OK;
}

int lnt_contract_attract(const uint64_t* keys, const double* vals, size_t n, int order, const int64_t* sdims,
                         int ncon_sets, const int* con_part, int natt_sets, const int* att_part, uint64_t* out_keys,
                         double* out_vals, uint64_t* d_nout, uint32_t* d_sorted, void* workspace,
                         size_t workspace_bytes, void* stream) {
  if (order < 1 || order > LNT_MAX_ORDER || !sdims || ncon_sets < 0 || natt_sets < 0 || !d_nout) return LNT_BAD_ARG;
  if ((ncon_sets && !con_part) || (natt_sets && !att_part)) return LNT_BAD_ARG;
  if (n && (!keys || !vals || !out_keys || !out_vals)) return LNT_BAD_ARG;
  UnaryParams P{};
  P.order = order;
  P.ncon_sets = ncon_sets;
  P.natt_sets = natt_sets;
  unsigned __int128 total = 1;
  for (int q = 0; q < order; ++q) {
    if (sdims[q] <= 0) return LNT_BAD_DIMS;
    P.sd[q] = make_divider((u64)sdims[q]);
    total *= (u64)sdims[q];
  }
  if (total >> 63) return LNT_OVERFLOW_KEYBITS;
  int m = 0;
  u64 cd = 1, ad = 1, od = 1;
  for (int p = 0; p < ncon_sets; ++p) {
    if (con_part[p] < 2 || m + con_part[p] > order) return LNT_BAD_ARG;
    for (int q = m; q < m + con_part[p]; ++q) {
      if (sdims[q] != sdims[m]) return LNT_BAD_DIMS;  // a contraction set runs over equal extents
      cd *= (u64)sdims[q];
    }
    P.con_part[p] = con_part[p];
    m += con_part[p];
  }
  P.ncon = m;
  for (int p = 0; p < natt_sets; ++p) {
    if (att_part[p] < 2 || m + att_part[p] > order) return LNT_BAD_ARG;
    for (int q = m; q < m + att_part[p]; ++q) {
      if (sdims[q] != sdims[m]) return LNT_BAD_DIMS;
      ad *= (u64)sdims[q];
    }
    P.att_part[p] = att_part[p];
    m += att_part[p];
  }
  P.natt = m - P.ncon;
  for (int q = m; q < order; ++q) od *= (u64)sdims[q];
  P.cdim = make_divider(cd);
  P.afull = make_divider(ad);
  P.other_dim = od;
  const UnaryLayout L = unary_layout(n);
  if (!workspace || workspace_bytes < L.total || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  cudaStream_t s = as_stream(stream);
  unsigned char* W = static_cast<unsigned char*>(workspace);
  u64* gk = reinterpret_cast<u64*>(W + L.gk);
  double* gv = reinterpret_cast<double*>(W + L.gv);
  u64* ck = reinterpret_cast<u64*>(W + L.ck);
  double* cv = reinterpret_cast<double*>(W + L.cv);
  unsigned long long* pos = reinterpret_cast<unsigned long long*>(W + L.pos);
  u64* d_nc = reinterpret_cast<u64*>(W + L.misc);
  if (d_sorted && cudaMemsetAsync(d_sorted, 0xff, 4, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  if (n == 0) return cudaMemsetAsync(d_nout, 0, 8, s) == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
  {
    ProfScope prof("unary_map", s);
    unary_map_kernel<<<grid_n(n), 256, 0, s>>>((const u64*)keys, vals, n, P, gk, gv);
    count_launch();
  }
  int st = run_collect(gk, gv, n, 0, ck, cv, d_nc, W + L.coll, s);
  if (st != LNT_OK) return st;
  KeepKey kk{ck, cv, d_nc, P};
  st = scan::run(kk, n, pos, (unsigned long long*)d_nout, W + L.scan, s, "unary_scan");
  if (st != LNT_OK) return st;
  {
    ProfScope prof("unary_write", s);
    unary_write_kernel<<<grid_n(n), 256, 0, s>>>(kk, n, pos, (u64*)out_keys, out_vals);
    count_launch();
    if (d_sorted) {
      unary_sorted_kernel<<<grid_n(n), 256, 0, s>>>((const u64*)out_keys, (const u64*)d_nout, d_sorted);
      count_launch();
    }
  }
  return launch_status();
}

}  // extern "C"
