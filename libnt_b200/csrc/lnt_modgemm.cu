// Residue products of the dense contraction's Ozaki scheme II on the 5th
// generation tensor cores (tcgen05), with the reduction modulo m_l fused into
// the epilogue:
//
//     R_l = (A_l * B_l^T) mod m_l,   l = 0 .. nmod-1,
//
// A_l (Mp x Kp) and B_l (Np x Kp) are the INT8 residue planes of the scaled
// operands (K contiguous), R_l is written as uint8 in [0, m_l), column-major
// (i + Mp j), so that the Chinese remaindering reads 1 byte per modulus and
// entry instead of a 4-byte INT32 product.
//
// One persistent CTA per SM walks (modulus, 256 x 256 output tile) pairs:
//   warp 0      TMA producer: per 128-byte K step one 256 x 128 box of A_l and
//               one of B_l (128-byte swizzle, no multicast: every CTA loads its
//               own tiles of this GPU's memory) into a 3-stage ring;
//   warp 1      allocates the 512 TMEM columns; one thread issues
//               tcgen05.mma.kind::i8 (M 128, N 256, K 32; two M blocks share the
//               B tile) with INT32 accumulators in TMEM and commits each stage
//               back to the producer and each finished tile to the epilogue;
//   warps 2-9   epilogue: tcgen05.ld of the accumulators (warp w reads TMEM
//               lanes 32 (w mod 4) ..), r = P mod m_l by float quotients with
//               a correction step, byte stores (a warp writes 32 consecutive
//               rows of a column), then the TMEM is handed back.
// Every mbarrier wait is bounded (a poll count and a time): on expiry the CTA
// latches kErrDenseWait, stops issuing, waits (bounded) for its own copies and
// products in flight, frees its TMEM and returns.
#include <cuda.h>

#include <algorithm>
#include <mutex>

#include "lnt_common.cuh"

namespace lnt {
namespace {

constexpr int kBM = 256;              // output rows per tile (two UMMA M blocks of 128)
constexpr int kBN = 256;              // output columns per tile (UMMA N)
constexpr int kBK = 128;              // K bytes per stage (one 128-byte swizzle row)
constexpr int kStages = 3;
constexpr int kStageA = kBM * kBK;    // 32 KB
constexpr int kStageB = kBN * kBK;    // 32 KB
constexpr int kStageBytes = kStageA + kStageB;
constexpr int kThreads = 320;         // 10 warps
constexpr int kEpiWarps = 8;
constexpr int kTmemCols = 512;        // two 128 x 256 INT32 accumulators
constexpr u32 kWaitPolls = 1u << 26;  // bound of every mbarrier wait: try_wait polls ...
constexpr u64 kWaitNs = 4000000000ull;  // ... and nanoseconds (a tile's main loop takes ~100 us)
constexpr int kGroupN = 8;            // tile raster: 8 output column tiles per band
constexpr size_t kSmemBytes = (size_t)kStages * kStageBytes + 1024 /* alignment */ + 256 /* barriers */;

struct ModGemmArgs {
  u64 Mp, Np, Kp;
  int nmod;
  int tiles_m, tiles_n;
  int mod[24];
  u32 off[24];     // m ceil(2^31 / m): makes a product non-negative without changing its residue
  u64 magic[24];   // floor(2^64 / m) + 1
  unsigned char* out;   // nmod planes of Mp x Np bytes, column-major
};

// ---- PTX wrappers ------------------------------------------------------------
__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(u32 bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(u32 bar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(u32 bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u32 bar, u32 parity) {
  u32 ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ u64 global_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase of parity `parity` of barrier `bar` (try_wait may
// suspend the thread for a while, so the bound is both a poll count and a
// time); gives up early when another role aborted (abort_flag may be null).
// Returns false on expiry or abort; expiry latches kErrDenseWait and raises
// the abort flag.
__device__ __forceinline__ bool mbar_wait(u32 bar, u32 parity, volatile int* abort_flag) {
  u64 t0 = 0;
  for (u32 i = 0; i < kWaitPolls; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 63u) {
      if (abort_flag && *abort_flag) return false;
      const u64 now = global_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > kWaitNs) break;
    }
  }
  latch_error(kErrDenseWait);
  if (abort_flag) *abort_flag = 1;
  return false;
}

__device__ __forceinline__ void tma_load_3d(u32 dst, const CUtensorMap* map, u32 bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(dst), "l"(reinterpret_cast<u64>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle:
// rows 128 bytes apart, 8-row groups 1024 bytes apart (stride byte offset),
// leading byte offset 16 (unused by swizzled K-major layouts), descriptor
// version 1, layout type 2 (128-byte swizzle).  The tile base is 1024-byte
// aligned; a K step inside the swizzle row advances the start address.
__device__ __forceinline__ u64 sw128_desc(u32 saddr) {
  return (u64)((saddr >> 4) & 0x3FFFu) | ((u64)1 << 16) | ((u64)(1024 >> 4) << 32) | ((u64)1 << 46) |
         ((u64)2 << 61);
}

// Instruction descriptor of tcgen05.mma.kind::i8: S32 accumulator (bits 4-5 =
// 2), signed A and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
constexpr u32 kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((u32)(kBN >> 3) << 17) | ((u32)(128 >> 4) << 24);

__device__ __forceinline__ void umma_i8(u32 d_tmem, u64 adesc, u64 bdesc, u32 accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(u32 bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(u32 taddr, u32 (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Tile t of the walk: modulus-major, then bands of kGroupN column tiles, row
// tiles inside a band (CTAs running at the same time share A and B panels).
__device__ __forceinline__ void tile_coords(int t, const ModGemmArgs& a, int& l, int& tm, int& tn) {
  const int per = a.tiles_m * a.tiles_n;
  l = t / per;
  const int u = t - l * per;
  const int band = u / (a.tiles_m * kGroupN);
  const int r = u - band * a.tiles_m * kGroupN;
  const int width = min(kGroupN, a.tiles_n - band * kGroupN);
  tm = r / width;
  tn = band * kGroupN + (r - tm * width);
}

// P mod m in [0, m) for |P| < 2^31 - 2^18 (so Kp < 2^17): u = P + off with
// off = m ceil(2^31 / m) is congruent to P and lies in [0, 2^32); then
// q = floor(u M / 2^64) with M = floor(2^64 / m) + 1 is floor(u / m) exactly,
// since u M / 2^64 exceeds u / m by less than u / 2^64 < 2^-32 < 1/m and the
// fraction of u / m is at most 1 - 1/m (division by an invariant integer,
// Granlund & Montgomery 1994); r = u - q m.
__device__ __forceinline__ u32 mod_small(int p, u32 m, u32 off, u64 magic) {
  const u32 u = (u32)p + off;
  const u32 q = (u32)__umul64hi((u64)u, magic);
  return u - q * m;
}

__global__ void __launch_bounds__(kThreads, 1) mod_gemm_kernel(const __grid_constant__ CUtensorMap map_a,
                                                               const __grid_constant__ CUtensorMap map_b,
                                                               const ModGemmArgs args) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + (size_t)kStages * kStageBytes);
  // bars[0..S): full, [S..2S): empty, [2S]: tmem full, [2S+1]: tmem empty, [2S+2]: drain
  u32* tmem_holder = reinterpret_cast<u32*>(bars + 2 * kStages + 3);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const u32 full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages);
  const u32 tfull = smem_u32(bars + 2 * kStages), tempty = smem_u32(bars + 2 * kStages + 1);
  const u32 drain = smem_u32(bars + 2 * kStages + 2);

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(tfull, 1);
    mbar_init(tempty, kEpiWarps);
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {  // the whole warp: .sync.aligned
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const u32 tmem = *tmem_holder;
  const int total = args.nmod * args.tiles_m * args.tiles_n;
  const int nk = (int)((args.Kp + kBK - 1) / kBK);

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int s = 0;
      u32 ph = 0;
      int issued[kStages] = {0};     // a copy was issued into the stage and not yet seen complete
      u32 issued_ph[kStages] = {0};  // the full-barrier phase that copy completes
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
        int l, tm, tn;
        tile_coords(t, args, l, tm, tn);
        for (int kb = 0; kb < nk; ++kb) {
          if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, abort_flag)) {
            ok = false;
            break;
          }
          issued[s] = 0;  // the MMA released it, so its previous copy completed
          const u32 fb = full0 + 8 * s;
          mbar_expect_tx(fb, kStageBytes);
          const u32 sa = smem_u32(smem + (size_t)s * kStageBytes);
          tma_load_3d(sa, &map_a, fb, kb * kBK, tm * kBM, l);
          tma_load_3d(sa + kStageA, &map_b, fb, kb * kBK, tn * kBN, l);
          issued[s] = 1;
          issued_ph[s] = ph;
          if (++s == kStages) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
      if (!ok) {  // stopped early: let this CTA's copies land before it exits
        for (int q = 0; q < kStages; ++q)
          if (issued[q]) mbar_wait(full0 + 8 * q, issued_ph[q], nullptr);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      int s = 0;
      u32 ph = 0;
      int it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < total && ok; t += gridDim.x, ++it) {
        if (it > 0) {  // the epilogue has read the previous tile's accumulators
          if (!mbar_wait(tempty, (u32)((it - 1) & 1), abort_flag)) break;
          tc_fence_after();
        }
        for (int kb = 0; kb < nk; ++kb) {
          if (!mbar_wait(full0 + 8 * s, ph, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const u32 sa = smem_u32(smem + (size_t)s * kStageBytes);
          const u32 sb = sa + kStageA;
#pragma unroll
          for (int kk = 0; kk < kBK / 32; ++kk) {
            const u32 acc = (kb > 0 || kk > 0) ? 1u : 0u;
            const u64 bdesc = sw128_desc(sb + 32 * kk);
            umma_i8(tmem, sw128_desc(sa + 32 * kk), bdesc, acc);
            umma_i8(tmem + kBN, sw128_desc(sa + 128 * kBK + 32 * kk), bdesc, acc);
          }
          umma_commit(empty0 + 8 * s);  // the stage is free once these products are done
          if (++s == kStages) {
            s = 0;
            ph ^= 1u;
          }
        }
        if (!ok) break;
        umma_commit(tfull);  // accumulators complete
      }
      // every product this thread issued has completed before the TMEM is freed
      // (on a normal exit the epilogue already waited for them)
      umma_commit(drain);
      mbar_wait(drain, 0, nullptr);
    }
  } else {
    // ---------------- epilogue ----------------
    const int q = warp & 3;             // TMEM lane quarter this warp may read
    const int half = (warp - 2) >> 2;   // column half of the tile
    int it = 0;
    for (int t = blockIdx.x; t < total; t += gridDim.x, ++it) {
      int l, tm, tn;
      tile_coords(t, args, l, tm, tn);
      // one lane waits, the warp follows its answer (tcgen05.ld needs the whole warp)
      const int got = lane == 0 ? (int)mbar_wait(tfull, (u32)(it & 1), abort_flag) : 0;
      if (!__shfl_sync(0xffffffffu, got, 0)) break;
      tc_fence_after();
      const u32 m = (u32)args.mod[l], off = args.off[l];
      const u64 magic = args.magic[l];
      unsigned char* plane = args.out + (size_t)l * args.Mp * args.Np;
#pragma unroll 1
      for (int mb = 0; mb < 2; ++mb) {
        const u64 row = (u64)tm * kBM + mb * 128 + q * 32 + lane;
#pragma unroll 1
        for (int cc = 0; cc < 4; ++cc) {
          const int c0 = half * 128 + cc * 32;
          u32 v[32];
          tmem_ld32(tmem + ((u32)(q * 32) << 16) + (u32)(mb * kBN + c0), v);
          const u64 col0 = (u64)tn * kBN + c0;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const u64 col = col0 + j;
            if (row < args.Mp && col < args.Np) plane[row + args.Mp * col] = (unsigned char)mod_small((int)v[j], m, off, magic);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tempty);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ---- host: tensor maps -------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// 3-D map over nmod planes of `rows` x Kp bytes (K contiguous), box 128 x 256 x 1.
bool make_plane_map(CUtensorMap* map, const void* base, u64 Kp, u64 rows, int nmod) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[3] = {Kp, rows, (cuuint64_t)nmod};
  const cuuint64_t strides[2] = {Kp, Kp * rows};
  const cuuint32_t box[3] = {(cuuint32_t)kBK, 256u, 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// The residue GEMMs of scheme II (see the file comment).  ra: nmod planes of
// Mp x Kp int8, rb: nmod planes of Np x Kp int8 (both 16-byte aligned, Kp a
// multiple of 16), out: nmod planes of Mp x Np uint8.  Returns an lnt_status.
int run_mod_gemm(const signed char* ra, const signed char* rb, int nmod, const int* moduli, u64 Mp, u64 Np, u64 Kp,
                 unsigned char* out, cudaStream_t s) {
  if (nmod < 1 || nmod > 24 || Kp % 16 || (uintptr_t)ra % 16 || (uintptr_t)rb % 16) return LNT_BAD_ARG;
  if (Kp >= (1ull << 17)) return LNT_UNSUPPORTED;  // |P| <= Kp 2^14 < 2^31
  ModGemmArgs a;
  a.Mp = Mp;
  a.Np = Np;
  a.Kp = Kp;
  a.nmod = nmod;
  a.tiles_m = (int)((Mp + kBM - 1) / kBM);
  a.tiles_n = (int)((Np + kBN - 1) / kBN);
  for (int l = 0; l < 24; ++l) {
    a.mod[l] = l < nmod ? moduli[l] : 1;
    const u64 m = (u64)a.mod[l];
    a.off[l] = (u32)(m * (((1ull << 31) + m - 1) / m));
    a.magic[l] = (u64)(~0ull / m) + (m == 1 ? 0ull : 1ull);  // floor(2^64 / m) + 1 (m = 1: any q works)
  }
  a.out = out;
  CUtensorMap ma, mb;
  if (!make_plane_map(&ma, ra, Kp, Mp, nmod) || !make_plane_map(&mb, rb, Kp, Np, nmod)) return LNT_DEVICE_ERROR;
  if (cudaFuncSetAttribute(mod_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes) !=
      cudaSuccess)
    return LNT_DEVICE_ERROR;
  const long long tiles = (long long)nmod * a.tiles_m * a.tiles_n;
  if (tiles >= (1ll << 31)) return LNT_UNSUPPORTED;
  const int grid = (int)std::min<long long>(tiles, sm_count());
  ProfScope prof("dense_mod_gemm", s);
  mod_gemm_kernel<<<grid, kThreads, kSmemBytes, s>>>(ma, mb, a);
  count_launch();
  return launch_status();
}

}  // namespace lnt
