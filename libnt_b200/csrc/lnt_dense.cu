// Dense lattice product C(:,:,t) = A(:,:,t) * B(:,:,t), column-major float64
// (the reference's DenseLatticeBase::operator*, DenseLatticeBase.h:404-430: an
// Eigen GEMM per tab), three ways:
//
// lnt_dense_lattice_mult_fp64: plain FP64 GEMM per tab (cuBLASLt DGEMM), the
// comparator of the emulated products.
//
// lnt_dense_lattice_mult_crt (scheme II below): the products on the INT8
// tensor cores through this library's own tcgen05 GEMM (lnt_modgemm.cu).
//
// lnt_dense_lattice_mult_split: error-free splitting onto the integer tensor
// cores (its INT8 GEMMs are cuBLASLt library GEMMs) (Ozaki, Ogita, Oishi, Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59 (2012), scheme I with integer slices):
//   1. each row of A and each column of B is scaled by a power of two so its
//      largest magnitude lies in [1/4, 1/2);
//   2. every scaled entry x is split into s signed 7-bit digits,
//      x = sum_p d_p 2^(-7(p+1)) + r, |d_p| <= 64, |r| <= 2^(-7s-1), all steps
//      exact in float64 (x*128 - rint(x*128) is exact);
//   3. the digit products d_p(A) d_q(B) are exact INT8 x INT8 -> INT32 tensor
//      core products; all (p, q) with p + q = L are one GEMM over a K axis of
//      (L+1) blocks (the slices of A are laid out [A_0|A_1|..] and those of B
//      [B_{s-1}|..|B_0] along K, so each level reads a contiguous prefix /
//      suffix); terms with p + q >= s lie below the kept precision and are
//      dropped;
//   4. one fused pass sums the s INT32 level results in float64 from the least
//      significant level up, with Neumaier compensation, and applies the row
//      and column scales.
// With s = 7 (49 bits per operand) the error is about 2^-48 |A||B|
// componentwise.  |d_p d_q| <= 2^12 and K' <= s*K keeps INT32 exact for
// K <= 2^31 / (2^12 s) (74,898 at s = 7).
#include <cublasLt.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "lnt_common.cuh"

namespace lnt {

int run_mod_gemm(const signed char* ra, const signed char* rb, int nmod, const int* moduli, u64 Mp, u64 Np, u64 Kp,
                 unsigned char* out, cudaStream_t s);

namespace {

constexpr int kDigitBits = 7;

// ---- per-device cuBLASLt handle -------------------------------------------
cublasLtHandle_t lt_handle() {
  static std::mutex mu;
  static cublasLtHandle_t handles[64] = {nullptr};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> g(mu);
  if (dev < 0 || dev >= 64) return nullptr;
  if (!handles[dev]) cublasLtCreate(&handles[dev]);
  return handles[dev];
}

// ---- scaling exponents ----------------------------------------------------
// eA[i]: A row i's scale exponent (entries * 2^-eA lie in [-1/2, 1/2]).
__global__ void row_exp_kernel(const double* __restrict__ A, u64 h, u64 w, int* __restrict__ eA) {
  const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= h) return;
  double m = 0.0;
  for (u64 k = 0; k < w; ++k) m = fmax(m, fabs(A[i + h * k]));
  int e = 0;
  if (m > 0.0) frexp(m, &e);  // m = f 2^e, f in [1/2, 1)
  eA[i] = m > 0.0 ? e + 1 : 0;
}

// eB[j]: B column j's scale exponent; one warp per column.
__global__ void col_exp_kernel(const double* __restrict__ B, u64 w, u64 wB, int* __restrict__ eB) {
  const u64 j = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= wB) return;
  double m = 0.0;
  for (u64 k = lane; k < w; k += 32) m = fmax(m, fabs(B[k + w * j]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) {
    int e = 0;
    if (m > 0.0) frexp(m, &e);
    eB[j] = m > 0.0 ? e + 1 : 0;
  }
}

// Splits x (already scaled into [-1/2, 1/2]) into s signed 7-bit digits.
__device__ __forceinline__ void split_digits(double x, int s, signed char* out, size_t stride) {
  for (int p = 0; p < s; ++p) {
    x *= 128.0;
    const double d = rint(x);
    x -= d;
    out[(size_t)p * stride] = (signed char)(int)d;
  }
}

// A (h x w col-major) -> Acat: h rows of s*Kp int8, slice p at columns [p*Kp, p*Kp + w).
// 32x32 tiles through shared memory: read coalesced along rows, write along K.
__global__ void split_a_kernel(const double* __restrict__ A, u64 h, u64 w, u64 Kp, int s,
                               const int* __restrict__ eA, signed char* __restrict__ Acat) {
  __shared__ double tile[32][33];
  const u64 i0 = (u64)blockIdx.x * 32, k0 = (u64)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const u64 i = i0 + tx, k = k0 + r;
    tile[r][tx] = (i < h && k < w) ? A[i + h * k] : 0.0;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const u64 i = i0 + r, k = k0 + tx;
    if (i < h && k < w) {
      const double x = ldexp(tile[tx][r], -eA[i]);
      split_digits(x, s, Acat + i * (u64)s * Kp + k, Kp);
    }
  }
}

// B (w x wB col-major) -> Bcat: wB rows of s*Kp int8, slice q at columns [(s-1-q)*Kp, ...).
__global__ void split_b_kernel(const double* __restrict__ B, u64 w, u64 wB, u64 Kp, int s,
                               const int* __restrict__ eB, signed char* __restrict__ Bcat) {
  const u64 total = w * wB;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
    const u64 j = t / w, k = t - j * w;
    const double x = ldexp(B[t], -eB[j]);
    signed char* row = Bcat + j * (u64)s * Kp;
    double y = x;
    for (int q = 0; q < s; ++q) {
      y *= 128.0;
      const double d = rint(y);
      y -= d;
      row[(u64)(s - 1 - q) * Kp + k] = (signed char)(int)d;
    }
  }
}

// C[i + h j] = 2^(eA_i + eB_j) * sum_L 2^(-7(L+2)) lev[L][i + Mp j], summed
// from the least significant level with Neumaier compensation.
__global__ void recombine_kernel(const int* __restrict__ lev, u64 Mp, u64 Np, int s, u64 h, u64 wB,
                                 const int* __restrict__ eA, const int* __restrict__ eB, double* __restrict__ C) {
  const u64 stride = (u64)gridDim.x * blockDim.x;
  const u64 mn = h * wB, plane = Mp * Np;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < mn; t += stride) {
    const u64 j = t / h, i = t - j * h;
    const u64 src = i + Mp * j;
    double sum = 0.0, comp = 0.0;
    for (int L = s - 1; L >= 0; --L) {
      const double term = ldexp((double)lev[(u64)L * plane + src], -kDigitBits * (L + 2));
      const double y = sum + term;
      comp += fabs(sum) >= fabs(term) ? (sum - y) + term : (term - y) + sum;
      sum = y;
    }
    C[t] = ldexp(sum + comp, eA[i] + eB[j]);
  }
}

// The integer GEMMs run on M, N, K padded to multiples of 16 (the INT8
// tensor-core GEMM needs 16-byte aligned leading dimensions); padding rows and
// columns of the slice operands are zero.
struct SplitLayout {
  u64 Kp, Mp, Np;
  size_t off_ea, off_eb, off_acat, off_bcat, off_lev, off_lt, lt_bytes, total;
};

SplitLayout split_layout(u64 h, u64 w, u64 wB, int s) {
  SplitLayout L;
  L.Kp = (w + 15) / 16 * 16;
  L.Mp = (h + 15) / 16 * 16;
  L.Np = (wB + 15) / 16 * 16;
  size_t off = 0;
  L.off_ea = off;
  off += align_up(h * 4, 256);
  L.off_eb = off;
  off += align_up(wB * 4, 256);
  L.off_acat = off;
  off += align_up(L.Mp * (u64)s * L.Kp, 256);
  L.off_bcat = off;
  off += align_up(L.Np * (u64)s * L.Kp, 256);
  L.off_lev = off;
  off += align_up((u64)s * L.Mp * L.Np * 4, 256);
  L.lt_bytes = 64ull << 20;
  L.off_lt = off;
  off += L.lt_bytes;
  L.total = off;
  return L;
}

int lt_int8_gemm(const signed char* A, int lda, const signed char* B, int ldb, int* C, u64 m, u64 n, u64 k,
                 void* ltws, size_t ltws_bytes, cudaStream_t s) {
  cublasLtHandle_t h = lt_handle();
  if (!h) return LNT_DEVICE_ERROR;
  cublasLtMatmulDesc_t op = nullptr;
  cublasLtMatrixLayout_t la = nullptr, lb = nullptr, lc = nullptr;
  cublasLtMatmulPreference_t pref = nullptr;
  int st = LNT_DEVICE_ERROR;
  do {
    if (cublasLtMatmulDescCreate(&op, CUBLAS_COMPUTE_32I, CUDA_R_32I) != CUBLAS_STATUS_SUCCESS) break;
    cublasOperation_t ta = CUBLAS_OP_T, tb = CUBLAS_OP_N;
    cublasLtMatmulDescSetAttribute(op, CUBLASLT_MATMUL_DESC_TRANSA, &ta, sizeof(ta));
    cublasLtMatmulDescSetAttribute(op, CUBLASLT_MATMUL_DESC_TRANSB, &tb, sizeof(tb));
    // A stored K x M (K-major rows of A), B stored K x N (K-major columns), C M x N
    if (cublasLtMatrixLayoutCreate(&la, CUDA_R_8I, k, m, lda) != CUBLAS_STATUS_SUCCESS) break;
    if (cublasLtMatrixLayoutCreate(&lb, CUDA_R_8I, k, n, ldb) != CUBLAS_STATUS_SUCCESS) break;
    if (cublasLtMatrixLayoutCreate(&lc, CUDA_R_32I, m, n, m) != CUBLAS_STATUS_SUCCESS) break;
    if (cublasLtMatmulPreferenceCreate(&pref) != CUBLAS_STATUS_SUCCESS) break;
    cublasLtMatmulPreferenceSetAttribute(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES, &ltws_bytes,
                                         sizeof(ltws_bytes));
    cublasLtMatmulHeuristicResult_t res;
    int found = 0;
    if (cublasLtMatmulAlgoGetHeuristic(h, op, la, lb, lc, lc, pref, 1, &res, &found) != CUBLAS_STATUS_SUCCESS ||
        !found) {
      st = LNT_UNSUPPORTED;
      break;
    }
    const int alpha = 1, beta = 0;
    ProfScope prof("dense_int8_gemm", s);
    if (cublasLtMatmul(h, op, &alpha, A, la, B, lb, &beta, C, lc, C, lc, &res.algo, ltws, ltws_bytes, s) !=
        CUBLAS_STATUS_SUCCESS)
      break;
    st = LNT_OK;
  } while (false);
  if (pref) cublasLtMatmulPreferenceDestroy(pref);
  if (lc) cublasLtMatrixLayoutDestroy(lc);
  if (lb) cublasLtMatrixLayoutDestroy(lb);
  if (la) cublasLtMatrixLayoutDestroy(la);
  if (op) cublasLtMatmulDescDestroy(op);
  return st;
}

int lt_dgemm(const double* A, const double* B, double* C, u64 m, u64 n, u64 k, void* ltws, size_t ltws_bytes,
             cudaStream_t s) {
  cublasLtHandle_t h = lt_handle();
  if (!h) return LNT_DEVICE_ERROR;
  cublasLtMatmulDesc_t op = nullptr;
  cublasLtMatrixLayout_t la = nullptr, lb = nullptr, lc = nullptr;
  cublasLtMatmulPreference_t pref = nullptr;
  int st = LNT_DEVICE_ERROR;
  do {
    if (cublasLtMatmulDescCreate(&op, CUBLAS_COMPUTE_64F, CUDA_R_64F) != CUBLAS_STATUS_SUCCESS) break;
    if (cublasLtMatrixLayoutCreate(&la, CUDA_R_64F, m, k, m) != CUBLAS_STATUS_SUCCESS) break;
    if (cublasLtMatrixLayoutCreate(&lb, CUDA_R_64F, k, n, k) != CUBLAS_STATUS_SUCCESS) break;
    if (cublasLtMatrixLayoutCreate(&lc, CUDA_R_64F, m, n, m) != CUBLAS_STATUS_SUCCESS) break;
    if (cublasLtMatmulPreferenceCreate(&pref) != CUBLAS_STATUS_SUCCESS) break;
    cublasLtMatmulPreferenceSetAttribute(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES, &ltws_bytes,
                                         sizeof(ltws_bytes));
    cublasLtMatmulHeuristicResult_t res;
    int found = 0;
    if (cublasLtMatmulAlgoGetHeuristic(h, op, la, lb, lc, lc, pref, 1, &res, &found) != CUBLAS_STATUS_SUCCESS ||
        !found) {
      st = LNT_UNSUPPORTED;
      break;
    }
    const double alpha = 1.0, beta = 0.0;
    ProfScope prof("dense_dgemm", s);
    if (cublasLtMatmul(h, op, &alpha, A, la, B, lb, &beta, C, lc, C, lc, &res.algo, ltws, ltws_bytes, s) !=
        CUBLAS_STATUS_SUCCESS)
      break;
    st = LNT_OK;
  } while (false);
  if (pref) cublasLtMatmulPreferenceDestroy(pref);
  if (lc) cublasLtMatrixLayoutDestroy(lc);
  if (lb) cublasLtMatrixLayoutDestroy(lb);
  if (la) cublasLtMatrixLayoutDestroy(la);
  if (op) cublasLtMatmulDescDestroy(op);
  return st;
}


// ===========================================================================
// Scheme II: integer moduli and Chinese remaindering (Ozaki, Uchino, Imamura,
// "Ozaki Scheme II: A GEMM-oriented emulation of floating-point matrix
// multiplication using an integer modular technique", 2024).
//   1. rows of A / columns of B are scaled by powers of two and rounded to
//      integers A', B' of at most beta bits (|A'| <= 2^(beta-1));
//   2. for each modulus m_l (pairwise coprime, <= 256) the symmetric residues
//      A' mod m_l, B' mod m_l fit INT8 and P_l = (A' mod m_l)(B' mod m_l) is an
//      exact INT8 tensor-core GEMM with INT32 accumulation (|P_l| <= 2^14 K),
//      run by the hand-written tcgen05 kernel of lnt_modgemm.cu, whose
//      epilogue stores only r_l = P_l mod m_l (one byte per entry);
//   3. per entry, X = sum_l r_l (M/m_l) ((M/m_l)^-1 mod m_l) reduced modulo M
//      into (-M/2, M/2] in exact integer limbs is A'B', as long as
//      |A'B'| < M/2 (M = prod m_l), which fixes beta:
//      2 beta <= log2 M - log2 K - 3.
// The error is the rounding of A and B to beta bits: about 2^(2-beta) |A||B|
// componentwise; N moduli give beta = floor((log2 M - log2 K - 3) / 2).
// ===========================================================================
constexpr int kMaxModuli = 20;
constexpr int kMaxLimbs = 6;  // 6 x 27 bits > log2 of the product of 20 moduli
// pairwise coprime, all <= 256 so symmetric residues fit in int8
constexpr int kModuli[kMaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                     223, 217, 211, 199, 197, 193, 191, 181, 179, 173};

struct CrtParams {
  int n;        // moduli used
  int beta;     // integer bits of A' and B'
  int m[kMaxModuli];
  double md[kMaxModuli];        // m_l as a double
  int u[kMaxModuli];            // (M/m_l)^-1 mod m_l
  double rinv_hi[kMaxModuli];   // 1/m_l as a double-double
  double rinv_lo[kMaxModuli];
  float rinv_f[kMaxModuli];     // 1/m_l in float
  double M_hi, M_lo;            // M as a double-double
  // exact remaindering: X = sum_l p_l V_l (mod M), V_l = (M/m_l) u_l < M, in
  // kLimbBits-bit limbs; M in the same limbs; 1/M for the quotient estimate
  int lv;                       // limbs of M
  u32 V[kMaxModuli][kMaxLimbs];
  u32 Ml[kMaxLimbs];
  double Minv;
};
constexpr int kLimbBits = 27;  // n * 2^31 * 2^27 < 2^63 for n <= 20 moduli

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// x mod m in [0, m) for an integer-valued double |x| < 2^56 and m <= 256:
// q = floor(x / m) is off by at most one, and fma(-q, m, x) is exact because
// the true remainder is a small integer.
__device__ __forceinline__ double dmod(double x, double m, double inv_m) {
  const double q = floor(x * inv_m);
  double r = fma(-q, m, x);
  if (r < 0.0) r += m;
  else if (r >= m) r -= m;
  return r;
}

// Same for an integer-valued float below 2^24.
__device__ __forceinline__ float fmod_small(float x, float m, float inv_m) {
  const float q = floorf(x * inv_m);
  float r = fmaf(-q, m, x);
  if (r < 0.f) r += m;
  else if (r >= m) r -= m;
  return r;
}

// 2^e as a double, exact for normal exponents (bit pattern built directly).
__device__ __forceinline__ double pow2(int e) {
  if (e >= -1022 && e <= 1023) return __longlong_as_double((long long)(1023 + e) << 52);
  return ldexp(1.0, e);
}

// x * 2^e, exact (two factors keep intermediate values normal).
__device__ __forceinline__ double scale2(double x, int e) {
  const int e1 = e / 2;
  return (x * pow2(e1)) * pow2(e - e1);
}

// A residue of the integer-valued double x (|x| <= 2^51, i.e. beta <= 52)
// modulo m_l, as a byte: q = x / m rounded to nearest by adding 1.5 * 2^52
// (exact integer spacing), r = x - q m exact by fma, and the low word of
// r + 1.5 * 2^52 is r as an int.  1/m rounded to double errs by 2^-53
// relatively, so x / m is off by at most 1/(4m) and |r| <= m/2 + 1/4: for odd
// m <= 255 that is |r| <= 127, for m = 256 |r| <= 128, and the byte of 128 is
// -128, congruent modulo 256.  Every modulus's byte is therefore an int8
// congruent to x, which is all the modular products need.
__device__ __forceinline__ int sym_res(double x, int l, const CrtParams& P) {
  constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
  const double q = fma(x, P.rinv_hi[l], kRound) - kRound;
  const double r = fma(-q, P.md[l], x);
  return __double2loint(r + kRound);
}

// Per-row maximum exponent of A (col-major) over a chunk of columns; eA must
// start below every double exponent (-4096; an all-zero row keeps it).  e = E + 1 for the row maximum f 2^E, f in [1/2, 1).
__global__ void row_exp_chunk_kernel(const double* __restrict__ A, u64 h, u64 w, u64 kchunk,
                                     int* __restrict__ eA) {
  const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= h) return;
  const u64 k0 = (u64)blockIdx.y * kchunk, k1 = min(w, k0 + kchunk);
  double m = 0.0;
  for (u64 k = k0; k < k1; ++k) m = fmax(m, fabs(A[i + h * k]));
  if (m > 0.0) {
    int e;
    frexp(m, &e);
    atomicMax(&eA[i], e + 1);
  }
}

__global__ void fill_int_kernel(int* __restrict__ p, u64 n, int v) {
  const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// Four residues (of four consecutive K entries) packed into one 32-bit word.
__device__ __forceinline__ u32 pack_res4(const double (&x)[4], int l, const CrtParams& P) {
  const u32 lo = __byte_perm((u32)sym_res(x[0], l, P), (u32)sym_res(x[1], l, P), 0x0040);
  const u32 hi = __byte_perm((u32)sym_res(x[2], l, P), (u32)sym_res(x[3], l, P), 0x0040);
  return __byte_perm(lo, hi, 0x5410);  // bytes x0, x1, x2, x3
}

// A (h x w col-major) -> residues res[l]: Mp rows of Kp int8 (row-major, K
// contiguous).  Tile of 32 rows x 128 columns through shared memory: read
// along rows (coalesced); each lane then turns four consecutive K entries of a
// row into one 4-byte word per modulus (a warp stores 128 consecutive bytes).
__global__ void __launch_bounds__(256) residue_a_kernel(const double* __restrict__ A, u64 h, u64 w, u64 Mp, u64 Kp,
                                                        const int* __restrict__ eA, CrtParams P,
                                                        signed char* __restrict__ res) {
  __shared__ double tile[32][129];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const u64 i0 = (u64)blockIdx.x * 32, k0 = (u64)blockIdx.y * 128;
  for (int kk = warp; kk < 128; kk += 8) {
    const u64 i = i0 + lane, k = k0 + kk;
    tile[lane][kk] = (i < h && k < w) ? A[i + h * k] : 0.0;
  }
  __syncthreads();
  const u64 k = k0 + 4 * lane;  // Kp is a multiple of 16, so k < Kp keeps all four in the row
  if (k >= Kp) return;
  for (int rr = warp; rr < 32; rr += 8) {
    const u64 i = i0 + rr;
    if (i >= h) continue;
    const int sc = P.beta - eA[i];
    double x[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) x[c] = rint(scale2(tile[rr][4 * lane + c], sc));
    u32* dst = reinterpret_cast<u32*>(res + i * Kp + k);
    const u64 plane = Mp * Kp / 4;
#pragma unroll
    for (int l = 0; l < kMaxModuli; ++l) {  // compile-time l: the moduli tables are direct constant operands
      if (l >= P.n) break;
      dst[(u64)l * plane] = pack_res4(x, l, P);
    }
  }
}

// B (w x wB col-major) -> residues res[l]: Np rows (columns of B) of Kp int8.
// Grid: y over columns of B, x over groups of four K entries (one 4-byte word
// per modulus; entries beyond w are zero).
__global__ void residue_b_kernel(const double* __restrict__ B, u64 w, u64 wB, u64 Np, u64 Kp,
                                 const int* __restrict__ eB, CrtParams P, signed char* __restrict__ res) {
  const u64 plane = Np * Kp / 4;
  for (u64 j = blockIdx.y; j < wB; j += gridDim.y) {
    const int sc = P.beta - eB[j];
    const double* col = B + w * j;
    u32* dst = reinterpret_cast<u32*>(res + j * Kp);
    for (u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x; 4 * g < Kp; g += (u64)gridDim.x * blockDim.x) {
      double x[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) x[c] = 4 * g + c < w ? rint(scale2(col[4 * g + c], sc)) : 0.0;
#pragma unroll
      for (int l = 0; l < kMaxModuli; ++l) {
        if (l >= P.n) break;
        dst[(u64)l * plane + g] = pack_res4(x, l, P);
      }
    }
  }
}

// Chinese remaindering of the residues r_l = (A'B' mod m_l) in [0, m_l), exact
// in integers, scaled back to float64.  Per entry: T = sum_l r_l V_l as LV+1
// signed 64-bit limb sums (27-bit limbs; r_l < 2^8, so each sum stays far
// below 2^63), carried into normalised limbs; q = round(T / M) from a double
// estimate, exact because A'B' = T - q M satisfies |A'B'| <= M/32 (the choice
// of beta) while the estimate errs by under 2^-15; X = T - q M in limbs,
// converted to double once (Horner from the top limb).  Each thread takes four
// consecutive rows (one 4-byte load per modulus); grid x over rows of C, y
// over columns.  (Unrolling the modulus loop to its compile-time bound, so
// that the moduli tables become direct constant operands, measured slower at
// 13 moduli: 5.35 against 4.69 ms at 16384^2.)
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

template <int LV>
__global__ void __launch_bounds__(256) crt_kernel(const unsigned char* __restrict__ res, u64 Mp, u64 Np, u64 h,
                                                  u64 wB, CrtParams P, const int* __restrict__ eA,
                                                  const int* __restrict__ eB, double* __restrict__ C) {
  const u64 i0 = ((u64)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i0 >= h) return;  // Mp is a multiple of 16: rows i0 .. i0+3 lie inside every plane
  const u64 plane = Mp * Np;
  int ea[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) ea[c] = i0 + c < h ? eA[i0 + c] - 2 * P.beta : 0;
  constexpr long long kMask = (1ll << kLimbBits) - 1;
  constexpr double kRadix = (double)(1ll << kLimbBits);
  const u64 w0 = i0 - 4 * (threadIdx.x & 31);  // the warp's first row: 128 rows, <= 128 bytes per plane
  for (u64 j = blockIdx.y; j < wB; j += gridDim.y) {
    // the next column's residue lines (one or two per plane) into L1 while
    // this column accumulates: the loads below otherwise wait on DRAM
    const u64 jn = j + gridDim.y;
    if (jn < wB) {
      for (int t = threadIdx.x & 31; t < 2 * P.n; t += 32) {
        const u64 r = (t & 1) && w0 + 127 < Mp ? w0 + 127 : w0;
        prefetch_l1(res + (u64)(t >> 1) * plane + r + Mp * jn);
      }
    }
    long long acc[4][LV + 1];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int b = 0; b <= LV; ++b) acc[c][b] = 0;
    const unsigned char* src = res + i0 + Mp * j;
    // (loading four moduli's words before using any measured slower: 72
    // registers instead of 60 cost a quarter of the resident warps)
#pragma unroll 2
    for (int l = 0; l < P.n; ++l) {
      const u32 w4 = __ldcs(reinterpret_cast<const u32*>(src + (u64)l * plane));
#pragma unroll
      for (int b = 0; b < LV; ++b) {
        const u32 v = P.V[l][b];
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[c][b] += (long long)((w4 >> (8 * c)) & 0xffu) * v;
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (i0 + c >= h) break;
      long long* a = acc[c];
#pragma unroll
      for (int b = 0; b < LV; ++b) {  // normalise: limbs in [0, 2^27), the top one signed
        const long long cy = a[b] >> kLimbBits;
        a[b] &= kMask;
        a[b + 1] += cy;
      }
      double td = (double)a[LV];
#pragma unroll
      for (int b = LV - 1; b >= 0; --b) td = fma(td, kRadix, (double)a[b]);
      const long long q = __double2ll_rn(td * P.Minv);
      const int qlo = (int)(q & kMask), qhi = (int)(q >> kLimbBits);  // |q| < 2^36
#pragma unroll
      for (int b = 0; b < LV; ++b) {
        a[b] -= (long long)qlo * (int)P.Ml[b];
        a[b + 1] -= (long long)qhi * (int)P.Ml[b];
      }
#pragma unroll
      for (int b = 0; b < LV; ++b) {
        const long long cy = a[b] >> kLimbBits;
        a[b] &= kMask;
        a[b + 1] += cy;
      }
      double x = (double)a[LV];
#pragma unroll
      for (int b = LV - 1; b >= 0; --b) x = fma(x, kRadix, (double)a[b]);
      C[i0 + c + h * j] = scale2(x, ea[c] + eB[j]);
    }
  }
}

// ---- choosing the number of moduli ------------------------------------------
// The rounding of A and B to beta-bit integers per row / column bounds the
// error of entry (i, j) by about 2^(1-beta) (max_k |a_ik| sum_k |b_kj| +
// sum_k |a_ik| max_k |b_kj|), so relative to (|A||B|)_ij it grows with the
// ratio of each row's (column's) largest magnitude to its mean magnitude.
// These kernels find the largest such ratio over the rows of A and the
// columns of B (all-zero rows and columns excluded).

// Per-row max |a| (as ordered bit patterns) and sum |a| over a chunk of columns.
__global__ void row_absstat_kernel(const double* __restrict__ A, u64 h, u64 w, u64 kchunk,
                                   unsigned long long* __restrict__ rmax, double* __restrict__ rsum) {
  const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= h) return;
  const u64 k0 = (u64)blockIdx.y * kchunk, k1 = min(w, k0 + kchunk);
  double m = 0.0, sm = 0.0;
  for (u64 k = k0; k < k1; ++k) {
    const double x = fabs(A[i + h * k]);
    m = fmax(m, x);
    sm += x;
  }
  atomicMax(&rmax[i], (unsigned long long)__double_as_longlong(m));  // non-negative: bit order = value order
  atomicAdd(&rsum[i], sm);
}

__global__ void row_ratio_kernel(const unsigned long long* __restrict__ rmax, const double* __restrict__ rsum, u64 h,
                                 u64 w, unsigned long long* __restrict__ out) {
  const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= h || !(rsum[i] > 0.0)) return;
  const double r = __longlong_as_double((long long)rmax[i]) * (double)w / rsum[i];
  atomicMax(out, (unsigned long long)__double_as_longlong(r));
}

// One warp per column of B (w x wB, col-major): max / mean of |b|.
__global__ void col_ratio_kernel(const double* __restrict__ B, u64 w, u64 wB, unsigned long long* __restrict__ out) {
  const u64 j = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= wB) return;
  double m = 0.0, sm = 0.0;
  for (u64 k = lane; k < w; k += 32) {
    const double x = fabs(B[k + w * j]);
    m = fmax(m, x);
    sm += x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    sm += __shfl_xor_sync(0xffffffffu, sm, o);
  }
  if (lane == 0 && sm > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m * (double)w / sm));
}

struct CrtLayout {
  u64 Kp, Mp, Np;
  size_t off_ea, off_eb, off_ra, off_rb, off_prod, total;
};

CrtLayout crt_layout(u64 h, u64 w, u64 wB, int n) {
  CrtLayout L;
  L.Kp = (w + 15) / 16 * 16;
  L.Mp = (h + 15) / 16 * 16;
  L.Np = (wB + 15) / 16 * 16;
  size_t off = 0;
  L.off_ea = off;
  off += align_up(h * 4, 256);
  L.off_eb = off;
  off += align_up(wB * 4, 256);
  L.off_ra = off;
  off += align_up((u64)n * L.Mp * L.Kp, 256);
  L.off_rb = off;
  off += align_up((u64)n * L.Np * L.Kp, 256);
  L.off_prod = off;  // residues of the products: n planes of Mp x Np bytes
  off += align_up((u64)n * L.Mp * L.Np, 256);
  L.total = off;
  return L;
}

// Host: moduli tables for n moduli and inner dimension K.
int make_crt_params(int n, u64 K, CrtParams* P) {
  if (n < 2 || n > kMaxModuli) return LNT_BAD_ARG;
  P->n = n;
  double log2M = 0.0;
  for (int l = 0; l < n; ++l) {
    P->m[l] = kModuli[l];
    P->md[l] = (double)kModuli[l];
    log2M += std::log2((double)kModuli[l]);
  }
  const int beta = (int)std::floor((log2M - std::log2((double)K) - 3.0) / 2.0);
  if (beta < 8) return LNT_UNSUPPORTED;
  // |A'|, |B'| <= 2^51: exact doubles, and symmetric residues that fit int8
  // without a range correction (sym_res)
  P->beta = std::min(beta, 52);
  for (int l = 0; l < n; ++l) {
    const int m = P->m[l];
    long long rest = 1;  // (M / m) mod m
    for (int q = 0; q < n; ++q)
      if (q != l) rest = rest * (P->m[q] % m) % m;
    int inv = 0;  // modular inverse by search (m <= 256)
    for (int x = 1; x < m; ++x)
      if (rest * x % m == 1) {
        inv = x;
        break;
      }
    if (!inv) return LNT_BAD_ARG;
    P->u[l] = inv;
    P->rinv_hi[l] = 1.0 / m;
    P->rinv_lo[l] = std::fma(-P->rinv_hi[l], (double)m, 1.0) / m;
    P->rinv_f[l] = 1.0f / (float)m;
  }
  // V_l = (M / m_l) u_l and M in 27-bit limbs (little-endian), 1/M as a double
  {
    constexpr int NL = kMaxLimbs + 1;
    const u64 mask = (1ull << kLimbBits) - 1;
    u64 Mb[NL] = {1};
    double Md = 1.0;
    for (int l = 0; l < n; ++l) {  // M *= m_l
      u64 carry = 0;
      for (int b = 0; b < NL; ++b) {
        const u64 t = Mb[b] * (u64)P->m[l] + carry;
        Mb[b] = t & mask;
        carry = t >> kLimbBits;
      }
      Md *= (double)P->m[l];
    }
    if (Mb[NL - 1] != 0) return LNT_UNSUPPORTED;
    P->lv = 0;
    for (int b = 0; b < kMaxLimbs; ++b) {
      P->Ml[b] = (u32)Mb[b];
      if (Mb[b]) P->lv = b + 1;
    }
    for (int l = 0; l < n; ++l) {
      u64 Q[NL] = {0};  // M / m_l: long division from the top limb
      u64 rem = 0;
      for (int b = NL - 1; b >= 0; --b) {
        const u64 cur = (rem << kLimbBits) | Mb[b];
        Q[b] = cur / (u64)P->m[l];
        rem = cur % (u64)P->m[l];
      }
      if (rem) return LNT_BAD_ARG;
      u64 carry = 0;  // V_l = Q u_l < M
      for (int b = 0; b < kMaxLimbs; ++b) {
        const u64 t = Q[b] * (u64)P->u[l] + carry;
        P->V[l][b] = (u32)(t & mask);
        carry = t >> kLimbBits;
      }
      if (carry) return LNT_BAD_ARG;
    }
    for (int l = n; l < kMaxModuli; ++l)
      for (int b = 0; b < kMaxLimbs; ++b) P->V[l][b] = 0;
    P->Minv = 1.0 / Md;
  }
  // M as a double-double (products of small integers, exact residual by fma)
  double mh = 1.0, ml = 0.0;
  for (int l = 0; l < n; ++l) {
    const double m = (double)P->m[l];
    const double ph = mh * m;
    const double pl = std::fma(mh, m, -ph) + ml * m;
    mh = ph + pl;
    ml = pl - (mh - ph);
  }
  P->M_hi = mh;
  P->M_lo = ml;
  return LNT_OK;
}

int check_dense(int64_t h, int64_t w, int64_t wB, int64_t d) {
  if (h <= 0 || w <= 0 || wB <= 0 || d <= 0) return LNT_BAD_DIMS;
  if (h > (1ll << 31) || w > (1ll << 31) || wB > (1ll << 31)) return LNT_UNSUPPORTED;
  return LNT_OK;
}

}  // namespace
}  // namespace lnt

using namespace lnt;

extern "C" {

int lnt_dense_split_workspace(int64_t h, int64_t w, int64_t wB, int slices, size_t* bytes) {
  int st = check_dense(h, w, wB, 1);
  if (st != LNT_OK) return st;
  if (!bytes || slices < 1 || slices > 8) return LNT_BAD_ARG;
  const u64 Kp = ((u64)w + 15) / 16 * 16;
  if ((u64)slices * Kp * 4096ull >= (1ull << 31)) return LNT_UNSUPPORTED;  // INT32 exactness bound
  *bytes = split_layout(h, w, wB, slices).total;
  return LNT_OK;
}

int lnt_dense_lattice_mult_split(const double* A, const double* B, double* C, int64_t h, int64_t w, int64_t wB,
                                 int64_t d, int slices, void* workspace, size_t workspace_bytes, void* stream) {
  int st = check_dense(h, w, wB, d);
  if (st != LNT_OK) return st;
  if (!A || !B || !C) return LNT_BAD_ARG;
  size_t need = 0;
  st = lnt_dense_split_workspace(h, w, wB, slices, &need);
  if (st != LNT_OK) return st;
  if (!workspace || workspace_bytes < need || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  const SplitLayout L = split_layout(h, w, wB, slices);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  int* eA = reinterpret_cast<int*>(ws + L.off_ea);
  int* eB = reinterpret_cast<int*>(ws + L.off_eb);
  signed char* Acat = reinterpret_cast<signed char*>(ws + L.off_acat);
  signed char* Bcat = reinterpret_cast<signed char*>(ws + L.off_bcat);
  int* lev = reinterpret_cast<int*>(ws + L.off_lev);
  cudaStream_t s = as_stream(stream);
  const int sms = sm_count();
  const u64 uh = h, uw = w, uwB = wB, Kp = L.Kp;
  for (int64_t t = 0; t < d; ++t) {
    const double* At = A + (u64)t * uh * uw;
    const double* Bt = B + (u64)t * uw * uwB;
    double* Ct = C + (u64)t * uh * uwB;
    {
      ProfScope prof("dense_split", s);
      row_exp_kernel<<<(unsigned)((uh + 255) / 256), 256, 0, s>>>(At, uh, uw, eA);
      col_exp_kernel<<<(unsigned)((uwB * 32 + 255) / 256), 256, 0, s>>>(Bt, uw, uwB, eB);
      if (Kp != uw || L.Mp != uh || L.Np != uwB) {  // zero every padding row and column
        if (cudaMemsetAsync(Acat, 0, L.Mp * (u64)slices * Kp, s) != cudaSuccess) return LNT_DEVICE_ERROR;
        if (cudaMemsetAsync(Bcat, 0, L.Np * (u64)slices * Kp, s) != cudaSuccess) return LNT_DEVICE_ERROR;
      }
      split_a_kernel<<<dim3((unsigned)((uh + 31) / 32), (unsigned)((uw + 31) / 32)), dim3(32, 8), 0, s>>>(
          At, uh, uw, Kp, slices, eA, Acat);
      split_b_kernel<<<sms * 16, 256, 0, s>>>(Bt, uw, uwB, Kp, slices, eB, Bcat);
      count_launch(4);
    }
    const int ld = (int)((u64)slices * Kp);
    for (int lvl = 0; lvl < slices; ++lvl) {
      // sum over p + q = lvl: A blocks [0, lvl], B blocks [slices-1-lvl, slices-1]
      st = lt_int8_gemm(Acat, ld, Bcat + (u64)(slices - 1 - lvl) * Kp, ld, lev + (u64)lvl * L.Mp * L.Np, L.Mp, L.Np,
                        (u64)(lvl + 1) * Kp, ws + L.off_lt, L.lt_bytes, s);
      if (st != LNT_OK) return st;
      count_launch();
    }
    {
      ProfScope prof("dense_recombine", s);
      recombine_kernel<<<sms * 16, 256, 0, s>>>(lev, L.Mp, L.Np, slices, uh, uwB, eA, eB, Ct);
      count_launch();
    }
  }
  return launch_status();
}


int lnt_dense_crt_moduli(const double* A, const double* B, int64_t h, int64_t w, int64_t wB, int64_t d, double tol,
                         void* workspace, size_t workspace_bytes, int* moduli, void* stream) {
  int st = check_dense(h, w, wB, d);
  if (st != LNT_OK) return st;
  if (!A || !B || !moduli || !(tol > 0.0)) return LNT_BAD_ARG;
  const size_t need = align_up((size_t)h * 8, 256) * 2 + 256;
  if (!workspace || workspace_bytes < need || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  auto* rmax = reinterpret_cast<unsigned long long*>(ws);
  auto* rsum = reinterpret_cast<double*>(ws + align_up((size_t)h * 8, 256));
  auto* out = reinterpret_cast<unsigned long long*>(ws + 2 * align_up((size_t)h * 8, 256));
  cudaStream_t s = as_stream(stream);
  const u64 uh = h, uw = w, uwB = wB, kchunk = 256;
  if (cudaMemsetAsync(out, 0, 8, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  for (int64_t t = 0; t < d; ++t) {
    if (cudaMemsetAsync(ws, 0, 2 * align_up((size_t)h * 8, 256), s) != cudaSuccess) return LNT_DEVICE_ERROR;
    row_absstat_kernel<<<dim3((unsigned)((uh + 255) / 256), (unsigned)((uw + kchunk - 1) / kchunk)), 256, 0, s>>>(
        A + (u64)t * uh * uw, uh, uw, kchunk, rmax, rsum);
    row_ratio_kernel<<<(unsigned)((uh + 255) / 256), 256, 0, s>>>(rmax, rsum, uh, uw, out);
    col_ratio_kernel<<<(unsigned)((uwB * 32 + 255) / 256), 256, 0, s>>>(B + (u64)t * uw * uwB, uw, uwB, out);
    count_launch(3);
  }
  unsigned long long bits = 0;
  if (cudaMemcpyAsync(&bits, out, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return LNT_DEVICE_ERROR;
  if (cudaStreamSynchronize(s) != cudaSuccess) return LNT_DEVICE_ERROR;
  double ratio = 0.0;
  std::memcpy(&ratio, &bits, 8);
  // |error_ij| <= 2^(1-beta) (max_k|a_ik| sum_k|b_kj| + sum_k|a_ik| max_k|b_kj|)
  //            <~ 2^(2-beta) R (|A||B|)_ij, with R the largest max / mean ratio
  const double lr = ratio > 1.0 ? std::log2(ratio) : 0.0;
  const int need_beta = (int)std::ceil(2.0 + lr - std::log2(tol));
  for (int n = 2; n <= kMaxModuli; ++n) {
    CrtParams P;
    if (make_crt_params(n, (u64)w, &P) == LNT_OK && P.beta >= std::min(need_beta, 52)) {
      *moduli = n;
      return LNT_OK;
    }
  }
  *moduli = kMaxModuli;
  return LNT_OK;
}

int lnt_dense_crt_workspace(int64_t h, int64_t w, int64_t wB, int moduli, size_t* bytes) {
  int st = check_dense(h, w, wB, 1);
  if (st != LNT_OK) return st;
  if (!bytes) return LNT_BAD_ARG;
  if ((u64)w >= (1ull << 17)) return LNT_UNSUPPORTED;  // INT32 exactness: K * 2^14 < 2^31
  CrtParams P;
  st = make_crt_params(moduli, (u64)w, &P);
  if (st != LNT_OK) return st;
  *bytes = crt_layout(h, w, wB, moduli).total;
  return LNT_OK;
}

int lnt_dense_lattice_mult_crt(const double* A, const double* B, double* C, int64_t h, int64_t w, int64_t wB,
                               int64_t d, int moduli, void* workspace, size_t workspace_bytes, void* stream) {
  int st = check_dense(h, w, wB, d);
  if (st != LNT_OK) return st;
  if (!A || !B || !C) return LNT_BAD_ARG;
  size_t need = 0;
  st = lnt_dense_crt_workspace(h, w, wB, moduli, &need);
  if (st != LNT_OK) return st;
  if (!workspace || workspace_bytes < need || (uintptr_t)workspace % 256) return LNT_WORKSPACE;
  CrtParams P;
  st = make_crt_params(moduli, (u64)w, &P);
  if (st != LNT_OK) return st;
  const CrtLayout L = crt_layout(h, w, wB, moduli);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  int* eA = reinterpret_cast<int*>(ws + L.off_ea);
  int* eB = reinterpret_cast<int*>(ws + L.off_eb);
  signed char* ra = reinterpret_cast<signed char*>(ws + L.off_ra);
  signed char* rb = reinterpret_cast<signed char*>(ws + L.off_rb);
  unsigned char* prod = ws + L.off_prod;
  cudaStream_t s = as_stream(stream);
  const int sms = sm_count();
  const u64 uh = h, uw = w, uwB = wB, Kp = L.Kp;
  for (int64_t t = 0; t < d; ++t) {
    const double* At = A + (u64)t * uh * uw;
    const double* Bt = B + (u64)t * uw * uwB;
    double* Ct = C + (u64)t * uh * uwB;
    {
      ProfScope prof("dense_residues", s);
      const u64 kchunk = 256;
      fill_int_kernel<<<(unsigned)((uh + 255) / 256), 256, 0, s>>>(eA, uh, -4096);  // below any double exponent
      {
        ProfScope prof_a("dense_exp_a", s);
        row_exp_chunk_kernel<<<dim3((unsigned)((uh + 255) / 256), (unsigned)((uw + kchunk - 1) / kchunk)), 256, 0,
                               s>>>(At, uh, uw, kchunk, eA);
      }
      {
        ProfScope prof_b("dense_exp_b", s);
        col_exp_kernel<<<(unsigned)((uwB * 32 + 255) / 256), 256, 0, s>>>(Bt, uw, uwB, eB);
      }
      if (Kp != uw || L.Mp != uh || L.Np != uwB) {  // zero every padding row and column
        if (cudaMemsetAsync(ra, 0, (u64)moduli * L.Mp * Kp, s) != cudaSuccess) return LNT_DEVICE_ERROR;
        if (cudaMemsetAsync(rb, 0, (u64)moduli * L.Np * Kp, s) != cudaSuccess) return LNT_DEVICE_ERROR;
      }
      {
        ProfScope prof_ra("dense_residue_a", s);
        residue_a_kernel<<<dim3((unsigned)((uh + 31) / 32), (unsigned)((Kp + 127) / 128)), 256, 0, s>>>(
            At, uh, uw, L.Mp, Kp, eA, P, ra);
      }
      const unsigned gx = (unsigned)std::min<u64>((Kp / 4 + 255) / 256, 64);
      const unsigned gyb = (unsigned)std::min<u64>(uwB, std::max<u64>(1, (u64)sms * 64 / gx));
      {
        ProfScope prof_rb("dense_residue_b", s);
        residue_b_kernel<<<dim3(gx, gyb), 256, 0, s>>>(Bt, uw, uwB, L.Np, Kp, eB, P, rb);
      }
      count_launch(5);
    }
    // all moduli's products on the tensor cores, reduced modulo m_l in the epilogue
    st = run_mod_gemm(ra, rb, moduli, P.m, L.Mp, L.Np, Kp, prod, s);
    if (st != LNT_OK) return st;
    {
      ProfScope prof("dense_crt", s);
      const u64 rows4 = (uh + 3) / 4;
      const unsigned gx = (unsigned)((rows4 + 255) / 256);
      const unsigned gy = (unsigned)std::min<u64>(uwB, std::max<u64>(1, (u64)sms * 32 / gx));
      const dim3 grid(gx, gy);
      switch (P.lv) {
        case 1:
        case 2:
        case 3:
        case 4:
          crt_kernel<4><<<grid, 256, 0, s>>>(prod, L.Mp, L.Np, uh, uwB, P, eA, eB, Ct);
          break;
        case 5:
          crt_kernel<5><<<grid, 256, 0, s>>>(prod, L.Mp, L.Np, uh, uwB, P, eA, eB, Ct);
          break;
        default:
          crt_kernel<6><<<grid, 256, 0, s>>>(prod, L.Mp, L.Np, uh, uwB, P, eA, eB, Ct);
          break;
      }
      count_launch();
    }
  }
  return launch_status();
}

int lnt_dense_fp64_workspace(size_t* bytes) {
  if (!bytes) return LNT_BAD_ARG;
  *bytes = 64ull << 20;
  return LNT_OK;
}

int lnt_dense_lattice_mult_fp64(const double* A, const double* B, double* C, int64_t h, int64_t w, int64_t wB,
                                int64_t d, void* workspace, size_t workspace_bytes, void* stream) {
  int st = check_dense(h, w, wB, d);
  if (st != LNT_OK) return st;
  if (!A || !B || !C) return LNT_BAD_ARG;
  if (!workspace || workspace_bytes < (64ull << 20)) return LNT_WORKSPACE;
  cudaStream_t s = as_stream(stream);
  for (int64_t t = 0; t < d; ++t) {
    st = lt_dgemm(A + (u64)t * h * w, B + (u64)t * w * wB, C + (u64)t * h * wB, h, wB, w, workspace,
                  workspace_bytes, s);
    if (st != LNT_OK) return st;
    count_launch();
  }
  return LNT_OK;
}

}  // extern "C"
