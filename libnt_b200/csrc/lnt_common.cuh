// Shared device/host helpers of the LNT CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/lnt.h"

namespace lnt {

typedef unsigned long long u64;
typedef unsigned int u32;

// ---------------------------------------------------------------------------
// Error latch.  A bounded device wait that gives up ORs its code in here and
// returns; the host reads it with lnt_device_status().
// ---------------------------------------------------------------------------
enum DeviceErr : u32 {
  kErrSortLookback = 1u << 0,
  kErrReduceLookback = 1u << 1,
  kErrMergeLookback = 1u << 2,
  kErrSpgemmLookback = 1u << 3,
  kErrBatchedQueue = 1u << 4,
  kErrDenseWait = 1u << 5,
};

// One error word per translation unit (no relocatable device code); each
// unit registers a reader at load time and lnt_device_status() ORs them.
static __device__ u32 g_lnt_device_error = 0;

typedef int (*ErrorReader)(int clear, u32* word);
void register_error_reader(ErrorReader f);

namespace {
inline int read_unit_error(int clear, u32* word) {
  *word = 0;
  if (cudaMemcpyFromSymbol(word, g_lnt_device_error, sizeof(u32)) != cudaSuccess) return LNT_DEVICE_ERROR;
  if (clear && *word) {
    u32 zero = 0;
    if (cudaMemcpyToSymbol(g_lnt_device_error, &zero, sizeof(u32)) != cudaSuccess) return LNT_DEVICE_ERROR;
  }
  return LNT_OK;
}
struct UnitErrorRegistration {
  UnitErrorRegistration() { register_error_reader(&read_unit_error); }
};
static UnitErrorRegistration s_unit_error_registration;
}  // namespace

// Poll budget of every spin-wait on a flag written by another CTA.  Each poll
// is an L2 round trip (~1 us worst case under load), so the default bounds a
// wait at well under a minute while never firing on a live predecessor.  The
// budget is a per-unit device word (like the error word) so that
// lnt_set_spin_limit can shorten it, e.g. to check the expiry path.
constexpr u32 kSpinLimit = 1u << 24;
static __device__ u32 g_lnt_spin_limit = kSpinLimit;

__device__ __forceinline__ u32 spin_limit() { return *reinterpret_cast<volatile u32*>(&g_lnt_spin_limit); }

typedef int (*SpinLimitWriter)(u32 polls);
void register_spin_limit_writer(SpinLimitWriter f);

namespace {
inline int write_unit_spin_limit(u32 polls) {
  return cudaMemcpyToSymbol(g_lnt_spin_limit, &polls, sizeof(u32)) == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
}
struct UnitSpinLimitRegistration {
  UnitSpinLimitRegistration() { register_spin_limit_writer(&write_unit_spin_limit); }
};
static UnitSpinLimitRegistration s_unit_spin_limit_registration;
}  // namespace

__device__ __forceinline__ void latch_error(u32 code) { atomicOr(&g_lnt_device_error, code); }

// Stream-ordered choice between two kernel sequences without a host round
// trip: an earlier kernel on the stream writes a gate word, and a kernel
// given (gate, want) returns at once unless *gate == want.  gate == nullptr
// means "always run".
__device__ __forceinline__ bool gated_off(const u32* gate, u32 want) { return gate && *gate != want; }

// Launch bookkeeping (host side).
void count_launch(int n = 1);

// Brackets one kernel launch with CUDA events when profiling is enabled
// (lnt_profile_enable); otherwise free.  Construct immediately before the
// launch, destroy right after it.
class ProfScope {
 public:
  ProfScope(const char* name, cudaStream_t s);
  ~ProfScope();
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

 private:
  const char* name_;
  cudaStream_t s_;
  void* start_;
};

// Status of the last launch (cudaGetLastError).
int launch_status();

// ---------------------------------------------------------------------------
// Division by a run-time invariant 64-bit divisor by multiply-high
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, section 4).  For d not a power of two:
//   l = ceil(log2 d), m = floor(2^64 (2^l - d) / d) + 1 (< 2^64),
//   q = (t + ((n - t) >> 1)) >> (l - 1),  t = mulhi(m, n)
// exact for every 64-bit n.  Powers of two use a shift.  The reference uses
// libdivide (libdivide.h) for the same purpose; results are identical to '/'.
// ---------------------------------------------------------------------------
struct Divider {
  u64 d;      // divisor
  u64 magic;  // 0 => power of two
  u32 shift;  // log2(d) for powers of two, l-1 otherwise
  u32 pad;
};

inline Divider make_divider(u64 d) {
  Divider r;
  r.d = d;
  r.pad = 0;
  if ((d & (d - 1)) == 0) {  // power of two (d >= 1)
    r.magic = 0;
    r.shift = (u32)__builtin_ctzll(d);
    return r;
  }
  u32 l = 64u - (u32)__builtin_clzll(d - 1);  // ceil(log2 d), 2..64
  u64 diff = (u64)(((unsigned __int128)1 << l) - d);  // 2^l - d < d
  unsigned __int128 num = (unsigned __int128)diff << 64;
  r.magic = (u64)(num / d) + 1ull;
  r.shift = l - 1u;
  return r;
}

__host__ __device__ __forceinline__ u64 mulhi64(u64 a, u64 b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (u64)(((unsigned __int128)a * b) >> 64);
#endif
}

__host__ __device__ __forceinline__ u64 divide(u64 n, const Divider& dv) {
  if (dv.magic == 0) return n >> dv.shift;
  u64 t = mulhi64(dv.magic, n);
  return (t + ((n - t) >> 1)) >> dv.shift;
}

// ---------------------------------------------------------------------------
// Re-keying (mixed-radix decode under the current sequence, encode under the
// new one).  Same arithmetic as create_shuffle_needs + reShuffleLinearIndex
// (IndexUtil.h:480-487, 567-589): for i = order-1 .. 1 take the quotient by
// the cumulative extent of the first i current-order modes, add quotient x
// (new stride of that mode), subtract; finally add the remainder x stride[0].
// ---------------------------------------------------------------------------
struct RekeyParams {
  int order;        // 0 or 1 => identity
  int pow2;         // every extent a power of two: `field` holds the bit-field moves
  Divider acc[LNT_MAX_ORDER];  // cumulative extents, current order
  u64 mult[LNT_MAX_ORDER];     // new stride of the mode at current position i
  u32 field[LNT_MAX_ORDER];    // pow2: source shift | bits << 8 | destination shift << 16
};

// With power-of-two extents the re-key is a permutation of bit fields: the
// mode at current position i occupies `bits` bits at its cumulative-extent
// shift and moves to its new stride's shift.
template <int N>
__host__ __device__ __forceinline__ u64 rekey_fields(u64 k, const RekeyParams& p) {
  u64 out = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const u32 f = p.field[i];
    out |= ((k >> (f & 63u)) & ((1ull << ((f >> 8) & 63u)) - 1ull)) << ((f >> 16) & 63u);
  }
  return out;
}

__host__ __device__ __forceinline__ u64 rekey(u64 k, const RekeyParams& p) {
  if (p.order <= 1) return k;
  if (p.pow2) {
    switch (p.order) {
      case 2: return rekey_fields<2>(k, p);
      case 3: return rekey_fields<3>(k, p);
      case 4: return rekey_fields<4>(k, p);
      case 5: return rekey_fields<5>(k, p);
      case 6: return rekey_fields<6>(k, p);
      default: break;
    }
  }
  u64 out = 0;
#pragma unroll 1
  for (int i = p.order - 1; i >= 1; --i) {
    u64 q = divide(k, p.acc[i]);
    out += q * p.mult[i];
    k -= q * p.acc[i].d;
  }
  return out + k * p.mult[0];
}

// Builds RekeyParams; returns an lnt_status.
int make_rekey_params(int order, const int64_t* dims, const int32_t* cur_seq,
                      const int32_t* new_seq, RekeyParams* out);
int make_rekey_params(const lnt_rekey_spec* spec, RekeyParams* out);

// Number of significant key bits for keys < max_key (ceil(log2(max_key))).
inline int key_bits_for(u64 max_key) {
  if (max_key <= 1) return 0;
  return 64 - __builtin_clzll(max_key - 1);
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs of the current device (cached per device).
int sm_count();

}  // namespace lnt
