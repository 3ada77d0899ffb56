// lnt_sort_pairs_noalloc: the pair sort of lnt_sort_pairs for callers that
// cannot allocate device memory.
//
// Who needs it: code that must not call cudaMalloc / cudaFree or any
// allocating library routine -- a latency-critical loop that cannot afford
// the device-wide synchronisation cudaFree (and at times cudaMalloc) implies,
// or a host environment (a plugin or foreign-function binding) that has no
// device allocator of its own from which to hand us a workspace.
//
// How: the sort's scratch (digit histograms, look-back states, one ping-pong
// pair buffer) lives in one file-scope __device__ array of fixed size, so the
// call needs only the caller's input and output buffers.  The array is
// created with the module on every device that loads this library and stays
// there until the process exits.  Limits and rules:
//   * at most LNT_SORT_NOALLOC_MAX_PAIRS pairs; larger requests return
//     LNT_UNSUPPORTED without touching the device;
//   * output ranges must not overlap the input ranges or each other
//     (LNT_BAD_ARG otherwise);
//   * every call on a device shares the one array and leaves its contents
//     behind; the control region that must start at zero is cleared by each
//     call on its stream, but two calls whose GPU work overlaps (different
//     streams, or several host threads) race on the array -- keep all calls
//     on a device ordered, e.g. on one stream;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and caches it; make that
//     first call before any stream capture.
#include <mutex>

#include "lnt_sort.cuh"

namespace lnt {
namespace {

// Room for the control block of any compiled sort variant at the maximum
// pair count and 64-bit keys, plus one ping-pong pair buffer.
constexpr size_t kNoAllocPairs = LNT_SORT_NOALLOC_MAX_PAIRS;
constexpr size_t kNoAllocCtrlBytes = 2u << 20;
constexpr size_t kNoAllocBytes = kNoAllocCtrlBytes + 2 * kNoAllocPairs * 8;

// Control block of a variant at the maximum pair count and 64-bit keys, laid
// out as make_sort_plan does (histograms, bin starts, look-back states per
// pass and tile, counters; each region 256-byte aligned).  Checked at compile
// time for every compiled variant, so a wider digit added later cannot
// silently exceed the fixed region.
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t ctrl_bytes_at_max(int bits, int threads, int items) {
  const size_t radix = (size_t)1 << bits, passes = (64 + bits - 1) / bits, tile = (size_t)threads * items;
  const size_t ntiles = (kNoAllocPairs + tile - 1) / tile;
  return 2 * align256(passes * radix * 4) + align256(passes * ntiles * radix * 4) + 256;
}
#define LNT_NOALLOC_FITS(B, T, I, W)                                              \
  static_assert(ctrl_bytes_at_max(B, T, I) <= kNoAllocCtrlBytes,                 \
                "sort variant (" #B ", " #T ", " #I ") needs a larger fixed control region");
LNT_SORT_VARIANTS(LNT_NOALLOC_FITS)
#undef LNT_NOALLOC_FITS

// [a, a + na) and [b, b + nb) share a byte.
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return x < y + nb && y < x + na;
}

static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array on the current device (cached per device).
int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LNT_DEVICE_ERROR;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_sort_scratch) != cudaSuccess || !p) return LNT_DEVICE_ERROR;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return LNT_OK;
}

}  // namespace
}  // namespace lnt

using namespace lnt;

extern "C" {

int lnt_sort_pairs_noalloc(const uint64_t* keys_in, const double* vals_in, uint64_t* keys_out, double* vals_out,
                           size_t n, uint64_t max_key, void* stream) {
  if (n == 0) return LNT_OK;
  if (!keys_in || !vals_in || !keys_out || !vals_out) return LNT_BAD_ARG;
  if (n > kNoAllocPairs) return LNT_UNSUPPORTED;
  // out of place: with an odd number of digit passes the first pass writes
  // the output while other tiles still read the input
  const size_t b = n * 8;
  if (overlaps(keys_out, b, keys_in, b) || overlaps(keys_out, b, vals_in, b) || overlaps(vals_out, b, keys_in, b) ||
      overlaps(vals_out, b, vals_in, b) || overlaps(keys_out, b, vals_out, b))
    return LNT_BAD_ARG;
  const SortPlan plan = make_sort_plan(n, max_key);
  if (plan.ctrl_bytes > kNoAllocCtrlBytes) return LNT_UNSUPPORTED;
  void* base = nullptr;
  int st = noalloc_scratch(&base);
  if (st != LNT_OK) return st;
  unsigned char* s = static_cast<unsigned char*>(base);
  u64* tk = reinterpret_cast<u64*>(s + kNoAllocCtrlBytes);
  double* tv = reinterpret_cast<double*>(s + kNoAllocCtrlBytes + kNoAllocPairs * 8);
  // run_sort clears the control block on the stream before its kernels read it
  return run_sort(plan, plain_source((const u64*)keys_in, vals_in, n), (u64*)keys_out, vals_out, tk, tv, s,
                  as_stream(stream));
}

}  // extern "C"
