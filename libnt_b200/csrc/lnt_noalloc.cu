// lnt_sort_pairs_noalloc: the pair sort of lnt_sort_pairs for callers that
// cannot allocate device memory.
//
// Who needs it: code that must not call cudaMalloc / cudaFree or any
// allocating library routine -- for example a path that runs while its
// stream is being captured into a CUDA graph (allocation calls are not
// allowed there, and cudaFree synchronises the device), a latency-critical
// loop that cannot afford the implicit synchronisation an allocation may
// cause, or a host environment (a plugin or foreign-function binding) that
// has no device allocator of its own to hand us a workspace.
//
// How: the sort's scratch (digit histograms, look-back states, one ping-pong
// pair buffer) lives in one file-scope __device__ array of fixed size, so the
// call needs only the caller's input and output buffers.  The array is
// created with the module on every device that loads this library and stays
// there until the process exits.  Limits and rules:
//   * at most LNT_SORT_NOALLOC_MAX_PAIRS pairs; larger requests return
//     LNT_UNSUPPORTED without touching the device;
//   * output buffers must not alias the inputs (LNT_BAD_ARG otherwise);
//   * every call on a device shares the one array and leaves its contents
//     behind; the control region that must start at zero is cleared by each
//     call on its stream, but two calls whose GPU work overlaps (different
//     streams, or several host threads) race on the array -- keep all calls
//     on a device ordered, e.g. on one stream;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and caches it; make that
//     first call outside any stream capture.
#include <mutex>

#include "lnt_sort.cuh"

namespace lnt {
namespace {

// Room for the control block of any compiled sort variant at the maximum
// pair count and 64-bit keys, plus one ping-pong pair buffer.
constexpr size_t kNoAllocPairs = LNT_SORT_NOALLOC_MAX_PAIRS;
constexpr size_t kNoAllocCtrlBytes = 2u << 20;
constexpr size_t kNoAllocBytes = kNoAllocCtrlBytes + 2 * kNoAllocPairs * 8;

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
  if ((const void*)keys_in == (const void*)keys_out || (const void*)vals_in == (const void*)vals_out)
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
