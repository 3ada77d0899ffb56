// Host-side helpers shared by every entry point, plus the re-key kernel
// (lnt_rekey) and the diagnostics entry points of include/lnt.h.
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

#include "lnt_common.cuh"

namespace lnt {

static std::atomic<uint64_t> g_launches{0};

static std::mutex& readers_mu() {
  static std::mutex mu;
  return mu;
}
static ErrorReader* readers() {
  static ErrorReader r[64];
  return r;
}
static int g_nreaders = 0;

void register_error_reader(ErrorReader f) {
  std::lock_guard<std::mutex> g(readers_mu());
  if (g_nreaders < 64) readers()[g_nreaders++] = f;
}

static SpinLimitWriter* spin_writers() {
  static SpinLimitWriter w[64];
  return w;
}
static int g_nspin_writers = 0;

void register_spin_limit_writer(SpinLimitWriter f) {
  std::lock_guard<std::mutex> g(readers_mu());
  if (g_nspin_writers < 64) spin_writers()[g_nspin_writers++] = f;
}

void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

// ---- per-kernel event timing ----------------------------------------------
namespace {
struct ProfRecord {
  const char* name;
  cudaEvent_t a, b;
};
std::mutex g_prof_mu;
std::atomic<bool> g_prof_on{false};
std::vector<ProfRecord> g_prof_records;
std::vector<cudaEvent_t> g_prof_pool;

cudaEvent_t prof_event() {
  if (!g_prof_pool.empty()) {
    cudaEvent_t e = g_prof_pool.back();
    g_prof_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}
}  // namespace

ProfScope::ProfScope(const char* name, cudaStream_t s) : name_(name), s_(s), start_(nullptr) {
  if (!g_prof_on.load(std::memory_order_relaxed)) return;
  std::lock_guard<std::mutex> g(g_prof_mu);
  cudaEvent_t e = prof_event();
  if (e && cudaEventRecord(e, s_) == cudaSuccess) start_ = e;
}

ProfScope::~ProfScope() {
  if (!start_) return;
  std::lock_guard<std::mutex> g(g_prof_mu);
  cudaEvent_t e = prof_event();
  if (e && cudaEventRecord(e, s_) == cudaSuccess) {
    g_prof_records.push_back({name_, (cudaEvent_t)start_, e});
  } else {
    g_prof_pool.push_back((cudaEvent_t)start_);
    if (e) g_prof_pool.push_back(e);
  }
}

int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LNT_OK : LNT_DEVICE_ERROR;
}

int sm_count() {
  static std::mutex mu;
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> g(mu);
  if (dev >= 0 && dev < 64 && cache[dev]) return cache[dev];
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
    n = 148;
  if (dev >= 0 && dev < 64) cache[dev] = n;
  return n;
}

static bool is_permutation(int order, const int32_t* seq) {
  unsigned seen = 0;
  for (int i = 0; i < order; ++i) {
    if (seq[i] < 0 || seq[i] >= order) return false;
    if (seen & (1u << seq[i])) return false;
    seen |= 1u << seq[i];
  }
  return true;
}

int make_rekey_params(int order, const int64_t* dims, const int32_t* cur_seq,
                      const int32_t* new_seq, RekeyParams* out) {
  if (!out) return LNT_BAD_ARG;
  out->order = 0;
  out->pow2 = 0;
  if (order <= 1) return order < 0 ? LNT_BAD_ARG : LNT_OK;
  if (order > LNT_MAX_ORDER || !dims || !cur_seq || !new_seq) return LNT_BAD_ARG;
  if (!is_permutation(order, cur_seq) || !is_permutation(order, new_seq)) return LNT_BAD_SEQ;
  unsigned __int128 total = 1;
  for (int i = 0; i < order; ++i) {
    if (dims[i] <= 0) return LNT_BAD_DIMS;
    total *= (unsigned __int128)dims[i];
    if (total >> 63) return LNT_OVERFLOW_KEYBITS;
  }
  bool same = true;
  for (int i = 0; i < order; ++i) same = same && (cur_seq[i] == new_seq[i]);
  if (same) return LNT_OK;  // identity
  // Cumulative extents under the current sequence.
  u64 acc = 1;
  for (int i = 0; i < order; ++i) {
    out->acc[i] = make_divider(acc);
    acc *= (u64)dims[cur_seq[i]];
  }
  // Stride of each mode under the new sequence.
  u64 stride_of_mode[LNT_MAX_ORDER];
  u64 s = 1;
  for (int i = 0; i < order; ++i) {
    stride_of_mode[new_seq[i]] = s;
    s *= (u64)dims[new_seq[i]];
  }
  for (int i = 0; i < order; ++i) out->mult[i] = stride_of_mode[cur_seq[i]];
  out->order = order;
  bool pow2 = true;
  for (int i = 0; i < order; ++i) pow2 = pow2 && ((u64)dims[i] & ((u64)dims[i] - 1)) == 0;
  out->pow2 = pow2 ? 1 : 0;
  for (int i = 0; i < LNT_MAX_ORDER; ++i) out->field[i] = 0;
  if (pow2) {
    for (int i = 0; i < order; ++i) {
      const u32 src = (u32)__builtin_ctzll(out->acc[i].d);
      const u32 bits = (u32)__builtin_ctzll((u64)dims[cur_seq[i]]);
      const u32 dst = (u32)__builtin_ctzll(out->mult[i]);
      out->field[i] = src | (bits << 8) | (dst << 16);
    }
  }
  return LNT_OK;
}

int make_rekey_params(const lnt_rekey_spec* spec, RekeyParams* out) {
  if (!spec) {
    out->order = 0;
    return LNT_OK;
  }
  return make_rekey_params(spec->order, spec->dims, spec->cur_seq, spec->new_seq, out);
}

// ---------------------------------------------------------------------------
// Re-key kernel: HBM-bound, 8 B read + 8 B written per key; two keys per
// thread per iteration through 16-byte vector accesses, grid-stride.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) rekey_kernel(const u64* __restrict__ in, u64* __restrict__ out,
                                                    size_t n, const RekeyParams p) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t npair = n / 2;
  const ulonglong2* in2 = reinterpret_cast<const ulonglong2*>(in);
  ulonglong2* out2 = reinterpret_cast<ulonglong2*>(out);
  for (size_t i = tid; i < npair; i += stride) {
    ulonglong2 v = in2[i];
    v.x = rekey(v.x, p);
    v.y = rekey(v.y, p);
    out2[i] = v;
  }
  if (tid == 0 && (n & 1)) out[n - 1] = rekey(in[n - 1], p);
}

__global__ void rekey_kernel_unaligned(const u64* __restrict__ in, u64* __restrict__ out, size_t n,
                                       const RekeyParams p) {
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = rekey(in[i], p);
}

}  // namespace lnt

using namespace lnt;

extern "C" {

const char* lnt_status_string(int s) {
  switch (s) {
    case LNT_OK: return "ok";
    case LNT_BAD_ARG: return "bad argument";
    case LNT_BAD_DIMS: return "dimension mismatch";
    case LNT_BAD_SEQ: return "sequence is not a permutation";
    case LNT_OVERFLOW_KEYBITS: return "dimensionality does not fit in 63 bits";
    case LNT_WORKSPACE: return "workspace too small";
    case LNT_TIMEOUT: return "device-side wait expired";
    case LNT_DEVICE_ERROR: return "CUDA error";
    case LNT_UNSUPPORTED: return "unsupported request";
    default: return "unknown status";
  }
}

int lnt_version(void) { return 100; }

uint64_t lnt_launch_count(void) { return g_launches.load(); }

int lnt_device_status(int clear, void* stream, uint32_t* detail) {
  cudaStream_t s = as_stream(stream);
  if (cudaStreamSynchronize(s) != cudaSuccess) return LNT_DEVICE_ERROR;
  u32 word = 0;
  std::lock_guard<std::mutex> g(readers_mu());
  for (int i = 0; i < g_nreaders; ++i) {
    u32 w = 0;
    if (readers()[i](clear, &w) != LNT_OK) return LNT_DEVICE_ERROR;
    word |= w;
  }
  if (detail) *detail = word;
  return word ? LNT_TIMEOUT : LNT_OK;
}

int lnt_set_spin_limit(uint32_t polls) {
  const u32 v = polls ? polls : kSpinLimit;
  std::lock_guard<std::mutex> g(readers_mu());
  for (int i = 0; i < g_nspin_writers; ++i)
    if (spin_writers()[i](v) != LNT_OK) return LNT_DEVICE_ERROR;
  return LNT_OK;
}

int lnt_profile_enable(int on) {
  g_prof_on.store(on != 0);
  return LNT_OK;
}

int lnt_profile_reset(void) {
  std::lock_guard<std::mutex> g(g_prof_mu);
  for (auto& r : g_prof_records) {
    cudaEventSynchronize(r.b);
    g_prof_pool.push_back(r.a);
    g_prof_pool.push_back(r.b);
  }
  g_prof_records.clear();
  return LNT_OK;
}

int lnt_profile_query(const char* kernel, double* total_ms, uint64_t* launches) {
  if (!kernel || !total_ms || !launches) return LNT_BAD_ARG;
  std::lock_guard<std::mutex> g(g_prof_mu);
  double t = 0.0;
  uint64_t c = 0;
  for (auto& r : g_prof_records) {
    if (std::strcmp(r.name, kernel) != 0) continue;
    if (cudaEventSynchronize(r.b) != cudaSuccess) return LNT_DEVICE_ERROR;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) return LNT_DEVICE_ERROR;
    t += ms;
    ++c;
  }
  *total_ms = t;
  *launches = c;
  return LNT_OK;
}

int lnt_rekey(const uint64_t* keys_in, uint64_t* keys_out, size_t n, int order, const int64_t* dims,
              const int32_t* cur_seq, const int32_t* new_seq, void* stream) {
  if (n == 0) return LNT_OK;
  if (!keys_in || !keys_out) return LNT_BAD_ARG;
  RekeyParams p;
  int st = make_rekey_params(order, dims, cur_seq, new_seq, &p);
  if (st != LNT_OK) return st;
  cudaStream_t s = as_stream(stream);
  if (p.order <= 1) {
    if (keys_in == keys_out) return LNT_OK;
    return cudaMemcpyAsync(keys_out, keys_in, n * sizeof(u64), cudaMemcpyDeviceToDevice, s) ==
                   cudaSuccess
               ? LNT_OK
               : LNT_DEVICE_ERROR;
  }
  int threads = 256;
  size_t want = (n / 2 + threads - 1) / threads;
  size_t cap = (size_t)sm_count() * 8;
  int blocks = (int)(want < cap ? (want ? want : 1) : cap);
  bool aligned = ((uintptr_t)keys_in % 16 == 0) && ((uintptr_t)keys_out % 16 == 0);
  {
    ProfScope prof("rekey", s);
    if (aligned)
      rekey_kernel<<<blocks, threads, 0, s>>>((const u64*)keys_in, (u64*)keys_out, n, p);
    else
      rekey_kernel_unaligned<<<blocks, threads, 0, s>>>((const u64*)keys_in, (u64*)keys_out, n, p);
  }
  count_launch();
  return launch_status();
}

}  // extern "C"
