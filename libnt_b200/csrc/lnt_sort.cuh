// LSD radix sort of (u64 key, f64 value) pairs, one-sweep style:
//   1. hist_kernel: one read of all keys builds the digit histograms of every
//      pass at once (shared-memory atomics, then one global add per bin);
//      the last block to finish turns them into exclusive bin starts.
//   2. per pass, onesweep_kernel: each CTA takes the next tile id, counts its
//      tile's digits and publishes them at once, starts the value copy into
//      shared memory (cp.async), ranks its keys stably (warp ballots +
//      per-warp counters) and stages them in digit order, then obtains its
//      global digit offsets by a windowed decoupled look-back over
//      predecessor tiles (after the ranking, so predecessors have had time to
//      publish inclusive prefixes) and writes keys and values in digit runs.
// Traffic per pass: 16 B read + 16 B written per pair (the HBM roofline).
// The first pass reads through a PairSource, which concatenates two arrays
// and re-keys each on the fly, so sortMerge's re-key + concatenation costs
// no extra pass.
//
// Several kernel variants (digit width, CTA size, items per thread, look-back
// window) are compiled in; the variant per (pair count, key width) comes from
// the table written by the autotuner (libnt_b200/tune.py -> lnt_tuned.h).
#pragma once

#include "lnt_common.cuh"

namespace lnt {

struct PairSource {
  const u64* ak;
  const double* av;
  size_t na;
  const u64* bk;
  const double* bv;
  size_t nb;
  double bscale;
  int pad;
  RekeyParams ra;
  RekeyParams rb;
  // Kernels reading this source run only when gate == nullptr or
  // *gate == gate_run (see gated_off); a gated sort uses persistent grids.
  const u32* gate;
  u32 gate_run;
  u32 pad2;
};

// Host: single-array source (no re-key).
inline PairSource plain_source(const u64* k, const double* v, size_t n) {
  PairSource s;
  s.ak = k;
  s.av = v;
  s.na = n;
  s.bk = nullptr;
  s.bv = nullptr;
  s.nb = 0;
  s.bscale = 1.0;
  s.pad = 0;
  s.ra.order = 0;
  s.rb.order = 0;
  s.gate = nullptr;
  s.gate_run = 0;
  s.pad2 = 0;
  return s;
}

// The same source, gated on (gate, run).
inline PairSource gated_source(PairSource s, const u32* gate, u32 run) {
  s.gate = gate;
  s.gate_run = run;
  return s;
}

// Compiled onesweep variants: (digit bits, CTA threads, items per thread,
// look-back window).  The autotuner's variant indices follow this order.
#define LNT_SORT_VARIANTS(X) \
  X(8, 256, 16, 16)          \
  X(8, 256, 16, 32)          \
  X(8, 512, 8, 16)           \
  X(8, 384, 12, 16)          \
  X(8, 256, 12, 16)          \
  X(9, 512, 8, 16)           \
  X(9, 512, 8, 32)           \
  X(9, 256, 12, 8)

// One compiled onesweep variant.
struct SortVariant {
  int bits;     // digit width
  int threads;  // CTA size
  int items;    // keys per thread (tile = threads * items)
  int window;   // predecessors read per look-back round trip
};

int sort_variant_count();
const SortVariant& sort_variant(int i);

struct SortPlan {
  int variant = 0;
  int key_bits = 0;
  int bits = 8;      // digit width
  int passes = 0;
  u32 n = 0;
  u32 tile = 0;      // pairs per onesweep tile
  u32 ntiles = 0;    // onesweep tiles per pass
  // byte offsets inside the control block
  size_t off_ghist = 0, off_bstart = 0, off_status = 0, off_counters = 0, ctrl_bytes = 0;
};

// Variant for a sort of n pairs with key_bits significant bits: the
// environment variable LNT_SORT_VARIANT when set (used by the autotuner),
// else the tuned table.
int choose_sort_variant(size_t n, int key_bits);

// Fills a plan for n pairs with keys < max_key (variant < 0: choose).
SortPlan make_sort_plan(size_t n, u64 max_key, int variant = -1);

// Runs the passes.  Pass p reads the previous pass's output (pass 0 reads
// src) and writes buffer ((passes-1-p) & 1): buf0 = final destination.
// `ctrl` points at plan.ctrl_bytes of scratch, zeroed here.
int run_sort(const SortPlan& plan, const PairSource& src, u64* buf0_k, double* buf0_v, u64* buf1_k,
             double* buf1_v, void* ctrl, cudaStream_t s);

// One digit pass of the 8-bit, 256-thread, 16-key onesweep kernel with
// caller-given digit (shift, mask), exclusive bin starts (256 entries) and a
// zeroed look-back array (kOnesweepPassTile-pair tiles x 256 digits) and tile
// counter.  Used by the bucketed sort.
constexpr u32 kOnesweepPassTile = 4096;
int run_onesweep_pass8(const PairSource& src, bool first, u64* out_k, double* out_v, u32 n, u32 shift, u32 mask,
                       const u32* bstart, u32* status, u32* tile_counter, cudaStream_t s);

// Bucketed sort + collect (lnt_bucket.cu): applies to n >= 2^20 pairs whose
// keys have at most 28 bits below the bucket bits.
bool bucket_path_applies(size_t n, int key_bits);
size_t bucket_ctrl_bytes(size_t n);
// Enqueues the bucketed path.  Its histogram kernel writes *gate: 0 when every
// bucket fits a CTA (the path's remaining kernels run), 1 when one does not
// (they return at once, and the caller's LSD path, gated on 1, runs instead).
// No host synchronisation.
int run_bucketed_sort_reduce(const PairSource& src, u32 n, int key_bits, int skip_zero_heads, u64* k0, double* v0,
                             u64* k1, double* v1, void* ctrl, u64* out_k, double* out_v, u64* d_nout, u32* gate,
                             cudaStream_t s);

// Duplicate collection gated on (gate, want); persistent grid when gated.
int run_collect_gated(const u64* keys, const double* vals, size_t n, int skip_zero_heads, u64* out_k,
                      double* out_v, u64* d_nout, void* ws, cudaStream_t s, const u32* gate, u32 want);

}  // namespace lnt
