// LSD radix sort of (u64 key, f64 value) pairs, one-sweep style:
//   1. hist_kernel: one read of all keys builds the digit histograms of every
//      pass at once (shared-memory atomics, then one global add per bin);
//      the last block to finish turns them into exclusive bin starts.
//   2. per pass, onesweep_kernel: each CTA takes the next tile id, ranks its
//      keys by digit with warp match-any + per-warp counters (stable), writes
//      its per-digit counts to a look-back array, obtains its global offsets
//      by decoupled look-back over predecessor tiles, reorders the tile in
//      shared memory by digit and writes keys and values out in digit runs.
// Traffic per pass: 16 B read + 16 B written per pair (the HBM roofline).
// The first pass reads through a PairSource, which concatenates two arrays
// and re-keys each on the fly, so sortMerge's re-key + concatenation costs
// no extra pass.
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
  return s;
}

struct SortPlan {
  int key_bits = 0;
  int bits = 8;      // digit width
  int passes = 0;
  u32 n = 0;
  u32 ntiles = 0;    // onesweep tiles per pass
  // byte offsets inside the control block
  size_t off_ghist = 0, off_bstart = 0, off_status = 0, off_counters = 0, ctrl_bytes = 0;
};

// Fills a plan for n pairs with keys < max_key and digit width `bits`.
SortPlan make_sort_plan(size_t n, u64 max_key, int bits);

// Runs the passes.  Pass p reads the previous pass's output (pass 0 reads
// src) and writes buffer ((passes-1-p) & 1): buf0 = final destination.
// `ctrl` points at plan.ctrl_bytes of scratch, zeroed here.
int run_sort(const SortPlan& plan, const PairSource& src, u64* buf0_k, double* buf0_v, u64* buf1_k,
             double* buf1_v, void* ctrl, cudaStream_t s);

// Digit width chosen for a sort of n pairs with key_bits significant bits
// (table written by the autotuner; defaults when absent).
int choose_sort_bits(size_t n, int key_bits);

}  // namespace lnt
