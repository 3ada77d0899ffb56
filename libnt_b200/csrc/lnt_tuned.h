// Autotuned kernel choices.  Written by libnt_b200/tune.py from timings on a
// B200 (the values come from lnt_tuned.json); sort entries are tried in
// order, the first whose ranges contain the request wins.  An empty table
// falls back to the untuned default.
#pragma once

namespace lnt {

struct TunedSortEntry {
  int key_bits_max;             // request key width <= this
  unsigned long long n_max;     // request pair count <= this
  int variant;                  // index into the compiled onesweep variants
};

static const TunedSortEntry kTunedSort[] = {
    {16, 16384ull, 2},  // 0.049 ms at n=2^14, 16 bits
    {16, 131072ull, 2},  // 0.052 ms at n=2^17, 16 bits
    {16, 1048576ull, 2},  // 0.070 ms at n=2^20, 16 bits
    {16, 8388608ull, 3},  // 0.244 ms at n=2^23, 16 bits
    {16, 67108864ull, 0},  // 1.598 ms at n=2^26, 16 bits
    {16, 4611686018427387904ull, 0},  // 3.130 ms at n=2^27, 16 bits
    {24, 16384ull, 4},  // 0.056 ms at n=2^14, 24 bits
    {24, 131072ull, 4},  // 0.058 ms at n=2^17, 24 bits
    {24, 1048576ull, 2},  // 0.086 ms at n=2^20, 24 bits
    {24, 8388608ull, 3},  // 0.339 ms at n=2^23, 24 bits
    {24, 67108864ull, 0},  // 2.288 ms at n=2^26, 24 bits
    {24, 4611686018427387904ull, 0},  // 4.485 ms at n=2^27, 24 bits
    {32, 16384ull, 2},  // 0.066 ms at n=2^14, 32 bits
    {32, 131072ull, 2},  // 0.067 ms at n=2^17, 32 bits
    {32, 1048576ull, 2},  // 0.102 ms at n=2^20, 32 bits
    {32, 8388608ull, 3},  // 0.439 ms at n=2^23, 32 bits
    {32, 67108864ull, 0},  // 2.977 ms at n=2^26, 32 bits
    {32, 4611686018427387904ull, 0},  // 5.850 ms at n=2^27, 32 bits
    {36, 16384ull, 5},  // 0.068 ms at n=2^14, 36 bits
    {36, 131072ull, 5},  // 0.075 ms at n=2^17, 36 bits
    {36, 1048576ull, 5},  // 0.117 ms at n=2^20, 36 bits
    {36, 8388608ull, 3},  // 0.538 ms at n=2^23, 36 bits
    {36, 67108864ull, 0},  // 3.659 ms at n=2^26, 36 bits
    {36, 4611686018427387904ull, 0},  // 7.205 ms at n=2^27, 36 bits
    {40, 16384ull, 4},  // 0.075 ms at n=2^14, 40 bits
    {40, 131072ull, 4},  // 0.079 ms at n=2^17, 40 bits
    {40, 1048576ull, 2},  // 0.122 ms at n=2^20, 40 bits
    {40, 8388608ull, 3},  // 0.542 ms at n=2^23, 40 bits
    {40, 67108864ull, 0},  // 3.694 ms at n=2^26, 40 bits
    {40, 4611686018427387904ull, 0},  // 7.263 ms at n=2^27, 40 bits
    {48, 16384ull, 4},  // 0.085 ms at n=2^14, 48 bits
    {48, 131072ull, 2},  // 0.091 ms at n=2^17, 48 bits
    {48, 1048576ull, 2},  // 0.140 ms at n=2^20, 48 bits
    {48, 8388608ull, 3},  // 0.645 ms at n=2^23, 48 bits
    {48, 67108864ull, 0},  // 4.385 ms at n=2^26, 48 bits
    {48, 4611686018427387904ull, 0},  // 8.625 ms at n=2^27, 48 bits
    {63, 16384ull, 5},  // 0.102 ms at n=2^14, 63 bits
    {63, 131072ull, 2},  // 0.113 ms at n=2^17, 63 bits
    {63, 1048576ull, 2},  // 0.180 ms at n=2^20, 63 bits
    {63, 8388608ull, 3},  // 0.839 ms at n=2^23, 63 bits
    {63, 67108864ull, 0},  // 5.742 ms at n=2^26, 63 bits
    {63, 4611686018427387904ull, 0},  // 11.304 ms at n=2^27, 63 bits
};

// digit-pass shape of the bucketed sort + collect (see run_onesweep_pass8)
constexpr int kTunedPass8Variant = 0;
// bucket geometry of the sort merge (0: 2^(lg n - 12) buckets, 1: 2^(lg n - 11))
constexpr int kTunedBucketSmall = 0;
// work-queue chunk of the batched contraction engine (units per grab)
constexpr unsigned kTunedBatchChunk = 1;
// dense-row threshold divisor of the tile engine
constexpr int kTunedTileDenseDiv = 8;

}  // namespace lnt
