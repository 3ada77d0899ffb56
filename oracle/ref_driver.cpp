/*
 * ref_driver.cpp - C entry points around the REFERENCE's own CPU kernels,
 * compiled in place from the reference tree (see oracle/Makefile), into
 * oracle/_ref/liblnt_ref.so.  TEST INFRASTRUCTURE: only tests/, the smoke
 * check and bench.py's CPU-baseline / reference arm load it.
 *
 * Which reference code runs:
 *   - re-keying: internal::create_shuffle_needs + internal::reShuffleLinearIndex
 *     (IndexUtil.h:480-487, 567-589) with the reference's libdivide dividers,
 *     exactly as SparseMIABase::change_linIdx_sequence calls them
 *     (SparseMIABase.h:768-814);
 *   - sorting: internal::_RadixSort_Unsigned_PowerOf2Radix_L1<2048,11,3000>
 *     (LibMIARadix.h:119-180), introsort_detail::IntrosortRec + DualSwapper
 *     (LibMIAAlgorithm.h:153-175, 752-766) and InsertionSortImproved
 *     (LibMIAAlgorithm.h:673-714).
 * The entry wrapper RadixSortInPlace_PowerOf2Radix_Unsigned
 * (LibMIARadix.h:444-484) does not compile at the reference's HEAD: line 470
 * passes the value InsertThreshold as the 4th template argument, a type
 * parameter.  lntr_radix_sort below restates that 20-line wrapper (top digit
 * shift from ceil(log2 max_size), the 3000-element threshold, the final
 * insertion sort) and calls the reference's L1 recursion directly.
 */
#include "IndexUtil.h"
#include "LibMIARadix.h"

#include <cstdint>

namespace {

using LibMIA::internal::create_shuffle_needs;
using LibMIA::internal::getShuffleSequence;
using LibMIA::internal::reorder_from;
using LibMIA::internal::reShuffleLinearIndex;

template <size_t N>
void rekey_n(int64_t* keys, size_t n, const int64_t* dims, const int32_t* cur, const int32_t* nw) {
    // SparseMIABase::change_linIdx_sequence (SparseMIABase.h:768-814)
    std::array<size_t, N> d, cs, ns;
    for (size_t i = 0; i < N; ++i) {
        d[i] = (size_t)dims[i];
        cs[i] = (size_t)cur[i];
        ns[i] = (size_t)nw[i];
    }
    if (cs == ns) return;
    auto reorder_Dims = d;
    auto new_reorder_Dims = d;
    reorder_from(d, cs, reorder_Dims);
    reorder_from(d, ns, new_reorder_Dims);
    auto index_order = getShuffleSequence(ns, cs);
    std::array<size_t, N> dim_accumulator;
    std::array<libdivide::divider<size_t>, N> fast_dim_accumulator;
    std::array<size_t, N> multiplier;
    create_shuffle_needs(reorder_Dims, new_reorder_Dims, index_order, dim_accumulator, fast_dim_accumulator,
                         multiplier);
    for (size_t i = 0; i < n; ++i)
        keys[i] = reShuffleLinearIndex(keys[i], multiplier, fast_dim_accumulator, dim_accumulator);
}

}  // namespace

extern "C" {

/* Re-key n keys in place; returns 0, or -1 for an unsupported order. */
int lntr_rekey(int64_t* keys, size_t n, int order, const int64_t* dims, const int32_t* cur_seq,
               const int32_t* new_seq) {
    switch (order) {
        case 1: return 0;
        case 2: rekey_n<2>(keys, n, dims, cur_seq, new_seq); return 0;
        case 3: rekey_n<3>(keys, n, dims, cur_seq, new_seq); return 0;
        case 4: rekey_n<4>(keys, n, dims, cur_seq, new_seq); return 0;
        case 5: rekey_n<5>(keys, n, dims, cur_seq, new_seq); return 0;
        case 6: rekey_n<6>(keys, n, dims, cur_seq, new_seq); return 0;
        case 7: rekey_n<7>(keys, n, dims, cur_seq, new_seq); return 0;
        case 8: rekey_n<8>(keys, n, dims, cur_seq, new_seq); return 0;
        default: return -1;
    }
}

/* In-place ascending sort of (key, value) pairs with the reference's MSD
 * radix sort (restated entry wrapper, LibMIARadix.h:444-484). */
void lntr_radix_sort(int64_t* keys, double* vals, size_t length, size_t max_size) {
    using namespace LibMIA::internal;
    typedef int64_t* ForwardIt;
    typedef double* FollowIt;
    const long Threshold = 3000;
    const unsigned long PowerOfTwoRadix = 2048;
    const unsigned long Log2ofPowerOfTwoRadix = 11;
    if (length == 0) return;
    auto current_bit_size = (unsigned long)std::ceil(std::log2((double)max_size));
    auto number_shifts = (unsigned long)std::ceil((double)current_bit_size / Log2ofPowerOfTwoRadix);
    unsigned long shiftRightAmount;
    if (current_bit_size >= Log2ofPowerOfTwoRadix)
        shiftRightAmount = (number_shifts - 1) * Log2ofPowerOfTwoRadix;
    else
        shiftRightAmount = 0;
    if ((long)length >= Threshold)
        _RadixSort_Unsigned_PowerOf2Radix_L1<PowerOfTwoRadix, Log2ofPowerOfTwoRadix, Threshold>(
            keys, vals, length, shiftRightAmount);
    else
        introsort_detail::IntrosortRec(keys, keys + length, introsort_detail::IntrosortDepth(keys, keys + length),
                                       std::less<int64_t>(), DualSwapper<ForwardIt, FollowIt>(keys, vals));
    InsertionSortImproved(keys, keys + length, vals, std::less<int64_t>());
}

/* Reference introsort with a key/value swapper (the n < 3000 branch of
 * SparseMIABase::sort(seq), SparseMIABase.h:615-618). */
void lntr_introsort(int64_t* keys, double* vals, size_t n) {
    using namespace LibMIA::internal;
    Introsort(keys, keys + n, std::less<int64_t>(), DualSwapper<int64_t*, double*>(keys, vals));
}

}  // extern "C"
