/*
 * lnt_mex.h - host-buffer gateways with the wire formats of the reference's
 * MATLAB mex functions (src/MATLAB/mex/*.cpp), so that a toolbox gateway can
 * hand its mxArray data straight to this library.
 *
 * Formats: int64 keys (non-negative; LCO linear indices), float64 values,
 * 1-based uint8 lexicographic orders, int64 [h w d] lattice shapes.  Every
 * array here is HOST memory.  Each call copies its inputs to the current CUDA
 * device, runs the include/lnt.h entry points, copies the result back and
 * returns when it is done (legacy default stream).  Unlike lnt.h, these calls
 * allocate and free device memory inside the call.  Results whose size is
 * known only after the computation are allocated with the caller's allocator
 * `alloc` (a MATLAB gateway passes mxMalloc; NULL means malloc, to be freed
 * with free); at least one element is always allocated.  Inputs are never
 * modified unless the function works in place, as its reference gateway does.
 * Returns an lnt_status code (lnt.h); LNT_BAD_ARG also for a negative key or
 * an allocator that returns NULL.
 */
#ifndef LNT_MEX_H
#define LNT_MEX_H

#include "lnt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef void* (*lnt_host_alloc)(size_t bytes);

/* SparseSortMex(vals, keys) (MATLAB/mex/sparse_sort.cpp:10-60): sorts the
 * pairs by key in place, ascending (stable here; the reference's introsort is
 * not, which only matters for equal keys). */
LNT_API int lnt_mex_sparse_sort(double* vals, int64_t* keys, size_t n);

/* SparseChangeLinIdxMex(keys, cur, desired, dims)
 * (MATLAB/mex/sparse_change_linIdx.cpp:14-72): re-linearises the keys in
 * place from the 1-based order `cur` to `desired` over `dims` (order modes). */
LNT_API int lnt_mex_sparse_change_linidx(int64_t* keys, size_t n, int order, const uint8_t* cur,
                                         const uint8_t* desired, const int64_t* dims);

/* SparsePermuteMex(vals, keys, cur, desired, dims)
 * (MATLAB/mex/sparse_permute.cpp:18-107): the keys were already re-linearised
 * to `desired` while the pairs are still in `cur`'s order; sorts the pairs by
 * key in place.  Nothing to do when cur == desired.  Keys must be below the
 * product of dims. */
LNT_API int lnt_mex_sparse_permute(double* vals, int64_t* keys, size_t n, int order, const uint8_t* cur,
                                   const uint8_t* desired, const int64_t* dims);

/* SparseMergeMex(a_vals, a_keys, b_vals, b_keys, op)
 * (MATLAB/mex/sparse_merge.cpp:50-163): both operands key-sorted in the same
 * order; C = A + B (op == 0) or A - B (op != 0) with
 * outside_merge_sparse_storage_containers semantics (lnt_merge_sorted). */
LNT_API int lnt_mex_sparse_merge(const double* a_vals, const int64_t* a_keys, size_t na, const double* b_vals,
                                 const int64_t* b_keys, size_t nb, int op, lnt_host_alloc alloc,
                                 double** c_vals, int64_t** c_keys, size_t* nc);

/* SparseLatticeMultMex(a_vals, a_keys, a_dims, b_vals, b_keys, b_dims, alg)
 * (MATLAB/mex/sparselattice_mul.cpp:14-137): A (a_dims = [h w d]) and B
 * ([w wB d]) key-sorted column-major; C = A * B per tab (csc_no_accum: keys
 * ascending, exact zero sums kept).  alg 0 (operator*), 1 (CSC: csc_times),
 * 2 (DCSC) and 3 (CSCNA) all compute this product with this pattern; alg 4
 * and 5 return LNT_UNSUPPORTED: in the reference both reach mtt_times (alg 4
 * falls through into 5), whose body computes and returns nothing
 * (SparseLatticeBase.h:1582-1640).  LNT_BAD_DIMS when a_dims[1] != b_dims[0]
 * or the depths differ. */
LNT_API int lnt_mex_sparselattice_mult(const double* a_vals, const int64_t* a_keys, size_t na,
                                       const int64_t* a_dims, const double* b_vals, const int64_t* b_keys,
                                       size_t nb, const int64_t* b_dims, int alg, lnt_host_alloc alloc,
                                       double** c_vals, int64_t** c_keys, size_t* nc);

/* SparseDenseLatticeMultMex(a_vals, a_keys, a_dims, B, dense_first)
 * (MATLAB/mex/sparse_denselattice_mul.cpp:8-106): sparse A (a_dims = [h w d],
 * column-major keys, any order) and dense B (b_dims, float64 column-major).
 * dense_first != 0: C = B * A (b_dims[1] == a_dims[0]), column-major keys;
 * else C = A * B (a_dims[1] == b_dims[0]), the reference's row-major lattice
 * keys.  Depths must match (LNT_BAD_DIMS otherwise).  The reference sorts the
 * caller's A in place; here A is left as it was. */
LNT_API int lnt_mex_sparse_denselattice_mult(const double* a_vals, const int64_t* a_keys, size_t na,
                                             const int64_t* a_dims, const double* B, const int64_t* b_dims,
                                             int dense_first, lnt_host_alloc alloc, double** c_vals,
                                             int64_t** c_keys, size_t* nc);

#ifdef __cplusplus
}
#endif
#endif /* LNT_MEX_H */
