/*
 * lnt.h - C ABI of the B200 sparse/dense multi-index-array (MIA) hot path.
 *
 * Plain pointers and sizes only.  Every array argument named *_keys / *_vals /
 * A / B / C is DEVICE memory on the current CUDA device; every function is
 * stream-ordered on `stream` (a cudaStream_t passed as void*, NULL = legacy
 * default stream) and returns an lnt_status code for argument errors and
 * launch failures.  Errors raised on the device (an expired bounded wait) are
 * latched in a per-device word read back by lnt_device_status().
 *
 * Sparse storage is the reference's LCO layout (SparseMIA.h:61-84, 203-206):
 * parallel arrays of 64-bit linear keys and float64 values, with
 *     key = sum_i idx[seq[i]] * prod_{j<i} dims[seq[j]]     (first listed mode fastest)
 * (IndexUtil.h:866-879).  Keys are unsigned here; the reference stores int64
 * but only ever holds non-negative keys below the dimensionality.
 *
 * Caller-allocated workspaces: each entry point that needs scratch memory has
 * a *_workspace() query giving the byte count; pass a device buffer at least
 * that large (256-byte aligned).  No entry point allocates device memory.
 */
#ifndef LNT_H
#define LNT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LNT_MAX_ORDER 16

#if defined(__GNUC__)
#define LNT_API __attribute__((visibility("default")))
#else
#define LNT_API
#endif

typedef enum lnt_status {
    LNT_OK = 0,
    LNT_BAD_ARG = 1,          /* null pointer, size out of range, misaligned workspace */
    LNT_BAD_DIMS = 2,         /* dimension mismatch (reference: DimensionMismatchException) */
    LNT_BAD_SEQ = 3,          /* a lexicographic sequence is not a permutation of 0..order-1 */
    LNT_OVERFLOW_KEYBITS = 4, /* product of dims does not fit in 63 bits */
    LNT_WORKSPACE = 5,        /* workspace smaller than the *_workspace() query */
    LNT_TIMEOUT = 6,          /* a bounded device-side wait expired (device status only) */
    LNT_DEVICE_ERROR = 7,     /* CUDA runtime error on launch */
    LNT_UNSUPPORTED = 8       /* valid request outside what this build implements */
} lnt_status;

/* Re-keying request: keys linearised under cur_seq are re-linearised under
 * new_seq.  order == 0 means "keys are used as they are". */
typedef struct lnt_rekey_spec {
    int32_t order;
    int32_t cur_seq[LNT_MAX_ORDER];
    int32_t new_seq[LNT_MAX_ORDER];
    int64_t dims[LNT_MAX_ORDER];
} lnt_rekey_spec;

/* ---- library info / diagnostics ---------------------------------------- */

/* Human-readable name of a status code. */
LNT_API const char* lnt_status_string(int status);

/* ABI version (major*10000 + minor*100 + patch). */
LNT_API int lnt_version(void);

/* Number of kernels this library has launched in the process so far. */
LNT_API uint64_t lnt_launch_count(void);

/* Reads (and, if clear != 0, resets) the device-side error word of the
 * current device after synchronising `stream`.  Returns LNT_OK when no
 * device-side wait expired since the last clear, else LNT_TIMEOUT.
 * *detail (may be NULL) receives the raw word (which kernel gave up). */
LNT_API int lnt_device_status(int clear, void* stream, uint32_t* detail);

/* Sets the poll budget of every bounded device-side wait (the look-backs of
 * the sort, collect, merge, scan and contraction kernels) on the current
 * device; polls == 0 restores the default (2^24 polls, well under a minute).
 * A wait that exhausts its budget latches its bit in the error word and
 * continues with the partial (too small) prefix it has summed, so its kernel
 * finishes with wrong results; lnt_device_status() then returns LNT_TIMEOUT
 * and the results of that call must be discarded.  Synchronous; do not call
 * it while this library's kernels run on the device.  The Python binding
 * applies LNT_SPIN_LIMIT from the environment when it loads. */
LNT_API int lnt_set_spin_limit(uint32_t polls);

/* Runs one bounded wait on a look-back state that nothing ever publishes
 * (the same look-back code as the collect kernels) on `stream`: it polls
 * through the budget of lnt_set_spin_limit, latches its bit and returns, so
 * that lnt_device_status() reports LNT_TIMEOUT afterwards.  It lets a caller
 * check its handling of an expired wait without a fault or a hang; shorten
 * the budget first (at the default it polls for several seconds). */
LNT_API int lnt_diag_expired_wait(void* stream);

/* Per-kernel timing: while enabled, every launch by this library is
 * bracketed by CUDA events on its own stream (a few microseconds of overhead
 * per launch; off by default). */
LNT_API int lnt_profile_enable(int on);
/* Clears all timing records. */
LNT_API int lnt_profile_reset(void);
/* Synchronises the recorded events and returns, for kernels of the given name
 * ("rekey", "sort_hist", "sort_onesweep", "sort_copy", "collect_lead",
 * "collect", ...), the summed device time in milliseconds and the launch
 * count since the last reset. */
LNT_API int lnt_profile_query(const char* kernel, double* total_ms, uint64_t* launches);

/* ---- key linearisation / permutation ----------------------------------- */

/* Re-linearise n keys from cur_seq to new_seq over `dims` (order modes).
 * keys_out may equal keys_in.  Replaces SparseMIABase::change_linIdx_sequence
 * (SparseMIABase.h:768-814: create_shuffle_needs + reShuffleLinearIndex,
 * IndexUtil.h:480-487, 567-589) and the mex gateway SparseChangeLinIdxMex
 * (MATLAB/mex/sparse_change_linIdx.cpp:16-72; 0-based sequences here). */
LNT_API int lnt_rekey(const uint64_t* keys_in, uint64_t* keys_out, size_t n, int order,
              const int64_t* dims, const int32_t* cur_seq, const int32_t* new_seq,
              void* stream);

/* ---- sorting ------------------------------------------------------------ */

/* Workspace bytes for lnt_sort_pairs on n pairs whose keys are < max_key. */
LNT_API int lnt_sort_pairs_workspace(size_t n, uint64_t max_key, size_t* bytes);

/* Ascending sort of (key, value) pairs by key; equal keys keep their input
 * order (stable).  keys_out/vals_out may equal keys_in/vals_in (in-place).
 * Only the ceil(log2(max_key)) low key bits are sorted, as the reference's
 * radix sort does with its `max_size` argument.  Replaces SparseMIABase::sort()
 * -> RadixSortInPlace_PowerOf2Radix_Unsigned (SparseMIABase.h:701-734,
 * LibMIARadix.h:444-484) and SparseSortMex (MATLAB/mex/sparse_sort.cpp:14-60). */
LNT_API int lnt_sort_pairs(const uint64_t* keys_in, const double* vals_in,
                   uint64_t* keys_out, double* vals_out, size_t n, uint64_t max_key,
                   void* workspace, size_t workspace_bytes, void* stream);

/* Kernel variants of the sort compiled into this library (digit width, CTA
 * threads, keys per thread, look-back window); the autotuner times each one.
 * The variant used is the tuned choice, or LNT_SORT_VARIANT=<index> from the
 * environment. */
LNT_API int lnt_sort_variant_count(void);
LNT_API int lnt_sort_variant(int index, int* bits, int* threads, int* items, int* window);

/* Largest pair count lnt_sort_pairs_noalloc accepts. */
#define LNT_SORT_NOALLOC_MAX_PAIRS 262144

/* lnt_sort_pairs for callers that cannot allocate device memory (a loop that
 * must not synchronise on an allocation, a plugin with no device allocator).
 * No counterpart in the reference, whose sort needs no workspace.  Same
 * result as lnt_sort_pairs, out of place only (LNT_BAD_ARG if an output range
 * overlaps an input range or the other output); n > LNT_SORT_NOALLOC_MAX_PAIRS
 * returns LNT_UNSUPPORTED; null pointers (n > 0) return LNT_BAD_ARG.  Its scratch is one
 * fixed 6 MiB array in device memory that every device loading this library
 * holds until exit; calls share it, so calls whose GPU work overlaps race --
 * order them on one stream.  The first call on a device looks the array up,
 * so make it before any stream capture.  Allocates nothing. */
LNT_API int lnt_sort_pairs_noalloc(const uint64_t* keys_in, const double* vals_in,
                                   uint64_t* keys_out, double* vals_out, size_t n,
                                   uint64_t max_key, void* stream);

/* ---- duplicate collection ----------------------------------------------- */

LNT_API int lnt_collect_duplicates_workspace(size_t n, size_t* bytes);

/* Fold runs of equal keys of a key-sorted array with +.  With skip_zero_heads
 * != 0 this is SparseMIA::collect_duplicates(std::plus) (SparseMIA.h:636-665):
 * a run whose raw values are all exactly 0.0 is dropped unless it starts at
 * position 0.  With skip_zero_heads == 0 it is collect_duplicates_function
 * (FunctionUtil.h:701-728): every run is kept.  *d_nout (device) receives the
 * output count.  Output buffers need room for n pairs and must not overlap
 * the input. */
LNT_API int lnt_collect_duplicates(const uint64_t* keys, const double* vals, size_t n,
                           int skip_zero_heads, uint64_t* keys_out, double* vals_out,
                           uint64_t* d_nout, void* workspace, size_t workspace_bytes,
                           void* stream);

/* ---- sort merge (both operands unsorted) -------------------------------- */

LNT_API int lnt_sort_reduce_workspace(size_t na, size_t nb, uint64_t max_key, size_t* bytes);

/* Concatenate A (re-keyed by a_rekey, may be NULL) and B (re-keyed by
 * b_rekey, values multiplied by b_scale, +1 or -1), sort by key and collect
 * duplicates (skip_zero_heads as in lnt_collect_duplicates).  This is
 * SparseMIA::sortMerge (SparseMIA.h:833-887) for op = + (b_scale = 1) and
 * op = - (b_scale = -1, the reference negates B while copying, :862-875);
 * with nb == 0 it is change_linIdx_sequence + collect_duplicates.
 * Output buffers need room for na+nb pairs; *d_nout (device) gets the count. */
LNT_API int lnt_sort_reduce(const uint64_t* a_keys, const double* a_vals, size_t na,
                    const lnt_rekey_spec* a_rekey,
                    const uint64_t* b_keys, const double* b_vals, size_t nb,
                    const lnt_rekey_spec* b_rekey, double b_scale,
                    uint64_t max_key, int skip_zero_heads,
                    uint64_t* keys_out, double* vals_out, uint64_t* d_nout,
                    void* workspace, size_t workspace_bytes, void* stream);

/* ---- scan merge (operands sorted in the same linearisation) ------------- */

LNT_API int lnt_merge_sorted_workspace(size_t na, size_t nb, size_t* bytes);

/* Merge two key-sorted operands: A-only entries are copied, B-only entries
 * become op(0, b), equal keys op(a, b) (op 0 = +, 1 = -); within a run of
 * equal keys the j-th A pairs with the j-th B.  Every entry is kept, exact
 * zeros included.  Replaces outside_merge_sparse_storage_containers
 * (FunctionUtil.h:373-419) on the SparseMIABase::outside_scanMerge path
 * (SparseMIABase.h:1404-1455) and the mex gateway SparseMergeMex
 * (MATLAB/mex/sparse_merge.cpp:15-163).  c arrays need room for na + nb
 * pairs; *d_nout (device) receives the output count. */
LNT_API int lnt_merge_sorted(const uint64_t* a_keys, const double* a_vals, size_t na,
                             const uint64_t* b_keys, const double* b_vals, size_t nb, int op,
                             uint64_t* c_keys, double* c_vals, uint64_t* d_nout,
                             void* workspace, size_t workspace_bytes, void* stream);

/* ---- re-key + sort (sort under a new linearisation) --------------------- */

LNT_API int lnt_permute_sort_workspace(size_t n, uint64_t max_key, size_t* bytes);

/* Re-key (may be NULL: keys as they are) and stable-sort n pairs, out of
 * place.  Replaces SparseMIABase::sort(seq) (SparseMIABase.h:590-645: re-key,
 * then radix sort or RadixShuffle::permute, LibMIARadix.h:705-927) and the mex
 * gateway SparsePermuteMex (MATLAB/mex/sparse_permute.cpp:15-117). */
LNT_API int lnt_permute_sort(const uint64_t* keys_in, const double* vals_in, size_t n,
                             const lnt_rekey_spec* rekey, uint64_t* keys_out, double* vals_out,
                             uint64_t max_key, void* workspace, size_t workspace_bytes, void* stream);

/* ---- sparse lattice product -------------------------------------------- */

/* A sparse lattice (3-D sparse array: rows x cols x tabs) in column-major LCO
 * form: key = row + rows*(col + cols*tab), keys ascending
 * (SparseLatticeBase / MappedSparseLattice, MappedSparseLattice.h:163-263). */
typedef struct lnt_lattice {
    const uint64_t* keys;
    const double* vals;
    uint64_t nnz;
    int64_t rows, cols, tabs;
} lnt_lattice;

/* C(:,:,t) = A(:,:,t) * B(:,:,t) for every tab; C is rows(A) x cols(B) x tabs,
 * keys ascending, duplicate products summed, exact zeros kept.  Replaces
 * SparseLatticeBase::operator* -> csc_no_accum<true> (SparseLatticeBase.h:
 * 1572-1576, 1854-1990) and the mex gateway SparseLatticeMultMex with alg 0
 * (MATLAB/mex/sparselattice_mul.cpp:14-137).  Two phases:
 *   1. lnt_lattice_mult_plan fills `plan` (size from *_plan_workspace) and
 *      writes d_counts[0] = number of products, d_counts[1] = capacity C needs
 *      (the exact output count, or an upper bound);
 *   2. lnt_lattice_mult (workspace from lnt_lattice_mult_workspace with the
 *      product count) writes C and *d_nc.
 * Errors: LNT_BAD_DIMS when cols(A) != rows(B) or the tab counts differ
 * (SparseLatticeBase::check_mult_dims). */
LNT_API int lnt_lattice_mult_plan_workspace(const lnt_lattice* A, const lnt_lattice* B, size_t* bytes);
LNT_API int lnt_lattice_mult_plan(const lnt_lattice* A, const lnt_lattice* B, void* plan,
                                  size_t plan_bytes, uint64_t* d_counts, void* stream);
LNT_API int lnt_lattice_mult_workspace(const lnt_lattice* A, const lnt_lattice* B, uint64_t products,
                                       size_t* bytes);
LNT_API int lnt_lattice_mult(const lnt_lattice* A, const lnt_lattice* B, const void* plan,
                             uint64_t products, void* workspace, size_t workspace_bytes,
                             uint64_t* c_keys, double* c_vals, uint64_t* d_nc, void* stream);

/* Products with no contracted index: outer and element-wise (inter) modes
 * only.  Replaces SparseMIABase::noLatticeMult / perform_noLatticeMult
 * (SparseMIABase.h:1701-1826), reached from MIA_Atom::operator* for pure
 * outer/inter products (MIA_Expr.h:1012-1057).  A is key-sorted under [its
 * outer modes, the inter modes] and passed as a lattice rows = outer size,
 * cols = 1, tabs = inter size; B is sorted under [its outer modes, the inter
 * modes] and passed as rows = 1, cols = its outer size, tabs = inter size.
 * C(l_outer, r_outer, inter) = a * b for every pair of entries with equal inter
 * index, key l_outer + |l_outer| (r_outer + |r_outer| inter), written in the
 * reference's emission order (ascending keys; B entries major, A entries
 * minor); equal keys are not folded.  Two phases sharing one workspace:
 * lnt_nolattice_mult_count writes the product count (the output count) to
 * *d_products, lnt_nolattice_mult writes C.  LNT_BAD_DIMS when cols(A) != 1,
 * rows(B) != 1 or the tab counts differ. */
LNT_API int lnt_nolattice_mult_workspace(const lnt_lattice* A, const lnt_lattice* B, size_t* bytes);
LNT_API int lnt_nolattice_mult_count(const lnt_lattice* A, const lnt_lattice* B, void* workspace,
                                     size_t workspace_bytes, uint64_t* d_products, void* stream);
LNT_API int lnt_nolattice_mult(const lnt_lattice* A, const lnt_lattice* B, uint64_t products, void* workspace,
                               size_t workspace_bytes, uint64_t* c_keys, double* c_vals, void* stream);

/* Mixed sparse / dense lattice products: the mex gateway
 * SparseDenseLatticeMultMex(a_vals, a_idx, a_dims, B, dense_first)
 * (MATLAB/mex/sparse_denselattice_mul.cpp:8-106).  S is the sparse operand,
 * D the dense one (float64 column-major, tabs one after another), `other` the
 * dense operand's extent that S does not share.  Every non-empty line of S
 * gives a full dense line of C (h or wB entries, exact zeros kept); each
 * entry is sum over the line's entries (k, v) of S, in key order, of
 * v * D(...), accumulated from 0 as c = c + v * d (no fused multiply-add).
 *   dense_first = 1: C = A * S, DenseLatticeBase::operator*(SparseLatticeBase)
 *     (DenseLatticeBase.h:436-500).  A is other x rows(S) x tabs(S); S keys
 *     sorted column-major (row + rows (col + cols tab)); C is other x cols(S)
 *     x tabs(S) with column-major keys i + other (col + cols tab), ascending.
 *   dense_first = 0: C = S * B, SparseLatticeBase::operator*(DenseLatticeBase)
 *     (SparseLatticeBase.h:1148-1162, evaluated as (B^T S^T)^T).  S keys sorted
 *     ROW-major (col + cols (row + rows tab), the order that product leaves its
 *     operand in); B is cols(S) x other x tabs(S); C is rows(S) x other x
 *     tabs(S) with the reference's row-major lattice keys
 *     j + other (row + rows tab), ascending.
 * Two phases sharing one workspace: lnt_sparse_dense_mult_count finds the
 * lines of S (kept in the workspace) and writes the output count to
 * *d_count; lnt_sparse_dense_mult, called after it with the same S and
 * workspace on the same stream, writes C.  Keys must lie below rows * cols * tabs (entries past the last
 * tab contribute nothing).  LNT_BAD_DIMS for non-positive extents. */
LNT_API int lnt_sparse_dense_mult_workspace(const lnt_lattice* S, int64_t other, int dense_first, size_t* bytes);
LNT_API int lnt_sparse_dense_mult_count(const lnt_lattice* S, int64_t other, int dense_first, void* workspace,
                                        size_t workspace_bytes, uint64_t* d_count, void* stream);
LNT_API int lnt_sparse_dense_mult(const double* D, const lnt_lattice* S, int64_t other, int dense_first,
                                  void* workspace, size_t workspace_bytes, uint64_t* c_keys, double* c_vals,
                                  void* stream);

/* Unary contraction / attraction: SparseMIABase::contract_attract
 * (SparseMIABase.h:1913-2053), which MIA_Atom applies to index labels repeated
 * inside one operand (perform_unary, MIA_Expr.h:690-735).  keys/vals: the
 * tensor sorted under the sequence [contraction modes, attraction modes, other
 * modes]; sdims[0..order): the extents in that sequence.  The first modes form
 * ncon_sets contraction sets of con_part[p] modes each (summed along their
 * diagonal), the next natt_sets attraction sets of att_part[p] modes (their
 * diagonal becomes one output mode); the rest are kept.  Output, in the
 * reference's emission order: one entry per group of equal kept and attracted
 * indices whose attraction sets agree and whose sum over the entries with
 * agreeing contraction sets is not zero; key = kept linear index + |kept| *
 * attraction linear index (output extents [kept..., one per attraction set]).
 * *d_nout = output count (<= n); *d_sorted (optional) = non-zero when the keys
 * written never decrease (the result's sorted flag).  LNT_BAD_DIMS when a set
 * spans different extents. */
LNT_API int lnt_contract_attract_workspace(size_t n, size_t* bytes);
LNT_API int lnt_contract_attract(const uint64_t* keys, const double* vals, size_t n, int order,
                                 const int64_t* sdims, int ncon_sets, const int* con_part, int natt_sets,
                                 const int* att_part, uint64_t* out_keys, double* out_vals, uint64_t* d_nout,
                                 uint32_t* d_sorted, void* workspace, size_t workspace_bytes, void* stream);

/* ---- batched lattice products ------------------------------------------- */

/* `count` independent products C_p = A_p * B_p, each as lnt_lattice_mult
 * (rows beyond 512 are accumulated in blocks of 512).  Host arrays: dims_host[4p..4p+3] =
 * (rows(A_p), cols(A_p) = rows(B_p), cols(B_p), tabs); a_off_host / b_off_host
 * (count+1 entries) delimit each problem's operand inside the concatenated
 * device arrays a_keys/a_vals, b_keys/b_vals (each lattice key-sorted).
 * C_p is written at c_keys/c_vals + c_off[p] (device, count+1 entries);
 * *c_capacity bounds the total output.  The reference has no batched form:
 * it is a loop of csc_no_accum calls (SparseLatticeBase.h:1854-1990).
 * Call lnt_batched_prepare once per batch layout (it uploads the descriptor
 * tables, including the problem of every output column, into the workspace,
 * synchronously), then lnt_batched_lattice_mult, which only enqueues kernels
 * and memsets on `stream` and can therefore be captured into a CUDA graph and
 * replayed.  Chunk size of the work queue: LNT_BATCH_CHUNK from the
 * environment, else the autotuned value (1 column). */
LNT_API int lnt_batched_workspace(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                                  const uint64_t* b_off_host, size_t* bytes, uint64_t* c_capacity);
LNT_API int lnt_batched_prepare(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                                const uint64_t* b_off_host, void* workspace, size_t workspace_bytes,
                                void* stream);
LNT_API int lnt_batched_lattice_mult(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                                     const uint64_t* b_off_host, const uint64_t* a_keys,
                                     const double* a_vals, const uint64_t* b_keys, const double* b_vals,
                                     void* workspace, size_t workspace_bytes, uint64_t* c_keys,
                                     double* c_vals, uint64_t* d_c_off, void* stream);

/* The same batch with the operands as the tensors store them: unsorted, each
 * key linearised in its tensor's own mode order.  Problem p's A keys are
 * re-keyed by a_rekey_host[p] and its B keys by b_rekey_host[p] into lattice
 * order (order 0 = already in lattice order; NULL array = all order 0), and
 * both are sorted inside the call -- the per-product toLatticeSort of the
 * reference (SparseMIABase.h:1457-1586; for c(i,l) = a(i,j,k) * b(k,l,j): A
 * as it is, B to the mode order {2,0,1}, SparseMIABase.h:1527-1586) done for
 * the whole batch by one radix sort over keys prefixed with the problem index
 * -- then multiplied as lnt_batched_lattice_mult does.  Keys must lie below
 * their lattice's size (rows x cols x tabs).  a_off_host[0] and b_off_host[0]
 * must be 0, and the batch holds fewer than 2^30 pairs.  Call
 * lnt_batched_contract_prepare once per batch layout (synchronous uploads),
 * then lnt_batched_contract, which only enqueues work on `stream` and can be
 * captured into a CUDA graph. */
LNT_API int lnt_batched_contract_workspace(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                                           const uint64_t* b_off_host, size_t* bytes, uint64_t* c_capacity);
LNT_API int lnt_batched_contract_prepare(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                                         const uint64_t* b_off_host, const lnt_rekey_spec* a_rekey_host,
                                         const lnt_rekey_spec* b_rekey_host, void* workspace,
                                         size_t workspace_bytes, void* stream);
LNT_API int lnt_batched_contract(int count, const int64_t* dims_host, const uint64_t* a_off_host,
                                 const uint64_t* b_off_host, const uint64_t* a_keys, const double* a_vals,
                                 const uint64_t* b_keys, const double* b_vals, void* workspace,
                                 size_t workspace_bytes, uint64_t* c_keys, double* c_vals, uint64_t* d_c_off,
                                 void* stream);

/* ---- dense lattice product ---------------------------------------------- */

/* Dense mode permutation, float64 column-major: out has extent dims[perm[k]]
 * in mode k and out(i_0, ..., i_{order-1}) = in(j) with j_{perm[k]} = i_k.
 * The copy that puts a dense operand's modes in lattice order before a
 * product: latticeCopy (FunctionUtil.h:195) and DenseMIA::inplace_permute
 * (DenseMIA.h:700-780, same reshuffle_order convention; here out of place).
 * out must not overlap in.  LNT_BAD_SEQ when perm is not a permutation of
 * 0..order-1. */
LNT_API int lnt_dense_permute(const double* in, double* out, int order, const int64_t* dims,
                              const int32_t* perm, void* stream);


/* C(:,:,t) = A(:,:,t) * B(:,:,t) for t < d; A is h x w, B is w x wB, C is
 * h x wB, all float64 column-major, tabs stored one after another.  Replaces
 * DenseLatticeBase::operator* (DenseLatticeBase.h:404-430, an Eigen GEMM per
 * tab) as used by DenseMIA products (DenseMIA.h:200, 1240-1255).
 * _fp64: plain float64 GEMM per tab (workspace from lnt_dense_fp64_workspace).
 * _split: float64 operands split into `slices` signed 7-bit integer slices
 * per row of A / column of B (power-of-two scaled), exact INT8 tensor-core
 * products with INT32 accumulation, float64 recombination with compensated
 * summation; error about 2^(-7 slices + 1) |A||B| per entry (slices = 7 for
 * float64-class accuracy, <= 1e-12 relative).  Requires slices * w < 2^19. */
LNT_API int lnt_dense_fp64_workspace(size_t* bytes);
LNT_API int lnt_dense_lattice_mult_fp64(const double* A, const double* B, double* C, int64_t h,
                                        int64_t w, int64_t wB, int64_t d, void* workspace,
                                        size_t workspace_bytes, void* stream);
LNT_API int lnt_dense_split_workspace(int64_t h, int64_t w, int64_t wB, int slices, size_t* bytes);
LNT_API int lnt_dense_lattice_mult_split(const double* A, const double* B, double* C, int64_t h,
                                         int64_t w, int64_t wB, int64_t d, int slices,
                                         void* workspace, size_t workspace_bytes, void* stream);

/* _crt: float64 operands rounded to beta-bit integers per row of A / column of
 * B (power-of-two scaled), products computed exactly modulo `moduli` pairwise
 * coprime integers <= 256 as INT8 tensor-core GEMMs (tcgen05) with INT32
 * accumulation, each product reduced modulo its modulus in the GEMM's
 * epilogue, and reconstructed by Chinese remaindering in exact integers;
 * beta = min(floor((log2 prod(moduli) - log2 w - 3) / 2), 52), error about
 * 2^(2-beta) |A||B| per entry (13 moduli: beta = 42 at w = 16384; 16 moduli:
 * beta = 52).  Requires w < 2^17 and 2 <= moduli <= 20. */
LNT_API int lnt_dense_crt_workspace(int64_t h, int64_t w, int64_t wB, int moduli, size_t* bytes);
/* The number of moduli for _crt that keeps every entry's error within
 * tol * (|A||B|)_ij (tol = 1e-12 for float64-class results): the error grows
 * with the largest ratio R of a row's (A) or column's (B) maximum magnitude
 * to its mean magnitude, which one pass over A and B measures here; the count
 * is the smallest with beta >= 2 + log2 R + log2(1/tol) (uniform data, R ~ 2:
 * 14 moduli at w = 16384, 13 at w = 4096; mantissas times 2^+-20, R ~ 30: 15
 * at w = 16384).  Synchronous on `stream` (the count is returned to the host);
 * workspace of at least 16 h + 768 bytes, 256-byte aligned. */
LNT_API int lnt_dense_crt_moduli(const double* A, const double* B, int64_t h, int64_t w, int64_t wB, int64_t d,
                                 double tol, void* workspace, size_t workspace_bytes, int* moduli, void* stream);
LNT_API int lnt_dense_lattice_mult_crt(const double* A, const double* B, double* C, int64_t h,
                                       int64_t w, int64_t wB, int64_t d, int moduli,
                                       void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LNT_H */
