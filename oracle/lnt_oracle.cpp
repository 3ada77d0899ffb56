/*
 * lnt_oracle.cpp - CPU restatement of the reference (extragoya/LibNT) hot
 * path, built into oracle/liblnt_oracle.so.
 *
 * TEST INFRASTRUCTURE ONLY.  This code is the checker: tests/, the smoke
 * check and bench.py's CPU-baseline leg call it to produce expected results.
 * No product code path links or calls it.
 *
 * Each function restates the reference lines it cites, written from their
 * behaviour (the reference's Boost/Eigen-bound glue cannot be compiled here).
 * Parity of these restatements is pinned by tests/test_oracle.py against
 * the reference's own compiled kernels (oracle/_ref), the reference's golden
 * fixtures (DenseLattice test1.bin, test2.bin, multtest_ddd.bin) and its known-answer tests.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

extern "C" {

/* Re-linearise keys from cur_seq to new_seq.  Restates
 * create_shuffle_needs + reShuffleLinearIndex (IndexUtil.h:480-487, 567-589)
 * with plain 64-bit division instead of libdivide (identical quotients). */
void lnto_rekey(const uint64_t* in, uint64_t* out, size_t n, int order, const int64_t* dims,
                const int32_t* cur_seq, const int32_t* new_seq) {
    if (order <= 1) {
        if (in != out) std::memmove(out, in, n * sizeof(uint64_t));
        return;
    }
    std::vector<uint64_t> acc(order), mult(order), stride_of_mode(order);
    uint64_t a = 1;
    for (int i = 0; i < order; ++i) {  // createDimAccumulator over current-order dims
        acc[i] = a;
        a *= (uint64_t)dims[cur_seq[i]];
    }
    uint64_t s = 1;
    for (int i = 0; i < order; ++i) {  // createMultiplier over new-order dims
        stride_of_mode[new_seq[i]] = s;
        s *= (uint64_t)dims[new_seq[i]];
    }
    for (int i = 0; i < order; ++i) mult[i] = stride_of_mode[cur_seq[i]];  // reorder by shuffle sequence
    for (size_t j = 0; j < n; ++j) {
        uint64_t idx = in[j], o = 0;
        for (int i = order - 1; i >= 1; --i) {
            uint64_t q = idx / acc[i];
            o += q * mult[i];
            idx -= q * acc[i];
        }
        out[j] = o + idx * mult[0];
    }
}

/* Ascending sort of (key, value) pairs by key, equal keys in input order.
 * The reference's sort (RadixSortInPlace_PowerOf2Radix_Unsigned,
 * LibMIARadix.h:444-484) orders keys identically; it is unstable, so the
 * order among equal keys is not part of its contract. */
void lnto_sort_pairs(uint64_t* keys, double* vals, size_t n) {
    std::vector<size_t> p(n);
    std::iota(p.begin(), p.end(), 0);
    std::stable_sort(p.begin(), p.end(), [&](size_t x, size_t y) { return keys[x] < keys[y]; });
    std::vector<uint64_t> k(n);
    std::vector<double> v(n);
    for (size_t i = 0; i < n; ++i) {
        k[i] = keys[p[i]];
        v[i] = vals[p[i]];
    }
    std::memcpy(keys, k.data(), n * 8);
    std::memcpy(vals, v.data(), n * 8);
}

/* Fold runs of equal keys of a key-sorted array with +, in place; returns
 * the new length.  skip_zero_heads != 0 restates SparseMIA::collect_duplicates
 * (SparseMIA.h:636-665): an element that would start a new key is skipped
 * when its value is exactly zero (`if(this->data_at(first))`, :650), the
 * element at position 0 always starts the output (:645-647).
 * skip_zero_heads == 0 restates collect_duplicates_function
 * (FunctionUtil.h:701-728), which keeps every run.
 * If abs_out is non-NULL it receives, per output element, the sum of |addend|
 * (the scale of the summation error). */
size_t lnto_collect_duplicates(uint64_t* keys, double* vals, size_t n, int skip_zero_heads, double* abs_out) {
    if (n == 0) return 0;
    size_t r = 0;  // result position
    if (abs_out) abs_out[0] = std::fabs(vals[0]);
    for (size_t f = 1; f < n; ++f) {
        if (keys[r] != keys[f]) {
            if (!skip_zero_heads || vals[f] != 0.0) {
                ++r;
                keys[r] = keys[f];
                vals[r] = vals[f];
                if (abs_out) abs_out[r] = std::fabs(vals[f]);
            }
        } else {
            vals[r] = vals[r] + vals[f];
            if (abs_out) abs_out[r] += std::fabs(vals[f]);
        }
    }
    return r + 1;
}

/* Two-way merge of two key-sorted operands in the same linearisation;
 * restates outside_merge_sparse_storage_containers (FunctionUtil.h:373-419):
 * A-only entries copied, B-only entries op(0, b), equal keys op(a, b) (one A
 * and one B consumed per step); every entry kept, exact zeros included.
 * op: 0 = +, 1 = -.  c arrays hold na + nb.  Returns the output length. */
size_t lnto_merge_sorted(const uint64_t* ak, const double* av, size_t na, const uint64_t* bk, const double* bv,
                         size_t nb, int op, uint64_t* ck, double* cv) {
    auto f = [op](double a, double b) { return op == 0 ? a + b : a - b; };
    size_t i = 0, j = 0, c = 0;
    while (i < na && j < nb) {
        if (ak[i] < bk[j]) {
            ck[c] = ak[i];
            cv[c++] = av[i++];
        } else if (bk[j] < ak[i]) {
            ck[c] = bk[j];
            cv[c++] = f(0.0, bv[j++]);
        } else {
            ck[c] = ak[i];
            cv[c++] = f(av[i++], bv[j++]);
        }
    }
    while (j < nb) {
        ck[c] = bk[j];
        cv[c++] = f(0.0, bv[j++]);
    }
    while (i < na) {
        ck[c] = ak[i];
        cv[c++] = av[i++];
    }
    return c;
}

/* Sparse lattice product C_t = A_t * B_t for every tab t present in both;
 * restates SparseLatticeBase::csc_no_accum<true> (SparseLatticeBase.h:1854-1990)
 * with mult_scatter (:1993-2031) and collect_duplicates_function.
 * A: h x w x d, keys row + h*(col + w*tab), sorted ascending.
 * B: w x wB x d, keys row + w*(col + wB*tab), sorted ascending.
 * C keys row + h*(col + wB*tab), ascending; duplicates summed, zeros kept.
 * Per B column the scattered products are ordered by row with a stable sort
 * (the reference uses its unstable radix sort there) and folded in order.
 * Call with ck == NULL to get the output length only.  cabs (optional)
 * receives per output element the sum of |products|. */
size_t lnto_lattice_mult(const uint64_t* ak, const double* av, size_t na, int64_t h, int64_t w, int64_t d,
                         const uint64_t* bk, const double* bv, size_t nb, int64_t wB, uint64_t* ck, double* cv,
                         double* cabs) {
    (void)d;
    const uint64_t H = (uint64_t)h, W = (uint64_t)w, WB = (uint64_t)wB;
    size_t out = 0;
    size_t ia = 0, ib = 0;
    std::vector<uint64_t> rows;
    std::vector<double> prods, mags;
    std::vector<size_t> perm;
    while (ia < na && ib < nb) {
        uint64_t ta = ak[ia] / (H * W), tb = bk[ib] / (W * WB);
        if (ta < tb) {  // advance A to B's tab
            while (ia < na && ak[ia] / (H * W) < tb) ++ia;
            continue;
        }
        if (tb < ta) {
            while (ib < nb && bk[ib] / (W * WB) < ta) ++ib;
            continue;
        }
        const uint64_t tab = ta;
        size_t ea = ia, eb = ib;
        while (ea < na && ak[ea] / (H * W) == tab) ++ea;
        while (eb < nb && bk[eb] / (W * WB) == tab) ++eb;
        // column pointers of A's tab (createJCCPIR / MultHelper, :121-193, :1462-1558)
        std::vector<size_t> colptr(W + 1, 0);
        for (size_t x = ia; x < ea; ++x) colptr[(ak[x] / H) % W + 1]++;
        for (uint64_t c = 0; c < W; ++c) colptr[c + 1] += colptr[c];
        size_t y = ib;
        while (y < eb) {
            const uint64_t col = (bk[y] / W) % WB;
            rows.clear();
            prods.clear();
            mags.clear();
            while (y < eb && (bk[y] / W) % WB == col) {
                const uint64_t brow = bk[y] % W;
                const double beta = bv[y];
                for (size_t x = ia + colptr[brow]; x < ia + colptr[brow + 1]; ++x) {
                    rows.push_back(ak[x] % H);
                    prods.push_back(beta * av[x]);
                    mags.push_back(std::fabs(beta * av[x]));
                }
                ++y;
            }
            if (rows.empty()) continue;
            perm.resize(rows.size());
            std::iota(perm.begin(), perm.end(), 0);
            std::stable_sort(perm.begin(), perm.end(), [&](size_t p, size_t q) { return rows[p] < rows[q]; });
            size_t k = 0;
            while (k < perm.size()) {
                const uint64_t r = rows[perm[k]];
                double s = prods[perm[k]], m = mags[perm[k]];
                size_t k2 = k + 1;
                while (k2 < perm.size() && rows[perm[k2]] == r) {
                    s = s + prods[perm[k2]];
                    m += mags[perm[k2]];
                    ++k2;
                }
                if (ck) {
                    ck[out] = r + H * (col + WB * tab);
                    cv[out] = s;
                    if (cabs) cabs[out] = m;
                }
                ++out;
                k = k2;
            }
        }
        ia = ea;
        ib = eb;
    }
    return out;
}

/* Dense lattice product, column-major per tab: C(:,:,t) = A(:,:,t) B(:,:,t)
 * (DenseLatticeBase::operator*, DenseLatticeBase.h:404-430, an Eigen GEMM per
 * tab).  A is h x w, B is w x wB, C is h x wB; k summed in ascending order. */
void lnto_dense_lattice_mult(const double* A, const double* B, double* C, int64_t h, int64_t w, int64_t wB,
                             int64_t d) {
    for (int64_t t = 0; t < d; ++t) {
        const double* At = A + (size_t)t * h * w;
        const double* Bt = B + (size_t)t * w * wB;
        double* Ct = C + (size_t)t * h * wB;
        for (int64_t c = 0; c < wB; ++c) {
            double* col = Ct + (size_t)c * h;
            for (int64_t r = 0; r < h; ++r) col[r] = 0.0;
            for (int64_t k = 0; k < w; ++k) {
                const double b = Bt[(size_t)c * w + k];
                const double* acol = At + (size_t)k * h;
                for (int64_t r = 0; r < h; ++r) col[r] += acol[r] * b;
            }
        }
    }
}

/* Selected entries of a single-tab dense product, each computed as an
 * error-free-transformed dot product (TwoProduct by fma + Neumaier's
 * compensated summation), plus sum |a_rk b_kc| per entry.  Used as the FP64
 * reference for measuring the error of split-precision products. */
void lnto_dense_entries(const double* A, const double* B, int64_t h, int64_t w, const int64_t* rows,
                        const int64_t* cols, size_t m, double* out, double* abs_out) {
    for (size_t e = 0; e < m; ++e) {
        const int64_t r = rows[e], c = cols[e];
        double s = 0.0, comp = 0.0, mag = 0.0;
        for (int64_t k = 0; k < w; ++k) {
            const double a = A[(size_t)k * h + r], b = B[(size_t)c * w + k];
            const double p = a * b;
            const double pe = std::fma(a, b, -p);  // exact low part of a*b
            const double t = s + p;
            if (std::fabs(s) >= std::fabs(p))
                comp += (s - t) + p;
            else
                comp += (p - t) + s;
            s = t;
            comp += pe;
            mag += std::fabs(p);
        }
        out[e] = s + comp;
        if (abs_out) abs_out[e] = mag;
    }
}

}  // extern "C"
