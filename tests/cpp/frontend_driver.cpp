// Drives the C++ index-label front end (libnt_b200/include/lnt/lnt.hpp) for
// tests/test_gpu_frontend.py: reads operands from raw files in a directory,
// evaluates one expression written exactly as a LibNT user would, and writes
// the result and the operands' post-states back.
//
//   frontend_driver <scenario> <dir>
// Files: <name>.keys (uint64), <name>.vals (float64), <name>.meta (text:
// order, dims..., seq..., sorted).  Scenarios: product, product_assign,
// elementwise, elementwise_decrement, ternary, elem_assign, repeated_elem,
// dense_assign_perm, push_back, outer_inter, outer, trace, attract, merge_add, merge_sub,
// merge_self, plus_equals, sort_seq, collect, dense, dense_perm, mixed_sd,
// mixed_sd_inter, mixed_ds, mixed_ds_inter, mixed_sd_perm, mixed_ds_perm.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "lnt/lnt.hpp"

namespace {

std::string g_dir;

template <class T>
std::vector<T> read_raw(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return {};
  const size_t n = (size_t)f.tellg() / sizeof(T);
  std::vector<T> v(n);
  f.seekg(0);
  f.read(reinterpret_cast<char*>(v.data()), n * sizeof(T));
  return v;
}

template <class T>
void write_raw(const std::string& path, const std::vector<T>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(T));
}

void load(lnt::SparseTensor& t, const std::string& name) {
  std::ifstream m(g_dir + "/" + name + ".meta");
  size_t order;
  m >> order;
  std::vector<int64_t> dims(order);
  std::vector<int> seq(order);
  for (auto& d : dims) m >> d;
  for (auto& s : seq) m >> s;
  int sorted;
  m >> sorted;
  t = lnt::SparseTensor(dims);
  t.assign_host(read_raw<uint64_t>(g_dir + "/" + name + ".keys"), read_raw<double>(g_dir + "/" + name + ".vals"),
                sorted != 0, seq);
}

void save(const lnt::SparseTensor& t, const std::string& name) {
  std::vector<uint64_t> k;
  std::vector<double> v;
  t.download(k, v);
  write_raw(g_dir + "/" + name + ".keys", k);
  write_raw(g_dir + "/" + name + ".vals", v);
  std::ofstream m(g_dir + "/" + name + ".meta");
  m << t.order();
  for (auto d : t.dims()) m << ' ' << d;
  for (auto s : t.linIdxSequence()) m << ' ' << s;
  m << ' ' << (t.is_sorted() ? 1 : 0) << '\n';
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::cerr << "usage: frontend_driver <scenario> <dir>\n";
    return 2;
  }
  const std::string sc = argv[1];
  g_dir = argv[2];
  try {
    lnt::Index i, j, k, l, m, n;
    if (sc == "product" || sc == "product_assign") {
      lnt::SparseNT<3> a, b;
      load(a, "a");
      load(b, "b");
      lnt::SparseNT<2> c;
      if (sc == "product")
        c(i, l) = a(i, j, k) * b(k, l, j);
      else
        c(l, i) = a(i, j, k) * b(k, l, j);
      save(c, "c");
      save(a, "a_after");
      save(b, "b_after");
    } else if (sc == "elementwise") {
      lnt::SparseNT<3> a, b, d;
      load(a, "a");
      load(b, "b");
      d(i, l, !n) = a(i, j, !n) * b(j, l, !n);
      save(d, "c");
    } else if (sc == "elementwise_decrement") {  // ~ turns the result's !n back into n
      lnt::SparseNT<3> a, b, d;
      load(a, "a");
      load(b, "b");
      d(i, l, n) = ~(a(i, j, !n) * b(j, l, !n));
      save(d, "c");
    } else if (sc == "ternary" || sc == "elem_assign" || sc == "repeated_elem") {
      lnt::SparseNT<4> a, b, c;
      lnt::SparseNT<2> b2, d2;
      lnt::SparseNT<1> d;
      load(a, "a");
      load(b, "b");
      load(b2, "b2");
      load(d2, "d2");
      load(d, "d");
      if (sc == "ternary")  // sparse_mia_mult_test.cpp:147-148
        c(i, k, m, n) = ~(a(i, !j, k, !l) * b(!j, !l, m, n)) * d2(j, l);
      else if (sc == "elem_assign")  // :123-124
        c(i, j, k, l) = a(i, !j, k, !l) * b2(!j, !l);
      else  // :142-143
        c(i, j, k, l) = ~(a(i, !j, k, !!l) * b2(!j, !!l)) * d(!l);
      save(c, "c");
    } else if (sc == "dense_assign_perm") {  // c(n,m,j,i) = a(i,j,k,l) * b(k,l,m,n)
      std::ifstream meta(g_dir + "/dense.meta");
      int64_t d1, d2;
      int slices;
      meta >> d1 >> d2 >> slices;
      lnt::DenseNT<4> a(d1, d1, d2, d2), b(d2, d2, d1, d1), c(d1, d1, d1, d1);
      a.upload(read_raw<double>(g_dir + "/A.vals"));
      b.upload(read_raw<double>(g_dir + "/B.vals"));
      c(n, m, j, i) = a(i, j, k, l) * b(k, l, m, n);
      std::vector<double> hv;
      c.download(hv);
      write_raw(g_dir + "/C.vals", hv);
    } else if (sc == "push_back") {  // build a tensor entry by entry
      lnt::SparseNT<3> a, b;
      load(a, "a");
      load(b, "b");
      std::vector<uint64_t> k;
      std::vector<double> v;
      a.download(k, v);
      lnt::SparseNT<3> t(a.dim(0), a.dim(1), a.dim(2));
      for (size_t q = 0; q < k.size(); ++q) t.push_back(v[q], k[q]);
      save(t, "c");
      t.sort();
      save(t, "c_sorted");
      b.download(k, v);
      for (size_t q = 0; q < k.size(); ++q) t.push_back(v[q], k[q]);
      save(t, "c3");
    } else if (sc == "outer_inter") {  // noLatticeMult: outer i, l with element-wise n
      lnt::SparseNT<2> a, b;
      lnt::SparseNT<3> d;
      load(a, "a");
      load(b, "b");
      d(i, l, !n) = a(i, !n) * b(!n, l);
      save(d, "c");
      save(a, "a_after");
      save(b, "b_after");
    } else if (sc == "outer") {  // noLatticeMult: pure outer product
      lnt::SparseNT<2> a, b;
      lnt::SparseNT<4> d;
      load(a, "a");
      load(b, "b");
      d(i, j, k, l) = a(i, j) * b(k, l);
      save(d, "c");
      save(a, "a_after");
      save(b, "b_after");
    } else if (sc == "trace") {  // contract_attract: double trace
      lnt::SparseNT<5> a;
      lnt::SparseNT<1> c;
      load(a, "a");
      c(k) = a(i, j, i, j, k);
      save(c, "c");
      save(a, "a_after");
    } else if (sc == "attract") {  // contract_attract: attraction of i, contraction of j
      lnt::SparseNT<5> a;
      lnt::SparseNT<2> c;
      load(a, "a");
      c(k, !i) = a(!i, j, !i, k, j);
      save(c, "c");
      save(a, "a_after");
    } else if (sc == "merge_add" || sc == "merge_sub") {
      lnt::SparseNT<4> a, b, c;
      load(a, "a");
      load(b, "b");
      if (sc == "merge_add")
        c(i, j, k, l) = a(i, j, k, l) + b(l, k, j, i);
      else
        c(i, j, k, l) = a(i, j, k, l) - b(l, k, j, i);
      save(c, "c");
      save(a, "a_after");
      save(b, "b_after");
    } else if (sc == "merge_self") {
      lnt::SparseNT<4> a, c;
      load(a, "a");
      c(i, j, k, l) = a(i, j, k, l) + a(l, k, j, i);
      save(c, "c");
    } else if (sc == "plus_equals") {
      lnt::SparseNT<4> a, b;
      load(a, "a");
      load(b, "b");
      a(i, j, k, l) += b(l, k, j, i);
      save(a, "c");
    } else if (sc == "sort_seq") {
      lnt::SparseNT<4> a;
      load(a, "a");
      a.sort({2, 0, 3, 1});
      save(a, "c");
    } else if (sc == "collect") {
      lnt::SparseNT<4> a;
      load(a, "a");
      a.collect_duplicates();
      save(a, "c");
    } else if (sc == "dense_perm") {  // dense operands whose modes are not in lattice order
      std::ifstream meta(g_dir + "/dense.meta");
      int64_t d1, d2;
      int slices;
      meta >> d1 >> d2 >> slices;
      lnt::DenseNT<4> a(d2, d1, d2, d1), b(d1, d2, d1, d2), c(d1, d1, d1, d1);
      a.upload(read_raw<double>(g_dir + "/A.vals"));
      b.upload(read_raw<double>(g_dir + "/B.vals"));
      lnt::DenseTensor::slices() = slices > 0 ? slices : 0;
      lnt::DenseTensor::precision() =
          slices < 0 ? lnt::DenseTensor::Precision::Float64 : lnt::DenseTensor::Precision::Emulated;
      c(i, j, m, n) = a(k, i, l, j) * b(m, k, n, l);
      std::vector<double> h;
      c.download(h);
      write_raw(g_dir + "/C.vals", h);
    } else if (sc.rfind("mixed_", 0) == 0) {  // sparse x dense / dense x sparse
      std::ifstream meta(g_dir + "/D.meta");
      int64_t e0, e1, e2;
      meta >> e0 >> e1 >> e2;
      lnt::DenseNT<3> D(e0, e1, e2);
      D.upload(read_raw<double>(g_dir + "/D.vals"));
      lnt::SparseNT<3> s;
      load(s, "a");
      if (sc == "mixed_sd") {
        lnt::SparseNT<2> c;
        c(i, l) = s(i, j, k) * D(j, k, l);
        save(c, "c");
      } else if (sc == "mixed_sd_inter") {
        lnt::SparseNT<3> c;
        c(i, l, !n) = s(i, j, !n) * D(j, l, !n);
        save(c, "c");
      } else if (sc == "mixed_sd_perm") {
        lnt::SparseNT<2> c;
        c(i, l) = s(i, j, k) * D(l, k, j);
        save(c, "c");
      } else if (sc == "mixed_ds_perm") {
        lnt::SparseNT<2> c;
        c(i, l) = D(j, i, k) * s(k, l, j);
        save(c, "c");
      } else if (sc == "mixed_ds") {
        lnt::SparseNT<2> c;
        c(i, l) = D(i, j, k) * s(k, l, j);
        save(c, "c");
      } else {
        lnt::SparseNT<3> c;
        c(i, l, !n) = D(i, j, !n) * s(l, j, !n);
        save(c, "c");
      }
      save(s, "a_after");
    } else if (sc == "dense") {
      std::ifstream meta(g_dir + "/dense.meta");
      int64_t d1, d2;
      int slices;
      meta >> d1 >> d2 >> slices;
      lnt::DenseNT<4> a(d1, d1, d2, d2), b(d2, d2, d1, d1), c(d1, d1, d1, d1);
      a.upload(read_raw<double>(g_dir + "/A.vals"));
      b.upload(read_raw<double>(g_dir + "/B.vals"));
      lnt::DenseTensor::slices() = slices > 0 ? slices : 0;
      lnt::DenseTensor::precision() =
          slices < 0 ? lnt::DenseTensor::Precision::Float64 : lnt::DenseTensor::Precision::Emulated;
      c(i, j, m, n) = a(i, j, k, l) * b(k, l, m, n);
      std::vector<double> h;
      c.download(h);
      write_raw(g_dir + "/C.vals", h);
    } else {
      std::cerr << "unknown scenario " << sc << "\n";
      return 2;
    }
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
