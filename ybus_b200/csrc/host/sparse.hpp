// Host-side sparse matrices and factorizations: the factor producer of the solve path.
//
// The GPU path solves against a factor made once on the host in FP64. In ybus that factor comes
// from ybus_sparse (Rust). This header holds the same algorithms, written for this library so it
// can make the factors it uploads by itself:
//
//   - triplet assembly with duplicates summed in input order
//       (ybus_sparse/src/compressed_matrix.rs:254-330, `assemble`)
//   - the symmetrised adjacency graph (ybus_sparse/src/compressed_matrix/ordering.rs:73-118)
//   - approximate minimum degree (ordering.rs:258-492), with the same tie rule (the node most
//     recently given its degree goes first) so the permutation is the one ybus_sparse computes
//   - COLAMD column ordering (ybus_sparse/src/compressed_matrix/colamd.rs:91-261)
//   - symbolic Cholesky: Liu's elimination tree and sorted row patterns (cholesky.rs:81-149)
//   - up-looking numeric Cholesky, L in CSR with the diagonal last and Lᴴ in CSR with the
//     diagonal first (cholesky.rs:206-311)
//   - Gilbert–Peierls LU with threshold partial pivoting, real or complex (lu.rs:268-417)
//
// Everything is FP64 (or complex128), templated on the scalar type.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <numeric>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace yb::host {

using idx_t = int64_t;
using c128 = std::complex<double>;

template <class T> struct is_complex : std::false_type {};
template <class R> struct is_complex<std::complex<R>> : std::true_type {};

inline double conj_of(double v) { return v; }
inline c128 conj_of(c128 v) { return std::conj(v); }
inline double abs_of(double v) { return std::fabs(v); }
inline double abs_of(c128 v) { return std::abs(v); }
inline double real_of(double v) { return v; }
inline double real_of(c128 v) { return v.real(); }
inline double magnitude_squared(double v) { return v * v; }
inline double magnitude_squared(c128 v) { return v.real() * v.real() + v.imag() * v.imag(); }

// An error the C ABI turns into a status code.
struct Error : std::runtime_error {
  int status;
  idx_t where;
  Error(int status_, const std::string &what, idx_t where_ = -1)
      : std::runtime_error(what), status(status_), where(where_) {}
};

// Status codes shared with the C ABI (include/ybgpu.h).
enum Status : int {
  kOk = 0,
  kInvalidArgument = 1,
  kShapeMismatch = 2,
  kTooLarge = 3,
  kNotPositiveDefinite = 4,
  kSingular = 5,
  kNoDevice = 6,
  kCuda = 7,
  kNotSymmetric = 8,
  kDeviceTimeout = 9,
  kInternal = 10,
};

// A compressed sparse matrix. `rows`/`cols` are the matrix's shape; `by_rows` says whether `ptr`
// runs over rows (CSR) or columns (CSC). Minor indices are sorted within each major slice.
template <class T> struct Compressed {
  idx_t rows = 0, cols = 0;
  bool by_rows = true;
  std::vector<idx_t> ptr, idx;
  std::vector<T> val;

  idx_t major() const { return by_rows ? rows : cols; }
  idx_t minor() const { return by_rows ? cols : rows; }
  idx_t stored() const { return (idx_t)idx.size(); }
};

template <class T> struct Triplet {
  idx_t row, col;
  T value;
};

// Triplets to a compressed matrix: grouped by major idx_t keeping input order, sorted stably by
// minor idx_t, duplicates summed in input order.
template <class T>
Compressed<T> from_triplets(idx_t rows, idx_t cols, const std::vector<Triplet<T>> &triplets,
                            bool by_rows = true) {
  Compressed<T> m;
  m.rows = rows;
  m.cols = cols;
  m.by_rows = by_rows;
  const idx_t major_dim = by_rows ? rows : cols;
  for (const auto &t : triplets) {
    if (t.row < 0 || t.row >= rows || t.col < 0 || t.col >= cols)
      throw Error(kInvalidArgument, "a triplet lies outside the matrix");
  }
  std::vector<idx_t> start(major_dim + 1, 0);
  for (const auto &t : triplets) start[(by_rows ? t.row : t.col) + 1]++;
  for (idx_t i = 0; i < major_dim; ++i) start[i + 1] += start[i];
  std::vector<idx_t> cursor(start.begin(), start.end() - 1);
  struct Entry {
    idx_t minor;
    T value;
  };
  std::vector<Entry> grouped(triplets.size());
  for (const auto &t : triplets) {
    idx_t major = by_rows ? t.row : t.col;
    grouped[cursor[major]++] = Entry{by_rows ? t.col : t.row, t.value};
  }
  m.ptr.assign(major_dim + 1, 0);
  m.idx.reserve(triplets.size());
  m.val.reserve(triplets.size());
  for (idx_t major = 0; major < major_dim; ++major) {
    auto first = grouped.begin() + start[major], last = grouped.begin() + start[major + 1];
    std::stable_sort(first, last, [](const Entry &a, const Entry &b) { return a.minor < b.minor; });
    const idx_t row_start = (idx_t)m.idx.size();
    for (auto it = first; it != last; ++it) {
      if ((idx_t)m.idx.size() > row_start && m.idx.back() == it->minor) {
        m.val.back() = m.val.back() + it->value;
      } else {
        m.idx.push_back(it->minor);
        m.val.push_back(it->value);
      }
    }
    m.ptr[major + 1] = (idx_t)m.idx.size();
  }
  return m;
}

// The other orientation of the same matrix (CSR <-> CSC), minor indices sorted.
template <class T> Compressed<T> reorient(const Compressed<T> &a) {
  Compressed<T> t;
  t.rows = a.rows;
  t.cols = a.cols;
  t.by_rows = !a.by_rows;
  const idx_t nmaj = a.minor();
  t.ptr.assign(nmaj + 1, 0);
  for (idx_t p = 0; p < a.stored(); ++p) t.ptr[a.idx[p] + 1]++;
  for (idx_t i = 0; i < nmaj; ++i) t.ptr[i + 1] += t.ptr[i];
  t.idx.resize(a.stored());
  t.val.resize(a.stored());
  std::vector<idx_t> cursor(t.ptr.begin(), t.ptr.end() - 1);
  for (idx_t j = 0; j < a.major(); ++j)
    for (idx_t p = a.ptr[j]; p < a.ptr[j + 1]; ++p) {
      idx_t q = cursor[a.idx[p]]++;
      t.idx[q] = j;
      t.val[q] = a.val[p];
    }
  return t;
}

// Rows `rows` and columns `cols` of `a`, in those orders (ybus_sparse access.rs:175-216).
template <class T>
Compressed<T> select(const Compressed<T> &a, const std::vector<idx_t> &rows,
                     const std::vector<idx_t> &cols) {
  const auto &majors = a.by_rows ? rows : cols;
  const auto &minors = a.by_rows ? cols : rows;
  std::vector<std::vector<idx_t>> positions(a.minor());
  for (idx_t pos = 0; pos < (idx_t)minors.size(); ++pos) positions.at(minors[pos]).push_back(pos);
  Compressed<T> s;
  s.rows = (idx_t)rows.size();
  s.cols = (idx_t)cols.size();
  s.by_rows = a.by_rows;
  s.ptr.push_back(0);
  std::vector<std::pair<idx_t, T>> segment;
  for (idx_t major : majors) {
    segment.clear();
    for (idx_t p = a.ptr.at(major); p < a.ptr.at(major + 1); ++p)
      for (idx_t pos : positions[a.idx[p]]) segment.push_back({pos, a.val[p]});
    std::stable_sort(segment.begin(), segment.end(),
                     [](const auto &x, const auto &y) { return x.first < y.first; });
    for (auto &e : segment) {
      s.idx.push_back(e.first);
      s.val.push_back(e.second);
    }
    s.ptr.push_back((idx_t)s.idx.size());
  }
  return s;
}

// Entry (i, j) of the result is entry (perm[i], perm[j]) of `a`.
template <class T> Compressed<T> permute_symmetric(const Compressed<T> &a, const std::vector<idx_t> &perm) {
  return select(a, perm, perm);
}

// The graph of A + Aᵀ without self loops: sorted, duplicate-free neighbour lists.
struct Adjacency {
  std::vector<idx_t> start, neighbours;
  idx_t size() const { return (idx_t)start.size() - 1; }
  idx_t degree(idx_t i) const { return start[i + 1] - start[i]; }
  const idx_t *begin(idx_t i) const { return neighbours.data() + start[i]; }
  const idx_t *end(idx_t i) const { return neighbours.data() + start[i + 1]; }
};

template <class T> Adjacency adjacency_of(const Compressed<T> &a) {
  const idx_t n = a.rows;
  Adjacency g;
  std::vector<idx_t> count(n + 1, 0);
  for (idx_t j = 0; j < a.major(); ++j)
    for (idx_t p = a.ptr[j]; p < a.ptr[j + 1]; ++p) {
      idx_t i = a.idx[p];
      if (i != j) {
        count[i + 1]++;
        count[j + 1]++;
      }
    }
  for (idx_t i = 0; i < n; ++i) count[i + 1] += count[i];
  std::vector<idx_t> cursor(count.begin(), count.end() - 1);
  std::vector<idx_t> raw(count[n]);
  for (idx_t j = 0; j < a.major(); ++j)
    for (idx_t p = a.ptr[j]; p < a.ptr[j + 1]; ++p) {
      idx_t i = a.idx[p];
      if (i != j) {
        raw[cursor[i]++] = j;
        raw[cursor[j]++] = i;
      }
    }
  g.start.assign(n + 1, 0);
  g.neighbours.reserve(raw.size());
  for (idx_t i = 0; i < n; ++i) {
    std::sort(raw.begin() + count[i], raw.begin() + count[i + 1]);
    for (idx_t k = count[i]; k < count[i + 1]; ++k)
      if (k == count[i] || raw[k] != raw[k - 1]) g.neighbours.push_back(raw[k]);
    g.start[i + 1] = (idx_t)g.neighbours.size();
  }
  return g;
}

// Approximate minimum degree ordering; returns perm with row i of P A Pᵀ = row perm[i] of A.
std::vector<idx_t> approximate_minimum_degree(const Adjacency &graph);

// COLAMD column ordering of a rows x cols pattern given as (row, col) pairs.
std::vector<idx_t> column_amd(idx_t rows, idx_t cols, const std::vector<std::pair<idx_t, idx_t>> &entries);

// Cholesky factor P A Pᵀ = L Lᴴ: L in CSR (rows sorted, diagonal last), Lᴴ in CSR (diagonal first).
template <class T> struct Cholesky {
  idx_t n = 0;
  std::vector<idx_t> perm;
  std::vector<idx_t> parent;  // elimination tree, -1 for a root
  Compressed<T> l, lh;
};

struct SymbolicCholesky {
  idx_t n = 0;
  std::vector<idx_t> perm, parent, l_ptr, l_idx;
};

SymbolicCholesky analyze_cholesky(const Adjacency &graph, std::vector<idx_t> perm);

template <class T> Cholesky<T> factor_cholesky(const Compressed<T> &a_csr, const SymbolicCholesky &sym);

// LU factor P A Q = L U: L unit lower in CSC (diagonal first), U upper in CSC (diagonal last).
template <class T> struct Lu {
  idx_t n = 0;
  std::vector<idx_t> row_perm, col_perm;
  Compressed<T> l, u;
};

template <class T>
Lu<T> factor_lu(const Compressed<T> &a_csc, const std::vector<idx_t> &col_perm, double tau,
                bool prefer_diagonal);

}  // namespace yb::host
