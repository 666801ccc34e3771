// C ABI of the host-side factor producer (libybhost.so, no GPU code): assemble a matrix from
// triplets, select rows and columns, factor by AMD-ordered Cholesky or by LU (AMD or COLAMD
// column order), and copy the factors out; and the thread-local last error every entry point of
// libybhost.so and libybgpu.so reports through. These stand in for the ybus_sparse calls whose results ybus_cuda uploads
// (ybus_cuda/src/factor.rs:103-133 takes a `Cholesky<f64>` or `Lu<f64>` made by ybus_sparse).
#include <memory>
#include <vector>

#include "../../include/ybhost.h"
#include "capi_common.hpp"
#include "host/sparse.hpp"

using namespace yb;
using host::c128;
using host::idx_t;

namespace {
thread_local std::string last_error;
}

namespace yb {
void set_last_error(const std::string &message) { last_error = message; }
void clear_last_error() { last_error.clear(); }
}  // namespace yb

struct yb_matrix {
  bool is_complex = false;
  host::Compressed<double> real;
  host::Compressed<c128> cplx;
};

struct yb_host_factor {
  int kind = 0;  // YB_CHOLESKY or YB_LU
  bool is_complex = false;
  host::Cholesky<double> chol;
  host::Lu<double> lu;
  host::Lu<c128> lu_c;
};

extern "C" {

int32_t yb_last_error_message(char *buffer, size_t length) {
  const size_t need = last_error.size() + 1;
  if (buffer && length) {
    const size_t copy = std::min(length - 1, last_error.size());
    std::memcpy(buffer, last_error.data(), copy);
    buffer[copy] = '\0';
  }
  return (int32_t)need;
}

int32_t yb_matrix_from_triplets(int64_t rows, int64_t cols, int64_t count, const int64_t *row_idx,
                                const int64_t *col_idx, const double *values, int32_t by_rows,
                                int32_t is_complex, yb_matrix **out) {
  return guard([&] {
    require(out != nullptr, "out is null");
    require(rows >= 0 && cols >= 0 && count >= 0, "negative size");
    require(count == 0 || (row_idx && col_idx && values), "null triplet arrays");
    auto m = std::make_unique<yb_matrix>();
    m->is_complex = is_complex != 0;
    if (m->is_complex) {
      std::vector<host::Triplet<c128>> t(count);
      for (int64_t k = 0; k < count; ++k) t[k] = {row_idx[k], col_idx[k], c128(values[2 * k], values[2 * k + 1])};
      m->cplx = host::from_triplets(rows, cols, t, by_rows != 0);
    } else {
      std::vector<host::Triplet<double>> t(count);
      for (int64_t k = 0; k < count; ++k) t[k] = {row_idx[k], col_idx[k], values[k]};
      m->real = host::from_triplets(rows, cols, t, by_rows != 0);
    }
    *out = m.release();
    return YB_OK;
  });
}

int32_t yb_matrix_select(const yb_matrix *m, int64_t n_rows, const int64_t *rows, int64_t n_cols,
                         const int64_t *cols, yb_matrix **out) {
  return guard([&] {
    require(m && out, "null argument");
    std::vector<idx_t> r(rows, rows + n_rows), c(cols, cols + n_cols);
    const idx_t R = m->is_complex ? m->cplx.rows : m->real.rows;
    const idx_t C = m->is_complex ? m->cplx.cols : m->real.cols;
    for (idx_t v : r) require(v >= 0 && v < R, "a selected row is out of range");
    for (idx_t v : c) require(v >= 0 && v < C, "a selected column is out of range");
    auto s = std::make_unique<yb_matrix>();
    s->is_complex = m->is_complex;
    if (m->is_complex)
      s->cplx = host::select(m->cplx, r, c);
    else
      s->real = host::select(m->real, r, c);
    *out = s.release();
    return YB_OK;
  });
}

int32_t yb_matrix_reorient(const yb_matrix *m, yb_matrix **out) {
  return guard([&] {
    require(m && out, "null argument");
    auto s = std::make_unique<yb_matrix>();
    s->is_complex = m->is_complex;
    if (m->is_complex)
      s->cplx = host::reorient(m->cplx);
    else
      s->real = host::reorient(m->real);
    *out = s.release();
    return YB_OK;
  });
}

int32_t yb_matrix_info(const yb_matrix *m, int64_t *rows, int64_t *cols, int64_t *stored,
                       int32_t *by_rows, int32_t *is_complex) {
  return guard([&] {
    require(m != nullptr, "null matrix");
    if (m->is_complex) {
      if (rows) *rows = m->cplx.rows;
      if (cols) *cols = m->cplx.cols;
      if (stored) *stored = m->cplx.stored();
      if (by_rows) *by_rows = m->cplx.by_rows;
    } else {
      if (rows) *rows = m->real.rows;
      if (cols) *cols = m->real.cols;
      if (stored) *stored = m->real.stored();
      if (by_rows) *by_rows = m->real.by_rows;
    }
    if (is_complex) *is_complex = m->is_complex;
    return YB_OK;
  });
}

int32_t yb_matrix_export(const yb_matrix *m, int64_t *ptr, int64_t *idx, double *values) {
  return guard([&] {
    require(m != nullptr, "null matrix");
    if (m->is_complex) {
      const auto &a = m->cplx;
      if (ptr) std::copy(a.ptr.begin(), a.ptr.end(), ptr);
      if (idx) std::copy(a.idx.begin(), a.idx.end(), idx);
      if (values)
        for (size_t k = 0; k < a.val.size(); ++k) {
          values[2 * k] = a.val[k].real();
          values[2 * k + 1] = a.val[k].imag();
        }
    } else {
      const auto &a = m->real;
      if (ptr) std::copy(a.ptr.begin(), a.ptr.end(), ptr);
      if (idx) std::copy(a.idx.begin(), a.idx.end(), idx);
      if (values) std::copy(a.val.begin(), a.val.end(), values);
    }
    return YB_OK;
  });
}

void yb_matrix_free(yb_matrix *m) { delete m; }

int32_t yb_ordering(const yb_matrix *m, int32_t ordering, int64_t *perm) {
  return guard([&] {
    require(m && perm, "null argument");
    std::vector<idx_t> p;
    const idx_t R = m->is_complex ? m->cplx.rows : m->real.rows;
    const idx_t C = m->is_complex ? m->cplx.cols : m->real.cols;
    if (ordering == YB_ORDER_NATURAL) {
      require(R == C, "the ordering needs a square matrix", YB_ERROR_SHAPE_MISMATCH);
      p.resize(R);
      std::iota(p.begin(), p.end(), 0);
    } else if (ordering == YB_ORDER_AMD) {
      require(R == C, "the ordering needs a square matrix", YB_ERROR_SHAPE_MISMATCH);
      p = host::approximate_minimum_degree(m->is_complex ? host::adjacency_of(m->cplx) : host::adjacency_of(m->real));
    } else if (ordering == YB_ORDER_COLAMD) {
      std::vector<std::pair<idx_t, idx_t>> entries;
      auto collect = [&](const auto &a) {
        for (idx_t j = 0; j < a.major(); ++j)
          for (idx_t q = a.ptr[j]; q < a.ptr[j + 1]; ++q)
            entries.push_back(a.by_rows ? std::make_pair(j, a.idx[q]) : std::make_pair(a.idx[q], j));
      };
      if (m->is_complex)
        collect(m->cplx);
      else
        collect(m->real);
      p = host::column_amd(R, C, entries);
    } else {
      require(false, "unknown ordering");
    }
    std::copy(p.begin(), p.end(), perm);
    return YB_OK;
  });
}

int32_t yb_host_cholesky(const yb_matrix *m, int32_t ordering, yb_host_factor **out) {
  return guard([&] {
    require(m && out, "null argument");
    require(!m->is_complex, "the Cholesky path is real");
    require(m->real.by_rows, "Cholesky takes a CSR matrix");
    require(m->real.rows == m->real.cols, "Cholesky needs a square matrix", YB_ERROR_SHAPE_MISMATCH);
    require(ordering != YB_ORDER_COLAMD, "COLAMD orders columns only, which does not apply to Cholesky");
    const auto graph = host::adjacency_of(m->real);
    std::vector<idx_t> perm;
    if (ordering == YB_ORDER_NATURAL) {
      perm.resize(m->real.rows);
      std::iota(perm.begin(), perm.end(), 0);
    } else {
      perm = host::approximate_minimum_degree(graph);
    }
    auto sym = host::analyze_cholesky(graph, std::move(perm));
    auto f = std::make_unique<yb_host_factor>();
    f->kind = YB_CHOLESKY;
    f->chol = host::factor_cholesky(m->real, sym);
    *out = f.release();
    return YB_OK;
  });
}

int32_t yb_host_lu(const yb_matrix *m, int32_t ordering, double pivot_threshold, yb_host_factor **out) {
  return guard([&] {
    require(m && out, "null argument");
    const bool cplx = m->is_complex;
    const bool by_rows = cplx ? m->cplx.by_rows : m->real.by_rows;
    require(!by_rows, "LU takes a CSC matrix");
    const idx_t R = cplx ? m->cplx.rows : m->real.rows;
    const idx_t C = cplx ? m->cplx.cols : m->real.cols;
    require(R == C, "LU needs a square matrix", YB_ERROR_SHAPE_MISMATCH);
    std::vector<idx_t> q;
    bool prefer_diagonal = true;
    if (ordering == YB_ORDER_NATURAL) {
      q.resize(C);
      std::iota(q.begin(), q.end(), 0);
    } else if (ordering == YB_ORDER_AMD) {
      q = host::approximate_minimum_degree(cplx ? host::adjacency_of(m->cplx) : host::adjacency_of(m->real));
    } else if (ordering == YB_ORDER_COLAMD) {
      std::vector<std::pair<idx_t, idx_t>> entries;
      auto collect = [&](const auto &a) {
        for (idx_t j = 0; j < a.cols; ++j)
          for (idx_t p = a.ptr[j]; p < a.ptr[j + 1]; ++p) entries.push_back({a.idx[p], j});
      };
      if (cplx)
        collect(m->cplx);
      else
        collect(m->real);
      q = host::column_amd(R, C, entries);
      prefer_diagonal = false;
    } else {
      require(false, "unknown ordering");
    }
    auto f = std::make_unique<yb_host_factor>();
    f->kind = YB_LU;
    f->is_complex = cplx;
    if (cplx)
      f->lu_c = host::factor_lu(m->cplx, q, pivot_threshold, prefer_diagonal);
    else
      f->lu = host::factor_lu(m->real, q, pivot_threshold, prefer_diagonal);
    *out = f.release();
    return YB_OK;
  });
}

int32_t yb_host_factor_info(const yb_host_factor *f, int32_t *kind, int32_t *is_complex, int64_t *n,
                            int64_t *lower_stored, int64_t *upper_stored) {
  return guard([&] {
    require(f != nullptr, "null factor");
    if (kind) *kind = f->kind;
    if (is_complex) *is_complex = f->is_complex;
    if (f->kind == YB_CHOLESKY) {
      if (n) *n = f->chol.n;
      if (lower_stored) *lower_stored = f->chol.l.stored();
      if (upper_stored) *upper_stored = f->chol.lh.stored();
    } else if (f->is_complex) {
      if (n) *n = f->lu_c.n;
      if (lower_stored) *lower_stored = f->lu_c.l.stored();
      if (upper_stored) *upper_stored = f->lu_c.u.stored();
    } else {
      if (n) *n = f->lu.n;
      if (lower_stored) *lower_stored = f->lu.l.stored();
      if (upper_stored) *upper_stored = f->lu.u.stored();
    }
    return YB_OK;
  });
}

// Cholesky: lower = L (CSR, diagonal last), upper = Lᴴ (CSR, diagonal first), row_perm = col_perm
// = P. LU: lower = L (CSC, unit diagonal first), upper = U (CSC, diagonal last), P and Q.
// Complex values are interleaved (re, im).
int32_t yb_host_factor_export(const yb_host_factor *f, int64_t *lower_ptr, int64_t *lower_idx,
                              double *lower_val, int64_t *upper_ptr, int64_t *upper_idx,
                              double *upper_val, int64_t *row_perm, int64_t *col_perm) {
  return guard([&] {
    require(f != nullptr, "null factor");
    auto put = [](const auto &m, int64_t *ptr, int64_t *idx, double *val) {
      if (ptr) std::copy(m.ptr.begin(), m.ptr.end(), ptr);
      if (idx) std::copy(m.idx.begin(), m.idx.end(), idx);
      if (val) {
        using T = typename std::decay_t<decltype(m.val)>::value_type;
        if constexpr (host::is_complex<T>::value) {
          for (size_t k = 0; k < m.val.size(); ++k) {
            val[2 * k] = m.val[k].real();
            val[2 * k + 1] = m.val[k].imag();
          }
        } else {
          std::copy(m.val.begin(), m.val.end(), val);
        }
      }
    };
    if (f->kind == YB_CHOLESKY) {
      put(f->chol.l, lower_ptr, lower_idx, lower_val);
      put(f->chol.lh, upper_ptr, upper_idx, upper_val);
      if (row_perm) std::copy(f->chol.perm.begin(), f->chol.perm.end(), row_perm);
      if (col_perm) std::copy(f->chol.perm.begin(), f->chol.perm.end(), col_perm);
    } else if (f->is_complex) {
      put(f->lu_c.l, lower_ptr, lower_idx, lower_val);
      put(f->lu_c.u, upper_ptr, upper_idx, upper_val);
      if (row_perm) std::copy(f->lu_c.row_perm.begin(), f->lu_c.row_perm.end(), row_perm);
      if (col_perm) std::copy(f->lu_c.col_perm.begin(), f->lu_c.col_perm.end(), col_perm);
    } else {
      put(f->lu.l, lower_ptr, lower_idx, lower_val);
      put(f->lu.u, upper_ptr, upper_idx, upper_val);
      if (row_perm) std::copy(f->lu.row_perm.begin(), f->lu.row_perm.end(), row_perm);
      if (col_perm) std::copy(f->lu.col_perm.begin(), f->lu.col_perm.end(), col_perm);
    }
    return YB_OK;
  });
}

int32_t yb_host_etree(const yb_host_factor *f, int64_t *parent) {
  return guard([&] {
    require(f && parent, "null argument");
    require(f->kind == YB_CHOLESKY, "only a Cholesky factor has an elimination tree here");
    std::copy(f->chol.parent.begin(), f->chol.parent.end(), parent);
    return YB_OK;
  });
}

void yb_host_factor_free(yb_host_factor *f) { delete f; }

}  // extern "C"
