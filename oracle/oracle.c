/* ORACLE — test infrastructure only.
 *
 * A plain-C restatement of ybus's CPU solve side, the reference the GPU path is checked
 * against. Only the tests, the smoke check and the bench's CPU-baseline leg use it; nothing in
 * the product links or calls it. Built with -ffp-contract=off so every multiply and add rounds
 * separately, as the reference's Rust code does (no fused multiply-add).
 *
 * Parity is pinned against the reference's own known-answer tests and fixtures (single-row
 * solves, the w = 0 singular column, the argmax tie rule, the LCG fixtures and the ring
 * networks) by the tests under tests/; the reference itself (Rust) cannot be built here.
 *
 * Each function names the reference code it restates.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---- real Cholesky --------------------------------------------------------------------- */

/* forward_by_rows (ybus_sparse/src/compressed_matrix/cholesky.rs:468-483): rows in order, the
 * off-diagonal terms subtracted left to right, then one division by the diagonal (stored last). */
static void forward_by_rows(int64_t n, const int64_t *ptr, const int64_t *idx, const double *val, double *y) {
  for (int64_t i = 0; i < n; ++i) {
    double remainder = y[i];
    double diagonal = 1.0;
    for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
      const int64_t col = idx[p];
      if (col < i) {
        remainder = remainder - val[p] * y[col];
      } else {
        diagonal = val[p];
        break;
      }
    }
    y[i] = remainder / diagonal;
  }
}

/* back_by_rows (cholesky.rs:487-501): rows from the last, the diagonal (stored first) found and
 * the entries right of it subtracted in stored order. */
static void back_by_rows(int64_t n, const int64_t *ptr, const int64_t *idx, const double *val, double *y) {
  for (int64_t i = n - 1; i >= 0; --i) {
    double remainder = y[i];
    double diagonal = 1.0;
    for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
      const int64_t col = idx[p];
      if (col == i)
        diagonal = val[p];
      else if (col > i)
        remainder = remainder - val[p] * y[col];
    }
    y[i] = remainder / diagonal;
  }
}

/* Cholesky::substitute (cholesky.rs:570-579): gather by P, forward with L, back with Lᵀ,
 * scatter by P. `scratch` holds n doubles. */
void or_cholesky_substitute(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                            const int64_t *lt_ptr, const int64_t *lt_idx, const double *lt_val, const int64_t *perm,
                            double *x, double *scratch) {
  for (int64_t i = 0; i < n; ++i) scratch[i] = x[perm[i]];
  forward_by_rows(n, l_ptr, l_idx, l_val, scratch);
  back_by_rows(n, lt_ptr, lt_idx, lt_val, scratch);
  for (int64_t i = 0; i < n; ++i) x[perm[i]] = scratch[i];
}

/* ---- real LU ------------------------------------------------------------------------------ */

/* Lu::back_substitute (lu.rs:640-649): U in CSC with the diagonal last, by columns from the last. */
static void lu_back_substitute(int64_t n, const int64_t *u_ptr, const int64_t *u_idx, const double *u_val, double *y) {
  for (int64_t j = n - 1; j >= 0; --j) {
    const int64_t diagonal = u_ptr[j + 1] - 1;
    y[j] = y[j] / u_val[diagonal];
    const double y_j = y[j];
    for (int64_t p = u_ptr[j]; p < diagonal; ++p) y[u_idx[p]] = y[u_idx[p]] - u_val[p] * y_j;
  }
}

/* Lu::substitute (lu.rs:770-785): gather by P, L (unit, CSC, diagonal first) by columns, U by
 * columns from the last, scatter by Q. */
void or_lu_substitute(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val, const int64_t *u_ptr,
                      const int64_t *u_idx, const double *u_val, const int64_t *row_perm, const int64_t *col_perm,
                      double *x, double *scratch) {
  for (int64_t i = 0; i < n; ++i) scratch[i] = x[row_perm[i]];
  for (int64_t j = 0; j < n; ++j) {
    const double y_j = scratch[j];
    for (int64_t p = l_ptr[j] + 1; p < l_ptr[j + 1]; ++p) scratch[l_idx[p]] = scratch[l_idx[p]] - l_val[p] * y_j;
  }
  lu_back_substitute(n, u_ptr, u_idx, u_val, scratch);
  for (int64_t i = 0; i < n; ++i) x[col_perm[i]] = scratch[i];
}

/* Lu::solve_transpose (lu.rs:506-533): Uᵀ y = Qᵀ b (column j of U is row j of Uᵀ, diagonal
 * last), then Lᵀ z = y (unit diagonal first), then x = Pᵀ z. */
void or_lu_solve_transpose(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                           const int64_t *u_ptr, const int64_t *u_idx, const double *u_val, const int64_t *row_perm,
                           const int64_t *col_perm, double *x, double *scratch) {
  for (int64_t i = 0; i < n; ++i) scratch[i] = x[col_perm[i]];
  for (int64_t j = 0; j < n; ++j) {
    const int64_t diagonal = u_ptr[j + 1] - 1;
    double remainder = scratch[j];
    for (int64_t p = u_ptr[j]; p < diagonal; ++p) remainder = remainder - u_val[p] * scratch[u_idx[p]];
    scratch[j] = remainder / u_val[diagonal];
  }
  for (int64_t j = n - 1; j >= 0; --j) {
    double remainder = scratch[j];
    for (int64_t p = l_ptr[j] + 1; p < l_ptr[j + 1]; ++p) remainder = remainder - l_val[p] * scratch[l_idx[p]];
    scratch[j] = remainder;
  }
  for (int64_t i = 0; i < n; ++i) x[row_perm[i]] = scratch[i];
}

/* ---- complex LU (num-complex arithmetic: textbook multiply and divide) -------------------- */

typedef struct {
  double re, im;
} c128;

static inline c128 cmul(c128 a, c128 b) {
  c128 r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}
static inline c128 csub(c128 a, c128 b) {
  c128 r = {a.re - b.re, a.im - b.im};
  return r;
}
/* num-complex's Div: (a conj(b)) / |b|² componentwise. */
static inline c128 cdiv(c128 a, c128 b) {
  const double norm = b.re * b.re + b.im * b.im;
  const double re = a.re * b.re + a.im * b.im;
  const double im = a.im * b.re - a.re * b.im;
  c128 r = {re / norm, im / norm};
  return r;
}

/* Lu::substitute for Complex<f64> (lu.rs:770-785), values interleaved (re, im). */
void or_lu_substitute_c128(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                           const int64_t *u_ptr, const int64_t *u_idx, const double *u_val, const int64_t *row_perm,
                           const int64_t *col_perm, double *x, double *scratch) {
  c128 *X = (c128 *)x, *Y = (c128 *)scratch;
  const c128 *L = (const c128 *)l_val, *U = (const c128 *)u_val;
  for (int64_t i = 0; i < n; ++i) Y[i] = X[row_perm[i]];
  for (int64_t j = 0; j < n; ++j) {
    const c128 y_j = Y[j];
    for (int64_t p = l_ptr[j] + 1; p < l_ptr[j + 1]; ++p) Y[l_idx[p]] = csub(Y[l_idx[p]], cmul(L[p], y_j));
  }
  for (int64_t j = n - 1; j >= 0; --j) {
    const int64_t diagonal = u_ptr[j + 1] - 1;
    Y[j] = cdiv(Y[j], U[diagonal]);
    const c128 y_j = Y[j];
    for (int64_t p = u_ptr[j]; p < diagonal; ++p) Y[u_idx[p]] = csub(Y[u_idx[p]], cmul(U[p], y_j));
  }
  for (int64_t i = 0; i < n; ++i) X[col_perm[i]] = Y[i];
}

/* ---- many right-hand sides on many threads ------------------------------------------------ */

/* Factorization::par_solve_many (ybus_sparse/src/compressed_matrix/factorization.rs:71-92):
 * each right-hand side is substituted independently with private scratch, so the result is bit
 * for bit the serial one whatever the thread count. `kind`: 1 Cholesky (lower = L CSR, upper =
 * Lᵀ CSR, perms P), 2 LU (lower = L CSC, upper = U CSC, P, Q), 3 LU transpose, 4 complex LU. */
typedef struct {
  int kind;
  int64_t n, count;
  const int64_t *a_ptr, *a_idx, *b_ptr, *b_idx, *p, *q;
  const double *a_val, *b_val;
  const double *rhs;
  double *out;
  int64_t next;
  pthread_mutex_t lock;
} SolveJob;

static void *solve_worker(void *arg) {
  SolveJob *job = (SolveJob *)arg;
  const int64_t width = job->kind == 4 ? 2 : 1;
  double *scratch = (double *)malloc(sizeof(double) * (size_t)(job->n * width + 1));
  for (;;) {
    pthread_mutex_lock(&job->lock);
    const int64_t k0 = job->next;
    job->next += 8;
    pthread_mutex_unlock(&job->lock);
    if (k0 >= job->count) break;
    const int64_t k1 = k0 + 8 < job->count ? k0 + 8 : job->count;
    for (int64_t k = k0; k < k1; ++k) {
      double *x = job->out + k * job->n * width;
      memcpy(x, job->rhs + k * job->n * width, sizeof(double) * (size_t)(job->n * width));
      switch (job->kind) {
        case 1:
          or_cholesky_substitute(job->n, job->a_ptr, job->a_idx, job->a_val, job->b_ptr, job->b_idx, job->b_val,
                                 job->p, x, scratch);
          break;
        case 2:
          or_lu_substitute(job->n, job->a_ptr, job->a_idx, job->a_val, job->b_ptr, job->b_idx, job->b_val, job->p,
                           job->q, x, scratch);
          break;
        case 3:
          or_lu_solve_transpose(job->n, job->a_ptr, job->a_idx, job->a_val, job->b_ptr, job->b_idx, job->b_val,
                                job->p, job->q, x, scratch);
          break;
        case 4:
          or_lu_substitute_c128(job->n, job->a_ptr, job->a_idx, job->a_val, job->b_ptr, job->b_idx, job->b_val,
                                job->p, job->q, x, scratch);
          break;
        default:
          break;
      }
    }
  }
  free(scratch);
  return NULL;
}

int or_solve_many(int kind, int64_t n, const int64_t *a_ptr, const int64_t *a_idx, const double *a_val,
                  const int64_t *b_ptr, const int64_t *b_idx, const double *b_val, const int64_t *p, const int64_t *q,
                  const double *rhs, int64_t count, double *out, int threads) {
  if (kind < 1 || kind > 4 || n < 0 || count < 0) return 1;
  if (n == 0 || count == 0) return 0;
  SolveJob job;
  memset(&job, 0, sizeof job);
  job.kind = kind, job.n = n, job.count = count;
  job.a_ptr = a_ptr, job.a_idx = a_idx, job.a_val = a_val;
  job.b_ptr = b_ptr, job.b_idx = b_idx, job.b_val = b_val;
  job.p = p, job.q = q, job.rhs = rhs, job.out = out, job.next = 0;
  pthread_mutex_init(&job.lock, NULL);
  if (threads < 1) threads = 1;
  if (threads == 1) {
    solve_worker(&job);
  } else {
    pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, solve_worker, &job);
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
    free(tid);
  }
  pthread_mutex_destroy(&job.lock);
  return 0;
}

/* ---- the device kernels' formulas, on the host --------------------------------------------- */

/* The rank-one update of one column (ybus_cuda/src/kernels.cu:24-58, and the host formula of
 * ybus_cuda/tests/gpu_pairs_test.rs:48-62): x = base + alpha y, w = inverse_weight − cᵀy,
 * z = cᵀx / w, out = x + z y; w = 0 is singular and gives x. Rows are natural; -1 is none. */
int or_pair_update(int64_t n, const double *base, const double *y, int64_t plus, int64_t minus, double alpha,
                   double inverse_weight, double *out) {
  double cy = 0.0, cx = 0.0;
  if (plus >= 0) {
    cy += y[plus];
    cx += base[plus] + alpha * y[plus];
  }
  if (minus >= 0) {
    cy -= y[minus];
    cx -= base[minus] + alpha * y[minus];
  }
  const double w = -cy + inverse_weight;
  for (int64_t i = 0; i < n; ++i) out[i] = base[i] + alpha * y[i];
  if (w == 0.0) return 1;
  const double z = cx / w;
  for (int64_t i = 0; i < n; ++i) out[i] = out[i] + z * y[i];
  return 0;
}

/* column_max (ybus_cuda/src/kernels.cu:78-128): the largest |v|·w, the smallest row on a tie,
 * -1 (and 0.0) if every product is zero; non-finite values take no part but set the flag. */
void or_column_max(int64_t n, const double *v, const double *weight, int64_t *row, double *value, int *not_finite) {
  double best = 0.0;
  int64_t best_row = -1;
  int bad = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (!isfinite(v[i])) {
      bad = 1;
      continue;
    }
    const double product = fabs(v[i]) * (weight ? weight[i] : 1.0);
    if (product > best) {
      best = product;
      best_row = i;
    }
  }
  *row = best_row;
  *value = best;
  *not_finite = bad;
}

/* CsrMatrix::mul_vec (ybus_sparse/src/compressed_matrix/product.rs:17-27): each entry a dot
 * product with its row, summed from zero in stored order. */
void or_csr_mul_vec(int64_t rows, const int64_t *ptr, const int64_t *idx, const double *val, const double *x,
                    double *out) {
  for (int64_t i = 0; i < rows; ++i) {
    double sum = 0.0;
    for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) sum = sum + val[p] * x[idx[p]];
    out[i] = sum;
  }
}

/* relative_residual (ybus_sparse/src/compressed_matrix/accuracy.rs:58-79): ‖b − A x‖∞ / ‖b‖∞,
 * 0 for a zero residual, infinity for a zero b with a nonzero residual. */
double or_relative_residual(int64_t n, const int64_t *ptr, const int64_t *idx, const double *val, const double *x,
                            const double *b) {
  double r_norm = 0.0, b_norm = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double ax = 0.0;
    for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) ax = ax + val[p] * x[idx[p]];
    const double r = fabs(b[i] - ax);
    if (r > r_norm) r_norm = r;
    if (fabs(b[i]) > b_norm) b_norm = fabs(b[i]);
  }
  if (b_norm > 0.0) return r_norm / b_norm;
  return r_norm > 0.0 ? INFINITY : 0.0;
}
