/* ybhost: the host side of ybgpu, with no GPU code in it.
 *
 * C ABI of libybhost.so: the status codes and the thread-local last-error message that every
 * ybgpu entry point shares, and the host factor producer, i.e. the ybus_sparse calls whose
 * results ybus_cuda uploads (ybus_cuda/src/factor.rs:103-133 takes a `Cholesky<f64>` or `Lu<f64>`
 * made by ybus_sparse). libybgpu.so depends on this library; a program that only assembles and
 * factors matrices on the host loads it alone. Conventions as ybgpu.h: an int32 status per call
 * (0 = success), opaque handles made by the producer and released by `_free`.
 */
#ifndef YBHOST_H
#define YBHOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (ybus_cuda's `CudaError` variants, ybus_cuda/src/lib.rs:89-124) ---------- */
#define YB_OK 0
#define YB_ERROR_INVALID_ARGUMENT 1 /* a contract violation (ybus_cuda panics) */
#define YB_ERROR_SHAPE_MISMATCH 2   /* CudaError::ShapeMismatch */
#define YB_ERROR_TOO_LARGE 3        /* CudaError::TooLarge */
#define YB_ERROR_NOT_POSITIVE_DEFINITE 4
#define YB_ERROR_SINGULAR 5
#define YB_NO_DEVICE 6              /* Gpu::new() -> Ok(None) */
#define YB_ERROR_CUDA 7             /* CudaError::Driver */
#define YB_ERROR_NOT_SYMMETRIC 8
#define YB_ERROR_DEVICE_TIMEOUT 9   /* a bounded device wait gave up */
#define YB_ERROR_INTERNAL 10

#define YB_CHOLESKY 1
#define YB_LU 2

#define YB_ORDER_NATURAL 0
#define YB_ORDER_AMD 1
#define YB_ORDER_COLAMD 3

/* The message of the calling thread's last failure, NUL-terminated and truncated to `length`;
 * returns the length needed including the NUL. */
int32_t yb_last_error_message(char *buffer, size_t length);

/* ---- host factor producer (the ybus_sparse calls whose results ybus_cuda uploads) --------- */
typedef struct yb_matrix yb_matrix;
typedef struct yb_host_factor yb_host_factor;

/* A compressed matrix from triplets, duplicates summed in input order
 * (ybus_sparse/src/compressed_matrix.rs:254-330). `by_rows` = 1 for CSR, 0 for CSC. Complex
 * values are interleaved (re, im), 2*count doubles. */
int32_t yb_matrix_from_triplets(int64_t rows, int64_t cols, int64_t count, const int64_t *row_idx,
                                const int64_t *col_idx, const double *values, int32_t by_rows,
                                int32_t is_complex, yb_matrix **out);
/* Rows and columns in the given orders (ybus_sparse/src/compressed_matrix/access.rs:175-216). */
int32_t yb_matrix_select(const yb_matrix *m, int64_t n_rows, const int64_t *rows, int64_t n_cols,
                         const int64_t *cols, yb_matrix **out);
/* The other orientation of the same matrix (to_csc / to_csr). */
int32_t yb_matrix_reorient(const yb_matrix *m, yb_matrix **out);
int32_t yb_matrix_info(const yb_matrix *m, int64_t *rows, int64_t *cols, int64_t *stored,
                       int32_t *by_rows, int32_t *is_complex);
int32_t yb_matrix_export(const yb_matrix *m, int64_t *ptr, int64_t *idx, double *values);
void yb_matrix_free(yb_matrix *m);
/* A fill-reducing ordering (ybus_sparse/src/compressed_matrix/ordering.rs:46-64). */
int32_t yb_ordering(const yb_matrix *m, int32_t ordering, int64_t *perm);

/* `CsrMatrix::analyze_cholesky(ordering)` then `factor` (cholesky.rs:50-311): P A Pᵀ = L Lᵀ. */
int32_t yb_host_cholesky(const yb_matrix *csr, int32_t ordering, yb_host_factor **out);
/* `CscMatrix::analyze_lu(ordering)` then `factor` with the pivot threshold (lu.rs:142-247). */
int32_t yb_host_lu(const yb_matrix *csc, int32_t ordering, double pivot_threshold, yb_host_factor **out);
int32_t yb_host_factor_info(const yb_host_factor *f, int32_t *kind, int32_t *is_complex, int64_t *n,
                            int64_t *lower_stored, int64_t *upper_stored);
/* Cholesky: lower = L (CSR, diagonal last), upper = Lᵀ (CSR, diagonal first), both perms = P.
 * LU: lower = L (CSC, unit diagonal first), upper = U (CSC, diagonal last), row_perm = P,
 * col_perm = Q. Any output may be NULL. */
int32_t yb_host_factor_export(const yb_host_factor *f, int64_t *lower_ptr, int64_t *lower_idx,
                              double *lower_val, int64_t *upper_ptr, int64_t *upper_idx,
                              double *upper_val, int64_t *row_perm, int64_t *col_perm);
int32_t yb_host_etree(const yb_host_factor *f, int64_t *parent);
void yb_host_factor_free(yb_host_factor *f);

#ifdef __cplusplus
}
#endif

#endif /* YBHOST_H */
