/* ybgpu: B200-native factor-once / solve-many sparse triangular solves.
 *
 * C ABI of libybgpu.so. It mirrors the public API of ybus's `ybus_cuda` crate
 * (ybus_cuda/src/lib.rs:73-75 re-exports `Gpu`, `GpuFactor`, `Timings`, `Pair`, `PairUpdate`,
 * `ColumnMax`, `GpuBlock`, `GpuOperator`) one entry point per method, in the conventions of
 * ybus's own C ABI (`ybus_ffi`): an int32 status per call (0 = success), a thread-local message
 * for the last failure, and opaque handles made by `_new` and released by `_free`
 * (ybus_ffi/src/lib.rs:44-73, ybus_ffi/src/status.rs:10-60).
 *
 * Contract violations that ybus_cuda answers with a panic (`assert!`) are reported here as
 * YB_ERROR_INVALID_ARGUMENT instead; nothing in this library aborts the caller.
 *
 * Arrays of right-hand sides and solutions are column-major: column k of an n-row array starts
 * at element k*n. Indices are int64 at the boundary and must fit 32 bits on the device
 * (YB_ERROR_TOO_LARGE otherwise, as ybus_cuda's `CudaError::TooLarge`, ybus_cuda/src/lib.rs:98).
 * A row index of -1 means "none" wherever ybus_cuda takes an `Option<usize>`.
 *
 * The status codes, the last-error message and the host factor producer are declared in
 * ybhost.h and live in libybhost.so, which libybgpu.so loads (a caller that only factors on the
 * host needs that library alone).
 */
#ifndef YBGPU_H
#define YBGPU_H

#include <stddef.h>
#include <stdint.h>

#include "ybhost.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- the GPU (ybus_cuda `Gpu`, ybus_cuda/src/lib.rs:168-219) ----------------------------- */
typedef struct yb_gpu yb_gpu;
typedef struct yb_factor yb_factor;

#define YB_FP64 0 /* substitutions in double */
#define YB_FP32 1 /* substitutions in float (no refinement) */

/* `Gpu::new()`: device `device`, or YB_NO_DEVICE where there is none (ybus returns Ok(None)). */
int32_t yb_gpu_new(int32_t device, yb_gpu **out);
void yb_gpu_free(yb_gpu *gpu);
/* `Gpu::name()` (lib.rs:210-212). */
int32_t yb_gpu_name(const yb_gpu *gpu, char *buffer, size_t length);
/* `Gpu::memory()`: free and total device memory in bytes (lib.rs:214-218). */
int32_t yb_gpu_memory(const yb_gpu *gpu, uint64_t *free_bytes, uint64_t *total_bytes);
/* No ybus counterpart: SM count, compute capability and L2 size, for sizing launches. */
int32_t yb_gpu_properties(const yb_gpu *gpu, int32_t *sm_count, int32_t *major, int32_t *minor, int64_t *l2_bytes);
/* The stream the host-array calls of this GPU run on (a cudaStream_t). */
void *yb_gpu_stream(const yb_gpu *gpu);
/* Waits for `stream` (NULL for the GPU's own) to finish; reports any asynchronous CUDA error. */
int32_t yb_gpu_synchronize(const yb_gpu *gpu, void *stream);

/* ---- an uploaded factorization (ybus_cuda `GpuFactor`, ybus_cuda/src/factor.rs) ------------ */
/* `GpuFactor::from_cholesky` (factor.rs:103-119): P A Pᵀ = L Lᵀ with L in CSR, each row's
 * diagonal last, and perm = P (row i of P A Pᵀ is row perm[i] of A). */
int32_t yb_factor_from_cholesky(yb_gpu *gpu, int64_t n, const int64_t *l_ptr, const int64_t *l_idx,
                                const double *l_val, const int64_t *perm, yb_factor **out);
/* `GpuFactor::from_lu` (factor.rs:123-133): P A Q = L U with L unit lower in CSC (diagonal
 * first), U upper in CSC (diagonal last), row_perm = P, col_perm = Q. */
int32_t yb_factor_from_lu(yb_gpu *gpu, int64_t n, const int64_t *l_ptr, const int64_t *l_idx,
                          const double *l_val, const int64_t *u_ptr, const int64_t *u_idx,
                          const double *u_val, const int64_t *row_perm, const int64_t *col_perm,
                          yb_factor **out);
/* `Lu::solve_transpose` (lu.rs:506-533) as a factor: the same arguments as yb_factor_from_lu, uploading
 * the factor of A' = Q U' L' P, so every solve of the result solves A' x = b (U' forward, then L'
 * backward). A Cholesky factor needs none: A' = A. */
int32_t yb_factor_from_lu_transposed(yb_gpu *gpu, int64_t n, const int64_t *l_ptr, const int64_t *l_idx,
                                     const double *l_val, const int64_t *u_ptr, const int64_t *u_idx,
                                     const double *u_val, const int64_t *row_perm, const int64_t *col_perm,
                                     yb_factor **out);
void yb_factor_free(yb_factor *f);
/* `GpuFactor::dim` and `block_width` (factor.rs:181-190); -1 for a null factor. */
int64_t yb_factor_dim(const yb_factor *f);
int64_t yb_factor_block_width(const yb_factor *f);
/* `GpuFactor::set_block_width` (factor.rs:192-201): at least 1, at most 64 for one row. */
int32_t yb_factor_set_block_width(yb_factor *f, int64_t width);
/* `GpuFactor::timings` / `reset_timings` (factor.rs:203-210), in seconds. */
int32_t yb_factor_timings(const yb_factor *f, double *upload_s, double *solve_s, double *download_s,
                          int64_t *blocks);
int32_t yb_factor_reset_timings(yb_factor *f);
/* No ybus counterpart (cuSPARSE's analysis is opaque there): the level schedule's shape. */
int32_t yb_factor_plan_info(const yb_factor *f, int32_t *fwd_levels, int32_t *bwd_levels,
                            int64_t *fwd_entries, int64_t *bwd_entries, int32_t *fwd_widest,
                            int32_t *bwd_widest);
/* No ybus counterpart: the tile solve's launch shape for a precision (tile width 1..32, a power
 * of two; threads a multiple of 32 up to 512; resident blocks per SM 1..8). */
int32_t yb_factor_set_tile(yb_factor *f, int32_t precision, int32_t tile_width, int32_t threads,
                           int32_t blocks_per_sm);
/* No ybus counterpart: which tile solve runs for a precision: 0 automatic (the lane solve for
 * solves of at least the lane threshold's right-hand sides when the factor admits it; else the
 * domain solve at the widest tile that fits in shared memory; else the streamed solve likewise;
 * else the global-scratch solve), 1 the level-sliced shared-memory solve, 2 the global-scratch
 * solve, 3 the streamed solve, 4 the domain solve, 5 the lane solve (1, 3, 4 and 5 give
 * YB_ERROR_INVALID_ARGUMENT at launch if the tile does not fit in shared memory or the factor
 * admits no domain or lane layout). The lane solve serves yb_solve_many_device and yb_solve_many;
 * the pair, refined and batched solves take the automatic choice among the others. */
int32_t yb_factor_set_tile_kind(yb_factor *f, int32_t precision, int32_t kind);
/* No ybus counterpart: the lane solve (one right-hand side per lane, a block of warps per 32; the
 * factor's rows in an elimination-tree postorder cut into subtree domains the warps take in
 * parallel under a top warp 0 takes, a few tens of live values per lane in shared memory; b, the
 * forward results and x streaming through a work array in HBM). info receives 12 values: {slots,
 * pages, page bytes, forward peak of live values, backward peak, entries of both sweeps, shared
 * memory per block, warps per block, domains, top rows, partial values per block, right-hand sides per lane};
 * YB_ERROR_INVALID_ARGUMENT if the factor admits no lane layout (too many live values). */
int32_t yb_factor_lane_info(yb_factor *f, int32_t precision, int64_t *info);
/* No ybus counterpart: the lane solve's shape for a precision: warps per block (1..16, default 8;
 * blocks of more than 8 warps run one to an SM, for blocks of fewer groups of 32 than SMs) and page
 * bytes (256..16384, a multiple of 16; default 0: the largest of 2048, 1024, 768, 512 with which
 * three blocks fit an SM). */
int32_t yb_factor_set_lane(yb_factor *f, int32_t precision, int32_t warps, int32_t page_bytes);
/* No ybus counterpart: how many right-hand sides each lane of the plain lane solve carries, 1 or 2
 * (a block then solves 32 or 64 right-hand sides; with two, each decoded record serves twice the
 * arithmetic, and two blocks share an SM instead of three). The refined solve's lane passes keep
 * one. yb_factor_lane_info reports it (its last value). */
int32_t yb_factor_set_lane_rhs_per_lane(yb_factor *f, int32_t precision, int32_t rhs_per_lane);
/* No ybus counterpart: the number of right-hand sides from which the automatic choice takes the
 * lane solve; -1 (the default): 1,536 when the domain solve's automatic tiles hold two or more
 * columns, else 64 (the measured crossovers). */
int32_t yb_factor_set_lane_min_count(yb_factor *f, int32_t precision, int64_t min_count);
/* No ybus counterpart: the number of right-hand sides from which yb_solve_many_refined_device takes
 * the FP32 lane solve (default 2048, the measured crossover with the refinement fused into the
 * domain solve on the 10,000-bus B'; the FP32 lane threshold of yb_factor_set_lane_min_count applies
 * too, whichever is higher). */
int32_t yb_factor_set_refine_lane_min_count(yb_factor *f, int64_t min_count);
/* No ybus counterpart: the thresholds the automatic choice applies for a precision: the plain
 * solve's lane threshold (the automatic one resolved for this factor) and the refined solve's
 * (either output may be NULL). */
int32_t yb_factor_lane_min_counts(const yb_factor *f, int32_t precision, int64_t *lane_min_count,
                                  int64_t *refine_lane_min_count);
/* No ybus counterpart: with on = 1, every lane-solve launch from now on records CUDA events around
 * its three kernels (gather, solve, scatter) on the caller's stream, for up to 4096 launches;
 * on = 0 stops. Either way the record so far is cleared. */
int32_t yb_factor_time_lane(yb_factor *f, int32_t on);
/* No ybus counterpart: waits for the recorded lane-solve launches and returns the total device
 * milliseconds of their gathers, solves and scatters, and how many launches they were; then clears
 * the record (timing stays on if it was). */
int32_t yb_factor_lane_times(yb_factor *f, double *gather_ms, double *solve_ms, double *scatter_ms,
                             int64_t *launches);
/* No ybus counterpart: the streamed solve's shape for a precision: warps per block (1..16), pages
 * in flight per warp (2..16), page bytes (512..16384, a multiple of 16), and the row count under
 * which a level is taken by one warp alone (0: twice a slice's rows). */
int32_t yb_factor_set_stream(yb_factor *f, int32_t precision, int32_t warps, int32_t ring,
                             int32_t page_bytes, int32_t narrow_rows);
/* No ybus counterpart: the forward level from which the streamed solve takes the top of the tree
 * as one dense block through its explicit inverse (-1: chosen from the factor, 0: none). */
int32_t yb_factor_set_tail_level(yb_factor *f, int32_t precision, int32_t tail_level);
/* No ybus counterpart: the streamed layout the automatic choice runs for a precision (building it
 * if needed); YB_ERROR_INVALID_ARGUMENT if that choice is not the streamed solve. */
int32_t yb_factor_stream_info(yb_factor *f, int32_t precision, int32_t *tile_width, int32_t *stages,
                              int64_t *records, int64_t *bytes, int32_t *fwd_wide, int32_t *bwd_wide,
                              int32_t *narrow_rows);
/* No ybus counterpart: the domain solve's shape for a precision: warps per block (1..16), pages in
 * flight per warp (2..8), page bytes (512..16384, a multiple of 16), and the cut, the first forward
 * level of the dense top block (-1: chosen by the layout's cost model). */
int32_t yb_factor_set_domain(yb_factor *f, int32_t precision, int32_t warps, int32_t ring, int32_t page_bytes,
                             int32_t cut);
/* No ybus counterpart: the domain layout the automatic choice runs for a precision (building it if
 * needed): tile width, cut, rows of the top block, records, bytes, shared memory per block and the
 * cost model's cycles per tile; YB_ERROR_INVALID_ARGUMENT if that choice is not the domain solve. */
int32_t yb_factor_domain_info(yb_factor *f, int32_t precision, int32_t *tile_width, int32_t *cut, int32_t *top_rows,
                              int64_t *records, int64_t *bytes, int64_t *smem_bytes, double *model_cycles);
/* No ybus counterpart: the autotuner. Times the solve of `count` right-hand sides for a precision
 * over the domain solve's shapes (warps 8/12/16, pages 1536/2048 bytes, 2 or 3 pages in flight, the
 * widest tile that fits and half of it), the global-scratch solve's (tile widths 1 to 32, 256 or
 * 512 threads) and the lane solve's (4, 6 or 8 warps per block with one or two right-hand sides
 * per lane, 12 or 16 with one, when the factor admits a lane layout) and keeps the fastest for the factor, for solves of
 * about that many right-hand sides. config receives {kind, tile width (0 for the lane solve),
 * warps, ring, page bytes} (for the global-scratch solve: {kind, tile width, warps, blocks per SM,
 * 0}) and best_ms its time (either may be NULL). With nothing to time, the configuration is left
 * as it was. */
int32_t yb_factor_autotune(yb_factor *f, int32_t precision, int64_t count, int32_t *config, double *best_ms);
/* No ybus counterpart, diagnostics on the host (no GPU needed): the lane solve's layout for a
 * Cholesky factor given as to yb_factor_from_cholesky, values of `value_bytes` (8 or 4), `warps`
 * warps per block, `rhs_per_lane` (1 or 2) right-hand sides per lane. info receives 12 values:
 * {slots, pages, page bytes, forward peak of live values, backward peak, forward entries, backward
 * entries, warps, domains, top rows, partial values per block, right-hand sides per lane}; blob
 * (pages * page_bytes bytes), warp_page (warps + 1), in_pos and out_pos (n each: the work-array
 * position of each row of b and of x) may be NULL. */
int32_t yb_lane_layout_cholesky(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                                const int64_t *perm, int32_t value_bytes, int32_t page_bytes, int32_t max_slots,
                                int32_t warps, int32_t rhs_per_lane, int64_t *info, uint8_t *blob, int32_t *warp_page,
                                int32_t *in_pos, int32_t *out_pos);
/* No ybus counterpart, diagnostics on the host (no GPU needed): the lane solve's layout for an LU
 * factor given as to yb_factor_from_lu (L and U in CSC, row and column permutations), the other
 * arguments and outputs as yb_lane_layout_cholesky's. */
int32_t yb_lane_layout_lu(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                          const int64_t *u_ptr, const int64_t *u_idx, const double *u_val, const int64_t *row_perm,
                          const int64_t *col_perm, int32_t value_bytes, int32_t page_bytes, int32_t max_slots,
                          int32_t warps, int32_t rhs_per_lane, int64_t *info, uint8_t *blob, int32_t *warp_page,
                          int32_t *in_pos, int32_t *out_pos);
/* No ybus counterpart, diagnostics on the host (no GPU needed): the domain layout a Cholesky factor
 * given as to yb_factor_from_cholesky gets for `value_bytes` (8 or 4). info receives {cut, top
 * rows, stages, warps, pages, records, entries, page bytes}, top_condition the worse infinity-norm
 * condition of the top block's two triangles; blob (pages * page_bytes bytes), warp_page (warps + 1),
 * top_slot (top rows) and top_condition may be NULL, so a first call can size them. A cut whose top
 * triangles have a condition above 1e4 is not used (their explicit inverses would lose accuracy). */
int32_t yb_domain_layout_cholesky(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                                  const int64_t *perm, int32_t value_bytes, int32_t warps, int32_t page_bytes,
                                  int32_t cut, int64_t *info, uint8_t *blob, int32_t *warp_page, int32_t *top_slot,
                                  double *top_condition);
/* Waits for the device and reports YB_ERROR_DEVICE_TIMEOUT (clearing it) if a bounded wait in a
 * kernel of this factor ran out since the last check; the host-array calls check by themselves. */
int32_t yb_factor_check_error(yb_factor *f);
/* No ybus counterpart, for tests of the device error path without a fault: the next plain lane
 * solve of this factor (its first launch only) does not issue the copy of page `page` of block 0's
 * first warp, so that warp's bounded wait (one second) runs out; the warp stops, waits (bounded)
 * for its copies in flight and takes its block's remaining barriers, and the solve reports
 * YB_ERROR_DEVICE_TIMEOUT (yb_factor_check_error, or the host-array call itself). -1 withholds
 * nothing; the setting applies once. */
int32_t yb_factor_withhold_lane_page(yb_factor *f, int32_t page);
/* No ybus counterpart, diagnostics: a device buffer of 512 int64 (or NULL to stop) into which block
 * 0 of the streamed or domain solve writes clock64() marks for its first 4 tiles, as
 * [tile][warp < 16][8]. Streamed solve: 0 tile loaded, 1 own records done, 2 all stages done,
 * 3 tile stored, 4 cycles waiting for pages, 5 cycles in block barriers, 6 pages taken. Domain
 * solve: 0 tile start, 1 tile loaded, 2 own records done, 3 tile stored, 4 cycles waiting for
 * pages, 5 cycles in block barriers, 6 pages taken, 7 records taken; a refined solve writes the
 * first 4 passes of block 0's first tile in place of 4 tiles. */
int32_t yb_factor_set_phase_clock(yb_factor *f, void *d_clock);
int32_t yb_factor_get_tile(const yb_factor *f, int32_t precision, int32_t *tile_width, int32_t *threads,
                           int32_t *blocks_per_sm);

/* `GpuFactor::solve_many` (factor.rs:234-289) with host arrays: `count` right-hand sides,
 * column-major n x count in the caller's order, solutions likewise, in FP64. Pinned (page-locked)
 * caller memory is copied directly; pageable memory goes through a pinned staging buffer. */
int32_t yb_solve_many(yb_factor *f, const double *rhs, int64_t count, double *out);
/* `Lu::solve_transpose` (lu.rs:506-533) for many right-hand sides, host arrays as yb_solve_many:
 * solves A' x = b with the factor of A. An LU factor makes the factor of A' = Q U' L' P from its
 * arrays at the first call and keeps it (yb_factor_from_lu_transposed's); a Cholesky factor solves
 * as yb_solve_many (A' = A). */
int32_t yb_solve_many_transpose(yb_factor *f, const double *rhs, int64_t count, double *out);
/* No ybus counterpart (ybus_sparse's `Cholesky::solve_refined` / `refine_normwise`, accuracy.rs:
 * 83-205, on the CPU): yb_solve_many_refined_device with host arrays, FP32 substitution and FP64
 * refinement against the attached matrix (yb_factor_attach_matrix), in blocks of at most the block
 * width; steps and ratio (either may be NULL) receive each column's corrections and relative
 * residual ||b - A x||inf / ||b||inf. */
int32_t yb_solve_many_mixed(yb_factor *f, const double *rhs, int64_t count, double *out, int32_t max_steps,
                            double tolerance, int32_t *steps, double *ratio);
/* The same solve on device arrays (leading dimensions ldb, ldx >= n) on `stream` (a
 * cudaStream_t, NULL for the GPU's own), asynchronous, in YB_FP64 or YB_FP32 substitution. */
int32_t yb_solve_many_device(yb_factor *f, const double *d_rhs, int64_t ldb, double *d_out, int64_t ldx,
                             int64_t count, int32_t precision, void *stream);

/* ---- blocks solved on the device (ybus_cuda `GpuBlock`, `GpuOperator`, pairs.rs) ------------- */
typedef struct yb_block yb_block;
typedef struct yb_operator yb_operator;

/* `GpuFactor::pair_solves` (pairs.rs:153-202): solves A y = e_plus - e_minus for each of `count`
 * pairs (unknowns, -1 for none; at most yb_factor_block_width of them; the two unknowns of a pair
 * differ), the right-hand sides built on the device, and keeps the solutions there. */
int32_t yb_pair_solves(yb_factor *f, int64_t count, const int64_t *plus, const int64_t *minus, yb_block **out);
/* `GpuFactor::pair_updates` (pairs.rs:204-253, kernels.cu:24-58): the pair solves, then each
 * column's rank-one update of `base` (n values): x = base + alpha y, w = inverse_weight - c'y,
 * z = c'x / w, result x + z y, each operation rounded on its own; w = 0 is singular and gives x. */
int32_t yb_pair_updates(yb_factor *f, const double *base, int64_t count, const int64_t *plus, const int64_t *minus,
                        const double *alpha, const double *inverse_weight, yb_block **out);
/* `GpuBlock::columns`; -1 for a null block. */
int64_t yb_block_columns(const yb_block *b);
/* `GpuBlock::singular`: one flag per column (all 0 for pair solves). */
int32_t yb_block_singular(const yb_block *b, int32_t *singular);
/* `GpuBlock::solutions`: n x columns, column-major, indexed by unknown. */
int32_t yb_block_solutions(yb_block *b, double *out);
/* `GpuBlock::maxima` (pairs.rs:293-308, kernels.cu:78-128): each column's largest |value|, its
 * unknown (the smallest on a tie, -1 if all are zero) and whether any value is not finite. Any
 * output may be NULL. */
int32_t yb_block_maxima(yb_block *b, int64_t *row, double *value, int32_t *not_finite);
/* `GpuBlock::product` (pairs.rs:373-392): the operator's M theta + offset for every column, with
 * column k's entry at zero_rows[k] set to 0 (-1: none; NULL: none at all), rows x columns
 * column-major. */
int32_t yb_block_product(yb_block *b, yb_operator *op, const int64_t *zero_rows, double *out);
/* `GpuBlock::product_maxima` (pairs.rs:396-413): the products reduced on the device to each
 * column's largest |value| * weight and its row (ties to the smaller row). */
int32_t yb_block_product_maxima(yb_block *b, yb_operator *op, const int64_t *zero_rows, int64_t *row, double *value,
                                int32_t *not_finite);
void yb_block_free(yb_block *b);
/* `GpuFactor::operator` (pairs.rs:112-149): a rows x n CSR matrix over the factor's unknowns,
 * with offset 0 and weights 1. */
int32_t yb_operator_new(yb_factor *f, int64_t rows, const int64_t *ptr, const int64_t *idx, const double *val,
                        yb_operator **out);
/* `GpuOperator::rows`; -1 for a null operator. */
int64_t yb_operator_rows(const yb_operator *op);
/* `GpuOperator::set_offset` / `set_weights` (pairs.rs:73-86): one value per row. */
int32_t yb_operator_set_offset(yb_operator *op, const double *offset);
int32_t yb_operator_set_weights(yb_operator *op, const double *weights);
void yb_operator_free(yb_operator *op);

/* ---- the DC callers (ybus_powerflow/src/dc/gpu.rs: `DcGpuStudy`, `DcGpuSensitivity`) ---------- */
typedef struct yb_dc_network yb_dc_network;

/* A DC network from its branch list (bus indices, reactances x; no taps or shifters): Bbus and Bf
 * stamped as ybus_powerflow's `Bdc::new` stamps them (dc.rs:79-113: b = 1/x, parallel branches
 * summed), B' = Bbus without the slack's row and column factored by AMD Cholesky on the host
 * (`DcModel::factor_over`, dc.rs:368-407) and uploaded with B' attached, Bf kept as an operator on
 * the solutions, and the bridges found (islands.rs:132-176). The unknowns are the buses other than
 * the slack, in bus order. */
int32_t yb_dc_network_new(yb_gpu *gpu, int64_t n_bus, int64_t n_branch, const int64_t *from, const int64_t *to,
                          const double *x, int64_t slack, yb_dc_network **out);
void yb_dc_network_free(yb_dc_network *net);
/* The network's uploaded factor (owned by the network). */
yb_factor *yb_dc_network_factor(yb_dc_network *net);
/* One flag per branch: whether it is a bridge (its outage islands the network). */
int32_t yb_dc_bridges(const yb_dc_network *net, uint8_t *bridge);
/* `DcGpuSensitivity::ptdf_columns` (gpu.rs:506-528; sensitivity.rs:233): for an injection at each
 * of `count` buses, withdrawn at the slack, every branch's flow: n_branch x count, column-major;
 * with slack weights set (yb_dc_set_slack_weights) each column less the shift H w. */
int32_t yb_dc_ptdf_columns(yb_dc_network *net, int64_t count, const int64_t *buses, double *out);
/* `DcGpuSensitivity::ptdf_transfers` (gpu.rs:532; sensitivity.rs:284): a transfer from each
 * from_bus to its to_bus. */
int32_t yb_dc_ptdf_transfers(yb_dc_network *net, int64_t count, const int64_t *from_bus, const int64_t *to_bus,
                             double *out);
/* `DcSensitivity::lodf_columns` on the GPU (sensitivity.rs:322-362): for the outage of each branch,
 * every branch's change in flow as a fraction of its flow before, -1 for itself, a NaN column for a
 * bridge; n_branch x count. */
int32_t yb_dc_lodf_columns(yb_dc_network *net, int64_t count, const int64_t *branches, double *out);
/* `DcSensitivity`'s distributed slack (`PtdfSlack::Weights`, dc/sensitivity.rs:101-126, 256-263;
 * on the GPU `DcGpuSensitivity::set_shifted`, gpu.rs:443-583): weights per bus (n_bus), normalized
 * to sum to 1, or NULL for the single slack again. The shift H w, every branch's flow for the
 * weighted injections, is computed here by one solve; yb_dc_ptdf_columns then subtracts it from
 * every column (PTDF - (PTDF w) 1'), while transfers and LODF columns do not depend on the slack.
 * YB_ERROR_INVALID_ARGUMENT when the weights' sum is zero or not finite. */
int32_t yb_dc_set_slack_weights(yb_dc_network *net, const double *weights);
/* `DcGpuStudy::solve_many` (gpu.rs:214-260) with the placement on the device: for each of `count`
 * injection scenarios (n_bus x count, column-major, by bus; the slack's entry is ignored), the
 * angles theta = B'^-1 p placed over the buses (the slack's angle 0; n_bus x count) and every
 * branch's flow b (theta_f - theta_t) (n_branch x count), and per scenario flags: 1 a flow not
 * finite, 2 an angle not finite or above 1e5 in magnitude (the check `DcStudy::place` makes before
 * it accepts a solution, dc.rs:558-564). Any output may be NULL. */
int32_t yb_dc_solve_many(yb_dc_network *net, int64_t count, const double *injections, double *theta, double *flows,
                         int32_t *flags);
/* `DcStudy::outage` for outages of several branches (dc/outage.rs:126-241: W = D^-1 - C'Y,
 * theta' = x + Y W^-1 C'x) and `DcGpuStudy::solve_branch_outages` (gpu.rs:273-322, one branch a
 * case) as whole solutions, on the device: case c takes out the branches branch_ptr[c] ..
 * branch_ptr[c+1] - 1 of `branches` (up to 16, sorted and repeats dropped as `outaged_branches`
 * does) and solves the scenario columns scenario_ptr[c] .. scenario_ptr[c+1] - 1 of `injections`
 * (n_bus x total). Per scenario the angles over the buses and the flows, the outaged branches'
 * zero, and the flags of yb_dc_solve_many; per case whether W is singular (the outage islands a
 * bus: the scenarios keep the base angles and the caller decides, as the reference's CPU fallback
 * would). Every output may be NULL. */
int32_t yb_dc_outage_solutions(yb_dc_network *net, int64_t cases, const int64_t *branch_ptr, const int64_t *branches,
                               const int64_t *scenario_ptr, const double *injections, double *theta, double *flows,
                               int32_t *flags, int32_t *singular);
/* No ybus counterpart as such (the reference screens one base per outage, `DcGpuStudy::
 * outage_loadings`, gpu.rs:334-430): N-1 screening of many injection scenarios per outage. Case c
 * takes out branch outaged[c] (a rank-one update of B', dc/outage.rs:126-241) and has the scenario
 * columns scenario_ptr[c] .. scenario_ptr[c+1] - 1 of `injections` (n_bus x total, column-major, by
 * bus; the slack's entry is ignored). For every scenario column: the branch with the largest
 * |flow| * weight (weights NULL: 1), the loading, and flags: 1 a flow not finite, 2 an angle not
 * finite or above 1e5 in magnitude (with a singular case, the reference's reasons to distrust a
 * screened outage and solve it again on the CPU, gpu.rs:406-410); per case whether the update is
 * singular (1/b - c'y = 0: a bridge). All cases run as one pair solve and one
 * scenario solve with the update, flows and maxima fused (YB_FP64), captured in a CUDA graph that
 * later calls of the same sizes replay; or with FP32 substitution and FP64 refinement, then the
 * same epilogue (YB_FP32; the slack must be bus 0). */
int32_t yb_dc_outage_loadings_batch(yb_dc_network *net, int64_t cases, const int64_t *outaged,
                                    const int64_t *scenario_ptr, const double *injections, const double *weights,
                                    int32_t precision, int64_t *max_branch, double *max_loading, int32_t *flags,
                                    int32_t *singular);

/* No ybus counterpart: the adjoint of a flow loss over a DC network, a forward/backward pair (the
 * analogue of an autograd function) for `count` injection scenarios (n_bus x count, column-major,
 * the slack's entries ignored). Forward: theta = B'^-1 p, flows f = diag(b) A theta (n_branch x
 * count, optional), loss = sum softplus(|f| - margin * limit)^2; theta and dL/df stay on the device.
 * Backward: lambda = B'^-T (Bf' dL/df) with the same factor; dL/dp = lambda (0 at the slack; n_bus x
 * count) and dL/db (n_branch), b = 1/x each branch's susceptance. Either output may be NULL. */
typedef struct yb_dc_adjoint yb_dc_adjoint;
int32_t yb_dc_adjoint_new(yb_dc_network *net, int64_t count, yb_dc_adjoint **out);
int32_t yb_dc_adjoint_forward(yb_dc_adjoint *adj, const double *injections, const double *limits, double margin,
                              double *loss, double *flows);
int32_t yb_dc_adjoint_backward(yb_dc_adjoint *adj, double *grad_injections, double *grad_susceptance);
void yb_dc_adjoint_free(yb_dc_adjoint *adj);

/* ---- complex LU factors and the multi-network batch (no ybus counterpart on the GPU) --------- */
/* A complex128 LU factor P A Q = L U as ybus_sparse's generic LU makes it for a Ybus (lu.rs:268-417):
 * L unit lower in CSC (diagonal first), U upper in CSC (diagonal last), values interleaved
 * (re, im), row_perm = P, col_perm = Q. Kept on the device in complex128 and complex64. */
int32_t yb_factor_from_lu_complex(yb_gpu *gpu, int64_t n, const int64_t *l_ptr, const int64_t *l_idx,
                                  const double *l_val, const int64_t *u_ptr, const int64_t *u_idx, const double *u_val,
                                  const int64_t *row_perm, const int64_t *col_perm, yb_factor **out);
/* Attaches the complex matrix A (CSR, n x n, natural order, interleaved values) to a complex factor,
 * for refinement and residuals. */
int32_t yb_factor_attach_matrix_complex(yb_factor *f, const int64_t *a_ptr, const int64_t *a_idx, const double *a_val);
/* Solves many complex factors' right-hand sides in one launch (a persistent work list of (network,
 * tile) items, largest networks first): network i solves counts[i] complex128 right-hand sides at
 * d_rhs[i] (column-major n_i x counts[i], interleaved) into d_out[i]. YB_FP64: complex128
 * substitution. YB_FP32: complex64 substitution, then complex128 residuals b - A x against the
 * attached matrices and complex64 corrections while any column is above `tolerance` and the worst
 * one at least halves, at most max_steps; `steps` (host, per network, may be NULL) receives the
 * corrections taken. d_ratio (NULL, or per network a device array of counts[i] doubles, entries may
 * be NULL) receives each column's final ||b - A x||inf / ||b||inf. All factors on one GPU. */
int32_t yb_solve_batch_complex(int64_t networks, yb_factor *const *factors, const double *const *d_rhs,
                               double *const *d_out, const int64_t *counts, int32_t precision, int32_t max_steps,
                               double tolerance, double *const *d_ratio, int32_t *steps, void *stream);

/* Attaches A, the matrix the factor factors (CSR, n x n, natural order, FP64), for refinement:
 * ybus_sparse's `solve_refined` takes it the same way (accuracy.rs:281-308). A copy with its
 * columns mapped to the factor's solution order is kept on the device. */
int32_t yb_factor_attach_matrix(yb_factor *f, const int64_t *a_ptr, const int64_t *a_idx, const double *a_val);
/* No ybus counterpart on the GPU; the CPU's is `solve_refined_normwise` (accuracy.rs:83-122):
 * the substitutions in FP32, the residual and the update x += d in FP64 against the attached A, up
 * to max_steps corrections per tile, until every column's ||r||inf / ||b||inf <= tolerance or the
 * residual stops halving. Each column keeps, as refine_normwise does, its best iterate: x, d_ratio
 * and d_steps are those of the iterate with the smallest relative residual. From 2,048 right-hand
 * sides on (yb_factor_set_refine_lane_min_count; or the FP32 lane threshold of
 * yb_factor_set_lane_min_count, if higher) the passes run on the lane solve, the stop rule applied
 * per column and the solve skipping groups of 32 columns that have all stopped, with each pass's
 * FP32 correction kept beside the work array (two work arrays of FP32, plus an FP64 one when
 * max_steps >= 2) and r = b - A x formed from them each pass; below it, or when the factor admits no
 * lane layout, on the domain solve with the refinement fused into its launch (r kept as r -= A d,
 * the residual of x to rounding). Device arrays as yb_solve_many_device; d_ratio (double, count) and
 * d_steps (int32, count) receive each column's relative residual and corrections (either may be
 * NULL).
 * YB_ERROR_INVALID_ARGUMENT when the factor admits neither solve. */
int32_t yb_solve_many_refined_device(yb_factor *f, const double *d_rhs, int64_t ldb, double *d_out, int64_t ldx,
                                     int64_t count, int32_t max_steps, double tolerance, double *d_ratio,
                                     int32_t *d_steps, void *stream);

/* No counterpart in ybus. The device-array solve for callers that must not have the library
 * allocate device memory: programs whose own pool allocator has reserved the GPU's memory (so a
 * cudaMalloc from here could fail or fragment their pool) and latency-bound loops that cannot take
 * an allocation's implicit synchronisation. It runs the level-scheduled tile solve with its working
 * vectors in a 16 MiB array compiled into the library, which every GPU that loads the library
 * holds until exit, and calls no cudaMalloc or cudaFree. Arguments as yb_solve_many_device; the
 * factor's upload (yb_factor_from_*) still allocates, once. The tile width is the one
 * yb_factor_set_tile gives the precision; YB_ERROR_TOO_LARGE if one block's working vectors
 * (order x tile width x value size) exceed the array. yb_gpu_new places the array on its device
 * and looks up its address (so the module that holds it is loaded then, not at this entry point's
 * first call under lazy module loading), and yb_gpu_new fails if that fails; this entry point
 * itself then loads and allocates nothing. Every call shares the array and
 * leaves its contents behind (no part needs to start at zero); calls that overlap on the GPU race
 * on it and must be serialised by the caller. */
int32_t yb_solve_many_device_noalloc(yb_factor *f, const double *d_rhs, int64_t ldb, double *d_out, int64_t ldx,
                                     int64_t count, int32_t precision, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* YBGPU_H */
