// Mixed-precision refinement around the lane solve, for blocks large enough to take it: the
// substitutions in FP32 through the lane solve (masked to the groups of 32 columns still
// refining), the update x += d and the residual R = b - A x in FP64, b and x kept in the lane
// layout [group][row][lane] (rows natural) so that the residual reads whole 256-byte rows and
// writes the next pass's FP32 right-hand side straight into the work array. The stop rule is the
// domain solve's refined one applied to each group of 32 columns (domain_solve.cuh, after
// ybus_sparse accuracy.rs:83-122): a group stops when none of its columns is above the tolerance,
// or none of those above it halved its relative residual in the last pass, or a relative
// residual is not a number, or after max_steps corrections.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "lane_solve.cuh"

namespace yb {

// The largest of non-negative doubles (and NaN above them all) by their bit patterns.
__device__ __forceinline__ void lane_atomic_max(unsigned long long *at, double v) {
  atomicMax(at, (unsigned long long)__double_as_longlong(v));
}

// x += d (or x = d on the first pass) for the groups still refining, in the lane layout: x in
// FP64 [group][row][lane], rows in x's natural order; d the lane solve's result in its work array
// (x's row i in work row out_pos[i]). One warp per 32 rows of a group, each lane a row.
template <class T>
__global__ void __launch_bounds__(256) lane_update_kernel(const T *__restrict__ work, const int32_t *__restrict__ out_pos,
                                                          double *__restrict__ xl, int32_t n, int64_t groups,
                                                          const uint8_t *__restrict__ group_active, bool first) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int64_t chunks = (n + 31) / 32, g = w / chunks;
  if (g >= groups || !group_active[g]) return;
  const int i = (int)(w % chunks) * 32 + lane;
  if (i >= n) return;
  double d[32];
  lane_row_load(work + ((size_t)g * n + __ldg(out_pos + i)) * 32, d);
  double *row = xl + ((size_t)g * n + i) * 32;
  if (!first) {
    double x[32];
    lane_row_load(row, x);
#pragma unroll
    for (int c = 0; c < 32; ++c) d[c] += x[c];
  }
  lane_row_store(row, d);
}

// R = b - A x for the groups still refining, in the lane layout (b and x FP64 [group][row][lane],
// rows natural): a warp takes a row of a group, its 32 lanes the group's 32 columns, so A's entries
// of the row are shared by the warp and every x row it reads is one 256-byte line. R goes in FP32
// into the work array's row in_pos[i] (the next pass's right-hand side) and each column's ||R||inf
// into rmax (and, when bmax is not null, ||b||inf into bmax), by atomic maximum. A in CSR, natural
// order. Blocks of 8 warps; a warp takes 32 rows of one group in turn.
__global__ void __launch_bounds__(256) lane_residual_kernel(const double *__restrict__ bl, const double *__restrict__ xl,
                                                            float *__restrict__ work, const int32_t *__restrict__ in_pos,
                                                            int32_t n, int64_t groups, int64_t count,
                                                            const int32_t *__restrict__ a_ptr,
                                                            const int32_t *__restrict__ a_idx,
                                                            const double *__restrict__ a_val,
                                                            const uint8_t *__restrict__ group_active,
                                                            unsigned long long *rmax, unsigned long long *bmax) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int64_t chunks = (n + 31) / 32, g = w / chunks;
  if (g >= groups || !group_active[g]) return;
  const int i0 = (int)(w % chunks) * 32, i1 = min(n, i0 + 32);
  const double *bg = bl + (size_t)g * n * 32 + lane, *xg = xl + (size_t)g * n * 32 + lane;
  double rm = 0.0, bm = 0.0;
  bool nan_seen = false;
  for (int i = i0; i < i1; ++i) {
    const double bv = bg[(size_t)i * 32];
    double acc = bv;
    const int p1 = __ldg(a_ptr + i + 1);
    for (int p = __ldg(a_ptr + i); p < p1; ++p) acc -= __ldg(a_val + p) * xg[(size_t)__ldg(a_idx + p) * 32];
    work[((size_t)g * n + __ldg(in_pos + i)) * 32 + lane] = (float)acc;
    rm = fmax(rm, fabs(acc));
    bm = fmax(bm, fabs(bv));
    nan_seen = nan_seen || (acc != acc);  // fmax drops NaN operands
  }
  const int64_t col = g * 32 + lane;
  if (col < count) {
    lane_atomic_max(rmax + col, nan_seen ? __longlong_as_double(0x7ff8000000000000LL) : rm);
    if (bmax) lane_atomic_max(bmax + col, bm);
  }
}

// One thread per group still refining: each column's relative residual after `pass` corrections,
// the group's decision, and for a group that stops, its columns' final relative residuals and
// correction counts. rmax is cleared for the next pass.
__global__ void lane_refine_decide_kernel(int64_t groups, int64_t count, int32_t pass, int32_t max_steps, double tolerance,
                                          unsigned long long *rmax, const unsigned long long *bmax, double *prev,
                                          uint8_t *group_active, double *ratio_out, int32_t *steps_out) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= groups || !group_active[g]) return;
  bool open = false, progress = false, bad = false;
  for (int c = 0; c < 32; ++c) {
    const int64_t col = g * 32 + c;
    if (col >= count) break;
    const double rn = __longlong_as_double((long long)rmax[col]), bn = __longlong_as_double((long long)bmax[col]);
    const double ratio = bn > 0.0 ? rn / bn : (rn > 0.0 ? __longlong_as_double(0x7ff0000000000000LL) : 0.0);
    bad = bad || (ratio != ratio);
    if (ratio > tolerance) {
      open = true;
      progress = progress || (ratio <= 0.5 * prev[col]);
    }
    prev[col] = ratio;
    rmax[col] = 0ull;
  }
  if (!open || !progress || bad || pass >= max_steps) {
    for (int c = 0; c < 32; ++c) {
      const int64_t col = g * 32 + c;
      if (col >= count) break;
      if (ratio_out) ratio_out[col] = prev[col];
      if (steps_out) steps_out[col] = pass;
    }
    group_active[g] = 0;
  }
}

// Every group refining, no maxima yet, no previous residual (+infinity).
__global__ void lane_refine_init_kernel(int64_t groups, int64_t count, unsigned long long *rmax, unsigned long long *bmax,
                                        double *prev, uint8_t *group_active) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count) rmax[k] = 0ull, bmax[k] = 0ull, prev[k] = __longlong_as_double(0x7ff0000000000000LL);
  if (k < groups) group_active[k] = 1;
}

}  // namespace yb
