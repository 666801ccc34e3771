// Mixed-precision refinement around the lane solve, for blocks large enough to take it: the
// substitutions in FP32 through the lane solve (masked to the groups of 32 columns still refining),
// the residual R = b - A x and the iterate x = x' + d in FP64 against the FP64 matrix, with the
// stop rule of ybus_sparse's refine_normwise (accuracy.rs:83-122) applied to every column.
//
// Data. b and x are the caller's (column-major). Each pass's correction d is the lane solve's
// output, FP32 in the work array's layout [group][work row][lane]; the iterate is never stored in
// full unless a third pass needs it: pass 0's iterate is d0 itself, pass 1's is d0 + d1 (both
// FP32, added in FP64 where they are read), and only from pass 2 on is x_k kept in FP64, in the
// same layout (X). The residual kernel forms x at every row it reads from those parts, so a pass
// reads b once, the parts of x once (plus the rows' neighbours from L2), and writes R in FP32 as
// the next pass's right-hand side and, for the columns still refining, x_k into the caller's x.
//
// Columns. Per column the state of refine_normwise: the current relative residual, the best one
// and its correction count (the x returned is the best iterate, not the last). From pass 1 on, x_k
// goes to the caller only for a column whose best iterate is x_{k-1}; if x_k turns out no better,
// x_{k-1} is put back. A column stops when its ratio is within the tolerance, is not a number,
// has not halved (ratio > ratio_before / 2), or after max_steps corrections; a group of 32 columns
// stops with its last column.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "lane_solve.cuh"

namespace yb {

// The state of one launch of the refined lane solve (a contiguous run of groups).
struct LaneRefineArgs {
  int32_t n;
  int64_t groups, count;                     // this launch's groups of 32 columns, and its columns
  const double *b;                           // the caller's right-hand sides (this launch's first column)
  int64_t ldb;
  double *x;                                 // the caller's solutions
  int64_t ldx;
  const int32_t *in_pos, *out_pos;           // rows of b and of x -> work rows
  // A by natural rows in slices of 32 (entry q of row 32 s + l at res_ptr[s] + 32 q + l, res_len[row]
  // entries), each entry's column as the work row that holds that unknown
  const int32_t *res_ptr, *res_len, *res_col;
  const double *res_val;
  float *work;                               // the next pass's right-hand side, R in FP32
  // per column
  unsigned long long *rmax, *bmax;           // ||R||inf and ||b||inf as bit patterns (atomic maxima)
  double *cur, *best;                        // the current and the best relative residual
  int32_t *best_steps;
  double *ratio_out;                         // null, or the caller's final relative residuals
  int32_t *steps_out;                        // null, or the caller's correction counts
  // per group
  uint8_t *active;                           // the group is still refining
  uint32_t *col_active, *write_mask, *restore_mask;
};

// The largest of |v| as an unsigned bit pattern: positive doubles order as their patterns, and a
// NaN (its sign cleared) lies above them all, so the maximum of a column holding a NaN is a NaN.
__device__ __forceinline__ unsigned long long abs_bits(double v) {
  return (unsigned long long)__double_as_longlong(fabs(v));
}

// Each lane holds 16 values, one per column of its half of the warp (lanes 0-15: columns 0-15,
// lanes 16-31: columns 16-31), for its row. Reduces every column to its maximum over the half's 16
// rows by a transposing butterfly: at each step a lane keeps half of its values and trades the
// other half with its partner; after four steps lane l holds column l's maximum.
__device__ __forceinline__ unsigned long long column_max16(unsigned long long (&v)[16]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 8, half = 8; s >= 1; s >>= 1, half >>= 1) {
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k < half) {
        const unsigned long long send = upper ? v[k] : v[k + half];
        const unsigned long long keep = upper ? v[k + half] : v[k];
        const unsigned long long got = __shfl_xor_sync(0xffffffffu, send, s);
        v[k] = keep > got ? keep : got;
      }
    }
  }
  return v[0];
}

// 16 FP32 values of a work row (64 bytes, 32-byte aligned) as doubles
__device__ __forceinline__ void load16(const float *p, double (&v)[16]) {
#pragma unroll
  for (int c = 0; c < 16; c += 8) {
    float f[8];
    asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(f[0]), "=f"(f[1]), "=f"(f[2]), "=f"(f[3]), "=f"(f[4]), "=f"(f[5]), "=f"(f[6]), "=f"(f[7])
                 : "l"(p + c));
#pragma unroll
    for (int k = 0; k < 8; ++k) v[c + k] = f[k];
  }
}
// 16 FP64 values of a row (128 bytes, 32-byte aligned), added to v
__device__ __forceinline__ void add16(const double *p, double (&v)[16]) {
#pragma unroll
  for (int c = 0; c < 16; c += 4) {
    double d[4];
    asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(d[0]), "=d"(d[1]), "=d"(d[2]), "=d"(d[3]) : "l"(p + c));
#pragma unroll
    for (int k = 0; k < 4; ++k) v[c + k] = d[k] + v[c + k];
  }
}

// The iterate's 16 values of this lane's half at work row `wr` of group g: d, plus the base
// (x_{k-1}) when there is one (BASE 1: FP32 parts, BASE 2: FP64), added in FP64 as base + d.
template <int BASE>
__device__ __forceinline__ void iterate16(size_t at, const float *__restrict__ d, const float *__restrict__ base32,
                                          const double *__restrict__ base64, double (&x)[16]) {
  load16(d + at, x);
  if constexpr (BASE == 1) {
    double bv[16];
    load16(base32 + at, bv);
#pragma unroll
    for (int c = 0; c < 16; ++c) x[c] = bv[c] + x[c];
  } else if constexpr (BASE == 2) {
    add16(base64 + at, x);
  }
}

// The residual R = b - A x of the groups still refining, in FP64, with x = base + d formed at every
// row read (BASE 0: x = d, pass 0). Two lanes per row, each the 16 columns of its half of the group;
// a warp takes 16 consecutive rows of one group, so b's and x's columns are read and written 16
// rows (128 bytes) at a time. R goes in FP32 to the work array (the next pass's right-hand side),
// each column's ||R||inf (and on the first pass ||b||inf) by atomic maximum of its bit pattern, and
// x_k to the caller's columns of write_mask.
template <int BASE>
__global__ void __launch_bounds__(256) lane_residual_kernel(LaneRefineArgs a, const float *__restrict__ d,
                                                            const float *__restrict__ base32,
                                                            const double *__restrict__ base64, bool first) {
  const int lane = threadIdx.x & 31, half = lane >> 4;
  const int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int64_t chunks = (a.n + 15) / 16, g = w / chunks;
  if (g >= a.groups || !a.active[g]) return;  // the whole warp
  const int i = (int)(w % chunks) * 16 + (lane & 15);
  const bool row = i < a.n;
  const int c0 = half * 16;                                   // this lane's first column in the group
  const int64_t col0 = g * 32 + c0;                           // ... in the launch
  const int64_t left = a.count - col0;
  const int cols = left <= 0 ? 0 : (left >= 16 ? 16 : (int)left);
  const size_t gw = (size_t)g * a.n;                          // the group's first work row
  double acc[16];
  const double *bc = a.b + col0 * a.ldb + i;
#pragma unroll
  for (int c = 0; c < 16; ++c) acc[c] = (row && c < cols) ? __ldg(bc + c * a.ldb) : 0.0;
  if (first) {
    unsigned long long bm[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) bm[c] = abs_bits(acc[c]);
    const unsigned long long m = column_max16(bm);
    if (g * 32 + lane < a.count) atomicMax(a.bmax + g * 32 + lane, m);
  }
  if (row) {
    const int len = __ldg(a.res_len + i);
    const int64_t e = __ldg(a.res_ptr + i / 32) + (i & 31);
    for (int q = 0; q < len; ++q) {
      const int32_t wj = __ldg(a.res_col + e + 32 * q);
      const double v = __ldg(a.res_val + e + 32 * q);
      double xj[16];
      iterate16<BASE>((gw + wj) * 32 + c0, d, base32, base64, xj);
#pragma unroll
      for (int c = 0; c < 16; ++c) acc[c] = fma(-v, xj[c], acc[c]);
    }
    // R into the work array, this half's 16 values in two 32-byte stores
    float *r = a.work + (gw + __ldg(a.in_pos + i)) * 32 + c0;
#pragma unroll
    for (int c = 0; c < 16; c += 8)
      asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(r + c), "f"((float)acc[c]),
                   "f"((float)acc[c + 1]), "f"((float)acc[c + 2]), "f"((float)acc[c + 3]), "f"((float)acc[c + 4]),
                   "f"((float)acc[c + 5]), "f"((float)acc[c + 6]), "f"((float)acc[c + 7])
                   : "memory");
  }
  unsigned long long rm[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) rm[c] = (row && c < cols) ? abs_bits(acc[c]) : 0ull;
  const unsigned long long m = column_max16(rm);
  if (g * 32 + lane < a.count) atomicMax(a.rmax + g * 32 + lane, m);
  if constexpr (BASE != 0) {
    const uint32_t mask = (a.write_mask[g] >> c0) & 0xffffu;
    if (row && mask) {  // x_k of this row for the caller
      double xi[16];
      iterate16<BASE>((gw + __ldg(a.out_pos + i)) * 32 + c0, d, base32, base64, xi);
      double *xc = a.x + col0 * a.ldx + i;
#pragma unroll
      for (int c = 0; c < 16; ++c)
        if ((mask >> c) & 1u) xc[c * a.ldx] = xi[c];
    }
  }
}

// One thread per group: each column's relative residual after `pass` corrections and the state of
// refine_normwise (accuracy.rs:93-118): pass 0 takes x0 as the best; a later pass keeps x_k if its
// ratio is below the best, else x_{k-1} is put back in the caller's x (restore_mask); a column stops
// within the tolerance, on a NaN ratio, when the ratio did not halve, or after max_steps, and then
// gets its best ratio and correction count. write_mask becomes the columns whose best is x_pass, the
// ones the next pass may overwrite; a column that stops at pass 0 has its x0 written by the restore.
__global__ void lane_refine_decide_kernel(LaneRefineArgs a, int32_t pass, int32_t max_steps, double tolerance) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.groups) return;
  if (!a.active[g]) {
    a.restore_mask[g] = 0;
    return;
  }
  uint32_t act = a.col_active[g], write = 0, restore = 0;
  const uint32_t wrote = a.write_mask[g];
  for (int c = 0; c < 32; ++c) {
    if (!((act >> c) & 1u)) continue;
    const int64_t col = g * 32 + c;
    const double rn = __longlong_as_double((long long)a.rmax[col]), bn = __longlong_as_double((long long)a.bmax[col]);
    const double ratio = bn > 0.0 ? rn / bn : (rn > 0.0 ? __longlong_as_double(0x7ff0000000000000LL) : 0.0);
    a.rmax[col] = 0ull;
    bool stop;
    if (pass == 0) {
      a.best[col] = ratio, a.best_steps[col] = 0, a.cur[col] = ratio;
      stop = ratio <= tolerance || max_steps < 1;
      if (stop) restore |= 1u << c;
    } else {
      const double previous = a.cur[col];
      a.cur[col] = ratio;
      const bool improved = ratio < a.best[col];
      if (improved) a.best[col] = ratio, a.best_steps[col] = pass;
      if (!improved && ((wrote >> c) & 1u)) restore |= 1u << c;
      stop = ratio != ratio || ratio > 0.5 * previous || ratio <= tolerance || pass >= max_steps;
    }
    if (stop) {
      act &= ~(1u << c);
      if (a.ratio_out) a.ratio_out[col] = a.best[col];
      if (a.steps_out) a.steps_out[col] = a.best_steps[col];
    } else if (a.best_steps[col] == pass) {
      write |= 1u << c;
    }
  }
  a.col_active[g] = act, a.write_mask[g] = write, a.restore_mask[g] = restore;
  if (!act) a.active[g] = 0;
}

// The caller's x of the columns in restore_mask set to the iterate `base` holds (FP32 parts or
// FP64, in the work array's layout): x_{pass-1} for the columns a pass made no better, x0 for the
// columns that stopped at pass 0. Two lanes per row as in the residual; groups with nothing to
// restore return at once.
template <class B>
__global__ void __launch_bounds__(256) lane_restore_kernel(LaneRefineArgs a, const B *__restrict__ base) {
  const int lane = threadIdx.x & 31, half = lane >> 4;
  const int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
  const int64_t chunks = (a.n + 15) / 16, g = w / chunks;
  if (g >= a.groups) return;
  const int c0 = half * 16;
  const uint32_t mask = (a.restore_mask[g] >> c0) & 0xffffu;
  const int i = (int)(w % chunks) * 16 + (lane & 15);
  if (!mask || i >= a.n) return;
  const B *src = base + ((size_t)g * a.n + __ldg(a.out_pos + i)) * 32 + c0;
  double *xc = a.x + (g * 32 + c0) * a.ldx + i;
#pragma unroll
  for (int c = 0; c < 16; ++c)
    if ((mask >> c) & 1u) xc[c * a.ldx] = (double)src[c];
}

// X = base + d over every work row of the groups still refining: the iterate kept in FP64 for a
// further pass (base FP32 parts on pass 1, X itself after).
template <class B>
__global__ void __launch_bounds__(256) lane_carry_kernel(LaneRefineArgs a, const B *base, const float *__restrict__ d,
                                                        double *X) {  // base may be X itself
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // one value of the launch's groups
  const int64_t g = k / ((int64_t)a.n * 32);
  if (g >= a.groups || !a.active[g]) return;
  X[k] = (double)base[k] + (double)d[k];
}

// Every group refining with every column below `count`, no maxima yet.
__global__ void lane_refine_init_kernel(LaneRefineArgs a) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < a.count) a.rmax[k] = 0ull, a.bmax[k] = 0ull;
  if (k < a.groups) {
    const int64_t left = a.count - k * 32, cols = left < 32 ? left : 32;
    a.active[k] = 1;
    a.col_active[k] = cols >= 32 ? 0xffffffffu : ((1u << cols) - 1u);
    a.write_mask[k] = 0, a.restore_mask[k] = 0;
  }
}

}  // namespace yb
