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

// The residual and restore kernels' lanes and blocks: a warp takes chunks of 8 consecutive rows of
// one group, four lanes per row, each lane 8 of the group's 32 columns (lane = quarter * 8 + row, so
// the 8 lanes of a quarter hold the chunk's 8 rows of the same 8 columns); a block of kResWarps
// warps, each taking kResChunks chunks in turn, covers kResRows rows of one group and returns at
// once, as a whole, when that group has stopped.
constexpr int kResWarps = 8, kResChunks = 8, kResRows = kResWarps * kResChunks * 8;
__host__ __device__ inline int64_t res_parts(int64_t n) { return (n + kResRows - 1) / kResRows; }

// Each lane holds 8 values, one per column of its quarter, for its row. Reduces every column to its
// maximum over the quarter's 8 rows by a transposing butterfly: at each step a lane keeps half of
// its values and trades the other half with its partner; after three steps lane l holds column l's
// maximum.
__device__ __forceinline__ unsigned long long column_max8(unsigned long long (&v)[8]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 4, half = 4; s >= 1; s >>= 1, half >>= 1) {
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
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

// 8 FP32 values (32 bytes, 32-byte aligned) in one load
__device__ __forceinline__ void load8(const float *p, float (&v)[8]) {
  asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
               : "l"(p));
}
// 8 FP64 values (64 bytes, 32-byte aligned) in two loads
__device__ __forceinline__ void load8(const double *p, double (&v)[8]) {
#pragma unroll
  for (int c = 0; c < 8; c += 4)
    asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v[c]), "=d"(v[c + 1]), "=d"(v[c + 2]), "=d"(v[c + 3])
                 : "l"(p + c));
}

// The iterate's 8 values of one lane's quarter at one work row, as loaded: the correction d and,
// when there is one, the base x_{k-1} (BASE 1: FP32 parts, BASE 2: FP64); value(c) = base + d in
// FP64. AT_ONCE: the neighbours whose loads the residual keeps in flight together.
template <int BASE> struct Iterate8 {
  static constexpr int AT_ONCE = 2;
  float d[8];
  __device__ __forceinline__ void load(size_t at, const float *dd, const float *, const double *) { load8(dd + at, d); }
  __device__ __forceinline__ double value(int c) const { return (double)d[c]; }
};
template <> struct Iterate8<1> {
  static constexpr int AT_ONCE = 2;
  float d[8], b[8];
  __device__ __forceinline__ void load(size_t at, const float *dd, const float *b32, const double *) {
    load8(dd + at, d);
    load8(b32 + at, b);
  }
  __device__ __forceinline__ double value(int c) const { return (double)b[c] + (double)d[c]; }
};
template <> struct Iterate8<2> {
  static constexpr int AT_ONCE = 1;
  float d[8];
  double b[8];
  __device__ __forceinline__ void load(size_t at, const float *dd, const float *, const double *b64) {
    load8(dd + at, d);
    load8(b64 + at, b);
  }
  __device__ __forceinline__ double value(int c) const { return b[c] + (double)d[c]; }
};

// The residual R = b - A x of the groups still refining, in FP64, with x = base + d formed at every
// row read (BASE 0: x = d, pass 0). Lanes as above: b's and x's columns are read and written 8 rows
// (64 bytes) at a time, and each row of x a lane reads is one 32-byte load, the four lanes of a row
// covering its 128-byte line, so an instruction touches 8 lines (against 16 with two lanes per row
// and 32 with one column per lane: L1's request rate, not DRAM, bounds this kernel). A row's
// neighbours are read AT_ONCE at a time. The first pass fits four blocks an SM (64 registers, a
// few bytes spilled: 955 to 773 us on the 10k-bus block); the later passes, whose iterates come in
// two parts, keep three (at four they spill 64 bytes and slow from 1.33 to 1.50 ms). R goes in FP32 to the work array (the next pass's
// right-hand side); each column's ||R||inf (and on the first pass ||b||inf) is reduced over the
// block's rows in shared memory and then taken by one atomic maximum of its bit pattern per block;
// x_k goes to the caller's columns of write_mask.
template <int BASE>
__global__ void __launch_bounds__(kResWarps * 32, BASE == 0 ? 4 : 3) lane_residual_kernel(LaneRefineArgs a, const float *__restrict__ d,
                                                                        const float *__restrict__ base32,
                                                                        const double *__restrict__ base64, bool first) {
  constexpr int AT = Iterate8<BASE>::AT_ONCE;
  __shared__ unsigned long long red[2][kResWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t parts = res_parts(a.n), g = blockIdx.x / parts, part = blockIdx.x - g * parts;
  if (g >= a.groups || !a.active[g]) return;  // the whole block
  const int c0 = (lane >> 3) * 8;                             // this lane's first column in the group
  const int64_t col0 = g * 32 + c0;                           // ... in the launch
  const int64_t left = a.count - col0;
  const int cols = left <= 0 ? 0 : (left >= 8 ? 8 : (int)left);
  const size_t gw = (size_t)g * a.n;                          // the group's first work row
  uint32_t write = 0;
  if constexpr (BASE != 0) write = (a.write_mask[g] >> c0) & 0xffu;
  unsigned long long rmax = 0ull, bmax = 0ull;  // column `lane`'s maxima over this warp's rows
  for (int k = 0; k < kResChunks; ++k) {
    const int64_t i0 = ((part * kResWarps + warp) * kResChunks + k) * 8;
    if (i0 >= a.n) break;  // the whole warp
    const int i = (int)i0 + (lane & 7);
    const bool row = i < a.n;
    double acc[8];
    const double *bc = a.b + col0 * a.ldb + i;
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = (row && c < cols) ? __ldg(bc + c * a.ldb) : 0.0;
    if (first) {
      unsigned long long bm[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) bm[c] = abs_bits(acc[c]);
      const unsigned long long m = column_max8(bm);
      bmax = m > bmax ? m : bmax;
    }
    if (row) {
      const int len = __ldg(a.res_len + i);
      const int64_t e = __ldg(a.res_ptr + i / 32) + (i & 31);
      for (int q = 0; q < len; q += AT) {  // in stored order
        int32_t w[AT];
        double v[AT];
#pragma unroll
        for (int t = 0; t < AT; ++t) {
          const bool ok = q + t < len;
          w[t] = ok ? __ldg(a.res_col + e + 32 * (q + t)) : 0;
          v[t] = ok ? __ldg(a.res_val + e + 32 * (q + t)) : 0.0;
        }
        Iterate8<BASE> x[AT];
#pragma unroll
        for (int t = 0; t < AT; ++t) x[t].load((gw + w[t]) * 32 + c0, d, base32, base64);
#pragma unroll
        for (int t = 0; t < AT; ++t)
          if (q + t < len) {
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[c] = fma(-v[t], x[t].value(c), acc[c]);
          }
      }
      // R into the work array, this quarter's 8 values in one 32-byte store
      float *r = a.work + (gw + __ldg(a.in_pos + i)) * 32 + c0;
      asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(r), "f"((float)acc[0]),
                   "f"((float)acc[1]), "f"((float)acc[2]), "f"((float)acc[3]), "f"((float)acc[4]), "f"((float)acc[5]),
                   "f"((float)acc[6]), "f"((float)acc[7])
                   : "memory");
    }
    unsigned long long rm[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) rm[c] = (row && c < cols) ? abs_bits(acc[c]) : 0ull;
    const unsigned long long m = column_max8(rm);
    rmax = m > rmax ? m : rmax;
    if constexpr (BASE != 0) {
      if (row && write) {  // x_k of this row for the caller
        Iterate8<BASE> xi;
        xi.load((gw + __ldg(a.out_pos + i)) * 32 + c0, d, base32, base64);
        double *xc = a.x + col0 * a.ldx + i;
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if ((write >> c) & 1u) xc[c * a.ldx] = xi.value(c);
      }
    }
  }
  // the block's maxima, one atomic per column
  red[0][warp][lane] = rmax;
  red[1][warp][lane] = bmax;
  __syncthreads();
  if (warp == 0 && g * 32 + lane < a.count) {
    unsigned long long mr = 0ull, mb = 0ull;
#pragma unroll
    for (int w = 0; w < kResWarps; ++w) {
      mr = red[0][w][lane] > mr ? red[0][w][lane] : mr;
      mb = red[1][w][lane] > mb ? red[1][w][lane] : mb;
    }
    if (mr) atomicMax(a.rmax + g * 32 + lane, mr);
    if (first && mb) atomicMax(a.bmax + g * 32 + lane, mb);
  }
}

// One warp per group, one lane per column: each column's relative residual after `pass`
// corrections and the state of refine_normwise (accuracy.rs:93-118): pass 0 takes x0 as the best; a
// later pass keeps x_k if its ratio is below the best, else x_{k-1} is put back in the caller's x
// (restore_mask); a column stops within the tolerance, on a NaN ratio, when the ratio did not
// halve, or after max_steps, and then gets its best ratio and correction count. write_mask becomes
// the columns whose best is x_pass, the ones the next pass may overwrite; a column that stops at
// pass 0 has its x0 written by the restore.
__global__ void lane_refine_decide_kernel(LaneRefineArgs a, int32_t pass, int32_t max_steps, double tolerance) {
  const int lane = threadIdx.x & 31;
  const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= a.groups) return;  // the whole warp
  if (!a.active[g]) {
    if (lane == 0) a.restore_mask[g] = 0;
    return;
  }
  const uint32_t act = a.col_active[g], wrote = a.write_mask[g];
  bool stop = false, write = false, restore = false;
  if ((act >> lane) & 1u) {
    const int64_t col = g * 32 + lane;
    const double rn = __longlong_as_double((long long)a.rmax[col]), bn = __longlong_as_double((long long)a.bmax[col]);
    const double ratio = bn > 0.0 ? rn / bn : (rn > 0.0 ? __longlong_as_double(0x7ff0000000000000LL) : 0.0);
    a.rmax[col] = 0ull;
    if (pass == 0) {
      a.best[col] = ratio, a.best_steps[col] = 0, a.cur[col] = ratio;
      stop = ratio <= tolerance || max_steps < 1;
      restore = stop;
    } else {
      const double previous = a.cur[col];
      a.cur[col] = ratio;
      const bool improved = ratio < a.best[col];
      if (improved) a.best[col] = ratio, a.best_steps[col] = pass;
      restore = !improved && ((wrote >> lane) & 1u);
      stop = ratio != ratio || ratio > 0.5 * previous || ratio <= tolerance || pass >= max_steps;
    }
    if (stop) {
      if (a.ratio_out) a.ratio_out[col] = a.best[col];
      if (a.steps_out) a.steps_out[col] = a.best_steps[col];
    } else {
      write = a.best_steps[col] == pass;
    }
  }
  const uint32_t stopped = __ballot_sync(0xffffffffu, stop), writes = __ballot_sync(0xffffffffu, write),
                 restores = __ballot_sync(0xffffffffu, restore);
  if (lane == 0) {
    const uint32_t left = act & ~stopped;
    a.col_active[g] = left, a.write_mask[g] = writes, a.restore_mask[g] = restores;
    if (!left) a.active[g] = 0;
  }
}

// The caller's x of the columns in restore_mask set to the iterate `base` holds (FP32 parts or
// FP64, in the work array's layout): x_{pass-1} for the columns a pass made no better, x0 for the
// columns that stopped at pass 0. Blocks and lanes as in the residual; a block whose group has
// nothing to restore returns at once.
template <class B>
__global__ void __launch_bounds__(kResWarps * 32) lane_restore_kernel(LaneRefineArgs a, const B *__restrict__ base) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t parts = res_parts(a.n), g = blockIdx.x / parts, part = blockIdx.x - g * parts;
  if (g >= a.groups) return;
  const uint32_t all = a.restore_mask[g];
  if (!all) return;  // the whole block
  const int c0 = (lane >> 3) * 8;
  const uint32_t mask = (all >> c0) & 0xffu;
  if (!mask) return;
  for (int k = 0; k < kResChunks; ++k) {
    const int64_t i0 = ((part * kResWarps + warp) * kResChunks + k) * 8;
    const int i = (int)i0 + (lane & 7);
    if (i >= a.n) break;
    const B *src = base + ((size_t)g * a.n + __ldg(a.out_pos + i)) * 32 + c0;
    double *xc = a.x + (g * 32 + c0) * a.ldx + i;
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if ((mask >> c) & 1u) xc[c * a.ldx] = (double)src[c];
  }
}

// X = base + d over the work rows of the groups still refining: the iterate kept in FP64 for a
// further pass (base FP32 parts on pass 1, X itself after). A block takes one of `parts` slices of
// one group's values and returns at once when the group has stopped.
template <class B>
__global__ void __launch_bounds__(256) lane_carry_kernel(LaneRefineArgs a, const B *base, const float *__restrict__ d,
                                                        double *X, int64_t parts) {  // base may be X itself
  const int64_t g = blockIdx.x / parts, part = blockIdx.x - g * parts;
  if (g >= a.groups || !a.active[g]) return;
  const int64_t gv = (int64_t)a.n * 32, per = (gv + parts - 1) / parts;
  const int64_t lo = g * gv + part * per, hi = g * gv + (gv < (part + 1) * per ? gv : (part + 1) * per);
  for (int64_t k = lo + threadIdx.x; k < hi; k += blockDim.x) X[k] = (double)base[k] + (double)d[k];
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
