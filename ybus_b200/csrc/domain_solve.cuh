// The domain solve: one thread block per SM holds a tile of W right-hand sides' whole working
// vector in shared memory and takes both sweeps through it, each warp reading its own stream of
// records (DomainLayout in plan.hpp) from pages that TMA bulk copies bring into a per-warp ring.
//
// Per tile:
//   load      b's W columns into slots (coalesced along each column), no scaling
//   stage 0   each warp solves its domains forward, level after level
//   stage 1   r_T = b_T - L_TB y_B into the tail buffer (top rows dealt over the warps)
//   stage 2   y_T = L_TT^-1 r_T (dense rows) into the top rows' slots
//   stage 3   y_T copied into the tail buffer
//   stage 4   x_T = U_TT^-1 y_T (dense rows) into the top rows' slots
//   stage 5   each warp solves its domains backward
//   store     the slots into x's W columns
// A block barrier separates stages; within a stage a warp orders its own records with
// __syncwarp. Without a top block, stages 1-5 collapse into stage 0: every warp's domains are
// closed under both sweeps, so no warp waits for another.
//
// The load and store policies (IO) give the tile its right-hand sides and take its solutions: dense
// columns of b and x here; other policies build right-hand sides on the device or fuse epilogues.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"
#include "plan.hpp"
#include "stream_solve.cuh"

namespace yb {

struct DomainArgs {
  int32_t n;
  int64_t count, tiles;
  const uint8_t *__restrict__ blob;
  const int32_t *__restrict__ warp_page;  // [warps + 1]
  int32_t page_bytes, ring, stages;
  int32_t tail;                           // rows of the top block (0: none)
  const int32_t *__restrict__ tail_slot;  // [tail]
  int32_t *error;                         // set to 1 if a wait ran out
  // diagnostics: if set, block 0 writes clock64() marks for its first 4 tiles as [tile][warp][8]:
  // 0 tile start, 1 load done, 2 last record done, 3 store done, 4 cycles waiting for pages,
  // 5 cycles in stage barriers, 6 pages taken, 7 records taken
  long long *phase_clock;
};

// Shared memory an IO policy may declare statically (its reductions), kept free beside the
// dynamic shared memory.
constexpr size_t kIoStaticSmem = 2048;

// The shared-memory footprint of a domain solve block.
__host__ __device__ inline size_t domain_smem_bytes(int32_t n, int32_t W, int32_t value_bytes, int32_t tail,
                                                    int32_t warps, int32_t ring, int32_t page_bytes) {
  const size_t y = (((size_t)(n + 2) * W * value_bytes) + 127) & ~(size_t)127;
  const size_t tb = (((size_t)(tail + 1) * W * value_bytes) + 15) & ~(size_t)15;
  const size_t ts = (((size_t)(tail + 1) * 4) + 127) & ~(size_t)127;
  return y + tb + ts + (size_t)warps * ring * page_bytes + (size_t)warps * ring * 8 + kIoStaticSmem;
}

// Dense columns of b in, dense columns of x out (column-major, natural row order; the
// permutations are applied on the shared-memory side). While a tile is solved, the columns of the
// block's next tile are prefetched into L2 by bulk prefetches, so its load finds them there.
struct DenseIO {
  static constexpr bool kRefine = false;
  const double *__restrict__ b;
  int64_t ldb;
  double *__restrict__ x;
  int64_t ldx;
  const int32_t *__restrict__ in_slot;
  const int32_t *__restrict__ out_slot;

  template <class T, int W>
  __device__ __forceinline__ void load(int64_t col0, int64_t count, int n, T *Ys) const {
    load_columns<T, W>(b, ldb, in_slot, col0, count, n, Ys);
  }

  template <class T, int W>
  __device__ __forceinline__ static void load_columns(const double *__restrict__ b, int64_t ldb,
                                                      const int32_t *__restrict__ in_slot, int64_t col0,
                                                      int64_t count, int n, T *Ys) {
    constexpr int U = W >= 4 ? 2 : 8 / W;  // loads in flight per thread and column
#pragma unroll 1
    for (int r0 = threadIdx.x; r0 < n; r0 += blockDim.x * U) {
      double v[U][W];
      int s[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = r0 + u * blockDim.x;
        s[u] = r < n ? __ldg(in_slot + r) : n + 1;
#pragma unroll
        for (int cc = 0; cc < W; ++cc)
          v[u][cc] = (r < n && col0 + cc < count) ? __ldcs(b + (col0 + cc) * ldb + r) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        T t[W];
#pragma unroll
        for (int cc = 0; cc < W; ++cc) t[cc] = (T)v[u][cc];
        store_w<T, W>(Ys + (size_t)s[u] * W, t);
      }
    }
  }

  template <int W> __device__ __forceinline__ void prefetch(int64_t col0, int64_t count, int n) const {
    prefetch_columns<W>(b, ldb, col0, count, n);
  }

  // Prefetches the columns col0 .. col0 + W - 1 into L2 (one bulk prefetch per column and 64 KB).
  template <int W>
  __device__ __forceinline__ static void prefetch_columns(const double *b, int64_t ldb, int64_t col0, int64_t count,
                                                          int n) {
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const int64_t bytes = (int64_t)n * 8;
    const int chunks = (int)((bytes + 65535) / 65536);
    for (int i = lane; i < W * chunks; i += 32) {
      const int cc = i / chunks, ch = i % chunks;
      if (col0 + cc >= count) continue;
      const char *base = reinterpret_cast<const char *>(b + (col0 + cc) * ldb) + (int64_t)ch * 65536;
      const int64_t left = bytes - (int64_t)ch * 65536;
      // a bulk prefetch wants a 16-byte aligned start and a multiple of 16 bytes
      const uintptr_t a0 = reinterpret_cast<uintptr_t>(base);
      const uintptr_t lo = (a0 + 15) & ~(uintptr_t)15;
      const int64_t len = ((int64_t)(a0 + (left < 65536 ? left : 65536)) - (int64_t)lo) & ~(int64_t)15;
      if (len > 0)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((uint32_t)len) : "memory");
    }
  }

  template <class T, int W>
  __device__ __forceinline__ void store(int64_t col0, int64_t count, int n, const T *Ys) const {
    store_columns<T, W>(x, ldx, out_slot, col0, count, n, Ys);
  }

  template <class T, int W>
  __device__ __forceinline__ static void store_columns(double *__restrict__ x, int64_t ldx,
                                                       const int32_t *__restrict__ out_slot, int64_t col0,
                                                       int64_t count, int n, const T *Ys) {
#pragma unroll 4
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      T t[W];
      load_w<T, W>(Ys + (size_t)__ldg(out_slot + r) * W, t);
#pragma unroll
      for (int cc = 0; cc < W; ++cc)
        if (col0 + cc < count) __stcs(x + (col0 + cc) * ldx + r, (double)t[cc]);
    }
  }
};

// Right-hand sides e_plus - e_minus built on the device (ybus_cuda/src/kernels.cu:5-17: the
// reference zeroes an n x width block and scatters the pairs; here the tile's slots are zeroed in
// shared memory), solutions stored in natural order. With UPDATE, each column's rank-one
// Sherman-Morrison update of `base` replaces the plain store (ybus_cuda/src/kernels.cu:24-58):
// x = base + alpha y, w = inverse_weight - c'y, z = c'x / w, out = x + z y, every operation
// rounded on its own as the reference's kernel (built with --fmad=false) rounds it; w = 0 flags the
// column singular and stores x. `plus`/`minus` are natural rows (-1: none), as right-hand-side rows
// for the load and as solution rows for the update.
template <bool UPDATE> struct PairIO {
  static constexpr bool kRefine = false;
  const int32_t *__restrict__ plus;
  const int32_t *__restrict__ minus;
  double *__restrict__ out;
  int64_t ldo;
  const int32_t *__restrict__ in_slot;
  const int32_t *__restrict__ out_slot;
  const double *__restrict__ base;            // UPDATE: [n], natural order
  const double *__restrict__ alpha;           // UPDATE: [count]
  const double *__restrict__ inverse_weight;  // UPDATE: [count]
  int32_t *__restrict__ singular;             // UPDATE: [count]

  template <class T, int W>
  __device__ __forceinline__ void load(int64_t col0, int64_t count, int n, T *Ys) const {
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      T t[W];
#pragma unroll
      for (int cc = 0; cc < W; ++cc) t[cc] = T(0);
      store_w<T, W>(Ys + (size_t)r * W, t);
    }
    __syncthreads();
    if (threadIdx.x < W && col0 + threadIdx.x < count) {
      const int64_t col = col0 + threadIdx.x;
      const int p = __ldg(plus + col), m = __ldg(minus + col);
      if (p >= 0) Ys[(size_t)__ldg(in_slot + p) * W + threadIdx.x] = T(1);
      if (m >= 0) Ys[(size_t)__ldg(in_slot + m) * W + threadIdx.x] = T(-1);
    }
  }

  template <int W> __device__ __forceinline__ void prefetch(int64_t, int64_t, int) const {}

  template <class T, int W>
  __device__ __forceinline__ void store(int64_t col0, int64_t count, int n, const T *Ys) const {
    if constexpr (!UPDATE) {
      DenseIO::store_columns<T, W>(out, ldo, out_slot, col0, count, n, Ys);
    } else {
#pragma unroll 1
      for (int cc = 0; cc < W; ++cc) {
        const int64_t col = col0 + cc;
        if (col >= count) break;
        const int p = __ldg(plus + col), m = __ldg(minus + col);
        const double a = __ldg(alpha + col);
        double cy = 0.0, cx = 0.0;
        if (p >= 0) {
          const double yp = (double)Ys[(size_t)__ldg(out_slot + p) * W + cc];
          cy = __dadd_rn(cy, yp);
          cx = __dadd_rn(cx, __dadd_rn(__ldg(base + p), __dmul_rn(a, yp)));
        }
        if (m >= 0) {
          const double ym = (double)Ys[(size_t)__ldg(out_slot + m) * W + cc];
          cy = __dsub_rn(cy, ym);
          cx = __dsub_rn(cx, __dadd_rn(__ldg(base + m), __dmul_rn(a, ym)));
        }
        const double w = __dadd_rn(-cy, __ldg(inverse_weight + col));
        const bool sing = (w == 0.0);
        const double z = sing ? 0.0 : __ddiv_rn(cx, w);
        if (threadIdx.x == 0) singular[col] = sing ? 1 : 0;
        double *o = out + col * ldo;
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
          const double y = (double)Ys[(size_t)__ldg(out_slot + r) * W + cc];
          const double xr = __dadd_rn(__ldg(base + r), __dmul_rn(a, y));
          o[r] = sing ? xr : __dadd_rn(xr, __dmul_rn(z, y));
        }
      }
    }
  }
};

// Keeps the larger (value, row): the larger value, the smaller row on a tie, row -1 never winning
// (the rule of ybus_cuda/src/kernels.cu:78-128)
__device__ __forceinline__ void better_max(double &v, int &r, double v2, int r2) {
  if (r2 >= 0 && (v2 > v || (v2 == v && (r < 0 || r2 < r)))) v = v2, r = r2;
}

// The N-1 screening of many scenarios (ybus_powerflow/src/dc/gpu.rs:334-430, with one right-hand
// side per scenario instead of one base): a column is a scenario's injections p over the buses
// (the slack's ignored), solved to theta = B'^-1 p; the epilogue applies its case's rank-one
// outage update theta' = theta + z y (y = B'^-1 c for c = e_from - e_to of the outaged branch,
// z = c'theta / (1/b - c'y); singular when 1/b - c'y is 0, which leaves theta), computes every
// branch's flow b (theta'_from - theta'_to) (the outaged branch carries nothing) and reduces it to
// the column's largest |flow| * weight with its branch (the smaller on a tie) and whether any flow
// is not finite. Only those maxima leave the GPU.
struct OutageIO {
  static constexpr bool kRefine = false;
  const double *__restrict__ inj;  // n_bus x S, column-major
  int64_t ldi;
  int32_t n_bus;
  const int32_t *__restrict__ bus_slot;  // [n_bus] slot of the bus's unknown; n + 1 for the slack
  const int32_t *__restrict__ case_of;   // [S]
  const int32_t *__restrict__ c_plus, *__restrict__ c_minus;  // per case: solution slots (n: none)
  const double *__restrict__ c_invb, *__restrict__ c_cy;      // per case: 1/b and c'y
  const int32_t *__restrict__ c_branch;                        // per case: the outaged branch
  const double *__restrict__ Y;                                // n x C, natural unknown order
  int64_t ldy;
  int32_t n_branch;
  const int32_t *__restrict__ br_slot_f, *__restrict__ br_slot_t;  // solution slots (n: slack)
  const int32_t *__restrict__ br_u_f, *__restrict__ br_u_t;        // unknowns (-1: slack)
  const double *__restrict__ br_b, *__restrict__ weight;
  int64_t *__restrict__ out_row;
  double *__restrict__ out_value;
  int32_t *__restrict__ out_bad;  // per column: 1 a flow not finite, 2 an angle not finite or above 1e5
  int32_t *__restrict__ case_singular;

  template <class T, int W>
  __device__ __forceinline__ void load(int64_t col0, int64_t count, int n, T *Ys) const {
    for (int r = threadIdx.x; r < n_bus; r += blockDim.x) {
      T t[W];
#pragma unroll
      for (int cc = 0; cc < W; ++cc) t[cc] = col0 + cc < count ? (T)__ldcs(inj + (col0 + cc) * ldi + r) : T(0);
      store_w<T, W>(Ys + (size_t)__ldg(bus_slot + r) * W, t);
    }
  }

  template <int W> __device__ __forceinline__ void prefetch(int64_t, int64_t, int) const {}

  template <class T, int W>
  __device__ __forceinline__ void store(int64_t col0, int64_t count, int n, const T *Ys) const {
    __shared__ double red_v[16];
    __shared__ int red_r[16], red_b[16];
#pragma unroll 1
    for (int cc = 0; cc < W; ++cc) {
      const int64_t col = col0 + cc;
      if (col >= count) break;
      const int c = __ldg(case_of + col);
      const double *y = Y + (int64_t)c * ldy;
      const double cx = __dsub_rn(__dadd_rn(0.0, (double)Ys[(size_t)__ldg(c_plus + c) * W + cc]),
                                  (double)Ys[(size_t)__ldg(c_minus + c) * W + cc]);
      const double w = __dadd_rn(-__ldg(c_cy + c), __ldg(c_invb + c));
      const bool sing = (w == 0.0);
      const double z = sing ? 0.0 : __ddiv_rn(cx, w);
      const int k = __ldg(c_branch + c);
      double v = 0.0;
      int row = -1, bad = 0;
      for (int l = threadIdx.x; l < n_branch; l += blockDim.x) {
        const int uf = __ldg(br_u_f + l), ut = __ldg(br_u_t + l);
        const double tf = uf < 0 ? 0.0 : __dadd_rn((double)Ys[(size_t)__ldg(br_slot_f + l) * W + cc], __dmul_rn(z, __ldg(y + uf)));
        const double tt = ut < 0 ? 0.0 : __dadd_rn((double)Ys[(size_t)__ldg(br_slot_t + l) * W + cc], __dmul_rn(z, __ldg(y + ut)));
        // an angle not finite or above 1e5 in magnitude (every unknown is some branch's end)
        if ((uf >= 0 && !(fabs(tf) <= 1e5)) || (ut >= 0 && !(fabs(tt) <= 1e5))) bad |= 2;
        const double b = __ldg(br_b + l);
        const double f = l == k ? 0.0 : __dadd_rn(__dmul_rn(b, tf), __dmul_rn(-b, tt));
        if (!isfinite(f)) {
          bad |= 1;
          continue;
        }
        const double load = fabs(f) * __ldg(weight + l);
        if (load > v) v = load, row = l;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, v, off);
        const int r2 = __shfl_xor_sync(0xffffffffu, row, off);
        bad |= __shfl_xor_sync(0xffffffffu, bad, off);
        better_max(v, row, v2, r2);
      }
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      if (lane == 0) red_v[warp] = v, red_r[warp] = row, red_b[warp] = bad;
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int w2 = 1; w2 < (int)(blockDim.x >> 5); ++w2) {
          better_max(v, row, red_v[w2], red_r[w2]);
          bad |= red_b[w2];
        }
        out_row[col] = row;
        out_value[col] = row >= 0 ? v : 0.0;
        out_bad[col] = bad;
        case_singular[c] = sing ? 1 : 0;
      }
      __syncthreads();
    }
  }
};

// Right-hand sides given over the buses (column-major, n_bus rows; bus_slot maps each bus to its
// unknown's slot, the slack to the spare slot n + 1, so its entry is ignored), solutions stored over
// the unknowns in natural order.
struct BusIO {
  static constexpr bool kRefine = false;
  const double *__restrict__ b;
  int64_t ldb;
  int32_t n_bus;
  const int32_t *__restrict__ bus_slot;
  double *__restrict__ x;
  int64_t ldx;
  const int32_t *__restrict__ out_slot;

  template <class T, int W>
  __device__ __forceinline__ void load(int64_t col0, int64_t count, int n, T *Ys) const {
    DenseIO::load_columns<T, W>(b, ldb, bus_slot, col0, count, n_bus, Ys);
  }
  template <int W> __device__ __forceinline__ void prefetch(int64_t col0, int64_t count, int n) const {}
  template <class T, int W>
  __device__ __forceinline__ void store(int64_t col0, int64_t count, int n, const T *Ys) const {
    DenseIO::store_columns<T, W>(x, ldx, out_slot, col0, count, n, Ys);
  }
};

// The adjoint solve's right-hand sides built in the load: q = Bf' g for each column of g (branch
// by scenario), Bf' given as each unknown's incident branches with their signed susceptances
// (inc_ptr over unknowns), summed in that order; solutions stored over the unknowns.
struct AdjointIO {
  static constexpr bool kRefine = false;
  const double *__restrict__ g;  // n_branch x count
  int64_t ldg;
  const int32_t *__restrict__ inc_ptr;  // [n + 1]
  const int32_t *__restrict__ inc_branch;
  const double *__restrict__ inc_value;
  const int32_t *__restrict__ in_slot;
  double *__restrict__ x;
  int64_t ldx;
  const int32_t *__restrict__ out_slot;

  template <class T, int W>
  __device__ __forceinline__ void load(int64_t col0, int64_t count, int n, T *Ys) const {
    for (int u = threadIdx.x; u < n; u += blockDim.x) {
      double q[W];
#pragma unroll
      for (int cc = 0; cc < W; ++cc) q[cc] = 0.0;
      const int p1 = __ldg(inc_ptr + u + 1);
      for (int p = __ldg(inc_ptr + u); p < p1; ++p) {
        const int l = __ldg(inc_branch + p);
        const double v = __ldg(inc_value + p);
#pragma unroll
        for (int cc = 0; cc < W; ++cc)
          if (col0 + cc < count) q[cc] = __dadd_rn(q[cc], __dmul_rn(v, __ldg(g + (col0 + cc) * ldg + l)));
      }
      T t[W];
#pragma unroll
      for (int cc = 0; cc < W; ++cc) t[cc] = (T)q[cc];
      store_w<T, W>(Ys + (size_t)__ldg(in_slot + u) * W, t);
    }
  }
  template <int W> __device__ __forceinline__ void prefetch(int64_t, int64_t, int) const {}
  template <class T, int W>
  __device__ __forceinline__ void store(int64_t col0, int64_t count, int n, const T *Ys) const {
    DenseIO::store_columns<T, W>(x, ldx, out_slot, col0, count, n, Ys);
  }
};

// Iterative refinement (ybus_sparse's `refine_normwise`, accuracy.rs:83-122): the substitutions in
// the precision of the tile (FP32); the residual and the update x += d in FP64 against the FP64
// matrix A. Pass 0 loads b into the slots and into the block's FP64 residual scratch R (natural row
// order, the W values of a row together). After each solve, `update` adds the solve's result d to
// x (x = d the first time) and updates R -= A d, both row by row in natural order, with A's
// columns mapped to solution slots so d is gathered from shared memory; then R goes into the slots
// for the next solve. R is updated rather than recomputed from x, so it is the residual of x up to
// rounding of the order of eps ||A|| ||x||. The tile is done when every column's relative residual
// ||r||inf / ||b||inf is at most the tolerance, after `max_steps` corrections, or when no column
// above the tolerance at least halved its residual in the last step (stagnation). Each column follows
// the CPU's refine_normwise (accuracy.rs:93-118) on its own: it stops within the tolerance, on a NaN
// ratio, when its ratio did not halve, or after max_steps; a column that has stopped is no longer
// updated; and a column that stops on a correction that made it no better gets its previous iterate
// back (kept for every column while it refines), so the x returned, the ratio and the corrections
// reported are the best iterate's. The tile is done when its last column stops.
struct RefineIO {
  static constexpr bool kRefine = true;
  const double *__restrict__ b;
  int64_t ldb;
  double *x;  // written and re-read within the launch: no read-only or streaming loads
  int64_t ldx;
  const int32_t *__restrict__ in_slot;
  const int32_t *__restrict__ out_slot;
  // A's rows in natural order, 32 rows to a slice (sliced ELL): slice g's entry q of row 32g + l
  // at a_ptr[g] + 32 q + l, with a_ptr[g + 1] - a_ptr[g] = 32 times the slice's longest row;
  // columns mapped to solution slots, padding pointing at the always-zero slot n with value 0
  const int32_t *__restrict__ a_ptr;  // [slices + 1]
  const int32_t *__restrict__ a_idx;
  const double *__restrict__ a_val;
  double *scratch;  // 2 gridDim.x blocks of n * W doubles: each block's R, then each block's previous x
  int32_t max_steps;
  double tolerance;
  double *__restrict__ ratio_out;  // [count] or null
  int32_t *__restrict__ steps_out;  // [count] or null

  template <int W> __device__ __forceinline__ double *residual(int n) const {
    return scratch + (size_t)blockIdx.x * n * W;
  }
  template <int W> __device__ __forceinline__ double *previous(int n) const {
    return scratch + ((size_t)gridDim.x + blockIdx.x) * n * W;
  }

  // x of the columns in `mask` back to the previous iterate (the columns a last correction made no
  // better), every thread of the block over the rows
  template <int W> __device__ __forceinline__ void restore(uint32_t mask, int64_t col0, int n) const {
    const double *P = previous<W>(n);
    for (int r = threadIdx.x; r < n; r += blockDim.x)
#pragma unroll
      for (int cc = 0; cc < W; ++cc)
        if ((mask >> cc) & 1u) x[(col0 + cc) * ldx + r] = P[(size_t)r * W + cc];
  }

  // b into the slots and into R, and ||b||inf of each column into bnorm (for all threads)
  template <class T, int W>
  __device__ __forceinline__ void load_b(int64_t col0, int64_t count, int n, T *Ys, double (&bnorm)[W]) const {
    constexpr int U = W >= 8 ? 1 : 4;  // rows in flight per thread
    __shared__ double red[32][W];
    double *R = residual<W>(n);
    double local[W];
#pragma unroll
    for (int cc = 0; cc < W; ++cc) local[cc] = 0.0;
#pragma unroll 1
    for (int r0 = threadIdx.x; r0 < n; r0 += blockDim.x * U) {
      double v[U][W];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = r0 + u * blockDim.x;
#pragma unroll
        for (int cc = 0; cc < W; ++cc) v[u][cc] = (r < n && col0 + cc < count) ? b[(col0 + cc) * ldb + r] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = r0 + u * blockDim.x;
        if (r >= n) break;
        T t[W];
#pragma unroll
        for (int cc = 0; cc < W; ++cc) {
          local[cc] = fmax(local[cc], fabs(v[u][cc]));
          t[cc] = (T)v[u][cc];
          R[(size_t)r * W + cc] = v[u][cc];
        }
        store_w<T, W>(Ys + (size_t)__ldg(in_slot + r) * W, t);
      }
    }
    block_max<W>(local, red, bnorm);
  }

  // x (first) or x += d from the slots for the columns still refining (`active`), the x before
  // kept; R -= A d; ||R||inf per column into rnorm; R into the slots
  template <class T, int W>
  __device__ __forceinline__ void update(bool first, uint32_t active, int64_t col0, int64_t count, int n, T *Ys,
                                         double (&rnorm)[W]) const {
    constexpr int U = W >= 8 ? 1 : 4;  // rows in flight per thread
    __shared__ double red[32][W];
    double *R = residual<W>(n);
    double *P = previous<W>(n);
    double local[W];
#pragma unroll
    for (int cc = 0; cc < W; ++cc) local[cc] = 0.0;
#pragma unroll 1
    for (int r0 = threadIdx.x; r0 < n; r0 += blockDim.x * U) {
      double acc[U][W], xo[U][W];
      int p0[U], p1[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = r0 + u * blockDim.x;
        const bool in = r < n;
        p0[u] = in ? __ldg(a_ptr + (r >> 5)) + (r & 31) : 0;
        p1[u] = in ? __ldg(a_ptr + (r >> 5) + 1) : 0;
#pragma unroll
        for (int cc = 0; cc < W; ++cc) {
          acc[u][cc] = in ? R[(size_t)r * W + cc] : 0.0;
          xo[u][cc] = (in && !first && col0 + cc < count) ? x[(col0 + cc) * ldx + r] : 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = r0 + u * blockDim.x;
        if (r >= n) break;
        T d[W];
        load_w<T, W>(Ys + (size_t)__ldg(out_slot + r) * W, d);
#pragma unroll
        for (int cc = 0; cc < W; ++cc)
          if (col0 + cc < count && ((active >> cc) & 1u)) {
            if (!first) P[(size_t)r * W + cc] = xo[u][cc];
            x[(col0 + cc) * ldx + r] = xo[u][cc] + (double)d[cc];
          }
        int p = p0[u];
#pragma unroll 1
        for (; p + 96 < p1[u]; p += 128) {  // four entries of the row at a time, their loads together
          int j[4];
          double v[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) j[e] = __ldg(a_idx + p + 32 * e), v[e] = __ldg(a_val + p + 32 * e);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            T y[W];
            load_w<T, W>(Ys + (size_t)j[e] * W, y);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[u][cc] -= v[e] * (double)y[cc];
          }
        }
        for (; p < p1[u]; p += 32) {
          const double v = __ldg(a_val + p);
          T y[W];
          load_w<T, W>(Ys + (size_t)__ldg(a_idx + p) * W, y);
#pragma unroll
          for (int cc = 0; cc < W; ++cc) acc[u][cc] -= v * (double)y[cc];
        }
#pragma unroll
        for (int cc = 0; cc < W; ++cc) {
          if (col0 + cc >= count) acc[u][cc] = 0.0;
          R[(size_t)r * W + cc] = acc[u][cc];
          local[cc] = fmax(local[cc], fabs(acc[u][cc]));
        }
      }
    }
    block_max<W>(local, red, rnorm);  // every gather of d is done past its barrier
#pragma unroll 1
    for (int r0 = threadIdx.x; r0 < n; r0 += blockDim.x * U) {
      double v[U][W];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = r0 + u * blockDim.x;
#pragma unroll
        for (int cc = 0; cc < W; ++cc) v[u][cc] = r < n ? R[(size_t)r * W + cc] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int r = r0 + u * blockDim.x;
        if (r >= n) break;
        T t[W];
#pragma unroll
        for (int cc = 0; cc < W; ++cc) t[cc] = (T)v[u][cc];
        store_w<T, W>(Ys + (size_t)__ldg(in_slot + r) * W, t);
      }
    }
    __syncthreads();
  }

  // The largest of every thread's values, per column, returned to all threads (NaN propagates).
  template <int W>
  __device__ __forceinline__ static void block_max(const double (&local)[W], double (&red)[32][W], double (&out)[W]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
#pragma unroll
    for (int cc = 0; cc < W; ++cc) {
      double v = local[cc];
      bool nan = v != v;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, off);
        nan = nan || (u != u);
        v = fmax(v, u);
      }
      if (lane == 0) red[warp][cc] = nan ? __longlong_as_double(0x7ff8000000000000LL) : v;
    }
    __syncthreads();
#pragma unroll
    for (int cc = 0; cc < W; ++cc) {
      double v = 0.0;
      bool nan = false;
      for (int w = 0; w < warps; ++w) {
        nan = nan || (red[w][cc] != red[w][cc]);
        v = fmax(v, red[w][cc]);
      }
      out[cc] = nan ? __longlong_as_double(0x7ff8000000000000LL) : v;
    }
    __syncthreads();
  }

  template <int W> __device__ __forceinline__ void prefetch(int64_t col0, int64_t count, int n) const {
    DenseIO::prefetch_columns<W>(b, ldb, col0, count, n);
  }
};

template <class T, int W, class IO>
__global__ void __launch_bounds__(512, 1) domain_tile_kernel(DomainArgs a, IO io) {
  static_assert(32 % W == 0, "W divides a warp");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int n = a.n;
  // the warp index through a shuffle from lane 0, so the compiler keeps what derives from it (the
  // warp's ring, its pages, the record headers) on the uniform datapath
  const int lane = threadIdx.x & 31, warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0),
            warps = blockDim.x >> 5;
  const int S = a.ring, PB = a.page_bytes;
  const int m = a.tail;
  const size_t y_bytes = (((size_t)(n + 2) * W * sizeof(T)) + 127) & ~(size_t)127;
  const size_t tb_bytes = (((size_t)(m + 1) * W * sizeof(T)) + 15) & ~(size_t)15;
  const size_t ts_bytes = (((size_t)(m + 1) * 4) + 127) & ~(size_t)127;
  T *Ys = reinterpret_cast<T *>(smem_raw);
  T *Tb = reinterpret_cast<T *>(smem_raw + y_bytes);
  int32_t *tslot = reinterpret_cast<int32_t *>(smem_raw + y_bytes + tb_bytes);
  uint8_t *ring = smem_raw + y_bytes + tb_bytes + ts_bytes + (size_t)warp * S * PB;
  uint64_t *full =
      reinterpret_cast<uint64_t *>(smem_raw + y_bytes + tb_bytes + ts_bytes + (size_t)warps * S * PB) + warp * S;

  // slot n is always zero (the target of padded split entries); slot n + 1 takes the load's spare writes
  if (threadIdx.x < 2 * W) Ys[n * W + threadIdx.x] = T(0);
  for (int t = threadIdx.x; t <= m; t += blockDim.x) tslot[t] = t < m ? __ldg(a.tail_slot + t) : n;
  if (lane == 0)
    for (int s = 0; s < S; ++s) mbar_init(full + s, 1);
  mbar_fence_init();
  __syncthreads();

  const int p0 = __ldg(a.warp_page + warp), np = __ldg(a.warp_page + warp + 1) - p0;
  const int64_t my_tiles = blockIdx.x < a.tiles ? (a.tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // The warp's stream is taken once per solve pass, np pages each, cyclically: page k of the run
  // is stream page k % np and lands in ring slot k % S. A refined solve takes a data-dependent
  // number of passes, so copies run S pages ahead of use and the last S are drained at the end.
  const bool streaming = np > 0 && my_tiles > 0;
  int slot_next = 0, page_next = 0;
  int64_t issued = 0, consumed = 0;
  auto issue_one = [&]() {
    fence_proxy_async();
    bulk_page(ring + (size_t)slot_next * PB, a.blob + (size_t)(p0 + page_next) * PB, (uint32_t)PB, full + slot_next);
    ++issued;
    if (++slot_next == S) slot_next = 0;
    if (++page_next == np) page_next = 0;
  };
  if (lane == 0 && streaming)
    for (int s = 0; s < S; ++s) issue_one();
  __syncwarp();

  int slot_cur = 0;
  uint32_t parity = 0;
  for (int64_t tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
    const int64_t col0 = tile * W;
    const int64_t it = (tile - blockIdx.x) / gridDim.x;
    // per column (the same in every thread): ||b||inf, the current and the best relative residual,
    // the best's corrections, and which columns still refine
    double bnorm[W], cur[W], best[W];
    int best_steps[W];
    uint32_t active = 0;
#pragma unroll
    for (int cc = 0; cc < W; ++cc) {
      bnorm[cc] = 0.0, cur[cc] = best[cc] = __longlong_as_double(0x7ff0000000000000LL), best_steps[cc] = 0;
      if (col0 + cc < a.count) active |= 1u << cc;
    }
    for (int pass = 0;; ++pass) {
    // diagnostics rows: the first 4 tiles, or for a refined solve the first 4 passes of tile 0
    const int64_t mark = IO::kRefine ? (it == 0 ? pass : 4) : it;
    long long *pc =
        (a.phase_clock && blockIdx.x == 0 && mark < 4 && lane == 0) ? a.phase_clock + (mark * 16 + warp) * 8 : nullptr;
    if (pc) pc[0] = clock64();
    if (pass == 0) {
      if constexpr (IO::kRefine)
        io.template load_b<T, W>(col0, a.count, n, Ys, bnorm);
      else
        io.template load<T, W>(col0, a.count, n, Ys);
    }
    if (pass == 0 && tile + gridDim.x < a.tiles) io.template prefetch<W>((tile + gridDim.x) * W, a.count, n);
    __syncthreads();
    if (pc) pc[1] = clock64();
    long long wait_cycles = 0, barrier_cycles = 0, pages_seen = 0, records_seen = 0;

    int done = 0;
    T acc[W];  // a split row's or a dense row's running sums, kept across its chunks
#pragma unroll
    for (int cc = 0; cc < W; ++cc) acc[cc] = T(0);
    for (int j = 0; j < np; ++j) {
      const long long w0 = pc ? clock64() : 0;
      const bool ready = mbar_wait_bounded(full + slot_cur, parity, a.error);
      if (pc) wait_cycles += clock64() - w0, ++pages_seen;
      const uint8_t *page = ring + (size_t)slot_cur * PB;
      int pos = ready ? 0 : PB;  // a page that never arrived is skipped
      while (pos + 16 <= PB) {
        const int4 hdr = *reinterpret_cast<const int4 *>(page + pos);
        const int kind = hdr.x, flags = hdr.w;
        if (kind < 0) break;
        const int stage = min(hdr.y, a.stages);
        if (done < stage) {
          const long long b0 = pc ? clock64() : 0;
          while (done < stage) {
            __syncthreads();
            ++done;
          }
          if (pc) barrier_cycles += clock64() - b0;
        }
        if (pc) ++records_seen;
        if (kind == kRecordRows) {
          // k = 2^kl lanes per row: each lane sums its share of the row's entries (two sums for
          // ILP), the k lanes reduce, and the row's first lane finishes the row
          const int4 h2 = *reinterpret_cast<const int4 *>(page + pos + 16);
          const int4 h3 = *reinterpret_cast<const int4 *>(page + pos + 32);
          const int rows = hdr.z, kl = h2.x, k = 1 << kl;
          const uint8_t *rec = page + pos;
          const int r = lane >> kl, sub = lane & (k - 1);
          const uint16_t *cols = reinterpret_cast<const uint16_t *>(rec + h3.z);
          const T *vals = reinterpret_cast<const T *>(rec + h3.w);
          int slot = 0, dest = 0, len = 0, start = 0;
          if (r < rows) {
            const int2 in = reinterpret_cast<const int2 *>(rec + h3.x)[r];
            slot = in.x & 0xffff, len = (int)((unsigned)in.x >> 16);
            start = in.y & 0xffff, dest = (int)((unsigned)in.y >> 16);
          }
          T s0[W], s1[W];
#pragma unroll
          for (int cc = 0; cc < W; ++cc) s0[cc] = T(0), s1[cc] = T(0);
          int q = sub;
          for (; q + k < len; q += 2 * k) {
            const int c0 = cols[start + q], c1 = cols[start + q + k];
            const T v0 = vals[start + q], v1 = vals[start + q + k];
            T y0[W], y1[W];
            load_w<T, W>(Ys + c0 * W, y0);
            load_w<T, W>(Ys + c1 * W, y1);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) s0[cc] += v0 * y0[cc], s1[cc] += v1 * y1[cc];
          }
          if (q < len) {
            const int c0 = cols[start + q];
            const T v0 = vals[start + q];
            T y0[W];
            load_w<T, W>(Ys + c0 * W, y0);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) s0[cc] += v0 * y0[cc];
          }
#pragma unroll
          for (int cc = 0; cc < W; ++cc) s0[cc] += s1[cc];
          for (int off = k >> 1; off > 0; off >>= 1)
#pragma unroll
            for (int cc = 0; cc < W; ++cc) s0[cc] += __shfl_xor_sync(0xffffffffu, s0[cc], off);
          if (r < rows && sub == 0) {
            T y[W];
            load_w<T, W>(Ys + slot * W, y);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) y[cc] -= s0[cc];
            if (flags & kRecordToTail) {
              store_w<T, W>(Tb + dest * W, y);
            } else {
              const T d = reinterpret_cast<const T *>(rec + h3.y)[r];
#pragma unroll
              for (int cc = 0; cc < W; ++cc) y[cc] *= d;
              store_w<T, W>(Ys + dest * W, y);
            }
          }
          pos += h2.z;
        } else if (kind == kRecordDense) {
          // a chunk of a dense inverse row: lanes split the columns, each lane keeps W sums
          const int len = hdr.z;
          const int t = *reinterpret_cast<const int32_t *>(page + pos + 16);
          const int j0 = *reinterpret_cast<const int32_t *>(page + pos + 20);
          const T *val = reinterpret_cast<const T *>(page + pos + 32);
          if (flags & kRecordFirst)
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] = T(0);
          for (int e = lane; e < len; e += 32) {
            const T v = val[e];
            T y[W];
            load_w<T, W>(Tb + (size_t)(j0 + e) * W, y);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] += v * y[cc];
          }
          if (flags & kRecordLast) {
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
              T v = acc[cc];
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
              if (lane == cc) Ys[(size_t)tslot[t] * W + cc] = v;
            }
          }
          pos += 32 + (int)(((int64_t)sizeof(T) * len + 15) & ~int64_t(15));
        } else if (kind == kRecordCopy) {
          // this warp's share of the top rows' slots into the tail buffer
          for (int idx = warp * 32 + lane; idx < m * W; idx += warps * 32)
            Tb[idx] = Ys[(size_t)tslot[idx / W] * W + idx % W];
          pos += 16;
        } else if (kind == kRecordSplit) {
          // one long row over the lanes: each lane's share of the entries, then a reduction
          const int len = hdr.z;
          const int row = *reinterpret_cast<const int32_t *>(page + pos + 16);
          const int dest = *reinterpret_cast<const int32_t *>(page + pos + 20);
          const T dinv = *reinterpret_cast<const T *>(page + pos + 32);
          const int32_t *col = reinterpret_cast<const int32_t *>(page + pos + 48);
          const int col_bytes = (4 * len + 15) & ~15;
          const T *val = reinterpret_cast<const T *>(page + pos + 48 + col_bytes);
          if (flags & kRecordFirst)
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] = T(0);
          for (int e = lane; e < len; e += 32) {
            const T v = val[e];
            T y[W];
            load_w<T, W>(Ys + (size_t)col[e] * W, y);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] += v * y[cc];
          }
          if (flags & kRecordLast) {
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
              T v = acc[cc];
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
              if (lane == cc) {
                if (flags & kRecordToTail)
                  Tb[(size_t)dest * W + cc] = Ys[(size_t)row * W + cc] - v;
                else
                  Ys[(size_t)row * W + cc] = (Ys[(size_t)row * W + cc] - v) * dinv;
              }
            }
          }
          pos += 48 + col_bytes + (int)(((int64_t)sizeof(T) * len + 15) & ~int64_t(15));
        } else {
          atomicExch(a.error, 2);  // an unknown record: stop reading this page
          break;
        }
        __syncwarp();
      }
      __syncwarp();
      ++consumed;
      if (lane == 0) issue_one();
      if (++slot_cur == S) slot_cur = 0, parity ^= 1u;
    }
    if (pc) pc[2] = clock64(), pc[4] = wait_cycles, pc[6] = pages_seen, pc[7] = records_seen;
    {
      const long long b0 = pc ? clock64() : 0;
      while (done < a.stages) {
        __syncthreads();
        ++done;
      }
      if (pc) pc[5] = barrier_cycles + (clock64() - b0);
    }
    if constexpr (IO::kRefine) {
      double rnorm[W];
      io.template update<T, W>(pass == 0, active, col0, a.count, n, Ys, rnorm);
      if (pc) pc[3] = clock64();
      // each refining column's relative residual after `pass` corrections (accuracy.rs:58-79) and
      // refine_normwise's decision for it (accuracy.rs:93-118)
      uint32_t restore = 0;
#pragma unroll
      for (int cc = 0; cc < W; ++cc) {
        if (!((active >> cc) & 1u)) continue;
        const double ratio = bnorm[cc] > 0.0 ? rnorm[cc] / bnorm[cc]
                                             : (rnorm[cc] > 0.0 ? __longlong_as_double(0x7ff0000000000000LL) : 0.0);
        bool stop;
        if (pass == 0) {
          best[cc] = cur[cc] = ratio;
          stop = ratio <= io.tolerance || io.max_steps < 1;
        } else {
          const double previous = cur[cc];
          cur[cc] = ratio;
          const bool improved = ratio < best[cc];
          if (improved) best[cc] = ratio, best_steps[cc] = pass;
          stop = ratio != ratio || ratio > 0.5 * previous || ratio <= io.tolerance || pass >= io.max_steps;
          if (stop && !improved && best_steps[cc] == pass - 1) restore |= 1u << cc;
        }
        if (stop) {
          active &= ~(1u << cc);
          if (threadIdx.x == cc) {
            if (io.ratio_out) io.ratio_out[col0 + cc] = best[cc];
            if (io.steps_out) io.steps_out[col0 + cc] = best_steps[cc];
          }
        }
      }
      if (restore) io.template restore<W>(restore, col0, n);
      if (!active) {
        __syncthreads();  // the restore's reads of the previous iterate, before the next tile
        break;
      }
    } else {
      io.template store<T, W>(col0, a.count, n, Ys);
      __syncthreads();
      if (pc) pc[3] = clock64();
      break;
    }
    }
  }
  // Every copy issued but not consumed (the S run ahead, or more after a wait that ran out) is
  // waited for, bounded, before the block's shared memory is released
  if (lane == 0 && streaming) {
    for (int64_t kk = consumed; kk < issued; ++kk) mbar_wait_bounded(full + (kk % S), (uint32_t)((kk / S) & 1), nullptr);
  }
}

}  // namespace yb
