// The level-scheduled tile solve: one thread block solves a tile of W right-hand sides through
// both sweeps of a factor, then takes the next tile (a persistent grid of blocks).
//
// Work layout inside a block. A tile's working vector Y lives in the block's own slice of a
// scratch buffer, as [slot][W] (the W right-hand sides of a slot contiguous, so each row read is
// one coalesced W*sizeof(T)-byte access). W lanes of a warp share one row: lane c owns
// right-hand side c, reading the row's factor entries as a broadcast and the rows it depends on
// from Y. Rows of one level are independent and spread over all the block's lane groups; a
// __syncthreads separates levels. The scratch slice is reused for every tile the block takes,
// so it stays resident in L2 and only b (read once, coalesced) and x (written once, coalesced)
// move through HBM.
//
// The permutations are folded into the prologue (Y[in_slot[r]] = b[r]) and epilogue
// (x[r] = Y[out_slot[r]]): reads of b and writes of x run along each column in its natural
// order and the scattered side of each copy hits the L2-resident tile.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"

namespace yb {

// How a tile's right-hand sides are formed.
enum class Load : int {
  Dense = 0,  // columns of b (double, column-major, natural row order)
  Pairs = 1,  // e_plus - e_minus per column (ybus_cuda/src/kernels.cu:5-17)
};

// What a tile's solutions become.
enum class Store : int {
  Dense = 0,       // columns of x (double, column-major, natural row order)
  PairUpdate = 1,  // the rank-one update of a base solution per column (ybus_cuda/src/kernels.cu:24-58)
};

template <class T> struct TileArgs {
  int32_t n;
  int64_t count;  // right-hand sides
  int64_t tiles;  // ceil(count / W)
  const double *__restrict__ b;  // Load::Dense
  int64_t ldb;                   // column stride of b
  double *__restrict__ x;
  int64_t ldx;
  const int32_t *__restrict__ plus;   // Load::Pairs, natural row or -1
  const int32_t *__restrict__ minus;
  const double *__restrict__ base;    // Store::PairUpdate, natural order
  const double *__restrict__ alpha;
  const double *__restrict__ inverse_weight;
  int32_t *__restrict__ singular;
  const int32_t *__restrict__ in_slot;
  const int32_t *__restrict__ out_slot;
  T *scratch;  // gridDim.x slices of n * W
  SweepView<T> fwd, bwd;
};

// One sweep over the tile in Y. Each lane group of W lanes takes rows of a level in turn.
template <class T, int W>
__device__ __forceinline__ void sweep_tile(const SweepView<T> &s, T *Y, int group, int groups, int c) {
  for (int l = 0; l < s.levels; ++l) {
    const int k0 = __ldg(s.level_ptr + l), k1 = __ldg(s.level_ptr + l + 1);
    int k = k0 + group;
    // Two rows per lane group per pass, so the loads of both are in flight together
    for (; k + groups < k1; k += 2 * groups) {
      const int ka = k, kb = k + groups;
      const int ra = __ldg(s.row + ka), rb = __ldg(s.row + kb);
      const int pa0 = __ldg(s.ptr + ka), pa1 = __ldg(s.ptr + ka + 1);
      const int pb0 = __ldg(s.ptr + kb), pb1 = __ldg(s.ptr + kb + 1);
      T acc_a = Y[(size_t)ra * W + c];
      T acc_b = Y[(size_t)rb * W + c];
      const int la = pa1 - pa0, lb = pb1 - pb0;
      const int common = la < lb ? la : lb;
      for (int q = 0; q < common; ++q) {
        const T va = __ldg(s.val + pa0 + q), vb = __ldg(s.val + pb0 + q);
        const int ja = __ldg(s.col + pa0 + q), jb = __ldg(s.col + pb0 + q);
        acc_a -= va * Y[(size_t)ja * W + c];
        acc_b -= vb * Y[(size_t)jb * W + c];
      }
      for (int q = common; q < la; ++q) acc_a -= __ldg(s.val + pa0 + q) * Y[(size_t)__ldg(s.col + pa0 + q) * W + c];
      for (int q = common; q < lb; ++q) acc_b -= __ldg(s.val + pb0 + q) * Y[(size_t)__ldg(s.col + pb0 + q) * W + c];
      Y[(size_t)ra * W + c] = acc_a * __ldg(s.dinv + ka);
      Y[(size_t)rb * W + c] = acc_b * __ldg(s.dinv + kb);
    }
    if (k < k1) {
      const int r = __ldg(s.row + k);
      const int p0 = __ldg(s.ptr + k), p1 = __ldg(s.ptr + k + 1);
      T acc = Y[(size_t)r * W + c];
#pragma unroll 4
      for (int p = p0; p < p1; ++p) acc -= __ldg(s.val + p) * Y[(size_t)__ldg(s.col + p) * W + c];
      Y[(size_t)r * W + c] = acc * __ldg(s.dinv + k);
    }
    __syncthreads();
  }
}

template <class T, int W, Load LOAD, Store STORE>
__global__ void __launch_bounds__(512) tile_solve_kernel(TileArgs<T> a) {
  static_assert(W == 1 || W == 2 || W == 4 || W == 8 || W == 16 || W == 32, "W divides a warp");
  constexpr int G = 32 / W;
  const int lane = threadIdx.x & 31;
  const int c = lane % W;
  const int group = (threadIdx.x >> 5) * G + lane / W;
  const int groups = (blockDim.x >> 5) * G;
  const int n = a.n;
  T *Y = a.scratch + (size_t)blockIdx.x * n * W;

  for (int64_t tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
    const int64_t col0 = tile * W;
    // Prologue: the tile's right-hand sides into Y, permuted into slots
    if constexpr (LOAD == Load::Dense) {
      for (int cc = 0; cc < W; ++cc) {
        const int64_t col = col0 + cc;
        const double *bc = a.b + col * a.ldb;
        if (col < a.count) {
          for (int r = threadIdx.x; r < n; r += blockDim.x) Y[(size_t)__ldg(a.in_slot + r) * W + cc] = (T)__ldg(bc + r);
        } else {
          for (int r = threadIdx.x; r < n; r += blockDim.x) Y[(size_t)r * W + cc] = T(0);
        }
      }
    } else {
      for (int i = threadIdx.x; i < n * W; i += blockDim.x) Y[i] = T(0);
      __syncthreads();
      if (threadIdx.x < W) {
        const int64_t col = col0 + threadIdx.x;
        if (col < a.count) {
          const int p = a.plus[col], m = a.minus[col];
          if (p >= 0) Y[(size_t)__ldg(a.in_slot + p) * W + threadIdx.x] = T(1);
          if (m >= 0) Y[(size_t)__ldg(a.in_slot + m) * W + threadIdx.x] = T(-1);
        }
      }
    }
    __syncthreads();
    sweep_tile<T, W>(a.fwd, Y, group, groups, c);
    sweep_tile<T, W>(a.bwd, Y, group, groups, c);
    // Epilogue: solutions out of slots into natural order
    if constexpr (STORE == Store::Dense) {
      for (int cc = 0; cc < W; ++cc) {
        const int64_t col = col0 + cc;
        if (col >= a.count) break;
        double *xc = a.x + col * a.ldx;
        for (int r = threadIdx.x; r < n; r += blockDim.x) xc[r] = (double)Y[(size_t)__ldg(a.out_slot + r) * W + cc];
      }
    } else {
      // x = base + alpha y, w = inverse_weight - c'y, z = c'x / w, out = x + z y, each
      // operation rounded separately as the CPU's update rounds it
      for (int cc = 0; cc < W; ++cc) {
        const int64_t col = col0 + cc;
        if (col >= a.count) break;
        const int p = a.plus[col], m = a.minus[col];
        const double al = a.alpha[col];
        double cy = 0.0, cx = 0.0;
        if (p >= 0) {
          const double yp = (double)Y[(size_t)__ldg(a.out_slot + p) * W + cc];
          cy = __dadd_rn(cy, yp);
          cx = __dadd_rn(cx, __dadd_rn(a.base[p], __dmul_rn(al, yp)));
        }
        if (m >= 0) {
          const double ym = (double)Y[(size_t)__ldg(a.out_slot + m) * W + cc];
          cy = __dsub_rn(cy, ym);
          cx = __dsub_rn(cx, __dadd_rn(a.base[m], __dmul_rn(al, ym)));
        }
        const double w = __dadd_rn(-cy, a.inverse_weight[col]);
        const bool singular = (w == 0.0);
        const double z = singular ? 0.0 : cx / w;
        if (threadIdx.x == 0) a.singular[col] = singular ? 1 : 0;
        double *xc = a.x + col * a.ldx;
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
          const double y = (double)Y[(size_t)__ldg(a.out_slot + r) * W + cc];
          const double xr = __dadd_rn(a.base[r], __dmul_rn(al, y));
          xc[r] = singular ? xr : __dadd_rn(xr, __dmul_rn(z, y));
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace yb
