// The multi-network batched solve (no ybus counterpart: ybus_cuda solves one real factor at a
// time): many factors of uneven orders and right-hand-side counts in one persistent launch. A
// work list of (network, tile) items, largest networks first, is dealt round-robin to the blocks;
// a block solves its item's tile of W right-hand sides through both sweeps of that network's
// factor, level by level with a block barrier between levels, its working vector in the block's
// slice of an L2-resident scratch buffer sized for the largest network. Values are complex here
// (cplx<float> or cplx<double>), for admittance (Ybus) LU factors; right-hand sides and solutions
// are complex128, column-major, natural order, interleaved (re, im).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cplx.cuh"
#include "device.cuh"

namespace yb {

template <class T> struct BatchNet {
  int32_t n;
  SweepView<T> fwd, bwd;
  const int32_t *__restrict__ in_slot;
  const int32_t *__restrict__ out_slot;
  const cplx<double> *b;  // right-hand sides (or residuals), ldb per column
  int64_t ldb;
  cplx<double> *x;        // solutions, ldx per column
  int64_t ldx;
  int64_t count;
};

struct BatchItem {
  int32_t net, tile;
};

// One sweep of a network's tile: lane groups of W lanes take the rows of a level, lane c the
// right-hand side c; a block barrier after each level.
template <class T, int W>
__device__ __forceinline__ void batch_sweep(const SweepView<T> &s, T *Y, int group, int groups, int c) {
  for (int l = 0; l < s.levels; ++l) {
    const int k1 = s.level_ptr[l + 1];
    for (int k = s.level_ptr[l] + group; k < k1; k += groups) {
      const int r = s.row[k];
      const int p1 = s.ptr[k + 1];
      T acc = Y[(size_t)r * W + c];
      for (int p = s.ptr[k]; p < p1; ++p) acc -= s.val[p] * Y[(size_t)s.col[p] * W + c];
      Y[(size_t)r * W + c] = acc * s.dinv[k];
    }
    __syncthreads();
  }
}

// ACCUMULATE: x += the solution (a refinement step's correction) instead of x = the solution.
template <class T, int W, bool ACCUMULATE>
__global__ void __launch_bounds__(512) batch_solve_kernel(const BatchNet<T> *__restrict__ nets,
                                                          const BatchItem *__restrict__ items, int64_t n_items,
                                                          T *scratch, int64_t slice) {
  static_assert(32 % W == 0, "W divides a warp");
  constexpr int G = 32 / W;
  const int lane = threadIdx.x & 31;
  const int c = lane % W;
  const int group = (threadIdx.x >> 5) * G + lane / W;
  const int groups = (blockDim.x >> 5) * G;
  T *Y = scratch + (size_t)blockIdx.x * slice;
  for (int64_t i = blockIdx.x; i < n_items; i += gridDim.x) {
    const BatchItem item = items[i];
    const BatchNet<T> &net = nets[item.net];
    const int n = net.n;
    const int64_t col0 = (int64_t)item.tile * W;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const int sl = net.in_slot[r];
#pragma unroll
      for (int cc = 0; cc < W; ++cc) {
        const int64_t col = col0 + cc;
        Y[(size_t)sl * W + cc] = col < net.count ? T(net.b[col * net.ldb + r]) : T(0);
      }
    }
    __syncthreads();
    batch_sweep<T, W>(net.fwd, Y, group, groups, c);
    batch_sweep<T, W>(net.bwd, Y, group, groups, c);
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
      const int sl = net.out_slot[r];
#pragma unroll
      for (int cc = 0; cc < W; ++cc) {
        const int64_t col = col0 + cc;
        if (col < net.count) {
          const cplx<double> v(Y[(size_t)sl * W + cc]);
          cplx<double> *xp = net.x + col * net.ldx + r;
          if (ACCUMULATE)
            *xp = *xp + v;
          else
            *xp = v;
        }
      }
    }
    __syncthreads();
  }
}

// The residual r = b - A x of every column of every network (A CSR in natural order, complex128,
// each row's products summed in stored order) and each column's ||r||inf / ||b||inf
// (accuracy.rs:58-79: 0 for a zero residual, infinity for a zero b with a nonzero residual). One
// block of 256 threads per (network, column) in `columns`.
struct ResidualNet {
  int32_t n;
  const int32_t *__restrict__ a_ptr;
  const int32_t *__restrict__ a_idx;
  const cplx<double> *__restrict__ a_val;
  const cplx<double> *b;
  int64_t ldb;
  const cplx<double> *x;
  int64_t ldx;
  cplx<double> *r;
  int64_t ldr;
  double *ratio;  // per column of this network
};

__global__ void batch_residual_kernel(const ResidualNet *__restrict__ nets, const BatchItem *__restrict__ columns) {
  __shared__ double sr[8], sb[8];
  const BatchItem it = columns[blockIdx.x];
  const ResidualNet &net = nets[it.net];
  const int64_t col = it.tile;
  const cplx<double> *b = net.b + col * net.ldb;
  const cplx<double> *x = net.x + col * net.ldx;
  cplx<double> *r = net.r + col * net.ldr;
  double rn = 0.0, bn = 0.0;
  for (int i = threadIdx.x; i < net.n; i += blockDim.x) {
    cplx<double> ax(0.0);
    for (int p = net.a_ptr[i]; p < net.a_ptr[i + 1]; ++p) ax += net.a_val[p] * x[net.a_idx[p]];
    const cplx<double> ri = b[i] - ax;
    r[i] = ri;
    rn = fmax(rn, magnitude(ri));
    bn = fmax(bn, magnitude(b[i]));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    rn = fmax(rn, __shfl_xor_sync(0xffffffffu, rn, off));
    bn = fmax(bn, __shfl_xor_sync(0xffffffffu, bn, off));
  }
  if ((threadIdx.x & 31) == 0) sr[threadIdx.x >> 5] = rn, sb[threadIdx.x >> 5] = bn;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) rn = fmax(rn, sr[w]), bn = fmax(bn, sb[w]);
    net.ratio[col] = bn > 0.0 ? rn / bn : (rn > 0.0 ? __longlong_as_double(0x7ff0000000000000LL) : 0.0);
  }
}

}  // namespace yb
