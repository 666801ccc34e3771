// The shared-memory tile solve: one thread block holds a tile of W right-hand sides' whole
// working vector in shared memory and takes both sweeps through it, level by level.
//
//   shared memory: Ys[(n + 2) * W], slot-major (the W values of a slot contiguous); slot n is
//   always zero (the target of padded entries), slot n + 1 absorbs padded rows' writes.
//
// Each sweep is a list of slices (see SliceSweep in plan.hpp): G = 32 / W rows of one level,
// their entries stored entry-major. A warp takes a level's slices round-robin; lane (g, c) owns
// row g of the slice and right-hand side c. The warp prefetches the next slice's row, diagonal
// and first CH entries into registers while it computes the current one, and the first slice of
// the next level before the level barrier, so the factor's L2 latency overlaps the gathers.
// Gathers of Y are shared-memory loads. b is read and x written once per tile, along columns
// (coalesced), with the permutations applied on the shared-memory side.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"

namespace yb {

template <class T> struct SliceView {
  int32_t levels;
  const int32_t *__restrict__ level_slice;
  const int2 *__restrict__ span;  // {entry offset, padded length} per slice
  const int32_t *__restrict__ row;
  const T *__restrict__ dinv;
  const int32_t *__restrict__ col;
  const T *__restrict__ val;
};

template <class T> struct SmemArgs {
  int32_t n;
  int64_t count, tiles;
  const double *__restrict__ b;
  int64_t ldb;
  double *__restrict__ x;
  int64_t ldx;
  const int32_t *__restrict__ in_slot;
  const int32_t *__restrict__ out_slot;
  SliceView<T> fwd, bwd;
};

template <class T, int CH> struct SliceRegs {
  int row, off, len;
  T dinv;
  int col[CH];
  T val[CH];
};

template <class T, int W, int CH>
__device__ __forceinline__ void load_slice(const SliceView<T> &v, int s, int g, SliceRegs<T, CH> &r) {
  constexpr int G = 32 / W;
  const int2 sp = __ldg(v.span + s);
  r.off = sp.x;
  r.len = sp.y;
  r.row = __ldg(v.row + s * G + g);
  r.dinv = __ldg(v.dinv + s * G + g);
#pragma unroll
  for (int q = 0; q < CH; ++q) {
    if (q < r.len) {
      r.col[q] = __ldg(v.col + r.off + q * G + g);
      r.val[q] = __ldg(v.val + r.off + q * G + g);
    }
  }
}

template <class T, int W, int CH>
__device__ __forceinline__ void compute_slice(const SliceView<T> &v, T *Ys, const SliceRegs<T, CH> &r, int g, int c) {
  constexpr int G = 32 / W;
  T acc = Ys[r.row * W + c];
#pragma unroll
  for (int q = 0; q < CH; ++q)
    if (q < r.len) acc -= r.val[q] * Ys[r.col[q] * W + c];
  for (int q = CH; q < r.len; ++q) {
    const int p = r.off + q * G + g;
    acc -= __ldg(v.val + p) * Ys[__ldg(v.col + p) * W + c];
  }
  Ys[r.row * W + c] = acc * r.dinv;
}

// One sweep over the tile in shared memory; ends with a barrier after its last level.
template <class T, int W, int CH>
__device__ __forceinline__ void sweep_slices(const SliceView<T> &v, T *Ys, int warp, int nwarps, int g, int c) {
  if (v.levels <= 0) return;
  SliceRegs<T, CH> cur, nxt;
  int s = __ldg(v.level_slice) + warp;
  int e = __ldg(v.level_slice + 1);
  bool have = s < e;
  if (have) load_slice<T, W, CH>(v, s, g, cur);
  for (int l = 0; l < v.levels; ++l) {
    while (have) {
      const int sn = s + nwarps;
      const bool hn = sn < e;
      if (hn) load_slice<T, W, CH>(v, sn, g, nxt);
      compute_slice<T, W, CH>(v, Ys, cur, g, c);
      s = sn;
      have = hn;
      if (hn) cur = nxt;
    }
    if (l + 1 < v.levels) {
      s = __ldg(v.level_slice + l + 1) + warp;
      e = __ldg(v.level_slice + l + 2);
      have = s < e;
      if (have) load_slice<T, W, CH>(v, s, g, cur);
    }
    __syncthreads();
  }
}

template <class T, int W, int CH>
__global__ void __launch_bounds__(512) smem_tile_kernel(SmemArgs<T> a) {
  static_assert(32 % W == 0, "W divides a warp");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *Ys = reinterpret_cast<T *>(smem_raw);
  const int n = a.n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane / W, c = lane % W;
  if (threadIdx.x < 2 * W) Ys[n * W + threadIdx.x] = T(0);
  for (int64_t tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
    const int64_t col0 = tile * W;
    // b's columns into slots (coalesced global reads)
#pragma unroll 1
    for (int cc = 0; cc < W; ++cc) {
      const int64_t col = col0 + cc;
      if (col < a.count) {
        const double *bc = a.b + col * a.ldb;
#pragma unroll 8
        for (int r = threadIdx.x; r < n; r += blockDim.x) Ys[__ldg(a.in_slot + r) * W + cc] = (T)__ldg(bc + r);
      } else {
        for (int r = threadIdx.x; r < n; r += blockDim.x) Ys[r * W + cc] = T(0);
      }
    }
    __syncthreads();
    sweep_slices<T, W, CH>(a.fwd, Ys, warp, nwarps, g, c);
    sweep_slices<T, W, CH>(a.bwd, Ys, warp, nwarps, g, c);
    // slots into x's columns (coalesced global writes)
#pragma unroll 1
    for (int cc = 0; cc < W; ++cc) {
      const int64_t col = col0 + cc;
      if (col >= a.count) break;
      double *xc = a.x + col * a.ldx;
#pragma unroll 8
      for (int r = threadIdx.x; r < n; r += blockDim.x) xc[r] = (double)Ys[__ldg(a.out_slot + r) * W + cc];
    }
    __syncthreads();
  }
}

}  // namespace yb
