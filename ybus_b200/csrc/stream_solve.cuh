// The streamed tile solve: a tile's working vector lives in shared memory, and each warp reads its
// share of the factor as a stream of fixed-size pages that TMA bulk copies bring into a per-warp
// shared-memory ring several pages ahead of use (see StreamLayout in plan.hpp).
//
// Shared memory of a block:
//   Ys[(n + 2) * W]            the tile, slot-major; slot n stays zero, slot n + 1 absorbs padding
//   ring[warps][S][page]       each warp's pages in flight
//   full[warps][S]             one mbarrier per ring slot: the bulk copy's completion
//
// Lane 0 of a warp issues `cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes`
// for page k + S once page k is consumed; the warp waits on the slot's mbarrier with
// `mbarrier.try_wait.parity`, a bounded number of times (a wait that runs out sets the error word
// and the kernel carries on to its end, so no barrier is left unmatched). A page's records are
// walked in order: before a record of stage s the warp takes block barriers until s have passed;
// slice records give each lane group a row, split records spread one row over the lane groups and
// reduce with shuffles. The stream is the same for every tile, so the prefetch runs on from one
// tile into the next.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.cuh"
#include "plan.hpp"

namespace yb {

struct StreamArgs {
  int32_t n;
  int64_t count, tiles;
  const double *__restrict__ b;
  int64_t ldb;
  double *__restrict__ x;
  int64_t ldx;
  const int32_t *__restrict__ in_slot;
  const int32_t *__restrict__ out_slot;
  const void *__restrict__ load_scale;  // [n] T, by row of b
  const uint8_t *__restrict__ blob;
  const int32_t *__restrict__ warp_page;  // [warps + 1]
  int32_t page_bytes, ring, stages;
  int32_t tail;                           // rows of the dense tail (0: none)
  const int32_t *__restrict__ tail_slot;  // [tail] their slots
  int32_t *error;  // set to 1 if a wait ran out
  // diagnostics: if set, block 0 records clock64() at phase boundaries of its first tiles:
  // [tile][warp][mark], marks 0 load done, 1 first record, 2 stage-barrier entries..., see kernel
  long long *phase_clock;
};

// How long a kernel waits for a copy before it gives up, records the failure and returns: one
// second of the GPU's global timer, far beyond any copy's latency, short enough that a copy that
// never lands costs a launch a second or two and leaves the context usable.
constexpr unsigned long long kWaitLimitNs = 1000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void bulk_page(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for a slot's copy; gives up after kWaitLimitNs, recording the failure in *error (if not
// null). Returns whether the copy completed. The timer is read only once a first try has failed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int32_t *error) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > kWaitLimitNs) {
      if (error) atomicExch(error, 1);
      return false;
    }
  }
  return true;
}

// Orders this thread's earlier shared-memory accesses before later async-proxy (bulk copy) writes.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// A slot's W values to and from registers, in 16-byte (or narrower) shared-memory accesses.
template <class T, int W> __device__ __forceinline__ void load_w(const T *p, T (&v)[W]) {
  if constexpr (sizeof(T) * W % 16 == 0) {
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) * W / 16); ++i) {
      const int4 q = reinterpret_cast<const int4 *>(p)[i];
      memcpy(&v[i * 16 / sizeof(T)], &q, 16);
    }
  } else if constexpr (sizeof(T) * W == 8) {
    const int2 q = *reinterpret_cast<const int2 *>(p);
    memcpy(&v[0], &q, 8);
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) v[i] = p[i];
  }
}

template <class T, int W> __device__ __forceinline__ void store_w(T *p, const T (&v)[W]) {
  if constexpr (sizeof(T) * W % 16 == 0) {
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) * W / 16); ++i) {
      int4 q;
      memcpy(&q, &v[i * 16 / sizeof(T)], 16);
      reinterpret_cast<int4 *>(p)[i] = q;
    }
  } else if constexpr (sizeof(T) * W == 8) {
    int2 q;
    memcpy(&q, &v[0], 8);
    *reinterpret_cast<int2 *>(p) = q;
  } else {
#pragma unroll
    for (int i = 0; i < W; ++i) p[i] = v[i];
  }
}

template <class T, int W>
__global__ void __launch_bounds__(512) stream_tile_kernel(StreamArgs a) {
  static_assert(32 % W == 0, "W divides a warp");
  constexpr int G = 32;  // rows of a slice record: one per lane
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int n = a.n;
  T *Ys = reinterpret_cast<T *>(smem_raw);
  const size_t y_bytes = (((size_t)(n + 2) * W * sizeof(T)) + 127) & ~(size_t)127;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  const int S = a.ring, PB = a.page_bytes;
  // the dense tail's buffer (tail + 1 rows) and slots (tail + 1: the spare maps to the zero slot)
  const int m = a.tail;
  T *Tb = reinterpret_cast<T *>(smem_raw + y_bytes);
  const size_t tb_bytes = (((size_t)(m + 1) * W * sizeof(T)) + 15) & ~(size_t)15;
  int32_t *tslot = reinterpret_cast<int32_t *>(smem_raw + y_bytes + tb_bytes);
  const size_t ts_bytes = (((size_t)(m + 1) * 4) + 127) & ~(size_t)127;
  uint8_t *ring = smem_raw + y_bytes + tb_bytes + ts_bytes + (size_t)warp * S * PB;
  uint64_t *full =
      reinterpret_cast<uint64_t *>(smem_raw + y_bytes + tb_bytes + ts_bytes + (size_t)warps * S * PB) + warp * S;
  const T *scale = reinterpret_cast<const T *>(a.load_scale);

  if (threadIdx.x < 2 * W) Ys[n * W + threadIdx.x] = T(0);
  for (int t = threadIdx.x; t <= m; t += blockDim.x) tslot[t] = t < m ? __ldg(a.tail_slot + t) : n;
  if (lane == 0)
    for (int s = 0; s < S; ++s) mbar_init(full + s, 1);
  mbar_fence_init();
  __syncthreads();

  const int p0 = __ldg(a.warp_page + warp), np = __ldg(a.warp_page + warp + 1) - p0;
  const int64_t my_tiles = blockIdx.x < a.tiles ? (a.tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int64_t total_pages = (int64_t)np * my_tiles;
  // Pages of this warp's stream, numbered across all its tiles: page k is stream page k % np
  auto issue = [&](int64_t k) {
    if (k < total_pages) {
      fence_proxy_async();
      const int slot = (int)(k % S);
      bulk_page(ring + (size_t)slot * PB, a.blob + (size_t)(p0 + (int)(k % np)) * PB, (uint32_t)PB, full + slot);
    }
  };
  if (lane == 0)
    for (int64_t k = 0; k < S; ++k) issue(k);
  __syncwarp();

  int64_t k = 0;  // next page to consume
  for (int64_t tile = blockIdx.x; tile < a.tiles; tile += gridDim.x) {
    const int64_t col0 = tile * W;
    // b's columns into slots, leaves (no forward entries) scaled by their diagonal
#pragma unroll 1
    for (int cc = 0; cc < W; ++cc) {
      const int64_t col = col0 + cc;
      if (col < a.count) {
        const double *bc = a.b + col * a.ldb;
#pragma unroll 8
        for (int r = threadIdx.x; r < n; r += blockDim.x)
          Ys[__ldg(a.in_slot + r) * W + cc] = (T)__ldg(bc + r) * __ldg(scale + r);
      } else {
        for (int r = threadIdx.x; r < n; r += blockDim.x) Ys[r * W + cc] = T(0);
      }
    }
    __syncthreads();
    const int64_t it = (tile - blockIdx.x) / gridDim.x;
    long long *pc = (a.phase_clock && blockIdx.x == 0 && it < 4 && lane == 0) ? a.phase_clock + (it * 16 + warp) * 8 : nullptr;
    if (pc) pc[0] = clock64();

    int done = 0;
    long long wait_cycles = 0, barrier_cycles = 0, pages_seen = 0;
    T acc[W];  // a row's W running sums (slice: this lane's row; split and dense: this lane's share)
#pragma unroll
    for (int cc = 0; cc < W; ++cc) acc[cc] = T(0);
    for (int j = 0; j < np; ++j, ++k) {
      const int slot = (int)(k % S);
      const long long w0 = pc ? clock64() : 0;
      const bool ready = mbar_wait_bounded(full + slot, (uint32_t)((k / S) & 1), a.error);
      if (pc) {
        wait_cycles += clock64() - w0;
        ++pages_seen;
      }
      const uint8_t *page = ring + (size_t)slot * PB;
      int pos = ready ? 0 : PB;  // a page that never arrived is skipped
      while (pos + 16 <= PB) {
        const int4 hdr = *reinterpret_cast<const int4 *>(page + pos);
        const int kind = hdr.x, len = hdr.z, flags = hdr.w;
        const int stage = min(hdr.y, a.stages);
        if (kind < 0 || len < 0 || len > PB) break;
        if (done < stage) {
          const long long b0 = pc ? clock64() : 0;
          while (done < stage) {
            __syncthreads();
            ++done;
          }
          if (pc) barrier_cycles += clock64() - b0;
        }
        const uint8_t *body = page + pos + 16;
        if (kind == kRecordSlice) {
          // this lane's row: W sums in registers, one vector load per entry
          const int32_t *rows = reinterpret_cast<const int32_t *>(body);
          const T *dinv = reinterpret_cast<const T *>(body + ((4 * G + 15) & ~15));
          const uint8_t *ent = body + ((4 * G + 15) & ~15) + ((sizeof(T) * G + 15) & ~15);
          const int32_t *col = reinterpret_cast<const int32_t *>(ent);
          const T *val = reinterpret_cast<const T *>(ent + ((4 * len * G + 15) & ~15));
          const int row = rows[lane];
          const bool to_tail = (flags & kRecordToTail) != 0;
          if (flags & kRecordFirst) load_w<T, W>(Ys + (to_tail ? tslot[row] : row) * W, acc);
          for (int q = 0; q < len; ++q) {
            const T v = val[q * G + lane];
            T y[W];
            load_w<T, W>(Ys + col[q * G + lane] * W, y);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] -= v * y[cc];
          }
          if (flags & kRecordLast) {
            if (to_tail) {
              store_w<T, W>(Tb + row * W, acc);
            } else {
              const T d = dinv[lane];
#pragma unroll
              for (int cc = 0; cc < W; ++cc) acc[cc] *= d;
              store_w<T, W>(Ys + row * W, acc);
            }
          }
          pos += 16 + ((4 * G + 15) & ~15) + ((sizeof(T) * G + 15) & ~15) + ((4 * len * G + 15) & ~15) +
                 ((sizeof(T) * len * G + 15) & ~15);
        } else if (kind == kRecordDense) {
          // one chunk of a dense tail row: lanes split the columns, each lane keeps W sums
          const int t = *reinterpret_cast<const int32_t *>(body);
          const int j0 = *reinterpret_cast<const int32_t *>(body + 4);
          const T *val = reinterpret_cast<const T *>(body + 16);
          if (flags & kRecordFirst)
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] = T(0);
          for (int e = lane; e < len; e += 32) {
            const T v = val[e];
            T y[W];
            load_w<T, W>(Tb + (j0 + e) * W, y);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] += v * y[cc];
          }
          if (flags & kRecordLast) {
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
              T v = acc[cc];
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
              if (lane == cc) Ys[tslot[t] * W + cc] = v;
            }
          }
          pos += 32 + ((sizeof(T) * len + 15) & ~15);
        } else if (kind == kRecordCopy) {
          // this warp's share of the tail's slots into the tail buffer
          for (int idx = warp * 32 + lane; idx < m * W; idx += warps * 32) Tb[idx] = Ys[tslot[idx / W] * W + idx % W];
          pos += 16;
        } else {
          // one long row split over the lanes: each lane's share of the entries, then a reduction
          const int row = *reinterpret_cast<const int32_t *>(body);
          const T dinv = *reinterpret_cast<const T *>(body + 16);
          const int32_t *col = reinterpret_cast<const int32_t *>(body + 32);
          const T *val = reinterpret_cast<const T *>(body + 32 + ((4 * len + 15) & ~15));
          if (flags & kRecordFirst)
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] = T(0);
          for (int e = lane; e < len; e += 32) {
            const T v = val[e];
            T y[W];
            load_w<T, W>(Ys + col[e] * W, y);
#pragma unroll
            for (int cc = 0; cc < W; ++cc) acc[cc] += v * y[cc];
          }
          if (flags & kRecordLast) {
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
              T v = acc[cc];
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
              if (lane == cc) Ys[row * W + cc] = (Ys[row * W + cc] - v) * dinv;
            }
          }
          pos += 48 + ((4 * len + 15) & ~15) + ((sizeof(T) * len + 15) & ~15);
        }
        __syncwarp();
      }
      __syncwarp();
      if (lane == 0) issue(k + S);
    }
    if (pc) {
      pc[1] = clock64();
      pc[4] = wait_cycles;
      pc[5] = barrier_cycles;
      pc[6] = pages_seen;
    }
    while (done < a.stages) {
      __syncthreads();
      ++done;
    }
    if (pc) pc[2] = clock64();
    // slots into x's columns
#pragma unroll 1
    for (int cc = 0; cc < W; ++cc) {
      const int64_t col = col0 + cc;
      if (col >= a.count) break;
      double *xc = a.x + col * a.ldx;
#pragma unroll 8
      for (int r = threadIdx.x; r < n; r += blockDim.x) xc[r] = (double)Ys[__ldg(a.out_slot + r) * W + cc];
    }
    __syncthreads();
    if (pc) pc[3] = clock64();
  }
  // Every copy issued was waited for above; after a wait that ran out, wait (bounded) for the
  // last copy into each slot before the block's shared memory is released
  if (lane == 0 && total_pages > 0) {
    const int64_t first = total_pages > S ? total_pages - S : 0;
    for (int64_t kk = first; kk < total_pages; ++kk) mbar_wait_bounded(full + (kk % S), (uint32_t)((kk / S) & 1), nullptr);
  }
}

}  // namespace yb
