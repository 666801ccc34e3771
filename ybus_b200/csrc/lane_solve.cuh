// The lane solve: one right-hand side per lane, a block of `warps` warps per group of 32. Every
// lane of a warp runs the same rows in the same order (the factor's records are read once per warp,
// from shared memory, at addresses all lanes share), each on its own right-hand side, so the rows
// need no barriers, no reductions across lanes and no divergence. The warps of a block take
// different subtree domains of the elimination tree on the same 32 right-hand sides; warp 0 takes
// the top above them between two block barriers, with the domains' updates of top rows handed over
// through a partial array and the top's solutions handed back through the work array (LaneLayout in
// plan.hpp). The order keeps a few tens of values alive per lane, in shared memory; the right-hand
// sides, the forward results and the solutions stream through the work array in HBM laid out
// [group][position][lane], so every row a warp reads or writes is one contiguous 32-value line.
//
// Three launches make a solve: the gather of b (natural rows, column-major) into the work array in
// solve order, the lane solve in place, and the scatter of the work array into x. Each warp's
// records stream into its ring of pages by TMA bulk copies (no multicast); the work rows come
// through a per-warp ring of cp.async copies, a batch of kLaneBatch rows at a time, one to two
// batches ahead of use.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"
#include "stream_solve.cuh"

namespace yb {

constexpr int kLaneBatch = 4;                // rows per prefetch batch
constexpr int kLaneRows = 2 * kLaneBatch;    // rows of the per-warp prefetch ring
constexpr int kLaneBarriers = 2;             // block barriers in every warp's stream
constexpr int kLaneMaxWarps = 8;             // warps per block at most

struct LaneArgs {
  int32_t n, slots, page_bytes, ring, partials;
  const uint8_t *__restrict__ blob;       // every warp's pages
  const int32_t *__restrict__ warp_page;  // [warps + 1]
  int32_t *error;                         // set to 1 if a wait ran out or a stream is malformed
};

// A warp's shared memory: live slots, the prefetch ring, the page ring and its barriers.
template <class T> __host__ __device__ inline size_t lane_warp_bytes(int32_t slots, int32_t ring, int32_t page_bytes) {
  const size_t b = (size_t)slots * 32 * sizeof(T) + (size_t)kLaneRows * 32 * sizeof(T) + (size_t)ring * page_bytes +
                   (size_t)ring * 8;
  return (b + 127) & ~(size_t)127;
}

template <int BYTES> __device__ __forceinline__ void cp_async_lane(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One entry {val or a 32-bit word, byte offset}: 16 bytes for FP64, 8 for FP32.
__device__ __forceinline__ void lane_entry(const uint8_t *p, double &v, uint32_t &o) {
  const double2 e = *reinterpret_cast<const double2 *>(p);
  v = e.x;
  o = (uint32_t)__double_as_longlong(e.y);
}
__device__ __forceinline__ void lane_entry(const uint8_t *p, float &v, uint32_t &o) {
  const float2 e = *reinterpret_cast<const float2 *>(p);
  v = e.x;
  o = __float_as_uint(e.y);
}
template <class T> __device__ __forceinline__ void lane_word(const uint8_t *p, uint32_t &word, uint32_t &o) {
  const uint2 *q = reinterpret_cast<const uint2 *>(p);
  if constexpr (sizeof(T) == 8) {
    const uint4 e = *reinterpret_cast<const uint4 *>(p);
    word = e.x, o = e.z;
  } else {
    const uint2 e = *q;
    word = e.x, o = e.y;
  }
}

// The block barrier, in its form that warps may reach from different instructions (the error path
// takes the barriers its stream did not reach at the kernel's end).
__device__ __forceinline__ void lane_barrier() { asm volatile("barrier.sync 0;" ::: "memory"); }

template <class T> __device__ __forceinline__ T &lane_slot(uint8_t *live_lane, uint32_t off) {
  return *reinterpret_cast<T *>(live_lane + off);
}

// acc[offset] -= val * z for a record's entries; the offsets of one record are distinct, so all of
// a group's accumulators are read before any is written.
template <class T> __device__ __forceinline__ void lane_scatter(const uint8_t *e, int count, T z, uint8_t *live_lane) {
  constexpr int E = sizeof(T) == 8 ? 16 : 8;
  int i = 0;
  for (; i + 4 <= count; i += 4) {
    T v[4], a[4];
    uint32_t o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) lane_entry(e + (i + q) * E, v[q], o[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) a[q] = lane_slot<T>(live_lane, o[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) lane_slot<T>(live_lane, o[q]) = fma(-v[q], z, a[q]);
  }
  const int left = count - i;
  if (left > 0) {
    T v[3], a[3];
    uint32_t o[3];
#pragma unroll
    for (int q = 0; q < 3; ++q)
      if (q < left) lane_entry(e + (i + q) * E, v[q], o[q]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      if (q < left) a[q] = lane_slot<T>(live_lane, o[q]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      if (q < left) lane_slot<T>(live_lane, o[q]) = fma(-v[q], z, a[q]);
  }
}

// acc -= val * x[offset] over a record's entries, in stored order.
template <class T> __device__ __forceinline__ T lane_gather(const uint8_t *e, int count, T acc, uint8_t *live_lane) {
  constexpr int E = sizeof(T) == 8 ? 16 : 8;
  int i = 0;
  for (; i + 4 <= count; i += 4) {
    T v[4], x[4];
    uint32_t o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) lane_entry(e + (i + q) * E, v[q], o[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) x[q] = lane_slot<T>(live_lane, o[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) acc = fma(-v[q], x[q], acc);
  }
  const int left = count - i;
  if (left > 0) {
    T v[3], x[3];
    uint32_t o[3];
#pragma unroll
    for (int q = 0; q < 3; ++q)
      if (q < left) lane_entry(e + (i + q) * E, v[q], o[q]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      if (q < left) x[q] = lane_slot<T>(live_lane, o[q]);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      if (q < left) acc = fma(-v[q], x[q], acc);
  }
  return acc;
}

// Block g solves the 32 right-hand sides of group g in `work` in place; `partial` holds each
// block's partial array.
template <class T>
__global__ void __launch_bounds__(kLaneMaxWarps * 32) lane_solve_kernel(LaneArgs a, T *__restrict__ work,
                                                                       T *__restrict__ partial) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int B = kLaneBatch, R = kLaneRows, E = sizeof(T) == 8 ? 16 : 8;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = a.n, S = a.ring, PB = a.page_bytes;
  uint8_t *base = smem_raw + (size_t)warp * lane_warp_bytes<T>(a.slots, S, PB);
  uint8_t *live_lane = base + lane * sizeof(T);
  T *rows = reinterpret_cast<T *>(base + (size_t)a.slots * 32 * sizeof(T));
  uint8_t *ring = reinterpret_cast<uint8_t *>(rows + R * 32);
  uint64_t *full = reinterpret_cast<uint64_t *>(ring + (size_t)S * PB);
  T *w = work + (size_t)blockIdx.x * n * 32;
  T *part = partial + (size_t)blockIdx.x * a.partials * 32;
  const int p0 = __ldg(a.warp_page + warp), np = __ldg(a.warp_page + warp + 1) - p0;
  const uint8_t *stream = a.blob + (size_t)p0 * PB;

  for (int s = 0; s < a.slots; ++s) lane_slot<T>(live_lane, s * 32 * sizeof(T)) = T(0);
  if (lane == 0) {
    for (int s = 0; s < S; ++s) mbar_init(full + s, 1);
    mbar_fence_init();
  }
  __syncwarp();
  if (lane == 0)
    for (int s = 0; s < S && s < np; ++s) bulk_page(ring + (size_t)s * PB, stream + (size_t)s * PB, (uint32_t)PB, full + s);
  int issued = min(S, np);
  __syncwarp();

  int k = 0;  // the page being read
  const uint8_t *page = ring;
  int off = 0;
  bool ok = np > 0 && mbar_wait_bounded(full, 0, a.error);
  auto advance = [&]() {  // the finished page's slot takes page k + S
    __syncwarp();
    if (k + S < np) {
      if (lane == 0) {
        fence_proxy_async();
        bulk_page(ring + (size_t)(k % S) * PB, stream + (size_t)(k + S) * PB, (uint32_t)PB, full + k % S);
      }
      issued = k + S + 1;
    }
    ++k;
    ok = k < np && mbar_wait_bounded(full + k % S, (uint32_t)((k / S) & 1), a.error);
    page = ring + (size_t)(k % S) * PB;
    off = 0;
  };

  // the phase: rows from `start` up (forward) or down (backward); row i of the phase is prefetched
  // into ring row i % R by batch i / B
  int start = 0, len = 0, i = 0, cur = 0, barriers = 0;
  bool backward = false, ended = false;
  auto issue_batch = [&](int batch) {
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int r = batch * B + q;
      if (r < len)
        cp_async_lane<sizeof(T)>(rows + (r & (R - 1)) * 32 + lane, w + (size_t)(backward ? start - r : start + r) * 32 + lane);
    }
    cp_async_commit();
  };
  auto next_row = [&]() -> T {
    if ((i & (B - 1)) == 0) {
      if (i > 0) issue_batch(i / B + 1);
      cp_async_wait<1>();
    }
    cur = backward ? start - i : start + i;
    return rows[(i++ & (R - 1)) * 32 + lane];
  };

  T z = T(0);  // the row's forward result, or its backward running sum
  while (ok && !ended) {
    if (off + 16 > PB) {
      advance();
      continue;
    }
    const uint2 h = *reinterpret_cast<const uint2 *>(page + off);
    const uint32_t kind = h.y >> 16;
    const int count = (int)(h.y & 0xffffu);
    const uint8_t *e = page + off + 16;
    if (kind <= kLaneRowEnd) {
      const T dinv = *reinterpret_cast<const T *>(page + off + 8);
      if (!backward) {
        if (kind <= kLaneRowBegin) {
          T b = next_row();
          T &acc = lane_slot<T>(live_lane, h.x);
          b += acc;
          acc = T(0);
          z = b * dinv;
          w[(size_t)cur * 32 + lane] = z;
        }
        lane_scatter<T>(e, count, z, live_lane);
      } else {
        if (kind <= kLaneRowBegin) z = next_row();
        z = lane_gather<T>(e, count, z, live_lane);
        if (kind == kLaneRow || kind == kLaneRowEnd) {
          const T x = z * dinv;
          lane_slot<T>(live_lane, h.x) = x;
          w[(size_t)cur * 32 + lane] = x;
        }
      }
      off += 16 + ((count * E + 15) & ~15);
      continue;
    }
    switch (kind & 0xffu) {
      case kLanePhase: {
        cp_async_wait<0>();
        __threadfence();  // the rows this lane stored are what the phase's copies read
        start = (int)h.x;
        len = (int)*reinterpret_cast<const uint32_t *>(page + off + 8);
        backward = (kind & kLaneBackward) != 0;
        i = 0;
        issue_batch(0);
        issue_batch(1);
        off += 16;
        break;
      }
      case kLanePartials: {
        T acc = lane_slot<T>(live_lane, h.x);
        for (int q = 0; q < count; ++q) {
          uint32_t word, o;
          lane_word<T>(e + q * E, word, o);
          acc += part[(size_t)word * 32 + lane];
        }
        lane_slot<T>(live_lane, h.x) = acc;
        off += 16 + ((count * E + 15) & ~15);
        break;
      }
      case kLaneFlush: {
        for (int q = 0; q < count; ++q) {
          uint32_t word, o;
          lane_word<T>(e + q * E, word, o);
          part[(size_t)word * 32 + lane] = lane_slot<T>(live_lane, o);
          lane_slot<T>(live_lane, o) = T(0);
        }
        off += 16 + ((count * E + 15) & ~15);
        break;
      }
      case kLaneImport: {
        for (int q = 0; q < count; ++q) {
          uint32_t word, o;
          lane_word<T>(e + q * E, word, o);
          lane_slot<T>(live_lane, o) = w[(size_t)word * 32 + lane];
        }
        off += 16 + ((count * E + 15) & ~15);
        break;
      }
      case kLaneBarrier:
        lane_barrier();
        ++barriers;
        off += 16;
        break;
      case kLaneEnd:
        ended = true;
        break;
      case kLanePageEnd:
        advance();
        break;
      default:  // a malformed stream
        if (lane == 0) atomicExch(a.error, 1);
        ok = false;
        break;
    }
  }
  cp_async_wait<0>();
  if (!ended) {
    // a wait that ran out: let the copies still in flight land before the block's memory is reused
    if (lane == 0) atomicExch(a.error, 1);
    for (int p = k; p < issued; ++p) mbar_wait_bounded(full + p % S, (uint32_t)((p / S) & 1), a.error);
  }
  while (barriers < kLaneBarriers) {  // every warp takes the same barriers, whatever happened
    lane_barrier();
    ++barriers;
  }
}

// b (natural rows, column-major, ldb) into the work array [group][position][lane] in solve order;
// right-hand sides past `count` are zero. Blocks of 256 threads take 64 rows of one group.
template <class T>
__global__ void __launch_bounds__(256) lane_in_kernel(const double *__restrict__ b, int64_t ldb, int64_t count, int32_t n,
                                                      int64_t groups, const int32_t *__restrict__ in_pos,
                                                      T *__restrict__ work) {
  __shared__ T tile[64][33];
  const int i0 = blockIdx.x * 64;
  for (int64_t g = blockIdx.y; g < groups; g += gridDim.y) {
    for (int e = threadIdx.x; e < 64 * 32; e += 256) {
      const int c = e >> 6, q = e & 63, i = i0 + q;
      const int64_t col = g * 32 + c;
      tile[q][c] = (i < n && col < count) ? T(b[col * ldb + i]) : T(0);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 64 * 32; e += 256) {
      const int q = e >> 5, c = e & 31, i = i0 + q;
      if (i < n) work[((size_t)g * n + __ldg(in_pos + i)) * 32 + c] = tile[q][c];
    }
    __syncthreads();
  }
}

// The work array (solutions in solve order) into x (natural rows, column-major, ldx).
template <class T>
__global__ void __launch_bounds__(256) lane_out_kernel(const T *__restrict__ work, int64_t count, int32_t n,
                                                       int64_t groups, const int32_t *__restrict__ out_pos,
                                                       double *__restrict__ x, int64_t ldx) {
  __shared__ T tile[64][33];
  const int i0 = blockIdx.x * 64;
  for (int64_t g = blockIdx.y; g < groups; g += gridDim.y) {
    for (int e = threadIdx.x; e < 64 * 32; e += 256) {
      const int q = e >> 5, c = e & 31, i = i0 + q;
      tile[q][c] = i < n ? work[((size_t)g * n + __ldg(out_pos + i)) * 32 + c] : T(0);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 64 * 32; e += 256) {
      const int c = e >> 6, q = e & 63, i = i0 + q;
      const int64_t col = g * 32 + c;
      if (i < n && col < count) x[col * ldx + i] = (double)tile[q][c];
    }
    __syncthreads();
  }
}

}  // namespace yb
