// The lane solve: one right-hand side per lane, a block of `warps` warps per group of 32. Every
// lane of a warp runs the same rows in the same order (the factor's records are read once per warp,
// from shared memory, at addresses all lanes share), each on its own right-hand side, so the rows
// need no barriers, no reductions across lanes and no divergence. The warps of a block take
// different subtree domains of the elimination tree on the same 32 right-hand sides; the top above
// them is solved between the second and fourth of four block barriers, with the domains' updates
// of top rows handed over through a partial array (which all warps add into the top rows'
// right-hand sides between the first two barriers) and the top's solutions handed back through the
// work array (LaneLayout in plan.hpp). In FP64 the top is a dense map every warp takes a share of
// (its right-hand sides into each warp's slots, then each solution as a dense row over all warps'
// slots); otherwise warp 0 runs its rows as a chain. The order keeps a few tens of values alive
// per lane, in shared memory; the right-hand sides, the forward results and the solutions stream
// through the work array in HBM laid out [group][work row][lane], a row's values in the work row of
// the row of b that feeds it, so every row a warp reads or writes is one contiguous 32-value line
// (R = 2 right-hand sides per lane: 64 values, lane l's two adjacent).
//
// Three launches make a solve: the gather of b (natural rows, column-major) into the work array,
// the lane solve in place, and the scatter of the work array into x; with the work rows in b's own
// row order the gather and scatter are plain transposes of 32-column blocks. Each warp's
// records stream into its ring of pages by TMA bulk copies (no multicast); the work rows come
// through a per-warp ring of cp.async copies, a batch of kLaneBatch rows at a time, one to two
// batches ahead of use.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"
#include "stream_solve.cuh"

namespace yb {

constexpr int kLaneMaxWarps = 16;            // warps per block at most
constexpr int kLaneNarrowWarps = 8;          // at most these take the kernel bounded to three blocks per SM

struct LaneArgs {
  int32_t n, slots, page_bytes, partials;
  const uint8_t *__restrict__ blob;       // every warp's pages
  const int32_t *__restrict__ warp_page;  // [warps + 1]
  int32_t *error;                         // set to 1 if a wait ran out or a stream is malformed
  const uint8_t *group_active;            // [groups] 0: the group is skipped; null: every group runs
  void *xout;  // null: the solutions overwrite the work array; else an array of the work array's layout
               // that receives them (the backward rows' results and the top solutions the domains read)
  int32_t withhold;  // for tests of the error path: the page of block 0's first warp whose copy is never
                     // issued, so that warp's bounded wait runs out (-1: none)
};

// A warp's shared memory (lane_warp_bytes_of in plan.hpp) for values of type T.
template <class T>
__host__ __device__ inline size_t lane_warp_bytes(int32_t slots, int32_t ring, int32_t page_bytes, int32_t rpl = 1) {
  return lane_warp_bytes_of((int32_t)sizeof(T), slots, ring, page_bytes, rpl);
}

template <int BYTES> __device__ __forceinline__ void cp_async_lane(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The block's dynamic shared memory. Every shared access of the lane solve is a 32-bit byte offset
// into it, so the compiler addresses shared memory directly.
extern __shared__ __align__(128) unsigned char lane_shared[];

template <class T> __device__ __forceinline__ T &lane_at(uint32_t off) { return *reinterpret_cast<T *>(lane_shared + off); }

// An entry {val or a 32-bit word, offset} at shared offset e: 16 bytes for FP64, 8 for FP32.
__device__ __forceinline__ void lane_entry(uint32_t e, double &v, uint32_t &word, uint32_t &o) {
  const uint4 x = lane_at<uint4>(e);
  v = __hiloint2double((int)x.y, (int)x.x);
  word = x.x, o = x.z;
}
__device__ __forceinline__ void lane_entry(uint32_t e, float &v, uint32_t &word, uint32_t &o) {
  const uint2 x = lane_at<uint2>(e);
  v = __uint_as_float(x.x);
  word = x.x, o = x.y;
}

// The block barrier, in its form that warps may reach from different instructions (the error path
// takes the barriers its stream did not reach at the kernel's end).
__device__ __forceinline__ void lane_barrier() { asm volatile("barrier.sync 0;" ::: "memory"); }

// A lane's values: one per right-hand side it carries (R = 1 or 2, adjacent columns of the group),
// loaded and stored together, 8 or 16 bytes, in shared and in global memory.
template <class T, int R> struct Lv {
  T v[R];
};
template <class T, int R> __device__ __forceinline__ Lv<T, R> lv_load(const void *p) {
  Lv<T, R> x;
  if constexpr (R == 1) {
    x.v[0] = *reinterpret_cast<const T *>(p);
  } else if constexpr (sizeof(T) == 8) {
    const double2 q = *reinterpret_cast<const double2 *>(p);
    x.v[0] = q.x, x.v[1] = q.y;
  } else {
    const float2 q = *reinterpret_cast<const float2 *>(p);
    x.v[0] = q.x, x.v[1] = q.y;
  }
  return x;
}
template <class T, int R> __device__ __forceinline__ void lv_store(void *p, const Lv<T, R> &x) {
  if constexpr (R == 1)
    *reinterpret_cast<T *>(p) = x.v[0];
  else if constexpr (sizeof(T) == 8)
    *reinterpret_cast<double2 *>(p) = make_double2(x.v[0], x.v[1]);
  else
    *reinterpret_cast<float2 *>(p) = make_float2(x.v[0], x.v[1]);
}
template <class T, int R> __device__ __forceinline__ Lv<T, R> lv_ld(uint32_t off) { return lv_load<T, R>(lane_shared + off); }
template <class T, int R> __device__ __forceinline__ void lv_st(uint32_t off, const Lv<T, R> &x) {
  lv_store<T, R>(lane_shared + off, x);
}
template <class T, int R> __device__ __forceinline__ Lv<T, R> lv_zero() {
  Lv<T, R> x;
#pragma unroll
  for (int r = 0; r < R; ++r) x.v[r] = T(0);
  return x;
}

// acc[offset] -= val * z for C entries (C known at compile time) at shared offset e, for each of
// the lane's R right-hand sides; the offsets of one record are distinct, so every accumulator is
// read before any is written.
template <class T, int R, int C> __device__ __forceinline__ void lane_scatter_n(uint32_t e, const Lv<T, R> &z, uint32_t live) {
  constexpr uint32_t E = sizeof(T) == 8 ? 16 : 8;
  T v[C];
  Lv<T, R> a[C];
  uint32_t o[C], w;
#pragma unroll
  for (int c = 0; c < C; ++c) lane_entry(e + c * E, v[c], w, o[c]);
#pragma unroll
  for (int c = 0; c < C; ++c) a[c] = lv_ld<T, R>(live + o[c]);
#pragma unroll
  for (int c = 0; c < C; ++c) {
#pragma unroll
    for (int r = 0; r < R; ++r) a[c].v[r] = fma(-v[c], z.v[r], a[c].v[r]);
    lv_st<T, R>(live + o[c], a[c]);
  }
}

// acc -= val * x[offset] over C entries, in stored order.
template <class T, int R, int C> __device__ __forceinline__ Lv<T, R> lane_gather_n(uint32_t e, Lv<T, R> acc, uint32_t live) {
  constexpr uint32_t E = sizeof(T) == 8 ? 16 : 8;
  T v[C];
  Lv<T, R> x[C];
  uint32_t o[C], w;
#pragma unroll
  for (int c = 0; c < C; ++c) lane_entry(e + c * E, v[c], w, o[c]);
#pragma unroll
  for (int c = 0; c < C; ++c) x[c] = lv_ld<T, R>(live + o[c]);
#pragma unroll
  for (int c = 0; c < C; ++c)
#pragma unroll
    for (int r = 0; r < R; ++r) acc.v[r] = fma(-v[c], x[c].v[r], acc.v[r]);
  return acc;
}

// The same for any count, four at a time.
template <class T, int R>
__device__ __forceinline__ void lane_scatter(uint32_t e, uint32_t count, const Lv<T, R> &z, uint32_t live) {
  constexpr uint32_t E = sizeof(T) == 8 ? 16 : 8;
  uint32_t i = 0;
  for (; i + 4 <= count; i += 4) lane_scatter_n<T, R, 4>(e + i * E, z, live);
  for (; i < count; ++i) lane_scatter_n<T, R, 1>(e + i * E, z, live);
}
template <class T, int R>
__device__ __forceinline__ Lv<T, R> lane_gather(uint32_t e, uint32_t count, Lv<T, R> acc, uint32_t live) {
  constexpr uint32_t E = sizeof(T) == 8 ? 16 : 8;
  uint32_t i = 0;
  for (; i + 4 <= count; i += 4) acc = lane_gather_n<T, R, 4>(e + i * E, acc, live);
  for (; i < count; ++i) acc = lane_gather_n<T, R, 1>(e + i * E, acc, live);
  return acc;
}

// Block g solves the 32 R right-hand sides of group g in `work` in place (R per lane: the records'
// decoding then serves R times the arithmetic); `partial` holds each block's partial array. With
// R = 1 three blocks of up to 8 warps share an SM (as many as its shared memory holds), so the
// launch bound lets each thread take up to 80 registers: the compiler then keeps the records'
// fields and addresses in registers instead of recomputing them (13 % fewer instructions and 7 %
// less time than with the 44 registers it picks unbounded); with R = 2 two blocks do. WIDE blocks
// of 9 to 16 warps run one to an SM: for grids of fewer groups than SMs, where each warp's chain
// of rows, not the SM's issue, sets the time and more warps shorten the chains.
template <class T, int R, bool WIDE = false>
__global__ void __launch_bounds__(WIDE ? kLaneMaxWarps * 32 : kLaneNarrowWarps * 32, WIDE ? 1 : (R == 1 ? 3 : 2))
    lane_solve_kernel(LaneArgs a, T *__restrict__ work, T *__restrict__ partial) {
  constexpr uint32_t E = sizeof(T) == 8 ? 16 : 8, VB = sizeof(T) * R, ROW = 32 * VB;
  // The warp index through a shuffle from lane 0: the compiler then knows it (and the shared
  // offsets, record fields and branches derived from it) to be the same across the warp, and keeps
  // the records' decoding on the uniform datapath instead of every lane's registers.
  if (a.group_active && !a.group_active[blockIdx.x]) return;  // the whole block, before any barrier
  const int lane = threadIdx.x & 31, warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
  constexpr int S = kLaneRing;  // known here, so the ring's slot and phase are a mask and a shift
  const int PB = a.page_bytes;
  const uint32_t base = (uint32_t)(warp * lane_warp_bytes<T>(a.slots, S, PB, R));
  const uint32_t live = base + lane * VB;                     // this lane's slot 0
  const uint32_t rows = base + (uint32_t)a.slots * ROW + lane * VB;  // its ring slot 0
  const uint32_t ring = base + (uint32_t)a.slots * ROW + (uint32_t)kLaneRows * ROW;  // the page ring
  uint64_t *full = &lane_at<uint64_t>(ring + (uint32_t)S * PB);
  const uint32_t smem_s = smem_u32(lane_shared);  // the shared window address of offset 0
  uint8_t *w_lane = reinterpret_cast<uint8_t *>(work + ((size_t)blockIdx.x * a.n * 32 + lane) * R);
  uint8_t *x_lane =
      a.xout ? reinterpret_cast<uint8_t *>(static_cast<T *>(a.xout) + ((size_t)blockIdx.x * a.n * 32 + lane) * R) : w_lane;
  uint8_t *part_lane = reinterpret_cast<uint8_t *>(partial + ((size_t)blockIdx.x * a.partials * 32 + lane) * R);
  const int p0 = __ldg(a.warp_page + warp), np = __ldg(a.warp_page + warp + 1) - p0;
  const uint8_t *stream = a.blob + (size_t)p0 * PB;

  for (int s = 0; s < a.slots; ++s) lv_st<T, R>(live + s * ROW, lv_zero<T, R>());
  if (lane == 0) {
    for (int s = 0; s < S; ++s) mbar_init(full + s, 1);
    mbar_fence_init();
  }
  __syncwarp();
  // the page a test withholds from this warp, or -1
  const int withheld = (blockIdx.x == 0 && warp == 0) ? a.withhold : -1;
  if (lane == 0)
    for (int s = 0; s < S && s < np; ++s)
      if (s != withheld) bulk_page(lane_shared + ring + s * PB, stream + (size_t)s * PB, (uint32_t)PB, full + s);
  int issued = min(S, np);
  __syncwarp();

  int k = 0;               // the page being read
  uint32_t page = ring;    // the record being read
  // every lane waits; the warp goes on only if all of them saw the page
  bool ok = __all_sync(0xffffffffu, np > 0 && mbar_wait_bounded(full, 0, a.error));
  bool ended = false;
  int barriers = 0;
  Lv<T, R> z = lv_zero<T, R>();  // the forward row's result, or the backward row's running sum
  // the header of the record being read, loaded while the record before it runs (pages are written
  // only by the bulk copies, never by a record)
  uint4 hn = lane_at<uint4>(page);
  while (ok) {
    const uint4 h = hn;
    const uint32_t kind = (h.x >> 16) & 31u, count = h.x >> 24;
    const uint32_t self = live + ((h.x & 0xffffu) << 4);
    const uint32_t b_at = rows + ((h.x >> 21) & 7u) * ROW;
    const uint32_t e = page + 16;
    const uint32_t next = page + 16 + ((count * E + 15) & ~15u);
    if (kind != kLanePageEnd) hn = lane_at<uint4>(next);  // within the page: every page ends with its end record
    T dinv;
    if constexpr (sizeof(T) == 8)
      dinv = __hiloint2double((int)h.w, (int)h.z);
    else
      dinv = __uint_as_float(h.z);
    // the start of a forward row: z from b and the row's accumulator, into the work row
    auto forward = [&]() {
      const Lv<T, R> acc = lv_ld<T, R>(self), b = lv_ld<T, R>(b_at);
      lv_st<T, R>(self, lv_zero<T, R>());
#pragma unroll
      for (int r = 0; r < R; ++r) z.v[r] = (b.v[r] + acc.v[r]) * dinv;
      lv_store<T, R>(w_lane + h.y, z);
    };
    // the end of a backward row: x into its slot and its row of the output
    auto backward = [&]() {
      Lv<T, R> x;
#pragma unroll
      for (int r = 0; r < R; ++r) x.v[r] = z.v[r] * dinv;
      lv_st<T, R>(self, x);
      lv_store<T, R>(x_lane + h.y, x);
    };
    // a prefetch block: the batch's rows into their half of the ring, then the batch before waited for
    auto prefetch = [&](uint32_t at) {
      const uint4 o = lane_at<uint4>(at);
      const uint32_t nrows = o.x & 7u;
      const uint32_t dst = smem_s + rows + ((o.x & 8u) ? (uint32_t)kLaneBatch * ROW : 0u);
      const uint32_t off[kLaneBatch] = {o.x & ~15u, o.y, o.z, o.w};
#pragma unroll
      for (int q = 0; q < kLaneBatch; ++q)
        if (q < (int)nrows)
          asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(dst + q * ROW), "l"(w_lane + off[q]),
                       "n"(VB)
                       : "memory");
      cp_async_commit();
      cp_async_wait<1>();
    };
    // the entries' bytes of a row of c entries, to the 16-byte boundary
    auto padded = [&](uint32_t c) { return (c * E + 15) & ~15u; };
    // One switch over every kind, the rows of at most 4 entries (some opening a batch with its
    // prefetch) first: a single jump dispatches a record (5 % fewer instructions than range tests
    // followed by a switch on the count).
    switch (kind) {
// a forward (backward) row of C entries whose record carries a prefetch block if PRE
#define YB_LANE_FWD(K, C, PRE)                                            \
  case K: {                                                               \
    if (PRE) prefetch(e + padded(C));                                     \
    forward();                                                            \
    if (C > 0) lane_scatter_n<T, R, (C > 0 ? C : 1)>(e, z, live);         \
    page = next;                                                          \
    continue;                                                             \
  }
#define YB_LANE_BWD(K, C, PRE)                                            \
  case K: {                                                               \
    if (PRE) prefetch(e + padded(C));                                     \
    const Lv<T, R> b = lv_ld<T, R>(b_at);                                 \
    z = C > 0 ? lane_gather_n<T, R, (C > 0 ? C : 1)>(e, b, live) : b;     \
    backward();                                                           \
    page = next;                                                          \
    continue;                                                             \
  }
      YB_LANE_FWD(kLaneFwdRow0, 0, false)
      YB_LANE_FWD(kLaneFwdRow0 + 1, 1, false)
      YB_LANE_FWD(kLaneFwdRow0 + 2, 2, false)
      YB_LANE_FWD(kLaneFwdRow0 + 3, 3, false)
      YB_LANE_FWD(kLaneFwdRow0 + 4, 4, false)
      YB_LANE_FWD(kLaneFwdPre1, 1, true)
      YB_LANE_FWD(kLaneFwdPre1 + 1, 2, true)
      YB_LANE_FWD(kLaneFwdPre1 + 2, 3, true)
      YB_LANE_FWD(kLaneFwdPre1 + 3, 4, true)
      YB_LANE_BWD(kLaneBwdRow0, 0, false)
      YB_LANE_BWD(kLaneBwdRow0 + 1, 1, false)
      YB_LANE_BWD(kLaneBwdRow0 + 2, 2, false)
      YB_LANE_BWD(kLaneBwdRow0 + 3, 3, false)
      YB_LANE_BWD(kLaneBwdRow0 + 4, 4, false)
      YB_LANE_BWD(kLaneBwdPre1, 1, true)
      YB_LANE_BWD(kLaneBwdPre1 + 1, 2, true)
      YB_LANE_BWD(kLaneBwdPre1 + 2, 3, true)
      YB_LANE_BWD(kLaneBwdPre1 + 3, 4, true)
#undef YB_LANE_FWD
#undef YB_LANE_BWD
      case kLaneFwdRowN: forward(); lane_scatter<T, R>(e, count, z, live); break;
      case kLaneFwdMore: lane_scatter<T, R>(e, count, z, live); break;
      case kLaneBwdRowN: z = lane_gather<T, R>(e, count, lv_ld<T, R>(b_at), live); backward(); break;
      case kLaneBwdBegin: z = lane_gather<T, R>(e, count, lv_ld<T, R>(b_at), live); break;
      case kLaneBwdMore: z = lane_gather<T, R>(e, count, z, live); break;
      case kLaneBwdEnd: z = lane_gather<T, R>(e, count, z, live); backward(); break;
      case kLanePrefetch: prefetch(e); break;
      case kLanePhase:
        cp_async_wait<0>();
        __threadfence();  // the rows this lane stored are what the phase's copies read
        break;
      case kLaneTopSum: {  // the row and up to four partials in flight at a time, added in order
        if (h.z == kTopLoad) {  // the dense top: this warp's share of its right-hand sides into slots
          for (uint32_t c = 0; c < count; c += 4) {
            Lv<T, R> r[4];
            uint32_t o[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              T v;
              uint32_t w;
              lane_entry(e + min(c + q, count - 1) * E, v, w, o[q]);
              r[q] = lv_load<T, R>(w_lane + w);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (c + q < count) lv_st<T, R>(live + o[q], r[q]);
          }
          break;
        }
        if (h.z == kTopRow || h.z == kTopRowMore) {  // a dense top row over every warp's slots
          Lv<T, R> acc = h.z == kTopRow ? lv_zero<T, R>() : lv_load<T, R>(x_lane + h.y);
          const uint32_t lane_off = (uint32_t)lane * VB;  // the offsets are this block's, lane 0's
          for (uint32_t c = 0; c < count; c += 4) {
            T v[4];
            Lv<T, R> r[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              uint32_t w, o;
              lane_entry(e + min(c + q, count - 1) * E, v[q], w, o);
              r[q] = lv_ld<T, R>(lane_off + o);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (c + q < count) {
#pragma unroll
                for (int k = 0; k < R; ++k) acc.v[k] = fma(v[q], r[q].v[k], acc.v[k]);
              }
          }
          lv_store<T, R>(x_lane + h.y, acc);
          break;
        }
        uint8_t *row = w_lane + h.y;
        Lv<T, R> acc = lv_load<T, R>(row);
        for (uint32_t c = 0; c < count; c += 4) {
          Lv<T, R> p[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            T v;
            uint32_t w, o;
            lane_entry(e + min(c + q, count - 1) * E, v, w, o);
            p[q] = lv_load<T, R>(part_lane + w);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (c + q < count) {
#pragma unroll
              for (int r = 0; r < R; ++r) acc.v[r] += p[q].v[r];
            }
        }
        lv_store<T, R>(row, acc);
        break;
      }
      case kLaneFlush:
        for (uint32_t c = 0; c < count; ++c) {
          T v;
          uint32_t w, o;
          lane_entry(e + c * E, v, w, o);
          lv_store<T, R>(part_lane + w, lv_ld<T, R>(live + o));
          lv_st<T, R>(live + o, lv_zero<T, R>());
        }
        break;
      case kLaneImport:  // four loads in flight at a time
        for (uint32_t c = 0; c < count; c += 4) {
          Lv<T, R> x[4];
          uint32_t o[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            T v;
            uint32_t w;
            lane_entry(e + min(c + q, count - 1) * E, v, w, o[q]);
            x[q] = lv_load<T, R>(x_lane + w);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (c + q < count) lv_st<T, R>(live + o[q], x[q]);
        }
        break;
      case kLaneBarrier:
        lane_barrier();
        ++barriers;
        break;
      case kLaneEnd:
        ended = true;
        break;
      case kLanePageEnd: {  // the finished page's slot takes page k + S
        __syncwarp();
        if (k + S < np) {
          if (lane == 0 && k + S != withheld) {
            fence_proxy_async();
            bulk_page(lane_shared + ring + (k % S) * PB, stream + (size_t)(k + S) * PB, (uint32_t)PB, full + k % S);
          }
          issued = k + S + 1;
        }
        ++k;
        ok = __all_sync(0xffffffffu, k < np && mbar_wait_bounded(full + k % S, (uint32_t)((k / S) & 1), a.error));
        page = ring + (uint32_t)(k % S) * PB;
        if (ok) hn = lane_at<uint4>(page);
        continue;
      }
      default:  // a malformed stream
        ok = false;
        continue;
    }
    if (ended) break;
    page = next;
  }
  cp_async_wait<0>();
  if (!ended) {
    // a wait that ran out, or a malformed stream: let the copies still in flight land before the
    // block's memory is reused
    if (lane == 0) atomicExch(a.error, 1);
    for (int p = k; p < issued; ++p) mbar_wait_bounded(full + p % S, (uint32_t)((p / S) & 1), a.error);
  }
  while (barriers < kLaneBarriers) {  // every warp takes the same barriers, whatever happened
    lane_barrier();
    ++barriers;
  }
}

// A lane's work row in 32-byte pieces (256-bit global accesses): 8 for FP64, 4 for FP32.
__device__ __forceinline__ void lane_row_store(double *row, const double (&v)[32]) {
#pragma unroll
  for (int c = 0; c < 32; c += 4)
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(row + c), "d"(v[c]), "d"(v[c + 1]), "d"(v[c + 2]),
                 "d"(v[c + 3])
                 : "memory");
}
__device__ __forceinline__ void lane_row_store(float *row, const double (&v)[32]) {
#pragma unroll
  for (int c = 0; c < 32; c += 8)
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(row + c), "f"((float)v[c]),
                 "f"((float)v[c + 1]), "f"((float)v[c + 2]), "f"((float)v[c + 3]), "f"((float)v[c + 4]),
                 "f"((float)v[c + 5]), "f"((float)v[c + 6]), "f"((float)v[c + 7])
                 : "memory");
}
__device__ __forceinline__ void lane_row_load(const double *row, double (&v)[32]) {
#pragma unroll
  for (int c = 0; c < 32; c += 4)
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(v[c]), "=d"(v[c + 1]), "=d"(v[c + 2]), "=d"(v[c + 3])
                 : "l"(row + c));
}
__device__ __forceinline__ void lane_row_load(const float *row, double (&v)[32]) {
#pragma unroll
  for (int c = 0; c < 32; c += 8) {
    float f[8];
    asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(f[0]), "=f"(f[1]), "=f"(f[2]), "=f"(f[3]), "=f"(f[4]), "=f"(f[5]), "=f"(f[6]), "=f"(f[7])
                 : "l"(row + c));
#pragma unroll
    for (int k = 0; k < 8; ++k) v[c + k] = f[k];
  }
}

// The warps of the gather and the scatter: warp w takes rows 32 (w % chunks) + lane of group
// w / chunks, chunks = ceil(n / 32), each lane one row; blocks of kLaneIoWarps warps.
constexpr int kLaneIoWarps = 8;
__host__ __device__ inline int64_t lane_io_blocks(int64_t groups, int64_t n) {
  return (groups * ((n + 31) / 32) + kLaneIoWarps - 1) / kLaneIoWarps;
}

// b (natural rows, column-major, ldb) into the work array [group][work row][32 R values] (b's row i
// to work row in_pos[i]; the row's values are the group's 32 R columns in order, so lane l's R
// values are columns R l .. R l + R - 1); right-hand sides past `count` are zero. Each lane reads its
// row of the group's columns, 32 at a time, one coalesced load across the warp per column, and
// stores each 32-value piece of the work row in 32-byte pieces: no shared memory, no barrier.
template <class T, int R = 1>
__global__ void __launch_bounds__(kLaneIoWarps * 32) lane_in_kernel(const double *__restrict__ b, int64_t ldb, int64_t count,
                                                                   int32_t n, int64_t groups,
                                                                   const int32_t *__restrict__ in_pos,
                                                                   T *__restrict__ work,
                                                                   const uint8_t *__restrict__ group_active) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kLaneIoWarps + (threadIdx.x >> 5);
  const int64_t chunks = (n + 31) / 32, g = w / chunks;
  if (g >= groups || (group_active && !group_active[g])) return;
  const int i = (int)(w % chunks) * 32 + lane;
  if (i >= n) return;
  T *row = work + ((size_t)g * n + __ldg(in_pos + i)) * 32 * R;
#pragma unroll
  for (int h = 0; h < R; ++h) {
    double v[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) {
      const int64_t col = (g * R + h) * 32 + c;
      v[c] = col < count ? b[col * ldb + i] : 0.0;
    }
    lane_row_store(row + h * 32, v);
  }
}

// The work array (solutions in their work rows) into x (natural rows, column-major, ldx): x's
// row i from work row out_pos[i], the mirror of lane_in_kernel.
template <class T, int R = 1>
__global__ void __launch_bounds__(kLaneIoWarps * 32) lane_out_kernel(const T *__restrict__ work, int64_t count, int32_t n,
                                                                    int64_t groups, const int32_t *__restrict__ out_pos,
                                                                    double *__restrict__ x, int64_t ldx) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kLaneIoWarps + (threadIdx.x >> 5);
  const int64_t chunks = (n + 31) / 32, g = w / chunks;
  if (g >= groups) return;
  const int i = (int)(w % chunks) * 32 + lane;
  if (i >= n) return;
  const T *row = work + ((size_t)g * n + __ldg(out_pos + i)) * 32 * R;
#pragma unroll
  for (int h = 0; h < R; ++h) {
    double v[32];
    lane_row_load(row + h * 32, v);
#pragma unroll
    for (int c = 0; c < 32; ++c) {
      const int64_t col = (g * R + h) * 32 + c;
      if (col < count) x[col * ldx + i] = v[c];
    }
  }
}

}  // namespace yb
