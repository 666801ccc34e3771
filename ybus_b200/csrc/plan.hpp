// The symbolic phase of the GPU solve: from a factor's two triangles and its permutations, the
// level schedule of each sweep and the factor packed in that schedule's order.
//
// ybus_cuda hands its triangles to cuSPARSE's SpSM analysis once per (matrix, block width)
// (ybus_cuda/src/sparse.rs:228-300). Here the analysis is ours and independent of the width:
//
//   - forward sweep over the lower triangle: level(i) = 1 + max level(j) over its off-diagonal
//     columns j < i, rows grouped by level;
//   - backward sweep over the upper triangle: level(i) = 1 + max level(j) over j > i;
//   - each sweep's rows stored contiguously in level order: off-diagonal columns and values,
//     and the reciprocal of the diagonal (1 for a unit diagonal);
//   - the input permutation folded into the load (b's row r goes to slot in_slot[r]) and the
//     output permutation into the store (x's row r comes from slot out_slot[r]), so no host
//     packing or unpacking is needed (ybus_cuda/src/factor.rs:256-286 does both on the host).
#pragma once

#include <cstdint>
#include <vector>

#include "host/sparse.hpp"

namespace yb {

template <class T> struct Sweep {
  int32_t levels = 0;
  std::vector<int32_t> level_ptr;  // [levels + 1] positions
  std::vector<int32_t> row;        // [n] row at each position
  std::vector<int32_t> ptr;        // [n + 1] off-diagonal entries of each position
  std::vector<int32_t> col;        // [off-diagonal entries]
  std::vector<T> val;              // [off-diagonal entries]
  std::vector<T> dinv;             // [n] reciprocal of each position's diagonal
  std::vector<int32_t> level_of;   // [n] level of each row
  int32_t widest = 0;              // rows in the widest level
  int64_t entries() const { return (int64_t)col.size(); }
};

// A sweep cut into slices for the shared-memory tile solve: each level's rows, longest first,
// taken G at a time (one row per lane group of a warp). A slice's entries are stored entry-major
// (entry q of its G rows contiguous), so a warp reads entry q of all its rows in one coalesced
// access with no dependent index loads. Short rows are padded with (col = n, val = 0), which
// reads an always-zero slot; missing rows of a level's last slice write to slot n + 1.
template <class T> struct SliceSweep {
  int32_t G = 0, levels = 0;
  std::vector<int32_t> level_slice;  // [levels + 1] slice ranges
  std::vector<int32_t> offset, length;  // [slices] entry offset and padded row length
  std::vector<int32_t> row;          // [slices * G]
  std::vector<T> dinv;               // [slices * G]
  std::vector<int32_t> col;          // [entries]
  std::vector<T> val;                // [entries]
  int64_t slices() const { return (int64_t)offset.size(); }
};

// Cuts `s` into slices of G rows for a factor of order n.
template <class T> SliceSweep<T> slice_sweep(const Sweep<T> &s, int32_t n, int32_t G);

// The factor of both sweeps as per-warp streams of records in fixed-size pages, for the streamed
// tile solve. A record is a slice of up to 32 rows of one level (one row per lane, each lane
// keeping the tile's W sums in registers), or one long row split over the lanes, or a chunk of
// either (entries that do not fit one page
// continue in the next record). Each record carries the number of block barriers that must have
// passed before it runs (its stage). Levels with many rows ("wide") are dealt over all warps with a
// block barrier after each; the narrow levels at the top of the tree, at the end of the forward
// sweep and the start of the backward one, all go to warp 0, which takes them back to back with
// only warp-level synchronisation. Forward rows with no entries need no record: the load of b
// scales them by their diagonal (load_scale).
//
// With a dense tail (tail_level K > 0), the rows T at forward levels K and above (the top of the
// tree: every row that depends on a T row is in T) are solved as a block: forward, r_T = b_T −
// L_TB y_B for all T rows at once, then y_T = L_TT⁻¹ r_T; backward (when T is closed under the
// upper triangle's dependencies, as it is for a Cholesky factor), x_T = U_TT⁻¹ y_T first, then the
// remaining rows by their levels counted without T. The inverses are computed here in FP64 and
// applied as dense triangular matrix-vector products, which take one stage each instead of one
// per level of the chain of narrow levels at the top of the tree.
struct StreamLayout {
  int32_t G = 0, warps = 0, page_bytes = 0, stages = 0;
  int32_t fwd_wide = 0, bwd_wide = 0, fwd_narrow_rows = 0, bwd_narrow_rows = 0;
  int64_t records = 0;
  int32_t tail = 0;                 // |T|, 0 for no dense tail
  bool tail_backward = false;       // the backward sweep also takes T densely
  std::vector<int32_t> tail_slot;   // [tail] the slot of each T row, increasing
  std::vector<double> fwd_inv;      // packed lower triangle of L_TT⁻¹, row-major
  std::vector<double> bwd_inv;      // packed upper triangle of U_TT⁻¹, row-major
  std::vector<uint8_t> blob;        // pages of all warps
  std::vector<int32_t> warp_page;   // [warps + 1] page ranges in the blob
  std::vector<double> load_scale;   // [n] by row of b: the forward diagonal's reciprocal, or 1
};

enum RecordKind : int32_t {
  kRecordEnd = -1,
  kRecordSlice = 0,
  kRecordSplit = 1,
  kRecordDense = 2,
  kRecordCopy = 3,
  kRecordRows = 4
};
// kRecordToTail: a slice whose rows are tail indices; its results (unscaled) go to the tail buffer
enum RecordFlags : int32_t { kRecordFirst = 1, kRecordLast = 2, kRecordToTail = 4 };

// Builds the streams of a plan's sweeps for values of `value_bytes` (8 or 4) and tile width W.
template <class T> struct Plan;
template <class T>
StreamLayout stream_layout(const Plan<T> &plan, int32_t W, int32_t value_bytes, int32_t warps, int32_t page_bytes,
                           int32_t narrow_rows, int32_t tail_level = 0);

// The factor of both sweeps cut for the domain solve (domain_solve.cuh). The rows at forward level
// K and above form the top T; the rows below fall into domains, the connected groups of rows
// joined by dependencies of either sweep that avoid T (for a Cholesky factor, the subtrees of the
// elimination tree hanging under T). Each domain goes whole to one warp, balanced by work, and a
// warp takes its domains level by level with only warp synchronisation: no block barrier between
// the levels below K. T is solved as one dense block through the explicit inverses of L_TT and
// U_TT (computed here in FP64): forward r_T = b_T - L_TB y_B over all warps, then y_T =
// L_TT^-1 r_T; backward x_T = U_TT^-1 y_T, then the domains in their backward order. Valid when no
// upper-triangle entry of a T row reaches below T (always so for a Cholesky factor).
//
// Records, in each warp's pages (16-byte aligned parts):
//   kRecordRows:  int4 {kind, stage, rows, flags}, int4 {kl, entries, record bytes, 0},
//                 int4 {byte offsets of info, dinv, cols, vals in the record}, then int2 info per
//                 row {slot | len << 16, start | dest << 16}, T dinv per row, uint16 col per entry,
//                 T val per entry. 2^kl lanes take each row: r = Y[slot] - the sum of its len
//                 entries from `start`; then Y[dest] = r * dinv, or, with kRecordToTail, the tail
//                 buffer's entry dest = r.
//   kRecordSplit, kRecordDense, kRecordCopy: as for the streamed solve; a split record's second
//                 header word is its destination, with kRecordToTail an entry of the tail buffer.
struct DomainLayout {
  int32_t warps = 0, page_bytes = 0, value_bytes = 0, stages = 0;
  int32_t K = 0;                    // first forward level of T (levels of the tree cut)
  int32_t tail = 0;                 // |T|
  std::vector<int32_t> tail_slot;   // [tail] slot of each T row
  std::vector<uint8_t> blob;        // pages of all warps
  std::vector<int32_t> warp_page;   // [warps + 1]
  int64_t records = 0, entries = 0, dense_entries = 0;
  double cost = 0;                  // the cost model's estimate for the chosen K (cycles per tile)
  double top_condition = 0;         // infinity-norm condition of the worse of L_TT and U_TT (0: no T)
};

// Builds the domain layout of `plan` for values of `value_bytes` (8 or 4). K < 0 picks the cut by
// a cost model; K = 0 puts every row into T (a dense solve). Throws host::Error if the factor does
// not admit the cut (kInvalidArgument) or the order does not fit 16-bit slots (kTooLarge).
template <class T>
DomainLayout domain_layout(const Plan<T> &plan, int32_t value_bytes, int32_t warps, int32_t page_bytes, int32_t K);

// The factor for the lane solve (lane_solve.cuh: one right-hand side per lane, every lane of a warp
// taking the same rows, `warps` warps per block of 32 right-hand sides). The rows are in a postorder
// of the forward elimination forest with larger subtrees first, cut into subtree domains (dealt to
// the warps) under a top (between the first and second block barriers every warp adds the domains'
// partial sums of a share of the top rows into their right-hand sides; the top itself is solved
// between the second and fourth, as a dense map every warp takes a share of in FP64, else by warp
// 0 as a chain); each warp's part is one stream of records in fixed-size pages.
//
// A record is a 16-byte header, then `count` entries of 16 bytes (FP64) or 8 (FP32): {T val, or a
// 32-bit word in its place; uint32 offset}. The header: uint32 {self (16 bits), kind (5 bits), ring
// slot (3 bits), count (8 bits)}, uint32 word, then 8 bytes: T dinv for rows. Offsets are byte offsets of 32-value live slots (slot 0 is always zero, slot 1 a sink),
// `self` such an offset / 16; words are byte offsets of 32-value rows of the work or partial array.
//   kLaneFwdRow0 + c (c = 0..4 entries), kLaneFwdRowN, kLaneFwdMore: a forward row at work offset
//     `word`: read and zero acc at self, z = (b + acc) * dinv with b from its ring slot, z into the
//     work row, then acc[offset] -= val * z per entry (kLaneFwdMore: more entries of the last row).
//   kLaneBwdRow0 + c, kLaneBwdRowN, or kLaneBwdBegin, kLaneBwdMore..., kLaneBwdEnd: a backward row:
//     acc = z from its ring slot minus val * x[offset] per entry, x = acc * dinv into the work row
//     and into slot self.
//   kLaneFwdPre1 + c - 1, kLaneBwdPre1 + c - 1 (c = 1..4 entries): the row of kind kLaneFwdRow0 + c
//     (kLaneBwdRow0 + c) that opens a batch, its entries followed by a 16-byte prefetch block (the
//     header's count is c + 16 / entry bytes): the prefetch block's copies run first, as a
//     kLanePrefetch record's would.
//   kLanePrefetch: its 16 bytes of entries are a prefetch block: kLaneBatch uint32 work-row
//     offsets, the first with the row count (up to kLaneBatch) in bits 0-2 and the upper-half flag
//     in bit 3; the rows are copied into the ring's lower (or upper) kLaneBatch slots, then the
//     batch before them is waited for.
//   kLanePhase: a new run of rows: earlier copies are finished and this lane's stores are visible
//     to its copies.
//   kLaneFlush: per entry, the partial row `word` takes slot `offset`, which is zeroed.
//   kLaneTopSum: the work row `word` += the partial rows of its entries' words, in order (mode
//     kTopSums); mode kTopLoad: per entry, slot `offset` takes the work row `word`; modes kTopRow
//     and kTopRowMore: the output row `word` = (0, or its value so far) + val * the value at the
//     block-wide shared offset `offset` (another warp's slot), per entry in order.
//   kLaneImport: per entry, slot `offset` takes the work row `word`.
//   kLaneBarrier: a block barrier (every warp's stream has four); kLaneEnd ends the stream;
//   kLanePageEnd ends its page (every page has one).
enum LaneKind : uint32_t {
  kLaneFwdRow0 = 0,  // .. kLaneFwdRow0 + 4
  kLaneFwdPre1 = 5,  // .. kLaneFwdPre1 + 3
  kLaneBwdRow0 = 9,  // .. kLaneBwdRow0 + 4
  kLaneBwdPre1 = 14,  // .. kLaneBwdPre1 + 3
  kLaneFwdRowN = 18,
  kLaneFwdMore = 19,
  kLaneBwdRowN = 20,
  kLaneBwdBegin = 21,
  kLaneBwdMore = 22,
  kLaneBwdEnd = 23,
  kLanePrefetch = 24,
  kLanePhase = 25,
  kLaneTopSum = 26,
  kLaneFlush = 27,
  kLaneImport = 28,
  kLaneBarrier = 29,
  kLaneEnd = 30,
  kLanePageEnd = 31
};
// The modes of a kLaneTopSum record (the header's third word): the top rows' partial sums, or one
// of the dense top's records: a warp's share of the top's right-hand sides into its slots, or a
// top row's solution as a dense row over every warp's slots (the first record of the row, or one
// continuing it).
enum LaneTopMode : uint32_t { kTopSums = 0, kTopLoad = 1, kTopRow = 2, kTopRowMore = 3 };
constexpr int kLaneDenseTopMost = 192;  // the largest top taken as a dense map
constexpr double kLaneDenseTopCondition = 1e8;  // the largest condition of that map
constexpr int kLaneBatch = 4;              // work rows per prefetch
constexpr int kLaneRows = 2 * kLaneBatch;  // slots of a warp's prefetch ring
constexpr int kLaneRing = 2;               // pages in flight per warp (a power of two)
constexpr int kLaneBarriers = 4;           // block barriers in every warp's stream

#if defined(__CUDACC__)
#define YB_HOST_DEVICE __host__ __device__
#else
#define YB_HOST_DEVICE
#endif

// A lane-solve warp's shared memory: live slots, the prefetch ring, the page ring and its
// barriers, for values of `value_bytes` and `rpl` right-hand sides per lane (a slot and a ring row
// hold 32 * rpl values), rounded to 128 bytes; warp w's part starts at w times this. The layout
// builder writes offsets into other warps' slots from it, the kernel places each warp's part by it.
inline YB_HOST_DEVICE size_t lane_warp_bytes_of(int32_t value_bytes, int32_t slots, int32_t ring, int32_t page_bytes,
                                                int32_t rpl) {
  const size_t row = (size_t)32 * value_bytes * rpl;
  const size_t b = (size_t)slots * row + (size_t)kLaneRows * row + (size_t)ring * page_bytes + (size_t)ring * 8;
  return (b + 127) & ~(size_t)127;
}
struct LaneLayout {
  int32_t warps = 1, slots = 0, page_bytes = 0, value_bytes = 0;
  int32_t rpl = 1;  // right-hand sides per lane: a slot or row holds 32 * rpl values
  int32_t domains = 0, top = 0, partials = 0;  // partials: partial-array values per block
  bool dense_top = false;                      // the top is solved as a dense map by every warp
  double top_condition = 0;                    // that map's condition (0: not computed)
  int32_t fwd_live = 0, bwd_live = 0;          // the peak number of live values in each sweep
  int64_t fwd_entries = 0, bwd_entries = 0;
  double cost = 0;                             // the cut's estimate of a block's time (work units)
  std::vector<uint8_t> blob;                   // every warp's pages
  std::vector<int32_t> warp_page;              // [warps + 1] page ranges
  std::vector<int32_t> in_pos;                 // [n] by row of b: its position in the work array
  std::vector<int32_t> out_pos;                // [n] by row of x: its position
};

template <class T> struct Plan {
  int32_t n = 0;
  std::vector<int32_t> in_slot, out_slot;   // [n]
  std::vector<int32_t> in_row, out_row;     // [n] inverses: slot -> original row
  Sweep<T> fwd, bwd;
};

// Builds a plan from CSR triangles (both with every row's diagonal stored, unless `unit_lower`,
// whose diagonal is taken as 1 whether stored or not). `in_perm[i]` is the row of b that slot i
// takes; `out_perm[i]` the row of x that slot i gives. Throws host::Error on invalid input.
template <class T>
Plan<T> build_plan(int64_t n, const host::Compressed<T> &lower, bool unit_lower,
                   const host::Compressed<T> &upper, const std::vector<int64_t> &in_perm,
                   const std::vector<int64_t> &out_perm);

// Builds the lane layout of `plan` for values of `value_bytes` (8 or 4), `warps` warps per block and
// `rpl` (1 or 2) right-hand sides per lane: the records are the same but for their byte offsets,
// which count slots and rows of 32 * rpl values. Throws host::Error (kInvalidArgument) when no
// postorder serves both sweeps, or (kTooLarge) when more than `max_slots` slots would be needed.
template <class T>
LaneLayout lane_layout(const Plan<T> &plan, int32_t value_bytes, int32_t page_bytes, int32_t max_slots, int32_t warps,
                       int32_t rpl = 1);

}  // namespace yb
