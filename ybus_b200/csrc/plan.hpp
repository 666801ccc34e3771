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

}  // namespace yb
