// Host-side diagnostics of the GPU solves' layouts (no GPU needed): the domain solve's and the
// lane solve's records for a Cholesky factor given as yb_factor_from_cholesky takes it, and the
// lane solve's for an LU factor given as yb_factor_from_lu takes it, built by the same code the
// upload runs (domain.cpp, lane.cpp), so tests can interpret them on the CPU.
#include <algorithm>
#include <vector>

#include "../../include/ybgpu.h"
#include "capi_common.hpp"
#include "plan.hpp"

using namespace yb;

namespace {

// A square compressed matrix from caller arrays, checked (by rows or by columns).
host::Compressed<double> compressed(int64_t n, const int64_t *ptr, const int64_t *idx, const double *val,
                                    bool by_rows) {
  host::Compressed<double> m;
  m.rows = m.cols = n;
  m.by_rows = by_rows;
  m.ptr.assign(ptr, ptr + n + 1);
  require(m.ptr[0] == 0, "pointers must start at 0");
  for (int64_t i = 0; i < n; ++i) require(m.ptr[i + 1] >= m.ptr[i], "pointers must not decrease");
  const int64_t nnz = m.ptr[n];
  require(nnz == 0 || (idx && val), "null index or value array");
  m.idx.assign(idx, idx + nnz);
  m.val.assign(val, val + nnz);
  for (int64_t v : m.idx) require(v >= 0 && v < n, "an index is out of range");
  return m;
}

void lane_outputs(const LaneLayout &lay, int64_t *info, uint8_t *blob, int32_t *warp_page, int32_t *in_pos,
                  int32_t *out_pos) {
  const int64_t v[12] = {lay.slots, lay.warp_page.back(), lay.page_bytes, lay.fwd_live, lay.bwd_live, lay.fwd_entries,
                         lay.bwd_entries, lay.warps, lay.domains, lay.top, lay.partials, lay.rpl};
  std::copy(v, v + 12, info);
  if (blob) std::copy(lay.blob.begin(), lay.blob.end(), blob);
  if (warp_page) std::copy(lay.warp_page.begin(), lay.warp_page.end(), warp_page);
  if (in_pos) std::copy(lay.in_pos.begin(), lay.in_pos.end(), in_pos);
  if (out_pos) std::copy(lay.out_pos.begin(), lay.out_pos.end(), out_pos);
}

}  // namespace

extern "C" {

int32_t yb_domain_layout_cholesky(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                                  const int64_t *perm, int32_t value_bytes, int32_t warps, int32_t page_bytes,
                                  int32_t cut, int64_t *info, uint8_t *blob, int32_t *warp_page, int32_t *top_slot,
                                  double *top_condition) {
  return guard([&] {
    require(n >= 0 && l_ptr && perm && info, "null argument");
    host::Compressed<double> lower = compressed(n, l_ptr, l_idx, l_val, true);
    host::Compressed<double> upper = host::reorient(lower);
    upper.by_rows = true;
    std::vector<int64_t> p(perm, perm + n);
    const Plan<double> plan = build_plan<double>(n, lower, false, upper, p, p);
    const DomainLayout lay = domain_layout(plan, value_bytes, warps, page_bytes, cut);
    const int64_t pages = lay.warp_page.back();
    const int64_t v[8] = {lay.K, lay.tail, lay.stages, lay.warps, pages, lay.records, lay.entries, lay.page_bytes};
    std::copy(v, v + 8, info);
    if (blob) std::copy(lay.blob.begin(), lay.blob.end(), blob);
    if (warp_page) std::copy(lay.warp_page.begin(), lay.warp_page.end(), warp_page);
    if (top_slot) std::copy(lay.tail_slot.begin(), lay.tail_slot.end(), top_slot);
    if (top_condition) *top_condition = lay.top_condition;
    return YB_OK;
  });
}

int32_t yb_lane_layout_cholesky(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                                const int64_t *perm, int32_t value_bytes, int32_t page_bytes, int32_t max_slots,
                                int32_t warps, int32_t rhs_per_lane, int64_t *info, uint8_t *blob, int32_t *warp_page,
                                int32_t *in_pos, int32_t *out_pos) {
  return guard([&] {
    require(n >= 0 && l_ptr && perm && info, "null argument");
    host::Compressed<double> lower = compressed(n, l_ptr, l_idx, l_val, true);
    host::Compressed<double> upper = host::reorient(lower);
    upper.by_rows = true;
    std::vector<int64_t> p(perm, perm + n);
    const Plan<double> plan = build_plan<double>(n, lower, false, upper, p, p);
    lane_outputs(lane_layout(plan, value_bytes, page_bytes, max_slots, warps, rhs_per_lane), info, blob, warp_page,
                 in_pos, out_pos);
    return YB_OK;
  });
}

int32_t yb_lane_layout_lu(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                          const int64_t *u_ptr, const int64_t *u_idx, const double *u_val, const int64_t *row_perm,
                          const int64_t *col_perm, int32_t value_bytes, int32_t page_bytes, int32_t max_slots,
                          int32_t warps, int32_t rhs_per_lane, int64_t *info, uint8_t *blob, int32_t *warp_page,
                          int32_t *in_pos, int32_t *out_pos) {
  return guard([&] {
    require(n >= 0 && l_ptr && u_ptr && info && (n == 0 || (row_perm && col_perm)), "null argument");
    // as yb_factor_from_lu builds its plan: the CSC triangles read by rows, L's diagonal unit
    const host::Compressed<double> lower = host::reorient(compressed(n, l_ptr, l_idx, l_val, false));
    const host::Compressed<double> upper = host::reorient(compressed(n, u_ptr, u_idx, u_val, false));
    std::vector<int64_t> p(row_perm, row_perm + n), q(col_perm, col_perm + n);
    const Plan<double> plan = build_plan<double>(n, lower, true, upper, p, q);
    lane_outputs(lane_layout(plan, value_bytes, page_bytes, max_slots, warps, rhs_per_lane), info, blob, warp_page,
                 in_pos, out_pos);
    return YB_OK;
  });
}

}  // extern "C"
