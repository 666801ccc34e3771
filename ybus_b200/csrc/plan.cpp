#include "plan.hpp"

#include <limits>
#include <string>

namespace yb {

using host::Error;
using host::idx_t;

namespace {

void check_permutation(const std::vector<int64_t> &perm, int64_t n, const char *name) {
  if ((int64_t)perm.size() != n) throw Error(host::kShapeMismatch, std::string(name) + " has the wrong length");
  std::vector<char> seen(n, 0);
  for (int64_t v : perm) {
    if (v < 0 || v >= n || seen[v]) throw Error(host::kInvalidArgument, std::string(name) + " is not a permutation");
    seen[v] = 1;
  }
}

template <class T>
Sweep<T> pack(const host::Compressed<T> &m, bool lower, bool unit) {
  const idx_t n = m.rows;
  Sweep<T> s;
  s.level_of.assign(n, 0);
  std::vector<T> diag(n, T(0));
  std::vector<char> has_diag(n, 0);
  // Validate and find each row's diagonal
  for (idx_t i = 0; i < n; ++i) {
    for (idx_t p = m.ptr[i]; p < m.ptr[i + 1]; ++p) {
      const idx_t j = m.idx[p];
      if (j < 0 || j >= n) throw Error(host::kInvalidArgument, "a factor index is out of range");
      if (lower ? j > i : j < i)
        throw Error(host::kInvalidArgument, lower ? "the lower factor has an entry above its diagonal"
                                                   : "the upper factor has an entry below its diagonal");
      if (j == i) {
        if (has_diag[i]) throw Error(host::kInvalidArgument, "a factor row stores its diagonal twice");
        has_diag[i] = 1;
        diag[i] = m.val[p];
      }
    }
    if (unit) {
      diag[i] = T(1);
    } else if (!has_diag[i] || diag[i] == T(0)) {
      throw Error(host::kSingular, "a factor row has no nonzero diagonal", i);
    }
  }
  // Levels: lower in increasing row order, upper in decreasing
  int32_t levels = 0;
  auto level_row = [&](idx_t i) {
    int32_t l = 0;
    for (idx_t p = m.ptr[i]; p < m.ptr[i + 1]; ++p) {
      const idx_t j = m.idx[p];
      if (j != i) l = std::max(l, s.level_of[j] + 1);
    }
    s.level_of[i] = l;
    levels = std::max(levels, l + 1);
  };
  if (lower)
    for (idx_t i = 0; i < n; ++i) level_row(i);
  else
    for (idx_t i = n - 1; i >= 0; --i) level_row(i);
  s.levels = levels;
  s.level_ptr.assign(levels + 1, 0);
  for (idx_t i = 0; i < n; ++i) s.level_ptr[s.level_of[i] + 1]++;
  for (int32_t l = 0; l < levels; ++l) {
    s.widest = std::max(s.widest, s.level_ptr[l + 1]);
    s.level_ptr[l + 1] += s.level_ptr[l];
  }
  s.row.assign(n, 0);
  {
    std::vector<int32_t> cursor(s.level_ptr.begin(), s.level_ptr.end() - 1);
    // Rows of a level in increasing order for the lower sweep, decreasing for the upper
    if (lower)
      for (idx_t i = 0; i < n; ++i) s.row[cursor[s.level_of[i]]++] = (int32_t)i;
    else
      for (idx_t i = n - 1; i >= 0; --i) s.row[cursor[s.level_of[i]]++] = (int32_t)i;
  }
  s.ptr.assign(n + 1, 0);
  s.dinv.assign(n, T(0));
  for (idx_t k = 0; k < n; ++k) {
    const idx_t i = s.row[k];
    for (idx_t p = m.ptr[i]; p < m.ptr[i + 1]; ++p)
      if (m.idx[p] != i) {
        s.col.push_back((int32_t)m.idx[p]);
        s.val.push_back(m.val[p]);
      }
    if ((int64_t)s.col.size() > std::numeric_limits<int32_t>::max())
      throw Error(host::kTooLarge, "the factor has too many entries for 32-bit indices");
    s.ptr[k + 1] = (int32_t)s.col.size();
    s.dinv[k] = T(1) / diag[i];
  }
  return s;
}

}  // namespace

template <class T>
Plan<T> build_plan(int64_t n, const host::Compressed<T> &lower, bool unit_lower, const host::Compressed<T> &upper,
                   const std::vector<int64_t> &in_perm, const std::vector<int64_t> &out_perm) {
  if (n < 0) throw Error(host::kInvalidArgument, "negative order");
  if (n > std::numeric_limits<int32_t>::max() / 64) throw Error(host::kTooLarge, "the order is too large for 32-bit indices");
  for (const auto *m : {&lower, &upper}) {
    if (!m->by_rows || m->rows != n || m->cols != n || (int64_t)m->ptr.size() != n + 1)
      throw Error(host::kShapeMismatch, "a triangle does not have the factor's order");
    if (m->ptr[0] != 0) throw Error(host::kInvalidArgument, "a triangle's pointers do not start at 0");
    for (int64_t i = 0; i < n; ++i)
      if (m->ptr[i + 1] < m->ptr[i]) throw Error(host::kInvalidArgument, "a triangle's pointers decrease");
    if (m->ptr[n] != (int64_t)m->idx.size() || m->idx.size() != m->val.size())
      throw Error(host::kInvalidArgument, "a triangle's arrays disagree in length");
  }
  check_permutation(in_perm, n, "the row permutation");
  check_permutation(out_perm, n, "the column permutation");
  Plan<T> plan;
  plan.n = (int32_t)n;
  plan.in_row.assign(in_perm.begin(), in_perm.end());
  plan.out_row.assign(out_perm.begin(), out_perm.end());
  plan.in_slot.assign(n, 0);
  plan.out_slot.assign(n, 0);
  for (int64_t i = 0; i < n; ++i) {
    plan.in_slot[in_perm[i]] = (int32_t)i;
    plan.out_slot[out_perm[i]] = (int32_t)i;
  }
  plan.fwd = pack(lower, true, unit_lower);
  plan.bwd = pack(upper, false, false);
  return plan;
}

template <class T> SliceSweep<T> slice_sweep(const Sweep<T> &s, int32_t n, int32_t G) {
  if (G < 1 || G > 32) throw Error(host::kInvalidArgument, "slice width must be 1 to 32");
  SliceSweep<T> out;
  out.G = G;
  out.levels = s.levels;
  out.level_slice.assign(1, 0);
  std::vector<int32_t> rows;
  for (int32_t l = 0; l < s.levels; ++l) {
    rows.assign(s.row.begin() + s.level_ptr[l], s.row.begin() + s.level_ptr[l + 1]);
    // positions k of this level, longest rows first (stable by position)
    std::vector<int32_t> ks(rows.size());
    for (size_t t = 0; t < ks.size(); ++t) ks[t] = s.level_ptr[l] + (int32_t)t;
    std::stable_sort(ks.begin(), ks.end(), [&](int32_t a, int32_t b) {
      return (s.ptr[a + 1] - s.ptr[a]) > (s.ptr[b + 1] - s.ptr[b]);
    });
    for (size_t t0 = 0; t0 < ks.size(); t0 += G) {
      const size_t t1 = std::min(ks.size(), t0 + (size_t)G);
      int32_t len = 0;
      for (size_t t = t0; t < t1; ++t) len = std::max(len, s.ptr[ks[t] + 1] - s.ptr[ks[t]]);
      out.offset.push_back((int32_t)out.col.size());
      out.length.push_back(len);
      for (int32_t g = 0; g < G; ++g) {
        const size_t t = t0 + g;
        if (t < t1) {
          out.row.push_back(s.row[ks[t]]);
          out.dinv.push_back(s.dinv[ks[t]]);
        } else {
          out.row.push_back(n + 1);
          out.dinv.push_back(T(0));
        }
      }
      for (int32_t q = 0; q < len; ++q)
        for (int32_t g = 0; g < G; ++g) {
          const size_t t = t0 + g;
          if (t < t1 && q < s.ptr[ks[t] + 1] - s.ptr[ks[t]]) {
            const int32_t p = s.ptr[ks[t]] + q;
            out.col.push_back(s.col[p]);
            out.val.push_back(s.val[p]);
          } else {
            out.col.push_back(n);
            out.val.push_back(T(0));
          }
        }
      if ((int64_t)out.col.size() > std::numeric_limits<int32_t>::max())
        throw Error(host::kTooLarge, "the sliced factor has too many entries for 32-bit offsets");
    }
    out.level_slice.push_back((int32_t)out.offset.size());
  }
  return out;
}

template SliceSweep<double> slice_sweep(const Sweep<double> &, int32_t, int32_t);

template Plan<double> build_plan(int64_t, const host::Compressed<double> &, bool, const host::Compressed<double> &,
                                 const std::vector<int64_t> &, const std::vector<int64_t> &);
template Plan<host::c128> build_plan(int64_t, const host::Compressed<host::c128> &, bool,
                                     const host::Compressed<host::c128> &, const std::vector<int64_t> &,
                                     const std::vector<int64_t> &);

}  // namespace yb
