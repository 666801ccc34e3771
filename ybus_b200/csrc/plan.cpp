#include "plan.hpp"

#include <complex>
#include <cstring>
#include <limits>
#include <functional>
#include <memory>
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

namespace yb {

namespace {

inline int64_t align16(int64_t v) { return (v + 15) & ~int64_t(15); }

// Appends records to one warp's pages.
struct PageWriter {
  int32_t page_bytes;
  std::vector<uint8_t> &blob;
  int64_t page_start = -1, pos = 0;
  int32_t pages = 0;
  PageWriter(int32_t pb, std::vector<uint8_t> &b) : page_bytes(pb), blob(b) {}
  void close_page() {
    if (page_start < 0) return;
    if (pos + 16 <= page_bytes) {
      int32_t end[4] = {kRecordEnd, 0, 0, 0};
      std::memcpy(blob.data() + page_start + pos, end, 16);
    }
    page_start = -1;
  }
  uint8_t *reserve(int64_t bytes) {
    if (bytes > page_bytes) throw Error(host::kInternal, "a stream record does not fit a page");
    if (page_start < 0 || pos + bytes > page_bytes) {
      close_page();
      page_start = (int64_t)blob.size();
      blob.resize(blob.size() + page_bytes, 0);
      pos = 0;
      ++pages;
    }
    uint8_t *p = blob.data() + page_start + pos;
    pos += bytes;
    return p;
  }
};

template <class V> void put(uint8_t *&p, const V *v, int64_t count) {
  std::memcpy(p, v, sizeof(V) * count);
  p += align16(sizeof(V) * count);
}

}  // namespace

template <class T>
StreamLayout stream_layout(const Plan<T> &plan, int32_t W, int32_t value_bytes, int32_t warps, int32_t page_bytes,
                           int32_t narrow_rows, int32_t tail_level) {
  if (W < 1 || W > 32 || 32 % W) throw Error(host::kInvalidArgument, "tile width must divide 32");
  if (value_bytes != 8 && value_bytes != 4) throw Error(host::kInvalidArgument, "values are 4 or 8 bytes");
  if (warps < 1 || page_bytes < 256 || page_bytes % 16) throw Error(host::kInvalidArgument, "bad stream shape");
  const int32_t n = plan.n, G = 32;  // a slice: one row per lane, each lane holding all W sums
  StreamLayout out;
  out.G = G;
  out.warps = warps;
  out.page_bytes = page_bytes;
  out.load_scale.assign(n, 1.0);
  // values written at value_bytes: double or float
  auto put_values = [&](uint8_t *&p, const std::vector<double> &v) {
    if (value_bytes == 8) {
      put(p, v.data(), (int64_t)v.size());
    } else {
      std::vector<float> f(v.begin(), v.end());
      put(p, f.data(), (int64_t)f.size());
    }
  };
  const int64_t head = 16;
  const int64_t slice_fixed = head + align16(4 * G) + align16((int64_t)value_bytes * G);
  // entries per record so a chunk fits a page (both arrays padded to 16 bytes)
  const int64_t slice_len_max = (page_bytes - slice_fixed - 32) / ((int64_t)G * (4 + value_bytes));
  const int64_t split_fixed = head + 16 + 16;
  const int64_t split_ent_max = ((page_bytes - split_fixed - 32) / (4 + value_bytes)) / G * G;
  if (slice_len_max < 1 || split_ent_max < G) throw Error(host::kInvalidArgument, "pages too small for the tile width");

  std::vector<std::unique_ptr<PageWriter>> writers;
  std::vector<std::vector<uint8_t>> blobs(warps);
  for (int32_t w = 0; w < warps; ++w) writers.emplace_back(new PageWriter(page_bytes, blobs[w]));

  // Entries of position k of sweep s that a record takes: all, or (for the tail's partial sums)
  // only those in columns outside the tail
  std::vector<char> in_tail(n, 0);
  auto entries_of = [&](const Sweep<T> &s, int32_t k, bool outside_tail) {
    std::vector<int32_t> ps;
    for (int32_t p = s.ptr[k]; p < s.ptr[k + 1]; ++p)
      if (!outside_tail || !in_tail[s.col[p]]) ps.push_back(p);
    return ps;
  };
  // A slice record (chunked): rows ks (positions of sweep s). to_tail: rows become tail indices
  // `tail_index[g]`, only entries outside the tail are taken and the result is left unscaled.
  auto emit_slice = [&](int32_t w, const Sweep<T> &s, const std::vector<int32_t> &ks, int32_t stage,
                        const std::vector<int32_t> *tail_index = nullptr) {
    const bool to_tail = tail_index != nullptr;
    std::vector<std::vector<int32_t>> ents;
    int32_t len = 0;
    for (int32_t k : ks) {
      ents.push_back(entries_of(s, k, to_tail));
      len = std::max(len, (int32_t)ents.back().size());
    }
    std::vector<int32_t> rows(G, to_tail ? 0 : n + 1);
    std::vector<double> dinv(G, 0.0);
    for (size_t g = 0; g < ks.size(); ++g) {
      rows[g] = to_tail ? (*tail_index)[g] : s.row[ks[g]];
      dinv[g] = to_tail ? 1.0 : (double)std::real(s.dinv[ks[g]]);
    }
    if (to_tail)  // padded rows of a tail record accumulate nothing into a spare tail entry
      for (size_t g = ks.size(); g < (size_t)G; ++g) rows[g] = out.tail;
    int32_t q0 = 0;
    do {
      const int32_t q1 = (int32_t)std::min<int64_t>(len, q0 + slice_len_max);
      const int32_t m = q1 - q0;
      const int64_t bytes = slice_fixed + align16(4LL * m * G) + align16((int64_t)value_bytes * m * G);
      uint8_t *p = writers[w]->reserve(bytes);
      int32_t hdr[4] = {kRecordSlice, stage, m,
                        (q0 == 0 ? kRecordFirst : 0) | (q1 == len ? kRecordLast : 0) | (to_tail ? kRecordToTail : 0)};
      put(p, hdr, 4);
      put(p, rows.data(), G);
      put_values(p, dinv);
      std::vector<int32_t> col((size_t)m * G, n);
      std::vector<double> val((size_t)m * G, 0.0);
      for (int32_t q = q0; q < q1; ++q)
        for (size_t g = 0; g < ks.size(); ++g) {
          if (q < (int32_t)ents[g].size()) {
            const int32_t pp = ents[g][q];
            col[(size_t)(q - q0) * G + g] = s.col[pp];
            val[(size_t)(q - q0) * G + g] = (double)std::real(s.val[pp]);
          }
        }
      put(p, col.data(), (int64_t)col.size());
      put_values(p, val);
      ++out.records;
      q0 = q1;
    } while (q0 < len);
  };
  // A copy marker: the warp copies its share of the tail's slots into the tail buffer
  auto emit_marker = [&](int32_t w, int32_t kind, int32_t stage, int32_t sweep) {
    uint8_t *p = writers[w]->reserve(16);
    int32_t hdr[4] = {kind, stage, sweep, 0};
    put(p, hdr, 4);
    ++out.records;
  };
  // Dense rows of a tail inverse (chunked): row t, columns [j0, j0 + count) of `inv`, where
  // packed(t, j) gives a value's index; the product with the tail buffer goes to t's slot
  const int64_t dense_fixed = head + 16;
  const int64_t dense_max = (page_bytes - dense_fixed - 16) / value_bytes / 4 * 4;
  auto emit_dense_row = [&](int32_t w, const std::vector<double> &inv, int32_t t, int32_t j_first, int32_t count,
                            auto packed, int32_t stage) {
    int32_t e0 = 0;
    do {
      const int32_t e1 = (int32_t)std::min<int64_t>(count, e0 + dense_max);
      const int32_t m = e1 - e0;
      uint8_t *p = writers[w]->reserve(dense_fixed + align16((int64_t)value_bytes * m));
      int32_t hdr[4] = {kRecordDense, stage, m, (e0 == 0 ? kRecordFirst : 0) | (e1 == count ? kRecordLast : 0)};
      put(p, hdr, 4);
      int32_t where[4] = {t, j_first + e0, 0, 0};
      put(p, where, 4);
      std::vector<double> v(m);
      for (int32_t e = e0; e < e1; ++e) v[e - e0] = inv[packed(t, j_first + e)];
      put_values(p, v);
      ++out.records;
      e0 = e1;
    } while (e0 < count);
  };
  // A split-row record (chunked): one row's entries spread over the G lane groups
  auto emit_split = [&](int32_t w, const Sweep<T> &s, int32_t k, int32_t stage) {
    const int32_t len = s.ptr[k + 1] - s.ptr[k];
    int32_t e0 = 0;
    do {
      const int32_t e1 = (int32_t)std::min<int64_t>(len, e0 + split_ent_max);
      const int32_t m = (int32_t)(((e1 - e0) + G - 1) / G * G);
      const int64_t bytes = split_fixed + align16(4LL * m) + align16((int64_t)value_bytes * m);
      uint8_t *p = writers[w]->reserve(bytes);
      int32_t hdr[4] = {kRecordSplit, stage, m, (e0 == 0 ? kRecordFirst : 0) | (e1 == len ? kRecordLast : 0)};
      put(p, hdr, 4);
      int32_t row[4] = {s.row[k], 0, 0, 0};
      put(p, row, 4);
      std::vector<double> dv(16 / value_bytes, 0.0);
      dv[0] = (double)std::real(s.dinv[k]);
      put_values(p, dv);
      std::vector<int32_t> col(m, n);
      std::vector<double> val(m, 0.0);
      for (int32_t e = e0; e < e1; ++e) {
        col[e - e0] = s.col[s.ptr[k] + e];
        val[e - e0] = (double)std::real(s.val[s.ptr[k] + e]);
      }
      put(p, col.data(), m);
      put_values(p, val);
      ++out.records;
      e0 = e1;
    } while (e0 < len);
  };
  auto sorted_level = [](const Sweep<T> &s, int32_t l) {
    std::vector<int32_t> ks;
    for (int32_t k = s.level_ptr[l]; k < s.level_ptr[l + 1]; ++k) ks.push_back(k);
    std::stable_sort(ks.begin(), ks.end(),
                     [&](int32_t a, int32_t b) { return (s.ptr[a + 1] - s.ptr[a]) > (s.ptr[b + 1] - s.ptr[b]); });
    return ks;
  };
  auto rows_of = [](const Sweep<T> &s, int32_t l) { return s.level_ptr[l + 1] - s.level_ptr[l]; };
  const Sweep<T> &F = plan.fwd, &B = plan.bwd;
  // The dense tail: rows at forward level >= tail_level
  const bool dense_tail = tail_level > 0 && tail_level < F.levels;
  std::vector<int32_t> tail_index(n, -1);
  if (dense_tail) {
    for (int32_t i = 0; i < n; ++i)
      if (F.level_of[i] >= tail_level) {
        tail_index[i] = (int32_t)out.tail_slot.size();
        out.tail_slot.push_back(i);
        in_tail[i] = 1;
      }
    out.tail = (int32_t)out.tail_slot.size();
    // Backward closure: every upper-triangle dependency of a tail row is a tail row
    out.tail_backward = true;
    for (int32_t k = 0; k < n && out.tail_backward; ++k)
      if (in_tail[B.row[k]])
        for (int32_t p = B.ptr[k]; p < B.ptr[k + 1]; ++p)
          if (!in_tail[B.col[p]]) {
            out.tail_backward = false;
            break;
          }
    // L_TT and U_TT (dense, in tail order, diagonal included) and their inverses in FP64
    const int32_t m = out.tail;
    std::vector<double> Lt((size_t)m * m, 0.0), Ut((size_t)m * m, 0.0);
    for (int32_t k = 0; k < n; ++k) {
      const int32_t i = F.row[k];
      if (!in_tail[i]) continue;
      const int32_t a = tail_index[i];
      Lt[(size_t)a * m + a] = 1.0 / (double)std::real(F.dinv[k]);
      for (int32_t p = F.ptr[k]; p < F.ptr[k + 1]; ++p)
        if (in_tail[F.col[p]]) Lt[(size_t)a * m + tail_index[F.col[p]]] = (double)std::real(F.val[p]);
    }
    // inverse of a lower triangle by columns: solve L z = e_c
    out.fwd_inv.assign((size_t)m * (m + 1) / 2, 0.0);
    std::vector<double> z(m);
    for (int32_t col = 0; col < m; ++col) {
      std::fill(z.begin(), z.end(), 0.0);
      for (int32_t i = col; i < m; ++i) {
        double acc = (i == col) ? 1.0 : 0.0;
        for (int32_t j = col; j < i; ++j) acc -= Lt[(size_t)i * m + j] * z[j];
        z[i] = acc / Lt[(size_t)i * m + i];
        out.fwd_inv[(size_t)i * (i + 1) / 2 + col] = z[i];
      }
    }
    if (out.tail_backward) {
      for (int32_t k = 0; k < n; ++k) {
        const int32_t i = B.row[k];
        if (!in_tail[i]) continue;
        const int32_t a = tail_index[i];
        Ut[(size_t)a * m + a] = 1.0 / (double)std::real(B.dinv[k]);
        for (int32_t p = B.ptr[k]; p < B.ptr[k + 1]; ++p) Ut[(size_t)a * m + tail_index[B.col[p]]] = (double)std::real(B.val[p]);
      }
      // inverse of an upper triangle by columns: solve U z = e_c, rows from the last
      out.bwd_inv.assign((size_t)m * (m + 1) / 2, 0.0);
      auto up = [m](int32_t i, int32_t j) { return (size_t)i * m - (size_t)i * (i - 1) / 2 + (j - i); };
      for (int32_t col = m - 1; col >= 0; --col) {
        std::fill(z.begin(), z.end(), 0.0);
        for (int32_t i = col; i >= 0; --i) {
          double acc = (i == col) ? 1.0 : 0.0;
          for (int32_t j = i + 1; j <= col; ++j) acc -= Ut[(size_t)i * m + j] * z[j];
          z[i] = acc / Ut[(size_t)i * m + i];
          out.bwd_inv[up(i, col)] = z[i];
        }
      }
    }
  }
  // Narrow levels (taken by warp 0 alone): without a dense tail, the forward sweep's suffix of
  // levels with fewer than `narrow_rows` rows; the backward sweep's prefix likewise
  int32_t f_end = F.levels;  // forward levels handled by level (the rest are the tail)
  if (dense_tail) f_end = tail_level;
  int32_t f_first_narrow = f_end;
  if (!dense_tail)
    while (f_first_narrow > 1 && rows_of(F, f_first_narrow - 1) < narrow_rows) --f_first_narrow;

  // Forward level 0: no entries, folded into the load
  if (F.levels > 0)
    for (int32_t k = F.level_ptr[0]; k < F.level_ptr[1]; ++k) {
      if (F.ptr[k + 1] != F.ptr[k]) throw Error(host::kInternal, "a level-0 row has entries");
      out.load_scale[plan.in_row[F.row[k]]] = (double)std::real(F.dinv[k]);
    }
  int32_t stage = 0;
  auto deal = [&](const Sweep<T> &s, std::vector<int32_t> ks, int32_t st, int32_t rot,
                  const std::vector<int32_t> *tails = nullptr) {
    std::stable_sort(ks.begin(), ks.end(),
                     [&](int32_t a, int32_t b) { return (s.ptr[a + 1] - s.ptr[a]) > (s.ptr[b + 1] - s.ptr[b]); });
    int32_t slice = 0;
    for (size_t t0 = 0; t0 < ks.size(); t0 += G, ++slice) {
      std::vector<int32_t> part(ks.begin() + t0, ks.begin() + std::min(ks.size(), t0 + (size_t)G));
      if (tails) {
        std::vector<int32_t> ti;
        for (int32_t k : part) ti.push_back(tail_index[s.row[k]]);
        emit_slice((slice + rot) % warps, s, part, st, &ti);
      } else {
        emit_slice((slice + rot) % warps, s, part, st);
      }
    }
  };
  auto level_positions = [](const Sweep<T> &s, int32_t l) {
    std::vector<int32_t> ks;
    for (int32_t k = s.level_ptr[l]; k < s.level_ptr[l + 1]; ++k) ks.push_back(k);
    return ks;
  };
  // With a dense tail, the rows below it fall into independent groups (for a Cholesky factor,
  // the subtrees hanging under the tail): each goes whole to one warp, balanced by work, which
  // takes its rows level by level with only warp synchronisation
  std::vector<int32_t> owner(n, -1);
  bool by_warp = false;
  if (dense_tail) {
    std::vector<int32_t> parent_uf(n);
    for (int32_t i = 0; i < n; ++i) parent_uf[i] = i;
    std::function<int32_t(int32_t)> find = [&](int32_t x) {
      while (parent_uf[x] != x) x = parent_uf[x] = parent_uf[parent_uf[x]];
      return x;
    };
    auto join = [&](const Sweep<T> &s) {
      for (int32_t k = 0; k < n; ++k) {
        const int32_t i = s.row[k];
        if (in_tail[i]) continue;
        for (int32_t p = s.ptr[k]; p < s.ptr[k + 1]; ++p)
          if (!in_tail[s.col[p]]) parent_uf[find(i)] = find(s.col[p]);
      }
    };
    join(F);
    if (out.tail_backward) join(B);
    std::vector<int64_t> work(n, 0);
    for (int32_t k = 0; k < n; ++k) {
      if (!in_tail[F.row[k]]) work[find(F.row[k])] += 1 + F.ptr[k + 1] - F.ptr[k];
      if (!in_tail[B.row[k]]) work[find(B.row[k])] += 1 + B.ptr[k + 1] - B.ptr[k];
    }
    std::vector<int32_t> roots;
    for (int32_t i = 0; i < n; ++i)
      if (!in_tail[i] && find(i) == i) roots.push_back(i);
    std::stable_sort(roots.begin(), roots.end(), [&](int32_t a, int32_t b) { return work[a] > work[b]; });
    std::vector<int64_t> load(warps, 0);
    std::vector<int32_t> group_warp(n, -1);
    for (int32_t r : roots) {
      const int32_t w = (int32_t)(std::min_element(load.begin(), load.end()) - load.begin());
      group_warp[r] = w;
      load[w] += work[r];
    }
    for (int32_t i = 0; i < n; ++i)
      if (!in_tail[i]) owner[i] = group_warp[find(i)];
    by_warp = true;
  }
  // Emits positions `ks` of sweep s (in topological order, with their levels `lev`) as each
  // owner warp's slices, one level after another, all at stage `st`
  auto emit_owned = [&](const Sweep<T> &s, const std::vector<int32_t> &ks, const std::vector<int32_t> &lev,
                        int32_t st) {
    std::vector<std::vector<int32_t>> mine(warps);
    for (int32_t k : ks) mine[owner[s.row[k]]].push_back(k);
    for (int32_t w = 0; w < warps; ++w) {
      auto &v = mine[w];
      std::stable_sort(v.begin(), v.end(), [&](int32_t a, int32_t b) { return lev[s.row[a]] < lev[s.row[b]]; });
      size_t i0 = 0;
      while (i0 < v.size()) {
        size_t i1 = i0;
        while (i1 < v.size() && lev[s.row[v[i1]]] == lev[s.row[v[i0]]]) ++i1;
        std::vector<int32_t> same(v.begin() + i0, v.begin() + i1);
        std::stable_sort(same.begin(), same.end(), [&](int32_t a, int32_t b) {
          return (s.ptr[a + 1] - s.ptr[a]) > (s.ptr[b + 1] - s.ptr[b]);
        });
        for (size_t t0 = 0; t0 < same.size(); t0 += G) {
          std::vector<int32_t> part(same.begin() + t0, same.begin() + std::min(same.size(), t0 + (size_t)G));
          emit_slice(w, s, part, st);
        }
        i0 = i1;
      }
    }
  };
  if (by_warp) {
    // forward rows below the tail (level 0 is folded into the load)
    std::vector<int32_t> ks;
    for (int32_t l = 1; l < f_end; ++l)
      for (int32_t k = F.level_ptr[l]; k < F.level_ptr[l + 1]; ++k) ks.push_back(k);
    std::vector<int32_t> lev(F.level_of.begin(), F.level_of.end());
    emit_owned(F, ks, lev, stage);
    ++stage;
    out.fwd_wide = 1;
  } else {
    // forward levels 1 .. f_first_narrow - 1 dealt over the warps, a barrier after each
    for (int32_t l = 1; l < f_first_narrow; ++l) {
      deal(F, level_positions(F, l), stage, l);
      ++stage;
      ++out.fwd_wide;
    }
  }
  if (dense_tail) {
    // r_T = b_T - L_TB y_B into the tail buffer, then y_T = L_TT^-1 r_T into the slots
    std::vector<int32_t> ks;
    for (int32_t l = tail_level; l < F.levels; ++l)
      for (int32_t k = F.level_ptr[l]; k < F.level_ptr[l + 1]; ++k) ks.push_back(k);
    deal(F, ks, stage, 0, &ks);
    ++stage;
    const int32_t m = out.tail;
    auto lower_at = [](int32_t i, int32_t j) { return (size_t)i * (i + 1) / 2 + j; };
    for (int32_t t = 0; t < m; ++t) emit_dense_row(t % warps, out.fwd_inv, t, 0, t + 1, lower_at, stage);
    ++stage;
    out.fwd_narrow_rows = out.tail;
  } else {
    auto narrow_level = [&](const Sweep<T> &s, int32_t l, int32_t st) {
      const auto ks = sorted_level(s, l);
      if ((int32_t)ks.size() * 2 >= G) {
        for (size_t t0 = 0; t0 < ks.size(); t0 += G) {
          std::vector<int32_t> part(ks.begin() + t0, ks.begin() + std::min(ks.size(), t0 + (size_t)G));
          emit_slice(0, s, part, st);
        }
      } else {
        for (int32_t k : ks) emit_split(0, s, k, st);
      }
    };
    for (int32_t l = std::max(f_first_narrow, 1); l < F.levels; ++l) {
      narrow_level(F, l, stage);
      out.fwd_narrow_rows += rows_of(F, l);
    }
    // the backward prefix of narrow levels joins warp 0's run
    int32_t b_narrow = 0;
    while (b_narrow < B.levels && rows_of(B, b_narrow) < narrow_rows) ++b_narrow;
    for (int32_t l = 0; l < b_narrow; ++l) {
      narrow_level(B, l, stage);
      out.bwd_narrow_rows += rows_of(B, l);
    }
    ++stage;
    for (int32_t l = b_narrow; l < B.levels; ++l) {
      deal(B, level_positions(B, l), stage, l);
      ++stage;
      ++out.bwd_wide;
    }
  }
  if (dense_tail) {
    std::vector<char> done_b(n, 0);
    if (out.tail_backward) {
      // x_T = U_TT^-1 y_T: copy y_T to the tail buffer, then the product into the slots
      for (int32_t w = 0; w < warps; ++w) emit_marker(w, kRecordCopy, stage, 1);
      ++stage;
      const int32_t m = out.tail;
      auto upper_at = [m](int32_t i, int32_t j) { return (size_t)i * m - (size_t)i * (i - 1) / 2 + (j - i); };
      for (int32_t t = 0; t < m; ++t) emit_dense_row(t % warps, out.bwd_inv, t, t, m - t, upper_at, stage);
      ++stage;
      for (int32_t i = 0; i < n; ++i) done_b[i] = in_tail[i];
      out.bwd_narrow_rows = out.tail;
    }
    // the remaining backward rows by levels counted over rows not yet done
    std::vector<int32_t> lev(n, -1);
    int32_t levels = 0;
    for (int32_t k = 0; k < n; ++k) {  // B's positions are in topological order (level order)
      const int32_t i = B.row[k];
      if (done_b[i]) continue;
      int32_t l = 0;
      for (int32_t p = B.ptr[k]; p < B.ptr[k + 1]; ++p)
        if (!done_b[B.col[p]]) l = std::max(l, lev[B.col[p]] + 1);
      lev[i] = l;
      levels = std::max(levels, l + 1);
    }
    if (by_warp && out.tail_backward) {
      std::vector<int32_t> ks;
      for (int32_t k = 0; k < n; ++k)
        if (!done_b[B.row[k]]) ks.push_back(k);
      emit_owned(B, ks, lev, stage);
      ++stage;
      out.bwd_wide = 1;
    } else {
      std::vector<std::vector<int32_t>> by_level(levels);
      for (int32_t k = 0; k < n; ++k)
        if (!done_b[B.row[k]]) by_level[lev[B.row[k]]].push_back(k);
      for (int32_t l = 0; l < levels; ++l) {
        deal(B, by_level[l], stage, l);
        ++stage;
        ++out.bwd_wide;
      }
    }
  }
  out.stages = stage;
  out.warp_page.assign(1, 0);
  for (int32_t w = 0; w < warps; ++w) {
    writers[w]->close_page();
    out.warp_page.push_back(out.warp_page.back() + writers[w]->pages);
    out.blob.insert(out.blob.end(), blobs[w].begin(), blobs[w].end());
  }
  return out;
}

template StreamLayout stream_layout(const Plan<double> &, int32_t, int32_t, int32_t, int32_t, int32_t, int32_t);

}  // namespace yb
