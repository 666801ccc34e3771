// The domain layout (DomainLayout in plan.hpp): the rows of a factor cut into per-warp domains
// under a dense top block, and the records each warp streams through for one tile.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>

#include "plan.hpp"

namespace yb {

using host::Error;

namespace {

inline int64_t a16(int64_t v) { return (v + 15) & ~int64_t(15); }

template <class T> double real_of(const T &v) { return (double)std::real(v); }

// One warp's pages: records never cross a page; a page's unused tail starts with an end marker.
struct Pages {
  int32_t page_bytes;
  std::vector<uint8_t> blob;
  int64_t start = -1, pos = 0;
  int32_t count = 0;
  explicit Pages(int32_t pb) : page_bytes(pb) {}
  void close() {
    if (start < 0) return;
    if (pos + 16 <= page_bytes) {
      const int32_t end[4] = {kRecordEnd, 0, 0, 0};
      std::memcpy(blob.data() + start + pos, end, 16);
    }
    start = -1;
  }
  uint8_t *reserve(int64_t bytes) {
    if (bytes > page_bytes) throw Error(host::kInternal, "a record does not fit a page");
    if (start < 0 || pos + bytes > page_bytes) {
      close();
      start = (int64_t)blob.size();
      blob.resize(blob.size() + page_bytes, 0);
      pos = 0;
      ++count;
    }
    uint8_t *p = blob.data() + start + pos;
    pos += bytes;
    return p;
  }
};

template <class V> void put(uint8_t *&p, const V *v, int64_t count) {
  if (count) std::memcpy(p, v, sizeof(V) * count);
  p += a16((int64_t)sizeof(V) * count);
}

void put_values(uint8_t *&p, const std::vector<double> &v, int32_t value_bytes) {
  if (value_bytes == 8) {
    put(p, v.data(), (int64_t)v.size());
  } else {
    std::vector<float> f(v.begin(), v.end());
    put(p, f.data(), (int64_t)f.size());
  }
}

// A row of a record: its slot, its result's destination, its entries (positions in the sweep).
struct RowJob {
  int32_t slot, dest;
  double dinv;
  std::vector<int32_t> ps;
};

// The cost model's constants, in SM cycles per tile (latency of one warp's serial work).
constexpr double kRecordCycles = 60, kIterCycles = 22, kReduceCycles = 16, kDenseRowCycles = 70,
                 kDenseIterCycles = 10, kBarrierCycles = 120, kDenseByteCycles = 1.0 / 48;

}  // namespace

template <class T>
DomainLayout domain_layout(const Plan<T> &plan, int32_t value_bytes, int32_t warps, int32_t page_bytes, int32_t K_in) {
  if (value_bytes != 8 && value_bytes != 4) throw Error(host::kInvalidArgument, "values are 4 or 8 bytes");
  if (warps < 1 || warps > 32 || page_bytes < 512 || page_bytes % 16)
    throw Error(host::kInvalidArgument, "bad domain layout shape");
  const int32_t n = plan.n;
  if (n + 2 > 65536) throw Error(host::kTooLarge, "the order does not fit 16-bit slots");
  const Sweep<T> &F = plan.fwd, &B = plan.bwd;
  const int32_t levels = F.levels;
  // position of each row in each sweep
  std::vector<int32_t> fpos(n), bpos(n);
  for (int32_t k = 0; k < n; ++k) fpos[F.row[k]] = k, bpos[B.row[k]] = k;
  auto flen = [&](int32_t i) { return F.ptr[fpos[i] + 1] - F.ptr[fpos[i]]; };
  auto blen = [&](int32_t i) { return B.ptr[bpos[i] + 1] - B.ptr[bpos[i]]; };

  // Rows in T for cut K, and whether the cut is valid (no upper entry of a T row below T)
  auto in_top = [&](int32_t K) {
    std::vector<char> t(n, 0);
    for (int32_t i = 0; i < n; ++i) t[i] = F.level_of[i] >= K;
    return t;
  };
  auto valid = [&](const std::vector<char> &top) {
    for (int32_t i = 0; i < n; ++i)
      if (top[i]) {
        const int32_t k = bpos[i];
        for (int32_t p = B.ptr[k]; p < B.ptr[k + 1]; ++p)
          if (!top[B.col[p]]) return false;
      }
    return true;
  };

  // Domains of cut K: connected groups of non-T rows, assigned to warps by work (largest first)
  struct Cut {
    int32_t K = 0, tail = 0;
    std::vector<char> top;
    std::vector<int32_t> owner;     // warp of each non-T row
    std::vector<int32_t> blevel;    // backward level of each non-T row, counted from T
    std::vector<int32_t> tail_index;
  };
  auto make_cut = [&](int32_t K) {
    Cut c;
    c.K = K;
    c.top = in_top(K);
    std::vector<int32_t> up(n);
    std::iota(up.begin(), up.end(), 0);
    auto find = [&](int32_t x) {
      while (up[x] != x) x = up[x] = up[up[x]];
      return x;
    };
    for (int32_t k = 0; k < n; ++k) {
      const int32_t i = F.row[k];
      if (c.top[i]) continue;
      for (int32_t p = F.ptr[k]; p < F.ptr[k + 1]; ++p) up[find(i)] = find(F.col[p]);
    }
    for (int32_t k = 0; k < n; ++k) {
      const int32_t i = B.row[k];
      if (c.top[i]) continue;
      for (int32_t p = B.ptr[k]; p < B.ptr[k + 1]; ++p)
        if (!c.top[B.col[p]]) up[find(i)] = find(B.col[p]);
    }
    std::vector<int64_t> work(n, 0);
    for (int32_t i = 0; i < n; ++i)
      if (!c.top[i]) work[find(i)] += 2 + flen(i) + blen(i);
    std::vector<int32_t> roots;
    for (int32_t i = 0; i < n; ++i)
      if (!c.top[i] && find(i) == i) roots.push_back(i);
    std::stable_sort(roots.begin(), roots.end(), [&](int32_t a, int32_t b) { return work[a] > work[b]; });
    std::vector<int64_t> load(warps, 0);
    std::vector<int32_t> root_warp(n, -1);
    for (int32_t r : roots) {
      const int32_t w = (int32_t)(std::min_element(load.begin(), load.end()) - load.begin());
      root_warp[r] = w;
      load[w] += work[r];
    }
    c.owner.assign(n, -1);
    for (int32_t i = 0; i < n; ++i)
      if (!c.top[i]) c.owner[i] = root_warp[find(i)];
    // backward levels over non-T rows (the backward sweep's positions are in topological order)
    c.blevel.assign(n, -1);
    for (int32_t k = 0; k < n; ++k) {
      const int32_t i = B.row[k];
      if (c.top[i]) continue;
      int32_t l = 0;
      for (int32_t p = B.ptr[k]; p < B.ptr[k + 1]; ++p)
        if (!c.top[B.col[p]]) l = std::max(l, c.blevel[B.col[p]] + 1);
      c.blevel[i] = l;
    }
    // T rows in increasing order: L_TT is then lower and U_TT upper triangular
    c.tail_index.assign(n, -1);
    for (int32_t i = 0; i < n; ++i)
      if (c.top[i]) c.tail_index[i] = c.tail++;
    return c;
  };

  const int64_t rows_fixed = 48;
  auto rows_bytes = [&](int64_t r, int64_t e) {
    return rows_fixed + a16(8 * r) + a16((int64_t)value_bytes * r) + a16(2 * e) + a16((int64_t)value_bytes * e);
  };
  const int64_t split_fixed = 16 + 16 + 16;
  const int64_t split_max = ((page_bytes - split_fixed - 32) / (4 + value_bytes)) / 32 * 32;

  // Groups the jobs of one (warp, level) into rows records: longest rows first, 32 / k rows a
  // record with k lanes on each row, as many as fit a page, k the same for the group and chosen
  // by the cost model; a row too long for any page goes alone into chunked split records. Calls
  // emit_rows(jobs, k_log2) and emit_split(job) in order; returns the cost-model cycles.
  auto group = [&](std::vector<RowJob> &jobs, auto &&emit_rows, auto &&emit_split) {
    std::stable_sort(jobs.begin(), jobs.end(),
                     [](const RowJob &a, const RowJob &b) { return a.ps.size() > b.ps.size(); });
    double cycles = 0;
    size_t first = 0;
    while (first < jobs.size() && rows_bytes(1, (int64_t)jobs[first].ps.size()) > page_bytes) {
      emit_split(jobs[first]);
      cycles += kRecordCycles + kIterCycles * (double)((jobs[first].ps.size() + 31) / 32) + 5 * kReduceCycles;
      ++first;
    }
    if (first == jobs.size()) return cycles;
    // chunks of the remaining rows for 2^kl lanes per row
    auto chunks = [&](int32_t kl, double *cost) {
      std::vector<std::pair<size_t, size_t>> out;
      const size_t per = (size_t)32 >> kl;
      double c = 0;
      size_t i = first;
      while (i < jobs.size()) {
        size_t j = i;
        int64_t e = 0;
        while (j < jobs.size() && j - i < per &&
               rows_bytes((int64_t)(j - i + 1), e + (int64_t)jobs[j].ps.size()) <= page_bytes) {
          e += (int64_t)jobs[j].ps.size();
          ++j;
        }
        out.emplace_back(i, j);
        c += kRecordCycles + kIterCycles * (double)((jobs[i].ps.size() + ((size_t)1 << kl) - 1) >> kl) +
             kReduceCycles * kl;
        i = j;
      }
      if (cost) *cost = c;
      return out;
    };
    int32_t best_kl = 0;
    double best = std::numeric_limits<double>::infinity();
    for (int32_t kl = 0; kl <= 5; ++kl) {
      double c;
      chunks(kl, &c);
      if (c < best) best = c, best_kl = kl;
    }
    for (auto [i, j] : chunks(best_kl, nullptr)) {
      std::vector<RowJob> part(jobs.begin() + i, jobs.begin() + j);
      emit_rows(part, best_kl);
    }
    return cycles + best;
  };

  // Builds the records of cut c into `out` (emit = true) or only prices them. Returns cycles.
  auto build = [&](const Cut &c, bool emit, DomainLayout *out) {
    std::vector<Pages> pages(warps, Pages(page_bytes));
    std::vector<double> busy(warps, 0.0);
    int64_t records = 0, entries = 0;
    const int32_t m = c.tail;
    auto emit_rows = [&](int32_t w, int32_t stage, bool to_tail, const Sweep<T> &s, std::vector<RowJob> &part,
                         int32_t kl) {
      ++records;
      int64_t e = 0;
      for (auto &j : part) e += (int64_t)j.ps.size();
      entries += e;
      if (!emit) return;
      const int64_t r = (int64_t)part.size();
      const int64_t bytes = rows_bytes(r, e);
      uint8_t *p = pages[w].reserve(bytes);
      const int32_t off_info = (int32_t)rows_fixed, off_dinv = off_info + (int32_t)a16(8 * r),
                    off_cols = off_dinv + (int32_t)a16((int64_t)value_bytes * r), off_vals = off_cols + (int32_t)a16(2 * e);
      const int32_t h1[4] = {kRecordRows, stage, (int32_t)r, to_tail ? (int32_t)kRecordToTail : 0};
      const int32_t h2[4] = {kl, (int32_t)e, (int32_t)bytes, 0};
      const int32_t h3[4] = {off_info, off_dinv, off_cols, off_vals};
      put(p, h1, 4);
      put(p, h2, 4);
      put(p, h3, 4);
      std::vector<int32_t> info;
      std::vector<double> dinv, val;
      std::vector<uint16_t> col;
      int32_t start = 0;
      for (auto &j : part) {
        info.push_back(j.slot | ((int32_t)j.ps.size() << 16));
        info.push_back(start | (j.dest << 16));
        dinv.push_back(j.dinv);
        for (int32_t pp : j.ps) {
          col.push_back((uint16_t)s.col[pp]);
          val.push_back(real_of(s.val[pp]));
        }
        start += (int32_t)j.ps.size();
      }
      if (start >= 65536) throw Error(host::kInternal, "a rows record has too many entries");
      put(p, info.data(), (int64_t)info.size());
      put_values(p, dinv, value_bytes);
      put(p, col.data(), (int64_t)col.size());
      put_values(p, val, value_bytes);
    };
    auto emit_split = [&](int32_t w, int32_t stage, bool to_tail, const Sweep<T> &s, const RowJob &j) {
      const int32_t len = (int32_t)j.ps.size();
      entries += len;
      int32_t e0 = 0;
      do {
        const int32_t e1 = (int32_t)std::min<int64_t>(len, e0 + split_max);
        const int32_t mm = ((e1 - e0) + 31) / 32 * 32;
        ++records;
        if (emit) {
          uint8_t *p = pages[w].reserve(split_fixed + a16(4LL * mm) + a16((int64_t)value_bytes * mm));
          const int32_t hdr[4] = {kRecordSplit, stage, mm,
                                  (e0 == 0 ? kRecordFirst : 0) | (e1 == len ? kRecordLast : 0) |
                                      (to_tail ? kRecordToTail : 0)};
          put(p, hdr, 4);
          const int32_t row[4] = {j.slot, j.dest, 0, 0};
          put(p, row, 4);
          std::vector<double> dv(16 / value_bytes, 0.0);
          dv[0] = j.dinv;
          put_values(p, dv, value_bytes);
          std::vector<int32_t> col(mm, n);
          std::vector<double> val(mm, 0.0);
          for (int32_t e = e0; e < e1; ++e) {
            col[e - e0] = s.col[j.ps[e]];
            val[e - e0] = real_of(s.val[j.ps[e]]);
          }
          put(p, col.data(), mm);
          put_values(p, val, value_bytes);
        }
        e0 = e1;
      } while (e0 < len);
    };
    auto job_of = [&](const Sweep<T> &s, int32_t k, bool outside_top_only, int32_t dest) {
      RowJob j;
      j.slot = s.row[k];
      j.dest = dest;
      j.dinv = real_of(s.dinv[k]);
      for (int32_t p = s.ptr[k]; p < s.ptr[k + 1]; ++p)
        if (!outside_top_only || !c.top[s.col[p]]) j.ps.push_back(p);
      return j;
    };
    const bool has_top = m > 0;
    const int32_t st_fwd = 0, st_tpart = 1, st_dfwd = 2, st_copy = 3, st_dbwd = 4, st_bwd = has_top ? 5 : 0;
    // forward domains: each warp's rows by forward level
    for (int32_t w = 0; w < warps; ++w) {
      std::vector<std::vector<RowJob>> by_level(c.K);
      for (int32_t k = 0; k < n; ++k) {
        const int32_t i = F.row[k];
        if (!c.top[i] && c.owner[i] == w) by_level[F.level_of[i]].push_back(job_of(F, k, false, i));
      }
      for (auto &jobs : by_level)
        busy[w] += group(
            jobs, [&](std::vector<RowJob> &part, int32_t kl) { emit_rows(w, st_fwd, false, F, part, kl); },
            [&](const RowJob &j) { emit_split(w, st_fwd, false, F, j); });
    }
    double cycles = *std::max_element(busy.begin(), busy.end());
    std::vector<double> dense_inv_f, dense_inv_b;
    if (has_top) {
      // r_T = b_T - L_TB y_B into the tail buffer, T rows dealt over the warps, longest first to
      // the warp with the fewest entries so far
      std::vector<RowJob> tjobs;
      for (int32_t k = 0; k < n; ++k)
        if (c.top[F.row[k]]) tjobs.push_back(job_of(F, k, true, c.tail_index[F.row[k]]));
      std::stable_sort(tjobs.begin(), tjobs.end(),
                       [](const RowJob &a, const RowJob &b) { return a.ps.size() > b.ps.size(); });
      std::vector<std::vector<RowJob>> share(warps);
      std::vector<int64_t> ents(warps, 0);
      for (auto &j : tjobs) {
        const int32_t w = (int32_t)(std::min_element(ents.begin(), ents.end()) - ents.begin());
        ents[w] += 4 + (int64_t)j.ps.size();
        share[w].push_back(j);
      }
      std::fill(busy.begin(), busy.end(), 0.0);
      for (int32_t w = 0; w < warps; ++w)
        busy[w] += group(
            share[w], [&](std::vector<RowJob> &part, int32_t kl) { emit_rows(w, st_tpart, true, F, part, kl); },
            [&](const RowJob &j) { emit_split(w, st_tpart, true, F, j); });
      cycles += *std::max_element(busy.begin(), busy.end());
      // dense inverses of L_TT and U_TT, in T order (tail index), computed in FP64
      std::vector<double> Lt((size_t)m * m, 0.0), Ut((size_t)m * m, 0.0);
      for (int32_t k = 0; k < n; ++k) {
        const int32_t i = F.row[k];
        if (!c.top[i]) continue;
        const int32_t a = c.tail_index[i];
        Lt[(size_t)a * m + a] = 1.0 / real_of(F.dinv[k]);
        for (int32_t p = F.ptr[k]; p < F.ptr[k + 1]; ++p)
          if (c.top[F.col[p]]) Lt[(size_t)a * m + c.tail_index[F.col[p]]] = real_of(F.val[p]);
      }
      for (int32_t k = 0; k < n; ++k) {
        const int32_t i = B.row[k];
        if (!c.top[i]) continue;
        const int32_t a = c.tail_index[i];
        Ut[(size_t)a * m + a] = 1.0 / real_of(B.dinv[k]);
        for (int32_t p = B.ptr[k]; p < B.ptr[k + 1]; ++p) Ut[(size_t)a * m + c.tail_index[B.col[p]]] = real_of(B.val[p]);
      }
      if (emit) {
        for (int32_t a = 0; a < m; ++a)
          for (int32_t b = 0; b < m; ++b) {
            if (b > a && Lt[(size_t)a * m + b] != 0.0) throw Error(host::kInternal, "L_TT is not lower triangular");
            if (b < a && Ut[(size_t)a * m + b] != 0.0) throw Error(host::kInternal, "U_TT is not upper triangular");
          }
        // inverse of the lower triangle by columns: solve L z = e_col
        dense_inv_f.assign((size_t)m * (m + 1) / 2, 0.0);
        std::vector<double> z(m);
        for (int32_t col = 0; col < m; ++col) {
          std::fill(z.begin(), z.end(), 0.0);
          for (int32_t i = col; i < m; ++i) {
            double acc = (i == col) ? 1.0 : 0.0;
            for (int32_t j = col; j < i; ++j) acc -= Lt[(size_t)i * m + j] * z[j];
            z[i] = acc / Lt[(size_t)i * m + i];
            dense_inv_f[(size_t)i * (i + 1) / 2 + col] = z[i];
          }
        }
        // inverse of the upper triangle by columns: solve U z = e_col, rows from the last
        dense_inv_b.assign((size_t)m * (m + 1) / 2, 0.0);
        auto up = [m](int32_t i, int32_t j) { return (size_t)i * m - (size_t)i * (i - 1) / 2 + (j - i); };
        for (int32_t col = m - 1; col >= 0; --col) {
          std::fill(z.begin(), z.end(), 0.0);
          for (int32_t i = col; i >= 0; --i) {
            double acc = (i == col) ? 1.0 : 0.0;
            for (int32_t j = i + 1; j <= col; ++j) acc -= Ut[(size_t)i * m + j] * z[j];
            z[i] = acc / Ut[(size_t)i * m + i];
            dense_inv_b[up(i, col)] = z[i];
          }
        }
      }
      if (emit) {
        // the infinity-norm condition of each triangle: the explicit inverses stand in for
        // substitution only while it is small (their rounding grows with it)
        auto cond = [m](const std::vector<double> &tri, const std::vector<double> &inv, bool lower) {
          double tn = 0, in = 0;
          for (int32_t i = 0; i < m; ++i) {
            double ts = 0, is = 0;
            for (int32_t j = 0; j < m; ++j) ts += std::fabs(tri[(size_t)i * m + j]);
            for (int32_t j = lower ? 0 : i; j < (lower ? i + 1 : m); ++j)
              is += std::fabs(lower ? inv[(size_t)i * (i + 1) / 2 + j] : inv[(size_t)i * m - (size_t)i * (i - 1) / 2 + (j - i)]);
            tn = std::max(tn, ts), in = std::max(in, is);
          }
          return tn * in;
        };
        out->top_condition = std::max(cond(Lt, dense_inv_f, true), cond(Ut, dense_inv_b, false));
      }
      // dense rows, dealt to balance their lengths: forward row t has t + 1 entries, backward m - t
      const int64_t dense_fixed = 32;
      const int64_t dense_max = (page_bytes - dense_fixed - 16) / value_bytes / 4 * 4;
      auto emit_dense = [&](int32_t w, int32_t stage, const std::vector<double> &inv, int32_t t, int32_t j_first,
                            int32_t count, bool lower) {
        int32_t e0 = 0;
        do {
          const int32_t e1 = (int32_t)std::min<int64_t>(count, e0 + dense_max);
          ++records;
          if (emit) {
            uint8_t *p = pages[w].reserve(dense_fixed + a16((int64_t)value_bytes * (e1 - e0)));
            const int32_t hdr[4] = {kRecordDense, stage, e1 - e0,
                                    (e0 == 0 ? kRecordFirst : 0) | (e1 == count ? kRecordLast : 0)};
            put(p, hdr, 4);
            const int32_t where[4] = {t, j_first + e0, 0, 0};
            put(p, where, 4);
            std::vector<double> v(e1 - e0);
            for (int32_t e = e0; e < e1; ++e) {
              const int32_t j = j_first + e;
              v[e - e0] = lower ? inv[(size_t)t * (t + 1) / 2 + j] : inv[(size_t)t * m - (size_t)t * (t - 1) / 2 + (j - t)];
            }
            put_values(p, v, value_bytes);
          }
          e0 = e1;
        } while (e0 < count);
      };
      for (int pass = 0; pass < 2; ++pass) {
        const bool lower = pass == 0;
        std::fill(busy.begin(), busy.end(), 0.0);
        // longest rows first to the least busy warp
        std::vector<int32_t> order(m);
        std::iota(order.begin(), order.end(), 0);
        if (lower) std::reverse(order.begin(), order.end());
        for (int32_t t : order) {
          const int32_t count = lower ? t + 1 : m - t;
          const int32_t w = (int32_t)(std::min_element(busy.begin(), busy.end()) - busy.begin());
          busy[w] += kDenseRowCycles + kDenseIterCycles * (double)((count + 31) / 32) +
                     kDenseByteCycles * (double)count * value_bytes * warps;
          emit_dense(w, lower ? st_dfwd : st_dbwd, lower ? dense_inv_f : dense_inv_b, t, lower ? 0 : t, count, lower);
        }
        cycles += *std::max_element(busy.begin(), busy.end());
        if (lower)
          for (int32_t w = 0; w < warps; ++w) {  // every warp copies its share of y_T
            ++records;
            if (emit) {
              uint8_t *p = pages[w].reserve(16);
              const int32_t hdr[4] = {kRecordCopy, st_copy, 1, 0};
              put(p, hdr, 4);
            }
          }
      }
      cycles += 5 * kBarrierCycles;
    }
    // backward domains: each warp's rows by backward level counted from T
    std::fill(busy.begin(), busy.end(), 0.0);
    for (int32_t w = 0; w < warps; ++w) {
      int32_t top_level = -1;
      for (int32_t i = 0; i < n; ++i)
        if (!c.top[i] && c.owner[i] == w) top_level = std::max(top_level, c.blevel[i]);
      std::vector<std::vector<RowJob>> by_level(top_level + 1);
      for (int32_t k = 0; k < n; ++k) {
        const int32_t i = B.row[k];
        if (!c.top[i] && c.owner[i] == w) by_level[c.blevel[i]].push_back(job_of(B, k, false, i));
      }
      for (auto &jobs : by_level)
        busy[w] += group(
            jobs, [&](std::vector<RowJob> &part, int32_t kl) { emit_rows(w, st_bwd, false, B, part, kl); },
            [&](const RowJob &j) { emit_split(w, st_bwd, false, B, j); });
    }
    cycles += *std::max_element(busy.begin(), busy.end()) + 2 * kBarrierCycles;
    if (emit) {
      out->stages = has_top ? 6 : 1;
      out->records = records;
      out->entries = entries;
      out->dense_entries = has_top ? (int64_t)m * (m + 1) : 0;
      out->warp_page.assign(1, 0);
      for (int32_t w = 0; w < warps; ++w) {
        pages[w].close();
        out->warp_page.push_back(out->warp_page.back() + pages[w].count);
        out->blob.insert(out->blob.end(), pages[w].blob.begin(), pages[w].blob.end());
      }
    }
    return cycles;
  };

  // The cut: as asked, or the cheapest valid one with a top of at most kMaxTop rows whose dense
  // triangles are well conditioned
  constexpr int32_t kMaxTop = 768;
  constexpr double kMaxTopCondition = 1e4;
  auto emit_cut = [&](int32_t K) {
    const Cut c = make_cut(K);
    if (!valid(c.top)) throw Error(host::kInvalidArgument, "an upper-triangle entry of a top row reaches below the cut");
    if (c.tail > 4096) throw Error(host::kInvalidArgument, "the top block is too large");
    DomainLayout out;
    out.warps = warps;
    out.page_bytes = page_bytes;
    out.value_bytes = value_bytes;
    out.K = K;
    out.tail = c.tail;
    out.tail_slot.assign(c.tail, 0);
    for (int32_t i = 0; i < n; ++i)
      if (c.top[i]) out.tail_slot[c.tail_index[i]] = i;
    out.cost = build(c, true, &out);
    return out;
  };
  if (K_in >= 0) {
    DomainLayout out = emit_cut(std::min(K_in, levels));
    if (!(out.top_condition <= kMaxTopCondition))
      throw Error(host::kInvalidArgument, "the top block is too ill-conditioned for its explicit inverse");
    return out;
  }
  std::vector<std::pair<double, int32_t>> candidates;
  for (int32_t k = levels; k >= 1; --k) {
    int32_t top = 0;
    for (int32_t l = k; l < levels; ++l) top += F.level_ptr[l + 1] - F.level_ptr[l];
    if (top > kMaxTop) break;
    const Cut c = make_cut(k);
    if (!valid(c.top)) continue;
    candidates.emplace_back(build(c, false, nullptr), k);
  }
  std::stable_sort(candidates.begin(), candidates.end());
  for (auto [cost, k] : candidates) {
    DomainLayout out = emit_cut(k);
    if (out.top_condition <= kMaxTopCondition) return out;
  }
  throw Error(host::kInvalidArgument, "the factor admits no domain cut");
}

template DomainLayout domain_layout(const Plan<double> &, int32_t, int32_t, int32_t, int32_t);

}  // namespace yb
