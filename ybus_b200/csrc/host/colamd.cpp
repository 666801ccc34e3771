// COLAMD column ordering for LU of an unsymmetric pattern, following the steps of ybus_sparse's
// `column_approximate_minimum_degree` (ybus_sparse/src/compressed_matrix/colamd.rs:91-261) so the
// column order, and therefore the LU factor of a complex Ybus, is the one ybus computes:
// rows as elements, pivot rows formed as unions, approximate external-degree scores, aggressive
// absorption of rows inside the pivot row, supercolumns found by a (count, sum) key, dense rows
// ignored and dense or emptied columns ordered last.
#include "sparse.hpp"

#include <map>

namespace yb::host {

namespace {

enum class ColStatus : uint8_t { Live, Eliminated, Merged, SetAside };

struct ScoreBuckets {
  std::vector<idx_t> head, next, prev, score;
  idx_t lowest;
  explicit ScoreBuckets(idx_t n) : head(n + 1, -1), next(n, -1), prev(n, -1), score(n, 0), lowest(n) {}
  void insert(idx_t col, idx_t s) {
    score[col] = s;
    prev[col] = -1;
    next[col] = head[s];
    if (head[s] >= 0) prev[head[s]] = col;
    head[s] = col;
    lowest = std::min(lowest, s);
  }
  void remove(idx_t col) {
    const idx_t s = score[col];
    if (prev[col] >= 0)
      next[prev[col]] = next[col];
    else
      head[s] = next[col];
    if (next[col] >= 0) prev[next[col]] = prev[col];
  }
  idx_t pop_lowest() {
    while (lowest < (idx_t)head.size()) {
      if (head[lowest] >= 0) return head[lowest];
      ++lowest;
    }
    return -1;
  }
};

}  // namespace

std::vector<idx_t> column_amd(idx_t n_rows, idx_t n_cols, const std::vector<std::pair<idx_t, idx_t>> &entries) {
  std::vector<std::vector<idx_t>> col_rows(n_cols);
  for (const auto &e : entries) {
    if (e.first < 0 || e.first >= n_rows || e.second < 0 || e.second >= n_cols)
      throw Error(kInvalidArgument, "an entry lies outside the matrix");
    col_rows[e.second].push_back(e.first);
  }
  for (auto &rows : col_rows) {
    std::sort(rows.begin(), rows.end());
    rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
  }
  auto threshold = [](idx_t n) { return std::max<idx_t>(16, (idx_t)(10.0 * std::sqrt((double)n))); };
  const idx_t dense_col = threshold(std::min(n_rows, n_cols));
  const idx_t dense_row = threshold(n_cols);
  std::vector<ColStatus> status(n_cols, ColStatus::Live);
  std::vector<idx_t> dense_cols, null_cols;
  for (idx_t c = 0; c < n_cols; ++c)
    if ((idx_t)col_rows[c].size() > dense_col) {
      status[c] = ColStatus::SetAside;
      dense_cols.push_back(c);
    }
  std::vector<std::vector<idx_t>> row_cols(n_rows);
  for (idx_t c = 0; c < n_cols; ++c)
    if (status[c] == ColStatus::Live)
      for (idx_t r : col_rows[c]) row_cols[r].push_back(c);
  std::vector<char> row_alive(n_rows);
  for (idx_t r = 0; r < n_rows; ++r) row_alive[r] = !row_cols[r].empty() && (idx_t)row_cols[r].size() <= dense_row;
  for (idx_t c = 0; c < n_cols; ++c) {
    auto &rows = col_rows[c];
    rows.erase(std::remove_if(rows.begin(), rows.end(), [&](idx_t r) { return !row_alive[r]; }), rows.end());
    if (status[c] == ColStatus::Live && rows.empty()) {
      status[c] = ColStatus::SetAside;
      null_cols.push_back(c);
    }
  }
  std::vector<idx_t> weight(n_cols, 1);
  std::vector<std::vector<idx_t>> members(n_cols);
  std::vector<idx_t> row_size(n_rows);
  for (idx_t r = 0; r < n_rows; ++r) row_size[r] = (idx_t)row_cols[r].size();
  idx_t live_weight = 0;
  for (auto s : status) live_weight += (s == ColStatus::Live);
  ScoreBuckets buckets(n_cols);
  for (idx_t c = 0; c < n_cols; ++c)
    if (status[c] == ColStatus::Live) {
      idx_t score = 0;
      for (idx_t r : col_rows[c]) score += row_size[r] - 1;
      buckets.insert(c, std::min(score, live_weight - 1));
    }

  std::vector<idx_t> order;
  order.reserve(n_cols);
  std::vector<idx_t> col_mark(n_cols, 0), row_mark(n_rows, 0), outside(n_rows, 0);
  idx_t stamp = 0;
  for (;;) {
    const idx_t pivot = buckets.pop_lowest();
    if (pivot < 0) break;
    buckets.remove(pivot);
    status[pivot] = ColStatus::Eliminated;
    live_weight -= weight[pivot];
    order.push_back(pivot);
    order.insert(order.end(), members[pivot].begin(), members[pivot].end());

    ++stamp;
    std::vector<idx_t> pivot_cols;
    for (idx_t r : col_rows[pivot]) {
      if (!row_alive[r]) continue;
      for (idx_t c : row_cols[r])
        if (status[c] == ColStatus::Live && col_mark[c] != stamp) {
          col_mark[c] = stamp;
          pivot_cols.push_back(c);
        }
      row_alive[r] = 0;
    }
    const idx_t p = (idx_t)row_cols.size();
    idx_t psize = 0;
    for (idx_t c : pivot_cols) psize += weight[c];
    row_size.push_back(psize);
    row_cols.push_back(pivot_cols);
    row_alive.push_back(1);
    row_mark.push_back(0);
    outside.push_back(0);
    for (idx_t c : pivot_cols) {
      buckets.remove(c);
      auto &rows = col_rows[c];
      rows.erase(std::remove_if(rows.begin(), rows.end(), [&](idx_t r) { return !row_alive[r]; }), rows.end());
      rows.push_back(p);
    }
    for (idx_t c : pivot_cols)
      for (idx_t r : col_rows[c]) {
        if (r == p) continue;
        if (row_mark[r] != stamp) {
          row_mark[r] = stamp;
          outside[r] = row_size[r];
        }
        outside[r] -= weight[c];
      }
    for (idx_t c : pivot_cols)
      for (idx_t r : col_rows[c])
        if (r != p && row_mark[r] == stamp && outside[r] == 0) row_alive[r] = 0;
    std::vector<idx_t> scores;
    scores.reserve(pivot_cols.size());
    for (idx_t c : pivot_cols) {
      auto &rows = col_rows[c];
      rows.erase(std::remove_if(rows.begin(), rows.end(), [&](idx_t r) { return !row_alive[r]; }), rows.end());
      idx_t external = 0;
      for (idx_t r : rows)
        if (r != p) external += outside[r];
      scores.push_back(row_size[p] - weight[c] + external);
    }
    std::map<std::pair<idx_t, idx_t>, std::vector<size_t>> representatives;
    for (size_t k = 0; k < pivot_cols.size(); ++k) {
      const idx_t c = pivot_cols[k];
      std::sort(col_rows[c].begin(), col_rows[c].end());
      idx_t sum = 0;
      for (idx_t r : col_rows[c]) sum += r;
      const std::pair<idx_t, idx_t> key{(idx_t)col_rows[c].size(), sum % (n_cols + 1)};
      auto &candidates = representatives[key];
      size_t found = SIZE_MAX;
      for (size_t other : candidates)
        if (col_rows[pivot_cols[other]] == col_rows[c]) {
          found = other;
          break;
        }
      if (found != SIZE_MAX) {
        const idx_t into = pivot_cols[found];
        weight[into] += weight[c];
        members[into].push_back(c);
        members[into].insert(members[into].end(), members[c].begin(), members[c].end());
        members[c].clear();
        status[c] = ColStatus::Merged;
        scores[found] -= weight[c];
      } else {
        candidates.push_back(k);
      }
    }
    for (size_t k = 0; k < pivot_cols.size(); ++k) {
      const idx_t c = pivot_cols[k];
      if (status[c] == ColStatus::Live) {
        const idx_t cap = live_weight - weight[c];
        buckets.insert(c, std::min(std::max<idx_t>(scores[k], 0), cap));
      }
    }
  }
  order.insert(order.end(), null_cols.begin(), null_cols.end());
  order.insert(order.end(), dense_cols.begin(), dense_cols.end());
  return order;
}

}  // namespace yb::host
