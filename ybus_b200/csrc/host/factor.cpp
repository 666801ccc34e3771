// Host factorizations for the solve path: AMD, symbolic and numeric Cholesky, Gilbert–Peierls LU.
// The algorithms and their operation orders follow ybus_sparse so that the factor this library
// uploads is the factor ybus would upload (citations per function).
#include "sparse.hpp"

#include <limits>

namespace yb::host {

namespace {

// Doubly linked lists of the variables of each approximate degree; insertion at the head, so
// the node most recently given a degree is found first (ordering.rs:258-285).
struct DegreeLists {
  std::vector<idx_t> head, next, prev;
  explicit DegreeLists(idx_t n) : head(n + 1, -1), next(n, -1), prev(n, -1) {}
  void insert(idx_t node, idx_t degree) {
    next[node] = head[degree];
    prev[node] = -1;
    if (head[degree] >= 0) prev[head[degree]] = node;
    head[degree] = node;
  }
  void remove(idx_t node, idx_t degree) {
    if (prev[node] >= 0)
      next[prev[node]] = next[node];
    else
      head[degree] = next[node];
    if (next[node] >= 0) prev[next[node]] = prev[node];
  }
};

enum class Role : uint8_t { Variable, Merged, Element, Absorbed, Dense };

}  // namespace

// Approximate minimum degree on the quotient graph (ybus_sparse ordering.rs:306-492): element
// absorption, aggressive absorption, supervariables found by hashing their adjacency, dense
// rows (more than max(16, 10 sqrt n) neighbours) ordered last.
std::vector<idx_t> approximate_minimum_degree(const Adjacency &graph) {
  const idx_t n = graph.size();
  std::vector<idx_t> order;
  order.reserve(n);
  if (n == 0) return order;
  const idx_t dense_threshold = (idx_t)std::max(10.0 * std::sqrt((double)n), 16.0);
  std::vector<Role> role(n);
  for (idx_t i = 0; i < n; ++i)
    role[i] = (graph.degree(i) > dense_threshold && n > 2) ? Role::Dense : Role::Variable;

  std::vector<idx_t> weight(n, 1), element_size(n, 0), degree(n, 0);
  std::vector<std::vector<idx_t>> variables(n), elements(n), element_list(n), members(n);
  for (idx_t i = 0; i < n; ++i) {
    for (const idx_t *q = graph.begin(i); q != graph.end(i); ++q)
      if (role[*q] != Role::Dense) variables[i].push_back(*q);
    degree[i] = (idx_t)variables[i].size();
  }
  DegreeLists lists(n);
  idx_t remaining = 0;
  for (idx_t i = n - 1; i >= 0; --i)
    if (role[i] == Role::Variable) {
      lists.insert(i, degree[i]);
      ++remaining;
    }

  const idx_t unset = std::numeric_limits<idx_t>::max();
  std::vector<idx_t> in_pivot(n, unset), outside(n, 0), outside_stamp(n, unset), external(n, 0);
  idx_t min_degree = 0, step = 0;
  std::vector<idx_t> pivot_list;
  // Groups of candidate supervariables by hash, in first-seen order. Groups are disjoint and a
  // merge in one group reads nothing another group writes, so any group order gives one result.
  std::vector<std::pair<uint64_t, std::vector<idx_t>>> groups;
  std::vector<std::pair<uint64_t, idx_t>> hashed;

  while (remaining > 0) {
    while (lists.head[min_degree] < 0) ++min_degree;
    const idx_t p = lists.head[min_degree];
    lists.remove(p, min_degree);
    ++step;

    in_pivot[p] = step;
    pivot_list.clear();
    for (idx_t j : variables[p])
      if (role[j] == Role::Variable && in_pivot[j] != step) {
        in_pivot[j] = step;
        pivot_list.push_back(j);
      }
    std::vector<idx_t> absorbed_elements;
    absorbed_elements.swap(elements[p]);
    for (idx_t e : absorbed_elements) {
      if (role[e] != Role::Element) continue;
      for (idx_t j : element_list[e])
        if (role[j] == Role::Variable && in_pivot[j] != step) {
          in_pivot[j] = step;
          pivot_list.push_back(j);
        }
      role[e] = Role::Absorbed;
      element_list[e].clear();
      element_list[e].shrink_to_fit();
    }
    variables[p].clear();
    variables[p].shrink_to_fit();
    role[p] = Role::Element;
    remaining -= weight[p];
    order.push_back(p);
    order.insert(order.end(), members[p].begin(), members[p].end());
    members[p].clear();

    // |L_e \ L_p| for each element next to L_p
    for (idx_t i : pivot_list) {
      lists.remove(i, degree[i]);
      for (idx_t e : elements[i])
        if (role[e] == Role::Element) {
          if (outside_stamp[e] != step) {
            outside_stamp[e] = step;
            outside[e] = element_size[e];
          }
          outside[e] -= weight[i];
        }
    }

    // Update each variable of L_p, and hash its adjacency
    hashed.clear();
    for (idx_t i : pivot_list) {
      std::vector<idx_t> kept{p};
      idx_t from_elements = 0;
      for (idx_t e : elements[i]) {
        if (role[e] != Role::Element) continue;
        if (outside[e] == 0) {
          role[e] = Role::Absorbed;
          element_list[e].clear();
        } else {
          from_elements += outside[e];
          kept.push_back(e);
        }
      }
      std::vector<idx_t> near;
      idx_t from_variables = 0;
      for (idx_t j : variables[i])
        if (role[j] == Role::Variable && in_pivot[j] != step) {
          near.push_back(j);
          from_variables += weight[j];
        }
      external[i] = from_variables + from_elements;
      std::sort(kept.begin(), kept.end());
      std::sort(near.begin(), near.end());
      uint64_t h = 0;
      for (idx_t x : kept) h = h * 31u + (uint64_t)x;
      for (idx_t x : near) h = h * 31u + (uint64_t)x;
      elements[i] = std::move(kept);
      variables[i] = std::move(near);
      hashed.push_back({h, i});
    }

    // Supervariables: within each hash group, merge every later variable with identical
    // elements and variables into the first of its kind
    groups.clear();
    {
      std::vector<std::pair<uint64_t, idx_t>> sorted = hashed;
      std::stable_sort(sorted.begin(), sorted.end(),
                       [](const auto &a, const auto &b) { return a.first < b.first; });
      for (size_t k = 0; k < sorted.size();) {
        size_t e = k;
        while (e < sorted.size() && sorted[e].first == sorted[k].first) ++e;
        if (e - k > 1) {
          std::vector<idx_t> g;
          for (size_t t = k; t < e; ++t) g.push_back(sorted[t].second);
          groups.push_back({sorted[k].first, std::move(g)});
        }
        k = e;
      }
    }
    for (auto &grp : groups) {
      auto &group = grp.second;
      for (size_t a = 0; a < group.size(); ++a) {
        const idx_t i = group[a];
        if (role[i] != Role::Variable) continue;
        for (size_t b = a + 1; b < group.size(); ++b) {
          const idx_t j = group[b];
          if (role[j] == Role::Variable && elements[i] == elements[j] && variables[i] == variables[j]) {
            weight[i] += weight[j];
            weight[j] = 0;
            role[j] = Role::Merged;
            members[i].push_back(j);
            members[i].insert(members[i].end(), members[j].begin(), members[j].end());
            members[j].clear();
            elements[j].clear();
            variables[j].clear();
          }
        }
      }
    }

    // The new element over the principal variables left, and their approximate degrees
    pivot_list.erase(std::remove_if(pivot_list.begin(), pivot_list.end(),
                                    [&](idx_t i) { return role[i] != Role::Variable; }),
                     pivot_list.end());
    idx_t size = 0;
    for (idx_t i : pivot_list) size += weight[i];
    element_size[p] = size;
    for (idx_t i : pivot_list) {
      const idx_t others = size - weight[i];
      const idx_t bound = std::min({remaining - weight[i], degree[i] + others, external[i] + others});
      degree[i] = bound;
      lists.insert(i, bound);
      min_degree = std::min(min_degree, bound);
    }
    element_list[p] = pivot_list;
  }
  for (idx_t i = 0; i < n; ++i)
    if (role[i] == Role::Dense) order.push_back(i);
  if ((idx_t)order.size() != n) throw Error(kInternal, "AMD lost a node");
  return order;
}

// Liu's elimination tree with path compression, then each row's pattern as its row subtree,
// sorted, with the diagonal last (cholesky.rs:81-149).
SymbolicCholesky analyze_cholesky(const Adjacency &graph, std::vector<idx_t> perm) {
  SymbolicCholesky s;
  const idx_t n = (idx_t)perm.size();
  s.n = n;
  std::vector<idx_t> inverse(n);
  for (idx_t k = 0; k < n; ++k) inverse[perm[k]] = k;
  auto for_lower = [&](idx_t i, auto &&f) {
    const idx_t old = perm[i];
    for (const idx_t *q = graph.begin(old); q != graph.end(old); ++q) {
      const idx_t j = inverse[*q];
      if (j < i) f(j);
    }
  };
  s.parent.assign(n, -1);
  std::vector<idx_t> ancestor(n, -1);
  for (idx_t i = 0; i < n; ++i)
    for_lower(i, [&](idx_t j) {
      while (j != i) {
        const idx_t next = ancestor[j];
        ancestor[j] = i;
        if (next < 0) {
          s.parent[j] = i;
          break;
        }
        j = next;
      }
    });
  s.l_ptr.assign(1, 0);
  std::vector<idx_t> mark(n, -1);
  for (idx_t i = 0; i < n; ++i) {
    const size_t start = s.l_idx.size();
    mark[i] = i;
    for_lower(i, [&](idx_t j) {
      while (mark[j] != i) {
        mark[j] = i;
        s.l_idx.push_back(j);
        j = s.parent[j];
      }
    });
    std::sort(s.l_idx.begin() + start, s.l_idx.end());
    s.l_idx.push_back(i);
    s.l_ptr.push_back((idx_t)s.l_idx.size());
  }
  s.perm = std::move(perm);
  return s;
}

// Up-looking numeric Cholesky (cholesky.rs:206-311): row i of L solves against the rows above,
// taking its pattern's columns in increasing order; L's columns are filled as rows finish.
template <class T> Cholesky<T> factor_cholesky(const Compressed<T> &a, const SymbolicCholesky &s) {
  const idx_t n = s.n;
  if (!a.by_rows || a.rows != n || a.cols != n) throw Error(kShapeMismatch, "Cholesky needs a square CSR matrix of the analysed order");
  // A must equal Aᴴ (values judged exactly, as ybus_sparse's is_hermitian does)
  {
    Compressed<T> at = reorient(a);  // CSC of A = CSR of Aᵀ
    for (idx_t i = 0; i < n; ++i) {
      // compare row i of A with row i of Aᵀ (conjugated), ignoring stored zeros
      idx_t p = a.ptr[i], q = at.ptr[i];
      const idx_t pe = a.ptr[i + 1], qe = at.ptr[i + 1];
      while (p < pe || q < qe) {
        if (p < pe && a.val[p] == T(0)) { ++p; continue; }
        if (q < qe && at.val[q] == T(0)) { ++q; continue; }
        if (p >= pe || q >= qe || a.idx[p] != at.idx[q] || a.val[p] != conj_of(at.val[q]))
          throw Error(kNotSymmetric, "the matrix is not symmetric");
        ++p;
        ++q;
      }
    }
  }
  const Compressed<T> c = permute_symmetric(a, s.perm);
  std::vector<idx_t> col_start(n + 1, 0);
  for (idx_t j : s.l_idx) col_start[j + 1]++;
  for (idx_t j = 0; j < n; ++j) col_start[j + 1] += col_start[j];
  for (idx_t j = 0; j <= n; ++j) col_start[j] -= j;
  std::vector<idx_t> col_fill(col_start.begin(), col_start.end());
  const idx_t below = (idx_t)s.l_idx.size() - n;
  std::vector<idx_t> col_rows(below);
  std::vector<T> col_vals(below);
  std::vector<T> l_vals(s.l_idx.size()), diagonal(n), work(n, T(0));
  for (idx_t i = 0; i < n; ++i) {
    double remaining = 0.0;
    for (idx_t p = c.ptr[i]; p < c.ptr[i + 1]; ++p) {
      const idx_t col = c.idx[p];
      if (col < i) {
        work[col] = c.val[p];
      } else {
        if (col == i) remaining = real_of(c.val[p]);
        break;
      }
    }
    const idx_t diag_slot = s.l_ptr[i + 1] - 1;
    for (idx_t p = s.l_ptr[i]; p < diag_slot; ++p) {
      const idx_t j = s.l_idx[p];
      const T l_ij = work[j] / diagonal[j];
      work[j] = T(0);
      for (idx_t q = col_start[j]; q < col_fill[j]; ++q) {
        const idx_t m = col_rows[q];
        work[m] = work[m] - conj_of(col_vals[q]) * l_ij;
      }
      col_rows[col_fill[j]] = i;
      col_vals[col_fill[j]] = l_ij;
      col_fill[j]++;
      l_vals[p] = l_ij;
      remaining = remaining - magnitude_squared(l_ij);
    }
    if (std::isnan(remaining) || remaining <= 0.0)
      throw Error(kNotPositiveDefinite, "the matrix is not positive definite", s.perm[i]);
    diagonal[i] = T(std::sqrt(remaining));
    l_vals[diag_slot] = diagonal[i];
  }
  Cholesky<T> f;
  f.n = n;
  f.perm = s.perm;
  f.parent = s.parent;
  f.l.rows = f.l.cols = n;
  f.l.by_rows = true;
  f.l.ptr = s.l_ptr;
  f.l.idx = s.l_idx;
  f.l.val = std::move(l_vals);
  f.lh.rows = f.lh.cols = n;
  f.lh.by_rows = true;
  f.lh.ptr.assign(1, 0);
  f.lh.idx.reserve(s.l_idx.size());
  f.lh.val.reserve(s.l_idx.size());
  for (idx_t j = 0; j < n; ++j) {
    f.lh.idx.push_back(j);
    f.lh.val.push_back(diagonal[j]);
    for (idx_t q = col_start[j]; q < col_fill[j]; ++q) {
      f.lh.idx.push_back(col_rows[q]);
      f.lh.val.push_back(conj_of(col_vals[q]));
    }
    f.lh.ptr.push_back((idx_t)f.lh.idx.size());
  }
  return f;
}

// Left-looking Gilbert–Peierls LU with threshold partial pivoting (lu.rs:268-417). Column k
// solves L x = A[:, q[k]] over its reach, found by depth-first search in postorder; a pivot is
// the largest candidate, or the diagonal of the ordered matrix while it is at least tau times
// that. L's rows are renumbered by pivot step at the end and every column is sorted.
template <class T>
Lu<T> factor_lu(const Compressed<T> &a, const std::vector<idx_t> &q, double tau, bool prefer_diagonal) {
  if (a.by_rows || a.rows != a.cols || (idx_t)q.size() != a.cols)
    throw Error(kShapeMismatch, "LU needs a square CSC matrix and a column permutation of its order");
  if (!(tau > 0.0 && tau <= 1.0)) throw Error(kInvalidArgument, "the pivot threshold must be in (0, 1]");
  const idx_t n = a.cols;
  std::vector<idx_t> pinv(n, -1), l_ptr{0}, u_ptr{0}, l_idx, u_idx;
  std::vector<T> l_val, u_val, x(n, T(0));
  std::vector<idx_t> visited(n, -1), postorder;
  std::vector<std::pair<idx_t, idx_t>> stack;
  postorder.reserve(n);
  for (idx_t k = 0; k < n; ++k) {
    const idx_t col = q[k];
    postorder.clear();
    auto first_child = [&](idx_t row) { return pinv[row] >= 0 ? l_ptr[pinv[row]] + 1 : 0; };
    for (idx_t p = a.ptr[col]; p < a.ptr[col + 1]; ++p) {
      const idx_t start = a.idx[p];
      if (visited[start] == k) continue;
      visited[start] = k;
      stack.push_back({start, first_child(start)});
      while (!stack.empty()) {
        auto &top = stack.back();
        const idx_t row = top.first;
        idx_t next = top.second;
        const idx_t end = pinv[row] >= 0 ? l_ptr[pinv[row] + 1] : 0;
        idx_t unvisited = -1;
        while (next < end) {
          const idx_t child = l_idx[next++];
          if (visited[child] != k) {
            unvisited = child;
            break;
          }
        }
        top.second = next;
        if (unvisited >= 0) {
          visited[unvisited] = k;
          stack.push_back({unvisited, first_child(unvisited)});
        } else {
          stack.pop_back();
          postorder.push_back(row);
        }
      }
    }
    for (idx_t p = a.ptr[col]; p < a.ptr[col + 1]; ++p) x[a.idx[p]] = a.val[p];
    for (auto it = postorder.rbegin(); it != postorder.rend(); ++it) {
      const idx_t row = *it;
      if (pinv[row] >= 0) {
        const idx_t s = pinv[row];
        const T x_row = x[row];
        for (idx_t p = l_ptr[s] + 1; p < l_ptr[s + 1]; ++p) x[l_idx[p]] = x[l_idx[p]] - l_val[p] * x_row;
      }
    }
    double largest = 0.0;
    idx_t pivot_row = -1;
    for (auto it = postorder.rbegin(); it != postorder.rend(); ++it) {
      const idx_t row = *it;
      if (pinv[row] >= 0) {
        u_idx.push_back(pinv[row]);
        u_val.push_back(x[row]);
      } else {
        const double magnitude = abs_of(x[row]);
        if (magnitude > largest) {
          largest = magnitude;
          pivot_row = row;
        }
      }
    }
    if (pivot_row < 0) throw Error(kSingular, "the matrix is singular", col);
    if (prefer_diagonal && pinv[col] < 0 && visited[col] == k && abs_of(x[col]) >= tau * largest) pivot_row = col;
    const T pivot = x[pivot_row];
    u_idx.push_back(k);
    u_val.push_back(pivot);
    u_ptr.push_back((idx_t)u_idx.size());
    pinv[pivot_row] = k;
    l_idx.push_back(pivot_row);
    l_val.push_back(T(1));
    for (auto it = postorder.rbegin(); it != postorder.rend(); ++it) {
      const idx_t row = *it;
      if (pinv[row] < 0) {
        l_idx.push_back(row);
        l_val.push_back(x[row] / pivot);
      }
      x[row] = T(0);
    }
    l_ptr.push_back((idx_t)l_idx.size());
  }
  Lu<T> f;
  f.n = n;
  f.row_perm.assign(n, 0);
  for (idx_t row = 0; row < n; ++row) f.row_perm[pinv[row]] = row;
  for (auto &row : l_idx) row = pinv[row];
  auto sort_columns = [](const std::vector<idx_t> &ptr, std::vector<idx_t> &idx, std::vector<T> &val) {
    std::vector<std::pair<idx_t, T>> pairs;
    for (size_t c = 0; c + 1 < ptr.size(); ++c) {
      pairs.clear();
      for (idx_t p = ptr[c]; p < ptr[c + 1]; ++p) pairs.push_back({idx[p], val[p]});
      std::sort(pairs.begin(), pairs.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
      for (size_t o = 0; o < pairs.size(); ++o) {
        idx[ptr[c] + o] = pairs[o].first;
        val[ptr[c] + o] = pairs[o].second;
      }
    }
  };
  sort_columns(l_ptr, l_idx, l_val);
  sort_columns(u_ptr, u_idx, u_val);
  f.col_perm = q;
  auto fill = [n](Compressed<T> &m, std::vector<idx_t> &ptr, std::vector<idx_t> &idx, std::vector<T> &val) {
    m.rows = m.cols = n;
    m.by_rows = false;
    m.ptr = std::move(ptr);
    m.idx = std::move(idx);
    m.val = std::move(val);
  };
  fill(f.l, l_ptr, l_idx, l_val);
  fill(f.u, u_ptr, u_idx, u_val);
  return f;
}

template Cholesky<double> factor_cholesky(const Compressed<double> &, const SymbolicCholesky &);
template Cholesky<c128> factor_cholesky(const Compressed<c128> &, const SymbolicCholesky &);
template Lu<double> factor_lu(const Compressed<double> &, const std::vector<idx_t> &, double, bool);
template Lu<c128> factor_lu(const Compressed<c128> &, const std::vector<idx_t> &, double, bool);

}  // namespace yb::host
