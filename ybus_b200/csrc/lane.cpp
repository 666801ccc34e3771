// The lane solve's layout (lane_solve.cuh): the factor's rows in one order that serves both sweeps,
// cut into subtree domains that the warps of a block take in parallel under a top that one warp
// takes, and each warp's part as a stream of records that every lane of the warp runs on its own
// right-hand side.
//
// Order. The forest's parent of row c is the first row whose forward row reads c (for a Cholesky
// factor, the elimination tree). A postorder visits each subtree whole, children with the larger
// subtrees first, which keeps the values alive at any moment to a few tens for a power-network
// factor: the forward accumulators of rows that have started to receive updates, and in the
// backward sweep (the reverse order) the solutions that rows still to come will read.
//
// Cut. The subtrees whose work is at most a cap are the domains (the largest such subtrees); the
// rows above them are the top. The domains go to the warps by work, largest first, and the cap is
// the one whose estimate (the busiest warp's domains plus the top) is least. In the work array the
// rows sit warp by warp, each warp's domains in postorder, then the top in postorder.
//
// Forward, right-looking: at row j, z_j = (b_j + acc_j) * dinv_j, acc_j read and zeroed, then for
// every later row r that reads j, acc_r -= L_rj z_j. A domain's updates of top rows gather in its
// warp's slots and go to the block's partial array when the domain ends (a flush); once every
// domain has ended, the warps add each top row's partials, in a fixed order, into the row's right-
// hand side in the work array (the top rows dealt to the warps by their count of partials), so the
// top warp's chain of rows waits on no partial. Backward, left-looking, rows in
// reverse order: x_j = (z_j - sum of U_jc x_c) * dinv_j, x_j kept in a slot while rows still to
// come read it; a domain first imports the top solutions its rows read from the work array.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <tuple>
#include <vector>

#include "plan.hpp"

namespace yb {

namespace {

// Slot 0 is always zero (the accumulator of a row no update reaches), slot 1 takes solutions no
// row reads; live values take the lowest free slot from 2 (interval colouring in visiting order:
// exactly the peak of live values).
struct Slots {
  std::vector<uint8_t> used;
  int32_t live = 0, peak = 0;
  int32_t take() {
    int32_t s = 0;
    while (s < (int32_t)used.size() && used[s]) ++s;
    if (s == (int32_t)used.size()) used.push_back(0);
    used[s] = 1;
    peak = std::max(peak, ++live);
    return s + 2;
  }
  void give(int32_t s) {
    used[s - 2] = 0;
    --live;
  }
};

// Writes one warp's records into fixed-size pages. Every page ends with a kLanePageEnd record (room
// for it is always kept); a record never straddles a page, and a record whose entries do not fit one
// page continues in the next records. The writer follows the phase (first position, direction and
// length) so that each row record carries its work-row offset (the work row of the row at position
// p is work_row[p]) and prefetch-ring slot, and puts a kLanePrefetch record, with the offsets of the
// rows it copies, before every kLaneBatch rows.
template <class T> struct PageWriter {
  static constexpr uint32_t kEntry = sizeof(T) == 8 ? 16 : 8;
  uint32_t kRow;  // a live slot's, work row's or partial row's bytes: 32 lanes of rpl values
  int32_t page_bytes;
  std::vector<uint8_t> &blob;
  const std::vector<int32_t> &work_row;
  size_t pos = 0;
  int32_t start = 0, len = 0, step = 1, row_i = 0;
  PageWriter(std::vector<uint8_t> &b, int32_t pb, const std::vector<int32_t> &wr, uint32_t row_bytes)
      : kRow(row_bytes), page_bytes(pb), blob(b), work_row(wr) {
    open();
  }
  void open() {
    blob.resize(blob.size() + page_bytes, 0);
    pos = 0;
  }
  uint8_t *at() { return blob.data() + blob.size() - page_bytes + pos; }
  void put(uint32_t self, uint32_t kind, uint32_t count, uint32_t word, const void *tail, size_t tail_bytes) {
    uint8_t *p = at();
    const uint32_t h[2] = {self | kind << 16 | count << 24, word};
    std::memcpy(p, h, 8);
    if (tail_bytes) std::memcpy(p + 8, tail, tail_bytes);
  }
  void room(size_t bytes) {
    if (pos + bytes + 16 <= (size_t)page_bytes) return;
    put(0, kLanePageEnd, 0, 0, nullptr, 0);
    open();
  }
  size_t most_entries() const { return std::min<size_t>(255, (page_bytes - 32) / kEntry); }
  static size_t bytes_of(size_t count) { return 16 + ((count * kEntry + 15) & ~(size_t)15); }
  void entries_at(uint8_t *p, const std::vector<std::pair<T, uint32_t>> &entries, const uint32_t *words, size_t from,
                  size_t take) {
    for (size_t e = 0; e < take; ++e) {
      uint8_t *q = p + 16 + e * kEntry;
      if (words)
        std::memcpy(q, &words[from + e], 4);
      else
        std::memcpy(q, &entries[from + e].first, sizeof(T));
      std::memcpy(q + sizeof(T), &entries[from + e].second, 4);
    }
  }
  void simple(uint32_t kind) {
    room(16);
    put(0, kind, 0, 0, nullptr, 0);
    pos += 16;
  }
  // The work-row offsets of a batch of the phase (rows past its end: none), its row count and
  // whether it fills the ring's upper half.
  int32_t batch_rows(int32_t batch, uint32_t (&rows)[kLaneBatch], bool &upper) const {
    static_assert(kLaneBatch == 4, "a prefetch holds four row offsets");
    const int32_t r0 = batch * kLaneBatch;
    const int32_t count = std::max(0, std::min(kLaneBatch, len - r0));
    for (int32_t q = 0; q < kLaneBatch; ++q) rows[q] = q < count ? (uint32_t)work_row[start + step * (r0 + q)] * kRow : 0;
    upper = (r0 & (kLaneRows - 1)) != 0;
    return count;
  }
  // A batch's prefetch block: its four row offsets, the row count in bits 0-2 of the first and the
  // upper-half flag in bit 3 (row offsets are multiples of 128 bytes).
  void prefetch_block(int32_t batch, uint32_t (&block)[kLaneBatch]) const {
    bool upper;
    const int32_t count = batch_rows(batch, block, upper);
    block[0] |= (uint32_t)count | (upper ? 8u : 0u);
  }
  void prefetch(int32_t batch) {
    uint32_t block[kLaneBatch];
    prefetch_block(batch, block);
    room(32);
    put(0, kLanePrefetch, 16 / kEntry, 0, nullptr, 0);
    std::memcpy(at() + 16, block, 16);
    pos += 32;
  }
  void phase(int32_t first, int32_t rows, bool backward) {
    simple(kLanePhase);
    start = first, len = rows, step = backward ? -1 : 1, row_i = 0;
    prefetch(0);
    prefetch(1);
  }
  // A top row's partial sums: work row `row` += the partial rows `w`, split as the pages need (the
  // records of one row run in order, each adding into what the one before stored).
  void sums(uint32_t row, const std::vector<std::pair<T, uint32_t>> &entries, const std::vector<uint32_t> &w) {
    size_t done = 0;
    while (done < entries.size()) {
      const size_t take = std::min(most_entries(), entries.size() - done);
      room(bytes_of(take));
      put(0, kLaneTopSum, (uint32_t)take, row, nullptr, 0);
      entries_at(at(), entries, w.data(), done, take);
      pos += bytes_of(take);
      done += take;
    }
  }
  // The dense top's records (kLaneTopSum with a mode in the header's third word): entries {val or
  // a 32-bit word, offset}, split as the pages need, the first record of mode `first`, the rest of
  // mode `more`; returns the blob positions of the entries' offset fields, in order.
  std::vector<size_t> moded(uint32_t word, uint32_t first, uint32_t more, const std::vector<std::pair<T, uint32_t>> &entries,
                            const uint32_t *words) {
    std::vector<size_t> at_offset;
    size_t done = 0;
    while (done < entries.size()) {
      const size_t take = std::min(most_entries(), entries.size() - done);
      room(bytes_of(take));
      const uint32_t mode[2] = {done == 0 ? first : more, 0};
      put(0, kLaneTopSum, (uint32_t)take, word, mode, 8);
      entries_at(at(), entries, words, done, take);
      for (size_t e = 0; e < take; ++e)
        at_offset.push_back(blob.size() - (size_t)page_bytes + pos + 16 + e * kEntry + sizeof(T));
      pos += bytes_of(take);
      done += take;
    }
    return at_offset;
  }
  // Records with entries {a 32-bit word in val's place, offset}, split as the pages need.
  void words(uint32_t kind, uint32_t self, const std::vector<std::pair<T, uint32_t>> &entries,
             const std::vector<uint32_t> &w) {
    size_t done = 0;
    while (done < entries.size()) {
      const size_t take = std::min(most_entries(), entries.size() - done);
      room(bytes_of(take));
      put(self, kind, (uint32_t)take, 0, nullptr, 0);
      entries_at(at(), entries, w.data(), done, take);
      pos += bytes_of(take);
      done += take;
    }
  }
  // One row of the phase: its records carry its work-row offset, its ring slot and its diagonal's
  // reciprocal; rows of up to 4 entries take the kinds for their exact count.
  void row(uint32_t self, T dinv, const std::vector<std::pair<T, uint32_t>> &entries, bool backward) {
    const size_t count = entries.size();
    const bool opens_batch = row_i % kLaneBatch == 0 && row_i > 0;
    // a batch's prefetch rides on the row that opens it when that row has 1 to 4 entries
    const bool carries = opens_batch && count >= 1 && count <= 4;
    if (opens_batch && !carries) prefetch(row_i / kLaneBatch + 1);
    uint32_t pre[kLaneBatch] = {};
    if (carries) prefetch_block(row_i / kLaneBatch + 1, pre);
    const uint32_t ring = (uint32_t)(row_i & (kLaneRows - 1)) << 5;
    const uint32_t wpos = (uint32_t)work_row[start + step * row_i] * kRow;
    ++row_i;
    uint8_t tail[8] = {};
    std::memcpy(tail, &dinv, sizeof(T));
    if (carries) {
      const size_t body = ((count * kEntry + 15) & ~(size_t)15) + 16;
      room(16 + body);
      put(self, (backward ? kLaneBwdPre1 : kLaneFwdPre1) + (uint32_t)count - 1 + ring, (uint32_t)(count + 16 / kEntry),
          wpos, tail, 8);
      entries_at(at(), entries, nullptr, 0, count);
      std::memcpy(at() + 16 + body - 16, pre, 16);
      pos += 16 + body;
      return;
    }
    if (count <= 4) {
      room(bytes_of(count));
      put(self, (backward ? kLaneBwdRow0 : kLaneFwdRow0) + (uint32_t)count + ring, (uint32_t)count, wpos, tail, 8);
      entries_at(at(), entries, nullptr, 0, count);
      pos += bytes_of(count);
      return;
    }
    size_t done = 0;
    while (done < count) {
      const size_t take = std::min(most_entries(), count - done);
      const bool first = done == 0, last = done + take == count;
      uint32_t kind;
      if (!backward)
        kind = first ? kLaneFwdRowN : kLaneFwdMore;
      else
        kind = first && last ? kLaneBwdRowN : first ? kLaneBwdBegin : last ? kLaneBwdEnd : kLaneBwdMore;
      room(bytes_of(take));
      put(self, kind + ring, (uint32_t)take, wpos, tail, 8);
      entries_at(at(), entries, nullptr, done, take);
      pos += bytes_of(take);
      done += take;
    }
  }
};

struct Cut {
  std::vector<int32_t> roots;  // domain roots
  std::vector<std::vector<int32_t>> warp_domains;
  std::vector<uint8_t> is_top;
  double cost = 0;
};

template <class V, class T>
LaneLayout build(const Plan<V> &plan, int32_t page_bytes, int32_t max_slots, int32_t warps, int32_t rpl) {
  const int32_t n = plan.n;
  LaneLayout lay;
  lay.page_bytes = page_bytes;
  lay.value_bytes = (int32_t)sizeof(T);
  lay.rpl = rpl;
  lay.warps = warps;
  struct Row {
    int32_t p0 = 0, p1 = 0;
    double dinv = 1;
  };
  std::vector<Row> frow(n), brow(n);
  for (int32_t p = 0; p < n; ++p) {
    frow[plan.fwd.row[p]] = {plan.fwd.ptr[p], plan.fwd.ptr[p + 1], (double)plan.fwd.dinv[p]};
    brow[plan.bwd.row[p]] = {plan.bwd.ptr[p], plan.bwd.ptr[p + 1], (double)plan.bwd.dinv[p]};
  }
  // The forest: the elimination tree of the two triangles' joint pattern, by Liu's algorithm with
  // path compression over the entries (i, k), k < i, of the forward triangle and of the backward
  // one transposed. Every entry's larger index is then an ancestor of its smaller, so one
  // postorder serves the forward sweep and its reverse the backward. For a Cholesky factor this is
  // the factor's own elimination tree (each column's parent its first off-diagonal row); for an LU
  // factor it also covers U's entries, which L's tree alone need not order.
  std::vector<int32_t> below_ptr(n + 1, 0), below;  // backward entries by column: rows r < c with U(r, c)
  for (int32_t r = 0; r < n; ++r)
    for (int32_t q = brow[r].p0; q < brow[r].p1; ++q) {
      const int32_t c = plan.bwd.col[q];
      if (c <= r) throw host::Error(host::kInvalidArgument, "the backward sweep is not upper triangular");
      ++below_ptr[c + 1];
    }
  for (int32_t c = 0; c < n; ++c) below_ptr[c + 1] += below_ptr[c];
  below.resize(below_ptr[n]);
  {
    std::vector<int32_t> fill(below_ptr.begin(), below_ptr.end() - 1);
    for (int32_t r = 0; r < n; ++r)
      for (int32_t q = brow[r].p0; q < brow[r].p1; ++q) below[fill[plan.bwd.col[q]]++] = r;
  }
  std::vector<int32_t> parent(n, -1), ancestor(n, -1);
  for (int32_t i = 0; i < n; ++i) {
    auto join = [&](int32_t k) {
      while (ancestor[k] >= 0 && ancestor[k] != i) {
        const int32_t up = ancestor[k];
        ancestor[k] = i;
        k = up;
      }
      if (ancestor[k] < 0) ancestor[k] = i, parent[k] = i;
    };
    for (int32_t q = frow[i].p0; q < frow[i].p1; ++q) {
      const int32_t c = plan.fwd.col[q];
      if (c >= i) throw host::Error(host::kInvalidArgument, "the forward sweep is not lower triangular");
      join(c);
    }
    for (int32_t q = below_ptr[i]; q < below_ptr[i + 1]; ++q) join(below[q]);
  }
  std::vector<int64_t> size(n, 1);
  for (int32_t c = 0; c < n; ++c)
    if (parent[c] >= 0) size[parent[c]] += size[c];
  std::vector<int32_t> child_ptr(n + 2, 0), child(n);
  for (int32_t c = 0; c < n; ++c) ++child_ptr[(parent[c] < 0 ? n : parent[c]) + 1];
  for (int32_t i = 0; i <= n; ++i) child_ptr[i + 1] += child_ptr[i];
  {
    std::vector<int32_t> fill(child_ptr.begin(), child_ptr.end() - 1);
    for (int32_t c = 0; c < n; ++c) child[fill[parent[c] < 0 ? n : parent[c]]++] = c;
  }
  for (int32_t v = 0; v <= n; ++v)
    std::stable_sort(child.begin() + child_ptr[v], child.begin() + child_ptr[v + 1],
                     [&](int32_t a, int32_t b) { return size[a] > size[b]; });
  std::vector<int32_t> order;
  order.reserve(n);
  {
    std::vector<std::pair<int32_t, int32_t>> stack{{n, child_ptr[n]}};
    while (!stack.empty()) {
      auto &top = stack.back();
      const int32_t v = top.first;
      if (top.second < child_ptr[v + 1]) {
        const int32_t c = child[top.second++];
        stack.push_back({c, child_ptr[c]});
      } else {
        if (v < n) order.push_back(v);
        stack.pop_back();
      }
    }
  }
  std::vector<int32_t> pos(n);
  for (int32_t t = 0; t < n; ++t) pos[order[t]] = t;
  for (int32_t r = 0; r < n; ++r) {
    for (int32_t q = frow[r].p0; q < frow[r].p1; ++q)
      if (pos[plan.fwd.col[q]] >= pos[r]) throw host::Error(host::kInvalidArgument, "no postorder serves the forward sweep");
    for (int32_t q = brow[r].p0; q < brow[r].p1; ++q)
      if (pos[plan.bwd.col[q]] <= pos[r])
        throw host::Error(host::kInvalidArgument, "the backward sweep does not run in the reverse postorder");
  }
  // forward columns: the rows each row updates
  std::vector<int32_t> col_ptr(n + 1, 0), col_row;
  std::vector<double> col_val;
  for (int32_t r = 0; r < n; ++r)
    for (int32_t q = frow[r].p0; q < frow[r].p1; ++q) ++col_ptr[plan.fwd.col[q] + 1];
  for (int32_t c = 0; c < n; ++c) col_ptr[c + 1] += col_ptr[c];
  col_row.resize(col_ptr[n]);
  col_val.resize(col_ptr[n]);
  {
    std::vector<int32_t> fill(col_ptr.begin(), col_ptr.end() - 1);
    for (int32_t r = 0; r < n; ++r)
      for (int32_t q = frow[r].p0; q < frow[r].p1; ++q) {
        const int32_t c = plan.fwd.col[q];
        col_row[fill[c]] = r;
        col_val[fill[c]++] = (double)plan.fwd.val[q];
      }
  }
  // work of each row (both sweeps, in instruction-like units) and of each subtree
  constexpr double kRowWork = 60, kEntryWork = 7;
  std::vector<double> work(n), sub(n, 0.0);
  for (int32_t v = 0; v < n; ++v)
    work[v] = 2 * kRowWork + kEntryWork * ((col_ptr[v + 1] - col_ptr[v]) + (brow[v].p1 - brow[v].p0));
  for (int32_t t = 0; t < n; ++t) {
    const int32_t v = order[t];  // a postorder lists children first
    sub[v] += work[v];
    if (parent[v] >= 0) sub[parent[v]] += sub[v];
  }
  const double total = std::accumulate(work.begin(), work.end(), 0.0);
  auto cut_at = [&](double cap) {
    Cut c;
    c.is_top.assign(n, 0);
    double top_work = 0;
    for (int32_t v = 0; v < n; ++v)
      if (sub[v] > cap) c.is_top[v] = 1, top_work += work[v];
    for (int32_t v = 0; v < n; ++v)
      if (!c.is_top[v] && (parent[v] < 0 || c.is_top[parent[v]])) c.roots.push_back(v);
    std::vector<int32_t> by_work(c.roots);
    std::stable_sort(by_work.begin(), by_work.end(), [&](int32_t a, int32_t b) { return sub[a] > sub[b]; });
    std::vector<double> load(warps, 0.0);
    c.warp_domains.assign(warps, {});
    for (int32_t r : by_work) {
      const int32_t w = (int32_t)(std::min_element(load.begin(), load.end()) - load.begin());
      load[w] += sub[r] + kRowWork;
      c.warp_domains[w].push_back(r);
    }
    // each warp's domains in postorder, so its rows keep the whole postorder's order
    for (auto &d : c.warp_domains) std::sort(d.begin(), d.end(), [&](int32_t a, int32_t b) { return pos[a] < pos[b]; });
    c.cost = *std::max_element(load.begin(), load.end()) + top_work;
    return c;
  };
  Cut best = cut_at(total + 1);  // one domain per tree of the forest, no top
  if (warps > 1)
    for (int k = 0; k <= 48; ++k) {  // caps a quarter octave apart
      Cut c = cut_at(total / (warps * std::pow(2.0, k / 4.0)));
      if (c.cost < best.cost) best = std::move(c);
    }
  lay.cost = best.cost;
  lay.domains = (int32_t)best.roots.size();
  // the work array's order: warp by warp, each domain in postorder, then the top in postorder
  std::vector<int32_t> newpos(n, -1), warp_start(warps + 1, 0);
  std::vector<std::pair<int32_t, int32_t>> domain_range;  // first and last position of each domain
  std::vector<std::vector<int32_t>> warp_dom_index(warps);
  {
    int32_t next = 0;
    for (int32_t w = 0; w < warps; ++w) {
      warp_start[w] = next;
      for (int32_t r : best.warp_domains[w]) {
        const int32_t first = pos[r] - (int32_t)size[r] + 1, d0 = next;
        for (int32_t t = first; t <= pos[r]; ++t) newpos[order[t]] = next++;
        warp_dom_index[w].push_back((int32_t)domain_range.size());
        domain_range.push_back({d0, next - 1});
      }
    }
    warp_start[warps] = next;
    for (int32_t t = 0; t < n; ++t)
      if (best.is_top[order[t]]) newpos[order[t]] = next++;
    if (next != n) throw host::Error(host::kInternal, "the lane cut lost rows");
  }
  const int32_t top0 = warp_start[warps];
  lay.top = n - top0;
  std::vector<int32_t> at(n);
  for (int32_t v = 0; v < n; ++v) at[newpos[v]] = v;
  // the work array in b's own row order: row v's right-hand side, forward result and solution sit
  // in the work row of the row of b that feeds it, so the gather of b and (when b and x share
  // their permutation) the scatter of x copy whole runs of rows
  std::vector<int32_t> work_of(n, -1), work_row(n);
  for (int32_t i = 0; i < n; ++i) {
    const int32_t v = plan.in_slot[i];
    if (v < 0 || v >= n || work_of[v] >= 0) throw host::Error(host::kInvalidArgument, "the solve's input order is not a permutation");
    work_of[v] = i;
  }
  for (int32_t p = 0; p < n; ++p) work_row[p] = work_of[at[p]];
  // partials: one per (domain, top row it updates), domains in warp order, top rows by position
  std::vector<std::vector<uint32_t>> contributors(n);
  std::vector<std::vector<std::pair<int32_t, uint32_t>>> domain_partials(domain_range.size());
  {
    uint32_t k = 0;
    std::vector<int32_t> seen(n, -1);
    for (size_t d = 0; d < domain_range.size(); ++d) {
      std::vector<int32_t> tops;
      for (int32_t p = domain_range[d].first; p <= domain_range[d].second; ++p) {
        const int32_t j = at[p];
        for (int32_t q = col_ptr[j]; q < col_ptr[j + 1]; ++q) {
          const int32_t r = col_row[q];
          if (best.is_top[r] && seen[r] != (int32_t)d) seen[r] = (int32_t)d, tops.push_back(r);
        }
      }
      std::sort(tops.begin(), tops.end(), [&](int32_t a, int32_t b) { return newpos[a] < newpos[b]; });
      for (int32_t r : tops) {
        domain_partials[d].push_back({r, k});
        contributors[r].push_back(k++);
      }
    }
    lay.partials = (int32_t)k;
  }
  // the top rows with partials, dealt to the warps by their count of partials (largest first, each
  // to the warp with the fewest so far), each warp's share in position order
  std::vector<std::vector<int32_t>> top_sums(warps);
  {
    std::vector<int32_t> rows;
    for (int32_t p = top0; p < n; ++p)
      if (!contributors[at[p]].empty()) rows.push_back(at[p]);
    std::stable_sort(rows.begin(), rows.end(),
                     [&](int32_t a, int32_t b) { return contributors[a].size() > contributors[b].size(); });
    std::vector<size_t> load(warps, 0);
    for (int32_t j : rows) {
      const int32_t w = (int32_t)(std::min_element(load.begin(), load.end()) - load.begin());
      load[w] += 1 + contributors[j].size();
      top_sums[w].push_back(j);
    }
    for (auto &t : top_sums) std::sort(t.begin(), t.end(), [&](int32_t a, int32_t b) { return newpos[a] < newpos[b]; });
  }
  const uint32_t row_bytes = 32u * (uint32_t)sizeof(T) * (uint32_t)rpl;  // a live slot, or a work or partial row
  auto off = [&](int32_t s) { return (uint32_t)s * row_bytes; };
  auto self_of = [&](int32_t s) { return (uint32_t)s * row_bytes / 16; };  // headers hold slot offsets / 16
  // The dense top: in FP64, with several warps and a top of 2 to kLaneDenseTopMost rows, its forward and
  // backward substitution is one linear map x_T = M r_T from the top rows' right-hand sides (after
  // the partial sums) to their solutions; M is that substitution applied to the identity, in FP64
  // here, kept when its condition (||M||inf ||M^-1||inf) is at most kLaneDenseTopCondition.
  // Between the second and third barriers every warp loads its share of r_T (the top rows
  // `share` at a time, in position order) into its slots 2..; between the third and fourth it
  // forms its share of x_T from every warp's slots, so the top no longer runs as warp 0's chain.
  const int32_t t = n - top0;
  const int32_t share = warps > 1 ? (t + warps - 1) / warps : 0;
  std::vector<double> dense_m;
  // (FP64 only: in FP32 the map's rounding, about its condition times FP32's epsilon, slowed the
  // refined solve's convergence enough to cost it a third pass on the 10,000-bus block)
  bool dense = sizeof(T) == 8 && warps > 1 && t > 1 && t <= kLaneDenseTopMost && 2 + share <= std::min(max_slots, 255);
  if (dense) {
    std::vector<int32_t> tidx(n, -1);
    for (int32_t p = top0; p < n; ++p) tidx[at[p]] = p - top0;
    dense_m.assign((size_t)t * t, 0.0);
    std::vector<double> acc_t(t), z(t), x(t);
    for (int32_t e = 0; e < t && dense; ++e) {
      std::fill(acc_t.begin(), acc_t.end(), 0.0);
      for (int32_t p = 0; p < t; ++p) {
        const int32_t j = at[top0 + p];
        z[p] = ((p == e ? 1.0 : 0.0) + acc_t[p]) * frow[j].dinv;
        for (int32_t q = col_ptr[j]; q < col_ptr[j + 1]; ++q) {
          const int32_t r = tidx[col_row[q]];
          if (r < 0) dense = false;  // a top row updates no row below the top
          else acc_t[r] -= col_val[q] * z[p];
        }
      }
      for (int32_t p = t - 1; p >= 0; --p) {
        const int32_t j = at[top0 + p];
        double v = z[p];
        for (int32_t q = brow[j].p0; q < brow[j].p1; ++q) {
          const int32_t c = tidx[plan.bwd.col[q]];
          if (c < 0) dense = false;
          else v -= (double)plan.bwd.val[q] * x[c];
        }
        x[p] = v * brow[j].dinv;
      }
      for (int32_t i = 0; i < t; ++i) dense_m[(size_t)i * t + e] = x[i];
    }
    if (dense) {
      // ||M^-1||inf by Gauss-Jordan elimination with partial pivoting on a copy
      std::vector<double> a(dense_m), inv((size_t)t * t, 0.0);
      for (int32_t i = 0; i < t; ++i) inv[(size_t)i * t + i] = 1.0;
      for (int32_t k = 0; k < t && dense; ++k) {
        int32_t piv = k;
        for (int32_t i = k + 1; i < t; ++i)
          if (std::abs(a[(size_t)i * t + k]) > std::abs(a[(size_t)piv * t + k])) piv = i;
        if (a[(size_t)piv * t + k] == 0.0) {
          dense = false;
          break;
        }
        if (piv != k)
          for (int32_t j = 0; j < t; ++j) {
            std::swap(a[(size_t)k * t + j], a[(size_t)piv * t + j]);
            std::swap(inv[(size_t)k * t + j], inv[(size_t)piv * t + j]);
          }
        const double d = a[(size_t)k * t + k];
        for (int32_t j = 0; j < t; ++j) a[(size_t)k * t + j] /= d, inv[(size_t)k * t + j] /= d;
        for (int32_t i = 0; i < t; ++i) {
          if (i == k) continue;
          const double f = a[(size_t)i * t + k];
          if (f == 0.0) continue;
          for (int32_t j = 0; j < t; ++j) a[(size_t)i * t + j] -= f * a[(size_t)k * t + j], inv[(size_t)i * t + j] -= f * inv[(size_t)k * t + j];
        }
      }
      auto norm = [&](const std::vector<double> &m) {
        double most = 0;
        for (int32_t i = 0; i < t; ++i) {
          double row = 0;
          for (int32_t j = 0; j < t; ++j) row += std::abs(m[(size_t)i * t + j]);
          most = std::max(most, row);
        }
        return most;
      };
      if (dense) {
        lay.top_condition = norm(dense_m) * norm(inv);
        dense = std::isfinite(lay.top_condition) && lay.top_condition <= kLaneDenseTopCondition;
      }
    }
  }
  lay.dense_top = dense;
  // the dense rows' offsets into other warps' slots, patched when the slot count is known:
  // (blob position, warp, slot)
  std::vector<std::tuple<size_t, int32_t, int32_t>> patches;
  std::vector<std::pair<T, uint32_t>> entries;
  std::vector<uint32_t> words;
  std::vector<int32_t> acc(n, -1), xslot(n, -1), readers(n, 0);
  int32_t peak_f = 0, peak_b = 0;
  auto forward_rows = [&](PageWriter<T> &pw, Slots &slots, int32_t p0, int32_t p1) {
    for (int32_t p = p0; p <= p1; ++p) {
      const int32_t j = at[p];
      uint32_t self = self_of(0);
      if (acc[j] >= 0) {
        self = self_of(acc[j]);
        slots.give(acc[j]);
        acc[j] = -1;
      }
      entries.clear();
      for (int32_t q = col_ptr[j]; q < col_ptr[j + 1]; ++q) {
        const int32_t r = col_row[q];
        if (acc[r] < 0) acc[r] = slots.take();
        entries.push_back({(T)col_val[q], off(acc[r])});
      }
      lay.fwd_entries += (int64_t)entries.size();
      pw.row(self, (T)frow[j].dinv, entries, false);
    }
  };
  // readers[c]: the rows still to come that read x_c
  auto backward_rows = [&](PageWriter<T> &pw, Slots &slots, int32_t p0, int32_t p1) {
    for (int32_t p = p1; p >= p0; --p) {
      const int32_t j = at[p];
      entries.clear();
      for (int32_t q = brow[j].p0; q < brow[j].p1; ++q) entries.push_back({(T)plan.bwd.val[q], off(xslot[plan.bwd.col[q]])});
      for (int32_t q = brow[j].p0; q < brow[j].p1; ++q) {
        const int32_t c = plan.bwd.col[q];
        if (--readers[c] == 0) {
          slots.give(xslot[c]);
          xslot[c] = -1;
        }
      }
      uint32_t self = self_of(1);
      if (readers[j] > 0) {
        xslot[j] = slots.take();
        self = self_of(xslot[j]);
      }
      lay.bwd_entries += (int64_t)entries.size();
      pw.row(self, (T)brow[j].dinv, entries, true);
    }
  };
  lay.warp_page.assign(1, 0);
  for (int32_t w = 0; w < warps; ++w) {
    PageWriter<T> pw(lay.blob, page_bytes, work_row, row_bytes);
    const int32_t p0 = warp_start[w], p1 = warp_start[w + 1] - 1;
    {  // forward domains, each ending with its flush
      Slots slots;
      if (p1 >= p0) pw.phase(p0, p1 - p0 + 1, false);
      for (int32_t d : warp_dom_index[w]) {
        forward_rows(pw, slots, domain_range[d].first, domain_range[d].second);
        entries.clear();
        words.clear();
        for (auto [r, k] : domain_partials[d]) {
          entries.push_back({T(0), off(acc[r])});
          words.push_back(k * row_bytes);
          slots.give(acc[r]);
          acc[r] = -1;
        }
        pw.words(kLaneFlush, 0, entries, words);
      }
      peak_f = std::max(peak_f, slots.peak);
    }
    pw.simple(kLaneBarrier);
    for (int32_t j : top_sums[w]) {  // this warp's share of the top rows' partial sums
      entries.assign(contributors[j].size(), {T(0), 0u});
      words.clear();
      for (uint32_t k : contributors[j]) words.push_back(k * row_bytes);
      pw.sums((uint32_t)work_of[j] * row_bytes, entries, words);
    }
    pw.simple(kLaneBarrier);
    if (dense) {  // this warp's share of r_T into its slots 2..
      entries.clear();
      words.clear();
      for (int32_t i = w * share; i < std::min(t, (w + 1) * share); ++i) {
        entries.push_back({T(0), off(2 + i - w * share)});
        words.push_back((uint32_t)work_row[top0 + i] * row_bytes);
      }
      if (!entries.empty()) pw.moded(0, kTopLoad, kTopLoad, entries, words.data());
    } else if (w == 0 && top0 < n) {  // the top, forward then backward
      Slots slots;
      pw.phase(top0, n - top0, false);
      forward_rows(pw, slots, top0, n - 1);
      peak_f = std::max(peak_f, slots.peak);
      Slots bslots;
      for (int32_t p = top0; p < n; ++p)
        for (int32_t q = brow[at[p]].p0; q < brow[at[p]].p1; ++q) ++readers[plan.bwd.col[q]];
      pw.phase(n - 1, n - top0, true);
      backward_rows(pw, bslots, top0, n - 1);
      peak_b = std::max(peak_b, bslots.peak);
    }
    pw.simple(kLaneBarrier);
    if (dense)  // this warp's share of x_T, each a dense row over every warp's slots, into the output
      for (int32_t i = w * share; i < std::min(t, (w + 1) * share); ++i) {
        entries.clear();
        for (int32_t j = 0; j < t; ++j) entries.push_back({(T)dense_m[(size_t)i * t + j], 0u});
        const auto at_off = pw.moded((uint32_t)work_row[top0 + i] * row_bytes, kTopRow, kTopRowMore, entries, nullptr);
        for (int32_t j = 0; j < t; ++j) patches.push_back({at_off[(size_t)j], j / share, 2 + j % share});
      }
    pw.simple(kLaneBarrier);
    {  // backward domains in reverse, each starting with the top solutions it reads
      Slots slots;
      if (p1 >= p0) pw.phase(p1, p1 - p0 + 1, true);
      const auto &doms = warp_dom_index[w];
      for (auto it = doms.rbegin(); it != doms.rend(); ++it) {
        const int32_t d0 = domain_range[*it].first, d1 = domain_range[*it].second;
        std::vector<int32_t> imports;
        for (int32_t p = d0; p <= d1; ++p)
          for (int32_t q = brow[at[p]].p0; q < brow[at[p]].p1; ++q) {
            const int32_t c = plan.bwd.col[q];
            if (readers[c]++ == 0 && best.is_top[c]) imports.push_back(c);
          }
        if (!imports.empty()) {
          std::sort(imports.begin(), imports.end(), [&](int32_t a, int32_t b) { return newpos[a] < newpos[b]; });
          entries.clear();
          words.clear();
          for (int32_t c : imports) {
            xslot[c] = slots.take();
            entries.push_back({T(0), off(xslot[c])});
            words.push_back((uint32_t)work_of[c] * row_bytes);
          }
          pw.words(kLaneImport, 0, entries, words);
        }
        backward_rows(pw, slots, d0, d1);
      }
      peak_b = std::max(peak_b, slots.peak);
    }
    pw.simple(kLaneEnd);
    lay.warp_page.push_back((int32_t)(lay.blob.size() / page_bytes));
  }
  lay.fwd_live = peak_f;
  lay.bwd_live = peak_b;
  lay.slots = 2 + std::max(peak_f, peak_b);
  if (dense) lay.slots = std::max(lay.slots, 2 + share);
  if (lay.slots > std::min(max_slots, 255))
    throw host::Error(host::kTooLarge, "the lane solve would keep more live values than its shared memory holds");
  {  // the dense rows' block-wide offsets: warp w's slot s at w * (a warp's shared bytes) + s * row
    const size_t wb = lane_warp_bytes_of((int32_t)sizeof(T), lay.slots, kLaneRing, page_bytes, rpl);
    for (const auto &[at_blob, warp, slot] : patches) {
      const size_t v = (size_t)warp * wb + (size_t)slot * row_bytes;
      if (v > UINT32_MAX) throw host::Error(host::kTooLarge, "a dense top offset does not fit 32 bits");
      const uint32_t o = (uint32_t)v;
      std::memcpy(lay.blob.data() + at_blob, &o, 4);
    }
  }
  lay.in_pos.resize(n);
  lay.out_pos.resize(n);
  for (int32_t i = 0; i < n; ++i) {
    lay.in_pos[i] = work_of[plan.in_slot[i]];
    lay.out_pos[i] = work_of[plan.out_slot[i]];
  }
  return lay;
}

}  // namespace

template <class T>
LaneLayout lane_layout(const Plan<T> &plan, int32_t value_bytes, int32_t page_bytes, int32_t max_slots, int32_t warps,
                       int32_t rpl) {
  if (page_bytes < 256 || page_bytes % 16)
    throw host::Error(host::kInvalidArgument, "pages must be 16-byte multiples of at least 256 bytes");
  if (warps < 1 || warps > 32) throw host::Error(host::kInvalidArgument, "1 to 32 warps per block");
  if (rpl != 1 && rpl != 2) throw host::Error(host::kInvalidArgument, "1 or 2 right-hand sides per lane");
  if (value_bytes == 8) return build<T, double>(plan, page_bytes, max_slots, warps, rpl);
  if (value_bytes == 4) return build<T, float>(plan, page_bytes, max_slots, warps, rpl);
  throw host::Error(host::kInvalidArgument, "values must be 8 or 4 bytes");
}

template LaneLayout lane_layout(const Plan<double> &, int32_t, int32_t, int32_t, int32_t, int32_t);

}  // namespace yb
