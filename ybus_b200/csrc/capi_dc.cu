// C ABI of the DC callers of the solve path (ybus_powerflow/src/dc/gpu.rs: `DcGpuStudy`,
// `DcGpuSensitivity`), for networks given as branch lists: B' and Bf built from the branch
// stamps (ybus_powerflow/src/dc.rs:79-113: b = 1/x, parallel branches summed), B' factored by AMD
// Cholesky on the host and uploaded, Bf kept as an operator on the solutions. On top of the
// factor's pair solves and products: PTDF columns and transfers (dc/sensitivity.rs:233-300),
// LODF columns with bridges masked (dc/sensitivity.rs:322-362, islands.rs:132-176), and the
// batched N-1 screening of many injection scenarios per outage, in FP64 with the rank-one
// outage update, the flows and their maxima fused into the solve, or in FP32 with FP64
// refinement followed by the same epilogue.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/ybgpu.h"
#include "capi_common.hpp"
#include "device.cuh"
#include "domain_solve.cuh"
#include "factor_state.cuh"

using namespace yb;
using host::idx_t;

namespace yb {
// From capi_gpu.cu: the FP64 domain solve's launch for an IO policy.
template <class IO> void launch_domain_fp64(yb_factor *f, int64_t count, const IO &io, cudaStream_t stream);
}  // namespace yb

struct yb_dc_network {
  yb_gpu *gpu = nullptr;
  int64_t n_bus = 0, n_branch = 0, slack = 0, n = 0;
  std::vector<int64_t> from, to, unknown;  // unknown: per bus, -1 for the slack
  std::vector<double> b;
  std::vector<uint8_t> bridge;
  yb_factor *factor = nullptr;
  yb_operator *flows = nullptr;
  // the screening's device data: per branch, per bus, and the workspace of the last batch size
  DeviceArray<int32_t> br_slot_f, br_slot_t, br_u_f, br_u_t, bus_slot;
  DeviceArray<double> br_b;
  DeviceArray<double> d_weight, d_inj, d_y, d_theta, d_cy, d_invb, d_ratio;
  DeviceArray<int32_t> d_case_of, d_plus_u, d_minus_u, d_plus_slot, d_minus_slot, d_branch, d_bad, d_sing, d_steps;
  DeviceArray<int64_t> d_row;
  DeviceArray<double> d_value;
  // the whole-solution calls' workspace (dc_solutions)
  struct Solutions {
    DeviceArray<int32_t> case_of, bus_of, unknown, out_ptr, out_branch, col_ptr, pu, mu, p0, p1, piv, singular, flags;
    DeviceArray<double> inj, rhs, theta, theta_bus, flows, y, lu, s0, s1, invb;
  } sol;
  // the distributed slack's shift H w over the branches, negated (empty: the single slack)
  std::vector<double> negated_shift;
  // a captured graph of the FP64 screening for the sizes it was made for
  cudaGraphExec_t graph = nullptr;
  int64_t graph_cases = -1, graph_columns = -1;
  ~yb_dc_network() {
    if (graph) cudaGraphExecDestroy(graph);
    if (flows) yb_operator_free(flows);
    if (factor) yb_factor_free(factor);
  }
};

namespace {

// Bridges of a multigraph (ybus_powerflow/src/islands.rs:132-176): parallel branches are separate
// edges, so neither of a parallel pair is a bridge; a self-loop never is. Iterative DFS.
std::vector<uint8_t> find_bridges(int64_t n_bus, const std::vector<int64_t> &from, const std::vector<int64_t> &to) {
  const int64_t m = (int64_t)from.size();
  std::vector<std::vector<std::pair<int64_t, int64_t>>> adj(n_bus);
  for (int64_t k = 0; k < m; ++k)
    if (from[k] != to[k]) adj[from[k]].push_back({to[k], k}), adj[to[k]].push_back({from[k], k});
  std::vector<int64_t> disc(n_bus, -1), low(n_bus, 0);
  std::vector<uint8_t> bridge(m, 0);
  int64_t timer = 0;
  struct Frame {
    int64_t node, via;
    size_t next;
  };
  std::vector<Frame> stack;
  for (int64_t root = 0; root < n_bus; ++root) {
    if (disc[root] >= 0) continue;
    disc[root] = low[root] = timer++;
    stack.push_back({root, -1, 0});
    while (!stack.empty()) {
      Frame &fr = stack.back();
      if (fr.next < adj[fr.node].size()) {
        const auto [nxt, k] = adj[fr.node][fr.next++];
        if (k == fr.via) continue;
        if (disc[nxt] < 0) {
          disc[nxt] = low[nxt] = timer++;
          stack.push_back({nxt, k, 0});
        } else {
          low[fr.node] = std::min(low[fr.node], disc[nxt]);
        }
      } else {
        const Frame done = fr;
        stack.pop_back();
        if (!stack.empty()) {
          Frame &parent = stack.back();
          low[parent.node] = std::min(low[parent.node], low[done.node]);
          if (low[done.node] > disc[parent.node]) bridge[done.via] = 1;
        }
      }
    }
  }
  return bridge;
}

yb_dc_network *check(yb_dc_network *net) {
  require(net != nullptr, "null network");
  return net;
}

// Solves pairs in chunks of the factor's block width and returns the flows (n_branch x count).
std::vector<double> pair_flows(yb_dc_network *net, const std::vector<int64_t> &plus, const std::vector<int64_t> &minus) {
  const int64_t count = (int64_t)plus.size();
  std::vector<double> out((size_t)(net->n_branch * count));
  const int64_t width = std::max<int64_t>(1, yb_factor_block_width(net->factor));
  for (int64_t k0 = 0; k0 < count; k0 += width) {
    const int64_t k1 = std::min(count, k0 + width);
    yb_block *blk = nullptr;
    int32_t st = yb_pair_solves(net->factor, k1 - k0, plus.data() + k0, minus.data() + k0, &blk);
    if (st != YB_OK) throw host::Error(st, "pair solves failed");
    st = yb_block_product(blk, net->flows, nullptr, out.data() + k0 * net->n_branch);
    yb_block_free(blk);
    if (st != YB_OK) throw host::Error(st, "flow products failed");
  }
  return out;
}

// The epilogue of the FP32-and-refinement screening: as OutageIO's, with theta from an array in
// natural unknown order. One block of 256 threads per column.
__global__ void outage_epilogue_kernel(const double *__restrict__ theta, int64_t ldt, const int32_t *__restrict__ case_of,
                                       const int32_t *__restrict__ c_plus_u, const int32_t *__restrict__ c_minus_u,
                                       const double *__restrict__ c_invb, const double *__restrict__ c_cy,
                                       const int32_t *__restrict__ c_branch, const double *__restrict__ Y, int64_t ldy,
                                       int32_t n_branch, const int32_t *__restrict__ br_u_f,
                                       const int32_t *__restrict__ br_u_t, const double *__restrict__ br_b,
                                       const double *__restrict__ weight, int64_t *__restrict__ out_row,
                                       double *__restrict__ out_value, int32_t *__restrict__ out_bad,
                                       int32_t *__restrict__ case_singular) {
  __shared__ double red_v[8];
  __shared__ int red_r[8], red_b[8];
  const int64_t col = blockIdx.x;
  const double *th = theta + col * ldt;
  const int c = case_of[col];
  const double *y = Y + (int64_t)c * ldy;
  const int p = c_plus_u[c], m = c_minus_u[c];
  const double cx = __dsub_rn(__dadd_rn(0.0, p >= 0 ? th[p] : 0.0), m >= 0 ? th[m] : 0.0);
  const double w = __dadd_rn(-c_cy[c], c_invb[c]);
  const bool sing = (w == 0.0);
  const double z = sing ? 0.0 : __ddiv_rn(cx, w);
  const int k = c_branch[c];
  double v = 0.0;
  int row = -1, bad = 0;
  for (int l = threadIdx.x; l < n_branch; l += blockDim.x) {
    const int uf = br_u_f[l], ut = br_u_t[l];
    const double tf = uf < 0 ? 0.0 : __dadd_rn(th[uf], __dmul_rn(z, y[uf]));
    const double tt = ut < 0 ? 0.0 : __dadd_rn(th[ut], __dmul_rn(z, y[ut]));
    if ((uf >= 0 && !(fabs(tf) <= 1e5)) || (ut >= 0 && !(fabs(tt) <= 1e5))) bad |= 2;
    const double f = l == k ? 0.0 : __dadd_rn(__dmul_rn(br_b[l], tf), __dmul_rn(-br_b[l], tt));
    if (!isfinite(f)) {
      bad |= 1;
      continue;
    }
    const double load = fabs(f) * weight[l];
    if (load > v) v = load, row = l;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double v2 = __shfl_xor_sync(0xffffffffu, v, off);
    const int r2 = __shfl_xor_sync(0xffffffffu, row, off);
    bad |= __shfl_xor_sync(0xffffffffu, bad, off);
    better_max(v, row, v2, r2);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red_v[warp] = v, red_r[warp] = row, red_b[warp] = bad;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w2 = 1; w2 < (int)(blockDim.x >> 5); ++w2) {
      better_max(v, row, red_v[w2], red_r[w2]);
      bad |= red_b[w2];
    }
    out_row[col] = row;
    out_value[col] = row >= 0 ? v : 0.0;
    out_bad[col] = bad;
    case_singular[c] = sing ? 1 : 0;
  }
}

// c'y of each case, summed as the reference's update sums it: 0 + y_plus - y_minus
__global__ void case_cy_kernel(const double *__restrict__ Y, int64_t ldy, const int32_t *__restrict__ plus_u,
                               const int32_t *__restrict__ minus_u, int64_t cases, double *__restrict__ cy) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cases) return;
  const double *y = Y + c * ldy;
  double s = 0.0;
  if (plus_u[c] >= 0) s = __dadd_rn(s, y[plus_u[c]]);
  if (minus_u[c] >= 0) s = __dsub_rn(s, y[minus_u[c]]);
  cy[c] = s;
}

// ---- whole solutions: solves with placement, multi-branch outages ------------------------------

constexpr int kMaxOutageRank = 16;  // the branches one outage case may take out together

// The right-hand sides over the unknowns from injections over the buses: rhs[s][u] = inj[s][bus_of[u]].
__global__ void unknowns_of_buses_kernel(const double *__restrict__ inj, int64_t ldi, const int32_t *__restrict__ bus_of,
                                         int64_t n, int64_t S, double *__restrict__ rhs) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * S) return;
  const int64_t s = k / n, u = k - s * n;
  rhs[k] = inj[s * ldi + bus_of[u]];
}

// c'v for an outaged branch's c over the unknowns, summed as ybus_powerflow's outage update sums it
// (dc/outage.rs:200-202): from 0, each entry sign * v[position] in position order.
__device__ __forceinline__ double c_dot(int32_t p0, double s0, int32_t p1, double s1, const double *v) {
  double d = __dadd_rn(0.0, s0 * v[p0]);
  if (p1 >= 0) d = __dadd_rn(d, s1 * v[p1]);
  return d;
}

// Per case (one thread): W = D^-1 - C'Y over its m outaged branches that touch an unknown
// (dc/outage.rs:205-216: W_ij = -c_i'y_j, plus 1/b_i on the diagonal), factored in place by LU with
// partial pivoting into lu (kMaxOutageRank^2 per case, row-major) and piv; singular when a pivot is
// zero or not finite (reactances that cancel), besides the cases the host found to island a bus.
__global__ void outage_lu_kernel(const double *__restrict__ Y, int64_t ldy, const int32_t *__restrict__ col_ptr,
                                 const int32_t *__restrict__ pos0, const double *__restrict__ sign0,
                                 const int32_t *__restrict__ pos1, const double *__restrict__ sign1,
                                 const double *__restrict__ invb, int64_t cases, double *__restrict__ lu,
                                 int32_t *__restrict__ piv, int32_t *__restrict__ singular) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cases || singular[c]) return;  // a case that islands a bus, found on the host
  constexpr int R = kMaxOutageRank;
  const int q0 = col_ptr[c], m = col_ptr[c + 1] - q0;
  double *a = lu + c * R * R;
  int32_t *pv = piv + c * R;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      double w = -c_dot(pos0[q0 + i], sign0[q0 + i], pos1[q0 + i], sign1[q0 + i], Y + (int64_t)(q0 + j) * ldy);
      if (i == j) w = __dadd_rn(w, invb[q0 + i]);
      a[i * R + j] = w;
    }
  bool sing = false;
  for (int k = 0; k < m; ++k) {
    int p = k;
    for (int i = k + 1; i < m; ++i)
      if (fabs(a[i * R + k]) > fabs(a[p * R + k])) p = i;
    pv[k] = p;
    if (p != k)
      for (int j = 0; j < m; ++j) {
        const double t = a[k * R + j];
        a[k * R + j] = a[p * R + j], a[p * R + j] = t;
      }
    const double d = a[k * R + k];
    if (d == 0.0 || !isfinite(d)) {
      sing = true;
      break;
    }
    for (int i = k + 1; i < m; ++i) {
      const double l = __ddiv_rn(a[i * R + k], d);
      a[i * R + k] = l;
      for (int j = k + 1; j < m; ++j) a[i * R + j] = __dsub_rn(a[i * R + j], __dmul_rn(l, a[k * R + j]));
    }
  }
  singular[c] = sing ? 1 : 0;
}

// One block per scenario column of a case with outaged branches: ctx_i = c_i'theta0, z = W^-1 ctx by
// the case's LU, and theta = theta0 + sum_j z_j y_j over the unknowns in place, in j order with the
// products and sums rounded apart as the CPU's x_i += z_j y_i (dc/outage.rs:217-236). A singular
// case's columns keep theta0 (the case is flagged).
__global__ void outage_update_kernel(double *__restrict__ theta, int64_t n, const int32_t *__restrict__ case_of,
                                     const int32_t *__restrict__ col_ptr, const int32_t *__restrict__ pos0,
                                     const double *__restrict__ sign0, const int32_t *__restrict__ pos1,
                                     const double *__restrict__ sign1, const double *__restrict__ lu,
                                     const int32_t *__restrict__ piv, const int32_t *__restrict__ singular,
                                     const double *__restrict__ Y, int64_t ldy) {
  constexpr int R = kMaxOutageRank;
  __shared__ double z[R];
  const int64_t s = blockIdx.x;
  const int c = case_of[s];
  const int q0 = col_ptr[c], m = col_ptr[c + 1] - q0;
  if (m == 0 || singular[c]) return;  // the whole block
  double *th = theta + s * n;
  if (threadIdx.x == 0) {
    double v[R];
    for (int i = 0; i < m; ++i) v[i] = c_dot(pos0[q0 + i], sign0[q0 + i], pos1[q0 + i], sign1[q0 + i], th);
    const double *a = lu + (int64_t)c * R * R;
    const int32_t *pv = piv + (int64_t)c * R;
    for (int k = 0; k < m; ++k) {  // P: the row swaps in order, then L (unit) and U
      const int p = pv[k];
      if (p != k) {
        const double t = v[k];
        v[k] = v[p], v[p] = t;
      }
    }
    for (int i = 1; i < m; ++i)
      for (int j = 0; j < i; ++j) v[i] = __dsub_rn(v[i], __dmul_rn(a[i * R + j], v[j]));
    for (int i = m - 1; i >= 0; --i) {
      for (int j = i + 1; j < m; ++j) v[i] = __dsub_rn(v[i], __dmul_rn(a[i * R + j], v[j]));
      v[i] = __ddiv_rn(v[i], a[i * R + i]);
    }
    for (int i = 0; i < m; ++i) z[i] = v[i];
  }
  __syncthreads();
  for (int64_t r = threadIdx.x; r < n; r += blockDim.x) {
    double x = th[r];
    for (int j = 0; j < m; ++j) x = __dadd_rn(x, __dmul_rn(z[j], __ldg(Y + (int64_t)(q0 + j) * ldy + r)));
    th[r] = x;
  }
}

// One block per scenario column: theta over the buses (the slack's 0) and each branch's flow
// b_k theta_f + (-b_k) theta_t (the row of Bf), zero for the branches the column's case takes out;
// flags: 1 a flow not finite, 2 an angle not finite or above 1e5 in magnitude (the check of
// ybus_powerflow's DcStudy::place, dc.rs:558-564).
__global__ void place_flows_kernel(const double *__restrict__ theta, int64_t n, int32_t n_bus,
                                   const int32_t *__restrict__ unknown, int32_t nl, const int32_t *__restrict__ br_u_f,
                                   const int32_t *__restrict__ br_u_t, const double *__restrict__ br_b,
                                   const int32_t *__restrict__ case_of, const int32_t *__restrict__ out_ptr,
                                   const int32_t *__restrict__ out_branch, double *__restrict__ theta_bus,
                                   double *__restrict__ flows, int32_t *__restrict__ flags) {
  __shared__ int red[32];
  const int64_t s = blockIdx.x;
  const double *th = theta + s * n;
  int bad = 0;
  for (int i = threadIdx.x; i < n_bus; i += blockDim.x) {
    const int u = unknown[i];
    const double t = u < 0 ? 0.0 : th[u];
    if (u >= 0 && !(fabs(t) <= 1e5)) bad |= 2;
    if (theta_bus) theta_bus[s * n_bus + i] = t;
  }
  const int c = case_of ? case_of[s] : 0;
  const int o0 = case_of ? out_ptr[c] : 0, o1 = case_of ? out_ptr[c + 1] : 0;
  for (int l = threadIdx.x; l < nl; l += blockDim.x) {
    bool out = false;
    for (int o = o0; o < o1; ++o) out |= out_branch[o] == l;
    const int uf = br_u_f[l], ut = br_u_t[l];
    const double tf = uf < 0 ? 0.0 : th[uf], tt = ut < 0 ? 0.0 : th[ut];
    const double b = br_b[l];
    const double f = out ? 0.0 : __dadd_rn(__dmul_rn(b, tf), __dmul_rn(-b, tt));
    if (!isfinite(f)) bad |= 1;
    if (flows) flows[s * (int64_t)nl + l] = f;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = bad;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) bad |= red[w];
    flags[s] = bad;
  }
}

// Solutions of many scenarios with outages of several branches each: case c takes out the branches
// branch_ptr[c] .. branch_ptr[c+1] - 1 of `branches` (none: the plain solve) and has the scenario
// columns scenario_ptr[c] .. scenario_ptr[c+1] - 1 of `injections` (n_bus x S, by bus). On the
// device: theta0 = B'^-1 p of every scenario, Y = B'^-1 C of every outaged branch (pair solves),
// every case's W = D^-1 - C'Y factored, every scenario's theta updated, placed over the buses and
// turned into flows. Outputs (host arrays, each may be null): theta over the buses (n_bus x S),
// flows (n_branch x S), flags per scenario (place_flows_kernel's), singular per case.
void dc_solutions(yb_dc_network *net, int64_t cases, const int64_t *branch_ptr, const int64_t *branches,
                  const int64_t *scenario_ptr, const double *injections, double *theta, double *flows, int32_t *flags,
                  int32_t *singular) {
  require(cases >= 1 && scenario_ptr && scenario_ptr[0] == 0, "scenario pointers must start at 0");
  for (int64_t c = 0; c < cases; ++c) require(scenario_ptr[c + 1] >= scenario_ptr[c], "scenario pointers must not decrease");
  const int64_t S = scenario_ptr[cases];
  require(S == 0 || injections, "null injections");
  if (branch_ptr) {
    require(branch_ptr[0] == 0, "branch pointers must start at 0");
    for (int64_t c = 0; c < cases; ++c) require(branch_ptr[c + 1] >= branch_ptr[c], "branch pointers must not decrease");
    require(branch_ptr[cases] == 0 || branches, "null branches");
  }
  yb_factor *f = net->factor;
  const int64_t n = net->n, nl = net->n_branch, nb = net->n_bus;
  // per case: its outaged branches sorted without repeats (flows zeroed), and the columns of C of
  // those that touch an unknown, each with its entries in position order
  std::vector<int32_t> out_ptr(1, 0), out_branch, col_ptr(1, 0), pu, mu, p0, p1;
  std::vector<double> s0, s1, invb;
  for (int64_t c = 0; c < cases; ++c) {
    std::vector<int64_t> rows;
    if (branch_ptr)
      for (int64_t j = branch_ptr[c]; j < branch_ptr[c + 1]; ++j) {
        require(branches[j] >= 0 && branches[j] < nl, "an outaged branch is out of range");
        rows.push_back(branches[j]);
      }
    std::sort(rows.begin(), rows.end());
    rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
    require((int64_t)rows.size() <= kMaxOutageRank, "a case takes out more than 16 branches");
    for (const int64_t k : rows) {
      out_branch.push_back((int32_t)k);
      const int64_t pf = net->unknown[net->from[k]], pt = net->unknown[net->to[k]];
      if (net->from[k] == net->to[k] || (pf < 0 && pt < 0)) continue;
      pu.push_back((int32_t)pf), mu.push_back((int32_t)pt);
      // the entries (position, sign) in position order: the from end +1, the to end -1
      std::vector<std::pair<int64_t, double>> e;
      if (pf >= 0) e.push_back({pf, 1.0});
      if (pt >= 0) e.push_back({pt, -1.0});
      std::sort(e.begin(), e.end());
      p0.push_back((int32_t)e[0].first), s0.push_back(e[0].second);
      p1.push_back(e.size() > 1 ? (int32_t)e[1].first : -1), s1.push_back(e.size() > 1 ? e[1].second : 0.0);
      invb.push_back(1.0 / net->b[k]);
    }
    out_ptr.push_back((int32_t)out_branch.size());
    col_ptr.push_back((int32_t)pu.size());
  }
  const int64_t K = (int64_t)pu.size();
  // the cases whose outage leaves a bus without a path to the slack (`outaged_branches`' reach
  // check, dc/outage.rs:243+): W is singular in exact arithmetic, whatever rounding makes of it
  std::vector<int32_t> islands((size_t)cases, 0);
  {
    std::vector<int64_t> parent((size_t)nb);
    std::vector<uint8_t> out((size_t)nl, 0);
    auto find = [&](int64_t a) {
      while (parent[(size_t)a] != a) a = parent[(size_t)a] = parent[(size_t)parent[(size_t)a]];
      return a;
    };
    for (int64_t c = 0; c < cases; ++c) {
      const int32_t o0 = out_ptr[(size_t)c], o1 = out_ptr[(size_t)c + 1];
      if (o1 == o0) continue;
      if (o1 - o0 == 1) {
        islands[(size_t)c] = net->bridge[(size_t)out_branch[(size_t)o0]] ? 1 : 0;
        continue;
      }
      for (int32_t o = o0; o < o1; ++o) out[(size_t)out_branch[(size_t)o]] = 1;
      for (int64_t i = 0; i < nb; ++i) parent[(size_t)i] = i;
      int64_t parts = nb;
      for (int64_t k = 0; k < nl; ++k) {
        if (out[(size_t)k]) continue;
        const int64_t a = find(net->from[k]), b = find(net->to[k]);
        if (a != b) parent[(size_t)a] = b, --parts;
      }
      for (int32_t o = o0; o < o1; ++o) out[(size_t)out_branch[(size_t)o]] = 0;
      islands[(size_t)c] = parts > 1 ? 1 : 0;
    }
  }
  std::vector<int32_t> case_of(S), bus_of(n), unknown(nb);
  for (int64_t c = 0; c < cases; ++c)
    for (int64_t j = scenario_ptr[c]; j < scenario_ptr[c + 1]; ++j) case_of[j] = (int32_t)c;
  for (int64_t i = 0; i < nb; ++i) {
    unknown[i] = (int32_t)net->unknown[i];
    if (net->unknown[i] >= 0) bus_of[net->unknown[i]] = (int32_t)i;
  }
  cuda_check(cudaSetDevice(net->gpu->device), "cudaSetDevice");
  cudaStream_t s = net->gpu->stream;
  auto &w = net->sol;
  w.case_of.upload(case_of, s), w.bus_of.upload(bus_of, s), w.unknown.upload(unknown, s);
  w.out_ptr.upload(out_ptr, s), w.out_branch.upload(out_branch.empty() ? std::vector<int32_t>{0} : out_branch, s);
  w.col_ptr.upload(col_ptr, s);
  if (S == 0) {
    if (singular) std::copy(islands.begin(), islands.end(), singular);
    return;
  }
  w.inj.reserve((size_t)(nb * S)), w.rhs.reserve((size_t)(n * S)), w.theta.reserve((size_t)(n * S));
  w.flags.reserve((size_t)S);
  if (theta) w.theta_bus.reserve((size_t)(nb * S));
  if (flows) w.flows.reserve((size_t)(nl * S));
  cuda_check(cudaMemcpyAsync(w.inj.get(), injections, sizeof(double) * nb * S, cudaMemcpyHostToDevice, s),
             "upload injections");
  unknowns_of_buses_kernel<<<(unsigned)((n * S + 255) / 256), 256, 0, s>>>(w.inj.get(), nb, w.bus_of.get(), n, S,
                                                                          w.rhs.get());
  cuda_check(cudaGetLastError(), "unknowns_of_buses_kernel launch");
  int32_t st = yb_solve_many_device(f, w.rhs.get(), n, w.theta.get(), n, S, YB_FP64, s);
  if (st != YB_OK) throw host::Error(st, "the scenario solve failed");
  w.singular.upload(islands, s);
  if (K > 0) {
    w.pu.upload(pu, s), w.mu.upload(mu, s), w.p0.upload(p0, s), w.p1.upload(p1, s);
    w.s0.upload(s0, s), w.s1.upload(s1, s), w.invb.upload(invb, s);
    w.y.reserve((size_t)(n * K));
    w.lu.reserve((size_t)(cases * kMaxOutageRank * kMaxOutageRank));
    w.piv.reserve((size_t)(cases * kMaxOutageRank));
    solve_pairs_device(f, K, w.pu.get(), w.mu.get(), nullptr, nullptr, nullptr, nullptr, w.y.get(), n, s);
    outage_lu_kernel<<<(unsigned)((cases + 127) / 128), 128, 0, s>>>(w.y.get(), n, w.col_ptr.get(), w.p0.get(),
                                                                     w.s0.get(), w.p1.get(), w.s1.get(), w.invb.get(),
                                                                     cases, w.lu.get(), w.piv.get(), w.singular.get());
    cuda_check(cudaGetLastError(), "outage_lu_kernel launch");
    outage_update_kernel<<<(unsigned)S, 256, 0, s>>>(w.theta.get(), n, w.case_of.get(), w.col_ptr.get(), w.p0.get(),
                                                     w.s0.get(), w.p1.get(), w.s1.get(), w.lu.get(), w.piv.get(),
                                                     w.singular.get(), w.y.get(), n);
    cuda_check(cudaGetLastError(), "outage_update_kernel launch");
  }
  place_flows_kernel<<<(unsigned)S, 256, 0, s>>>(w.theta.get(), n, (int32_t)nb, w.unknown.get(), (int32_t)nl,
                                                 net->br_u_f.get(), net->br_u_t.get(), net->br_b.get(), w.case_of.get(),
                                                 w.out_ptr.get(), w.out_branch.get(), theta ? w.theta_bus.get() : nullptr,
                                                 flows ? w.flows.get() : nullptr, w.flags.get());
  cuda_check(cudaGetLastError(), "place_flows_kernel launch");
  if (theta)
    cuda_check(cudaMemcpyAsync(theta, w.theta_bus.get(), sizeof(double) * nb * S, cudaMemcpyDeviceToHost, s), "download");
  if (flows)
    cuda_check(cudaMemcpyAsync(flows, w.flows.get(), sizeof(double) * nl * S, cudaMemcpyDeviceToHost, s), "download");
  if (flags) cuda_check(cudaMemcpyAsync(flags, w.flags.get(), sizeof(int32_t) * S, cudaMemcpyDeviceToHost, s), "download");
  if (singular)
    cuda_check(cudaMemcpyAsync(singular, w.singular.get(), sizeof(int32_t) * cases, cudaMemcpyDeviceToHost, s),
               "download");
  cuda_check(cudaStreamSynchronize(s), "DC solutions");
}

}  // namespace

extern "C" int32_t yb_dc_network_new(yb_gpu *gpu, int64_t n_bus, int64_t n_branch, const int64_t *from,
                                     const int64_t *to, const double *x, int64_t slack, yb_dc_network **out) {
  return guard([&] {
    require(gpu && out, "null argument");
    require(n_bus >= 2 && n_branch >= 1, "a network needs two buses and a branch");
    require(from && to && x, "null branch arrays");
    require(slack >= 0 && slack < n_bus, "the slack bus is out of range");
    auto net = std::make_unique<yb_dc_network>();
    net->gpu = gpu;
    net->n_bus = n_bus, net->n_branch = n_branch, net->slack = slack, net->n = n_bus - 1;
    net->from.assign(from, from + n_branch);
    net->to.assign(to, to + n_branch);
    net->b.resize(n_branch);
    for (int64_t k = 0; k < n_branch; ++k) {
      require(from[k] >= 0 && from[k] < n_bus && to[k] >= 0 && to[k] < n_bus, "a branch end is out of range");
      require(x[k] != 0.0 && std::isfinite(x[k]), "a branch reactance is zero or not finite");
      net->b[k] = 1.0 / x[k];
    }
    net->unknown.assign(n_bus, -1);
    for (int64_t i = 0, u = 0; i < n_bus; ++i)
      if (i != slack) net->unknown[i] = u++;
    // Bbus stamps per branch (f,f,b), (f,t,-b), (t,f,-b), (t,t,b), duplicates summed in order;
    // B' is Bbus without the slack's row and column
    std::vector<host::Triplet<double>> t;
    t.reserve(4 * n_branch);
    for (int64_t k = 0; k < n_branch; ++k) {
      const int64_t f = from[k], g = to[k];
      const double bk = net->b[k];
      t.push_back({f, f, bk});
      t.push_back({f, g, -bk});
      t.push_back({g, f, -bk});
      t.push_back({g, g, bk});
    }
    const auto bbus = host::from_triplets<double>(n_bus, n_bus, t, true);
    std::vector<idx_t> keep;
    for (int64_t i = 0; i < n_bus; ++i)
      if (i != slack) keep.push_back(i);
    const auto bp = host::select(bbus, keep, keep);
    const auto graph = host::adjacency_of(bp);
    auto sym = host::analyze_cholesky(graph, host::approximate_minimum_degree(graph));
    const auto chol = host::factor_cholesky(bp, sym);
    const int64_t n = net->n;
    std::vector<int64_t> perm(chol.perm.begin(), chol.perm.end());
    int32_t st = yb_factor_from_cholesky(gpu, n, chol.l.ptr.data(), chol.l.idx.data(), chol.l.val.data(), perm.data(),
                                         &net->factor);
    if (st != YB_OK) throw host::Error(st, "uploading the factor failed");
    st = yb_factor_attach_matrix(net->factor, bp.ptr.data(), bp.idx.data(), bp.val.data());
    if (st != YB_OK) throw host::Error(st, "attaching B' failed");
    // Bf over the unknowns: per branch (f, b), (t, -b), the slack's column dropped
    std::vector<int64_t> ptr(1, 0), idx;
    std::vector<double> val;
    for (int64_t k = 0; k < n_branch; ++k) {
      if (net->unknown[from[k]] >= 0) idx.push_back(net->unknown[from[k]]), val.push_back(net->b[k]);
      if (net->unknown[to[k]] >= 0) idx.push_back(net->unknown[to[k]]), val.push_back(-net->b[k]);
      ptr.push_back((int64_t)idx.size());
    }
    st = yb_operator_new(net->factor, n_branch, ptr.data(), idx.data(), val.data(), &net->flows);
    if (st != YB_OK) throw host::Error(st, "uploading Bf failed");
    net->bridge = find_bridges(n_bus, net->from, net->to);
    // the screening's per-branch and per-bus device data
    const yb_factor *f = net->factor;
    std::vector<int32_t> sf(n_branch), stt(n_branch), uf(n_branch), ut(n_branch), bus_slot(n_bus);
    for (int64_t k = 0; k < n_branch; ++k) {
      uf[k] = (int32_t)net->unknown[from[k]];
      ut[k] = (int32_t)net->unknown[to[k]];
      sf[k] = uf[k] < 0 ? (int32_t)n : f->plan.out_slot[uf[k]];
      stt[k] = ut[k] < 0 ? (int32_t)n : f->plan.out_slot[ut[k]];
    }
    for (int64_t i = 0; i < n_bus; ++i)
      bus_slot[i] = net->unknown[i] < 0 ? (int32_t)(n + 1) : f->plan.in_slot[net->unknown[i]];
    cudaStream_t s = gpu->stream;
    cuda_check(cudaSetDevice(gpu->device), "cudaSetDevice");
    net->br_slot_f.upload(sf, s), net->br_slot_t.upload(stt, s);
    net->br_u_f.upload(uf, s), net->br_u_t.upload(ut, s);
    net->bus_slot.upload(bus_slot, s);
    net->br_b.upload(net->b, s);
    cuda_check(cudaStreamSynchronize(s), "network upload");
    *out = net.release();
    return YB_OK;
  });
}

extern "C" void yb_dc_network_free(yb_dc_network *net) {
  if (!net) return;
  cudaSetDevice(net->gpu->device);
  delete net;
}

extern "C" yb_factor *yb_dc_network_factor(yb_dc_network *net) { return net ? net->factor : nullptr; }

extern "C" int32_t yb_dc_bridges(const yb_dc_network *net, uint8_t *bridge) {
  return guard([&] {
    require(net && bridge, "null argument");
    std::copy(net->bridge.begin(), net->bridge.end(), bridge);
    return YB_OK;
  });
}

extern "C" int32_t yb_dc_ptdf_columns(yb_dc_network *net, int64_t count, const int64_t *buses, double *out) {
  return guard([&] {
    check(net);
    require(count >= 0 && (count == 0 || (buses && out)), "null argument");
    std::vector<int64_t> plus(count), minus(count, -1);
    for (int64_t k = 0; k < count; ++k) {
      require(buses[k] >= 0 && buses[k] < net->n_bus, "a bus is out of range");
      plus[k] = net->unknown[buses[k]];  // the slack injects nothing: its column is zero, or -H w
    }
    // with a distributed slack every column loses the shift H w (the operator's offset, -H w)
    const bool shifted = !net->negated_shift.empty();
    if (shifted) {
      const int32_t st = yb_operator_set_offset(net->flows, net->negated_shift.data());
      if (st != YB_OK) throw host::Error(st, "setting the shift failed");
    }
    std::vector<double> flows;
    try {
      flows = pair_flows(net, plus, minus);
    } catch (...) {
      if (shifted) yb_operator_set_offset(net->flows, std::vector<double>(net->n_branch, 0.0).data());
      throw;
    }
    if (shifted) {
      const int32_t st = yb_operator_set_offset(net->flows, std::vector<double>(net->n_branch, 0.0).data());
      if (st != YB_OK) throw host::Error(st, "clearing the shift failed");
    }
    std::copy(flows.begin(), flows.end(), out);
    return YB_OK;
  });
}

extern "C" int32_t yb_dc_set_slack_weights(yb_dc_network *net, const double *weights) {
  return guard([&] {
    check(net);
    if (!weights) {
      net->negated_shift.clear();
      return YB_OK;
    }
    // normalized to sum to 1, as DcSensitivity::new does (dc/sensitivity.rs:101-126)
    double total = 0.0;
    for (int64_t i = 0; i < net->n_bus; ++i) total += weights[i];
    require(total != 0.0 && std::isfinite(total), "the weights don't have a finite, nonzero sum");
    std::vector<double> rhs((size_t)net->n, 0.0);
    for (int64_t i = 0; i < net->n_bus; ++i)
      if (net->unknown[i] >= 0) rhs[(size_t)net->unknown[i]] = weights[i] / total;  // the slack's share drops
    // H w: the flows of the weighted injections (dc/sensitivity.rs:258-263), from one solve
    std::vector<double> theta((size_t)net->n);
    const int32_t st = yb_solve_many(net->factor, rhs.data(), 1, theta.data());
    if (st != YB_OK) throw host::Error(st, "the shift's solve failed");
    std::vector<double> shift((size_t)net->n_branch);
    for (int64_t k = 0; k < net->n_branch; ++k) {
      const int64_t uf = net->unknown[net->from[k]], ut = net->unknown[net->to[k]];
      const double tf = uf < 0 ? 0.0 : theta[(size_t)uf], tt = ut < 0 ? 0.0 : theta[(size_t)ut];
      shift[(size_t)k] = -(net->b[k] * (tf - tt));
    }
    net->negated_shift = std::move(shift);
    return YB_OK;
  });
}

extern "C" int32_t yb_dc_solve_many(yb_dc_network *net, int64_t count, const double *injections, double *theta,
                                    double *flows, int32_t *flags) {
  return guard([&] {
    check(net);
    require(count >= 0, "negative count");
    if (count == 0) return YB_OK;
    const int64_t sp[2] = {0, count};
    dc_solutions(net, 1, nullptr, nullptr, sp, injections, theta, flows, flags, nullptr);
    return YB_OK;
  });
}

extern "C" int32_t yb_dc_outage_solutions(yb_dc_network *net, int64_t cases, const int64_t *branch_ptr,
                                          const int64_t *branches, const int64_t *scenario_ptr,
                                          const double *injections, double *theta, double *flows, int32_t *flags,
                                          int32_t *singular) {
  return guard([&] {
    check(net);
    require(cases >= 0, "negative case count");
    if (cases == 0) return YB_OK;
    require(branch_ptr != nullptr, "null branch pointers");
    dc_solutions(net, cases, branch_ptr, branches, scenario_ptr, injections, theta, flows, flags, singular);
    return YB_OK;
  });
}

extern "C" int32_t yb_dc_ptdf_transfers(yb_dc_network *net, int64_t count, const int64_t *from_bus,
                                        const int64_t *to_bus, double *out) {
  return guard([&] {
    check(net);
    require(count >= 0 && (count == 0 || (from_bus && to_bus && out)), "null argument");
    std::vector<int64_t> plus(count), minus(count);
    for (int64_t k = 0; k < count; ++k) {
      require(from_bus[k] >= 0 && from_bus[k] < net->n_bus && to_bus[k] >= 0 && to_bus[k] < net->n_bus,
              "a bus is out of range");
      plus[k] = net->unknown[from_bus[k]];
      minus[k] = net->unknown[to_bus[k]];
      if (plus[k] >= 0 && plus[k] == minus[k]) plus[k] = minus[k] = -1;  // a transfer to itself moves nothing
    }
    const auto flows = pair_flows(net, plus, minus);
    std::copy(flows.begin(), flows.end(), out);
    return YB_OK;
  });
}

extern "C" int32_t yb_dc_lodf_columns(yb_dc_network *net, int64_t count, const int64_t *branches, double *out) {
  return guard([&] {
    check(net);
    require(count >= 0 && (count == 0 || (branches && out)), "null argument");
    std::vector<int64_t> plus, minus, which;
    for (int64_t k = 0; k < count; ++k) {
      const int64_t br = branches[k];
      require(br >= 0 && br < net->n_branch, "a branch is out of range");
      if (net->bridge[br]) continue;
      int64_t p = net->unknown[net->from[br]], m = net->unknown[net->to[br]];
      if (p >= 0 && p == m) p = m = -1;
      plus.push_back(p), minus.push_back(m), which.push_back(k);
    }
    const auto flows = pair_flows(net, plus, minus);
    const int64_t nl = net->n_branch;
    for (int64_t k = 0; k < count; ++k) std::fill(out + k * nl, out + (k + 1) * nl, std::nan(""));
    for (size_t j = 0; j < which.size(); ++j) {
      const int64_t k = which[j], row = branches[k];
      double *col = out + k * nl;
      std::copy(flows.begin() + (int64_t)j * nl, flows.begin() + ((int64_t)j + 1) * nl, col);
      // LODF = H / (1 - H_kk), -1 on the outaged branch (dc/sensitivity.rs:349-362)
      const double remaining = 1.0 - col[row];
      for (int64_t l = 0; l < nl; ++l) col[l] /= remaining;
      col[row] = -1.0;
    }
    return YB_OK;
  });
}

extern "C" int32_t yb_dc_outage_loadings_batch(yb_dc_network *net, int64_t cases, const int64_t *outaged,
                                               const int64_t *scenario_ptr, const double *injections,
                                               const double *weights, int32_t precision, int64_t *max_branch,
                                               double *max_loading, int32_t *flags, int32_t *singular) {
  return guard([&] {
    check(net);
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(cases >= 0 && (cases == 0 || (outaged && scenario_ptr)), "null argument");
    if (cases == 0) return YB_OK;
    require(scenario_ptr[0] == 0, "scenario pointers must start at 0");
    for (int64_t c = 0; c < cases; ++c) require(scenario_ptr[c + 1] >= scenario_ptr[c], "scenario pointers must not decrease");
    const int64_t S = scenario_ptr[cases];
    require(S == 0 || (injections && max_branch && max_loading && flags), "null output");
    yb_factor *f = net->factor;
    const int64_t n = net->n, nl = net->n_branch;
    // per case: the outaged branch's pair over the unknowns, its slots, 1/b
    std::vector<int32_t> case_of(S), pu(cases), mu(cases), ps(cases), ms(cases), br(cases);
    std::vector<double> invb(cases);
    for (int64_t c = 0; c < cases; ++c) {
      const int64_t k = outaged[c];
      require(k >= 0 && k < nl, "an outaged branch is out of range");
      int64_t p = net->unknown[net->from[k]], m = net->unknown[net->to[k]];
      if (p >= 0 && p == m) p = m = -1;
      pu[c] = (int32_t)p, mu[c] = (int32_t)m, br[c] = (int32_t)k;
      ps[c] = p < 0 ? (int32_t)n : f->plan.out_slot[p];
      ms[c] = m < 0 ? (int32_t)n : f->plan.out_slot[m];
      invb[c] = (p < 0 && m < 0) ? 1.0 : 1.0 / net->b[k];
      for (int64_t j = scenario_ptr[c]; j < scenario_ptr[c + 1]; ++j) case_of[j] = (int32_t)c;
    }
    std::vector<double> w(nl, 1.0);
    if (weights) w.assign(weights, weights + nl);
    cuda_check(cudaSetDevice(net->gpu->device), "cudaSetDevice");
    cudaStream_t s = net->gpu->stream;
    net->d_case_of.upload(case_of, s), net->d_plus_u.upload(pu, s), net->d_minus_u.upload(mu, s);
    net->d_plus_slot.upload(ps, s), net->d_minus_slot.upload(ms, s), net->d_branch.upload(br, s);
    net->d_invb.upload(invb, s), net->d_weight.upload(w, s);
    net->d_inj.reserve((size_t)(net->n_bus * S));
    net->d_y.reserve((size_t)(n * cases));
    net->d_cy.reserve((size_t)cases);
    net->d_row.reserve((size_t)S), net->d_value.reserve((size_t)S), net->d_bad.reserve((size_t)S);
    net->d_sing.reserve((size_t)cases);
    cuda_check(cudaMemcpyAsync(net->d_inj.get(), injections, sizeof(double) * net->n_bus * S, cudaMemcpyHostToDevice, s),
               "upload injections");
    OutageIO io{};
    io.inj = net->d_inj.get(), io.ldi = net->n_bus, io.n_bus = (int32_t)net->n_bus, io.bus_slot = net->bus_slot.get();
    io.case_of = net->d_case_of.get(), io.c_plus = net->d_plus_slot.get(), io.c_minus = net->d_minus_slot.get();
    io.c_invb = net->d_invb.get(), io.c_cy = net->d_cy.get(), io.c_branch = net->d_branch.get();
    io.Y = net->d_y.get(), io.ldy = n, io.n_branch = (int32_t)nl;
    io.br_slot_f = net->br_slot_f.get(), io.br_slot_t = net->br_slot_t.get();
    io.br_u_f = net->br_u_f.get(), io.br_u_t = net->br_u_t.get(), io.br_b = net->br_b.get(), io.weight = net->d_weight.get();
    io.out_row = net->d_row.get(), io.out_value = net->d_value.get(), io.out_bad = net->d_bad.get();
    io.case_singular = net->d_sing.get();
    // y = B'^-1 c of every case, then c'y; then the scenarios
    auto run = [&]() {
      solve_pairs_device(f, cases, net->d_plus_u.get(), net->d_minus_u.get(), nullptr, nullptr, nullptr, nullptr,
                         net->d_y.get(), n, s);
      case_cy_kernel<<<(unsigned)((cases + 255) / 256), 256, 0, s>>>(net->d_y.get(), n, net->d_plus_u.get(),
                                                                     net->d_minus_u.get(), cases, net->d_cy.get());
      cuda_check(cudaGetLastError(), "case_cy_kernel launch");
      if (S == 0) return;
      if (precision == YB_FP64) {
        launch_domain_fp64(f, S, io, s);
      } else {
        net->d_theta.reserve((size_t)(n * S));
        net->d_ratio.reserve((size_t)S), net->d_steps.reserve((size_t)S);
        // scenario right-hand sides over the unknowns, then FP32 substitution with FP64 refinement
        const int32_t st = yb_solve_many_refined_device(f, net->d_inj.get() + (net->slack == 0 ? 1 : 0), net->n_bus,
                                                        net->d_theta.get(), n, S, 3, 1e-10, net->d_ratio.get(),
                                                        net->d_steps.get(), s);
        if (st != YB_OK) throw host::Error(st, "the refined scenario solve failed");
        outage_epilogue_kernel<<<(unsigned)S, 256, 0, s>>>(
            net->d_theta.get(), n, net->d_case_of.get(), net->d_plus_u.get(), net->d_minus_u.get(), net->d_invb.get(),
            net->d_cy.get(), net->d_branch.get(), net->d_y.get(), n, (int32_t)nl, net->br_u_f.get(), net->br_u_t.get(),
            net->br_b.get(), net->d_weight.get(), net->d_row.get(), net->d_value.get(), net->d_bad.get(),
            net->d_sing.get());
        cuda_check(cudaGetLastError(), "outage_epilogue_kernel launch");
      }
    };
    if (precision == YB_FP32) require(net->slack == 0, "the FP32 screening takes the slack at bus 0");
    if (precision == YB_FP64 && net->graph && net->graph_cases == cases && net->graph_columns == S) {
      // the same sizes as the captured graph: its buffers hold this batch's inputs
      cuda_check(cudaGraphLaunch(net->graph, s), "cudaGraphLaunch");
    } else {
      run();  // makes every layout and buffer the launches need, outside any capture
      if (precision == YB_FP64) {
        if (net->graph) cudaGraphExecDestroy(net->graph), net->graph = nullptr;
        cudaGraph_t g = nullptr;
        cuda_check(cudaStreamSynchronize(s), "before capture");
        cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
        try {
          run();
        } catch (...) {
          cudaStreamEndCapture(s, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        cuda_check(cudaStreamEndCapture(s, &g), "cudaStreamEndCapture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        cuda_check(e, "cudaGraphInstantiate");
        net->graph = exec, net->graph_cases = cases, net->graph_columns = S;
      }
    }
    std::vector<int32_t> bad(S), sing(cases);
    cuda_check(cudaMemcpyAsync(max_branch, net->d_row.get(), sizeof(int64_t) * S, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaMemcpyAsync(max_loading, net->d_value.get(), sizeof(double) * S, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaMemcpyAsync(flags, net->d_bad.get(), sizeof(int32_t) * S, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaMemcpyAsync(sing.data(), net->d_sing.get(), sizeof(int32_t) * cases, cudaMemcpyDeviceToHost, s),
               "download");
    cuda_check(cudaStreamSynchronize(s), "outage screening");
    if (singular) std::copy(sing.begin(), sing.end(), singular);
    return YB_OK;
  });
}

// ---- the adjoint of a flow loss (no ybus counterpart) ---------------------------------------------

// A forward/backward pair over a DC network, the analogue of an autograd function: forward solves
// theta = B'^-1 p for `count` injection scenarios, computes the flows f = diag(b) A theta and the
// loss sum softplus(|f| - margin * limit)^2, and keeps theta and dL/df on the device; backward
// solves lambda = B'^-T (Bf' dL/df) with the same factor (B' is symmetric) and gives dL/dp =
// lambda (zero at the slack) and dL/db_k = sum over scenarios of dL/df_k (theta_f - theta_t) -
// (lambda_f - lambda_t)(theta_f - theta_t): the sensitivity of the flows' own b plus the chain of
// the outer-product accumulation -lambda theta' onto B''s pattern through dB'/db_k = a_k a_k'.
struct yb_dc_adjoint {
  yb_dc_network *net = nullptr;
  int64_t count = 0;
  bool forward_done = false;
  DeviceArray<double> p, limits, theta, g, lambda, flows, loss_part, gb_part, grad_b;
  DeviceArray<int32_t> inc_ptr, inc_branch;
  DeviceArray<double> inc_value;
  DeviceArray<int32_t> unknown;  // per bus: its unknown, -1 for the slack
  DeviceArray<double> grad_p;    // dL/dp by bus, count x n_bus
};

namespace {

constexpr int kLossThreads = 256;
constexpr int kGradChunk = 32;  // scenarios per partial sum of dL/db

// softplus(u) = log(1 + e^u), written to stay finite for large |u|
__device__ __forceinline__ double softplus(double u) { return fmax(u, 0.0) + log1p(exp(-fabs(u))); }
__device__ __forceinline__ double sigmoid(double u) {
  return u >= 0.0 ? 1.0 / (1.0 + exp(-u)) : exp(u) / (1.0 + exp(u));
}

// One thread per (branch, scenario): the flow, its loss term and dL/df; the block's loss terms
// summed in a fixed tree into loss_part[block]
__global__ void flow_loss_kernel(const double *__restrict__ theta, int64_t n, int32_t nl,
                                 const int32_t *__restrict__ uf, const int32_t *__restrict__ ut,
                                 const double *__restrict__ b, const double *__restrict__ limits, double margin,
                                 int64_t total, double *__restrict__ flows, double *__restrict__ g,
                                 double *__restrict__ loss_part) {
  __shared__ double part[kLossThreads];
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double term = 0.0;
  if (idx < total) {
    const int64_t r = idx / nl;
    const int l = (int)(idx % nl);
    const double *th = theta + r * n;
    const double tf = uf[l] < 0 ? 0.0 : th[uf[l]], tt = ut[l] < 0 ? 0.0 : th[ut[l]];
    const double f = __dadd_rn(__dmul_rn(b[l], tf), __dmul_rn(-b[l], tt));
    const double u = fabs(f) - margin * limits[l];
    const double s = softplus(u);
    term = s * s;
    const double sign = f > 0.0 ? 1.0 : (f < 0.0 ? -1.0 : 0.0);
    g[idx] = 2.0 * s * sigmoid(u) * sign;
    if (flows) flows[idx] = f;
  }
  part[threadIdx.x] = term;
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride /= 2) {
    if (threadIdx.x < stride) part[threadIdx.x] += part[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = part[0];
}

// Partial sums of dL/db over a chunk of scenarios: gb_part[chunk][l]
__global__ void grad_b_kernel(const double *__restrict__ theta, const double *__restrict__ lambda, int64_t n,
                              const double *__restrict__ g, int32_t nl, const int32_t *__restrict__ uf,
                              const int32_t *__restrict__ ut, int64_t count, double *__restrict__ gb_part) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nl) return;
  const int64_t r0 = (int64_t)blockIdx.y * kGradChunk, r1 = min(count, r0 + kGradChunk);
  double acc = 0.0;
  for (int64_t r = r0; r < r1; ++r) {
    const double *th = theta + r * n, *la = lambda + r * n;
    const double d = (uf[l] < 0 ? 0.0 : th[uf[l]]) - (ut[l] < 0 ? 0.0 : th[ut[l]]);
    const double e = (uf[l] < 0 ? 0.0 : la[uf[l]]) - (ut[l] < 0 ? 0.0 : la[ut[l]]);
    acc += g[r * nl + l] * d - e * d;
  }
  gb_part[(int64_t)blockIdx.y * nl + l] = acc;
}

// dL/db_l: the chunks' partial sums in chunk order
__global__ void grad_b_reduce_kernel(const double *__restrict__ gb_part, int32_t nl, int64_t chunks,
                                     double *__restrict__ grad_b) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nl) return;
  double s = 0.0;
  for (int64_t c = 0; c < chunks; ++c) s += gb_part[c * nl + l];
  grad_b[l] = s;
}

// dL/dp by bus: lambda's entry of the bus's unknown, 0 at the slack
__global__ void grad_p_kernel(const double *__restrict__ lambda, int64_t n, const int32_t *__restrict__ unknown,
                              int64_t n_bus, int64_t total, double *__restrict__ grad_p) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= total) return;
  const int64_t r = k / n_bus, i = k - r * n_bus;
  const int32_t u = unknown[i];
  grad_p[k] = u < 0 ? 0.0 : lambda[r * n + u];
}

}  // namespace

extern "C" int32_t yb_dc_adjoint_new(yb_dc_network *net, int64_t count, yb_dc_adjoint **out) {
  return guard([&] {
    check(net);
    require(out != nullptr && count >= 1, "bad argument");
    const int64_t n = net->n, nl = net->n_branch;
    require(count * nl < ((int64_t)1 << 40), "too many scenarios", host::kTooLarge);
    auto adj = std::make_unique<yb_dc_adjoint>();
    adj->net = net;
    adj->count = count;
    // Bf' over the unknowns: each unknown's incident branches in branch order, +b at the from end
    std::vector<std::vector<std::pair<int32_t, double>>> inc(n);
    for (int64_t l = 0; l < nl; ++l) {
      if (net->unknown[net->from[l]] >= 0) inc[net->unknown[net->from[l]]].push_back({(int32_t)l, net->b[l]});
      if (net->unknown[net->to[l]] >= 0) inc[net->unknown[net->to[l]]].push_back({(int32_t)l, -net->b[l]});
    }
    std::vector<int32_t> ptr(1, 0), br;
    std::vector<double> val;
    for (auto &v : inc) {
      for (auto [l, x] : v) br.push_back(l), val.push_back(x);
      ptr.push_back((int32_t)br.size());
    }
    cuda_check(cudaSetDevice(net->gpu->device), "cudaSetDevice");
    cudaStream_t s = net->gpu->stream;
    adj->inc_ptr.upload(ptr, s);
    adj->inc_branch.upload(br.empty() ? std::vector<int32_t>{0} : br, s);
    adj->inc_value.upload(val.empty() ? std::vector<double>{0.0} : val, s);
    std::vector<int32_t> unknown(net->unknown.begin(), net->unknown.end());
    adj->unknown.upload(unknown, s);
    adj->p.resize((size_t)(net->n_bus * count));
    adj->limits.resize((size_t)nl);
    adj->theta.resize((size_t)(n * count));
    adj->lambda.resize((size_t)(n * count));
    adj->g.resize((size_t)(nl * count));
    adj->loss_part.resize((size_t)((nl * count + kLossThreads - 1) / kLossThreads));
    adj->gb_part.resize((size_t)(((count + kGradChunk - 1) / kGradChunk) * nl));
    adj->grad_b.resize((size_t)nl);
    cuda_check(cudaStreamSynchronize(s), "adjoint set-up");
    *out = adj.release();
    return YB_OK;
  });
}

extern "C" void yb_dc_adjoint_free(yb_dc_adjoint *adj) {
  if (!adj) return;
  cudaSetDevice(adj->net->gpu->device);
  delete adj;
}

extern "C" int32_t yb_dc_adjoint_forward(yb_dc_adjoint *adj, const double *injections, const double *limits,
                                         double margin, double *loss, double *flows) {
  return guard([&] {
    require(adj && injections && limits && loss, "null argument");
    yb_dc_network *net = adj->net;
    const int64_t n = net->n, nl = net->n_branch, count = adj->count;
    cuda_check(cudaSetDevice(net->gpu->device), "cudaSetDevice");
    cudaStream_t s = net->gpu->stream;
    cuda_check(cudaMemcpyAsync(adj->p.get(), injections, sizeof(double) * net->n_bus * count, cudaMemcpyHostToDevice, s),
               "upload injections");
    cuda_check(cudaMemcpyAsync(adj->limits.get(), limits, sizeof(double) * nl, cudaMemcpyHostToDevice, s), "upload limits");
    BusIO io{adj->p.get(), net->n_bus, (int32_t)net->n_bus, net->bus_slot.get(), adj->theta.get(), n,
             net->factor->out_slot.get()};
    launch_domain_fp64(net->factor, count, io, s);
    if (flows) adj->flows.reserve((size_t)(nl * count));
    const int64_t total = nl * count, blocks = (total + kLossThreads - 1) / kLossThreads;
    flow_loss_kernel<<<(unsigned)blocks, kLossThreads, 0, s>>>(adj->theta.get(), n, (int32_t)nl, net->br_u_f.get(),
                                                               net->br_u_t.get(), net->br_b.get(), adj->limits.get(),
                                                               margin, total, flows ? adj->flows.get() : nullptr,
                                                               adj->g.get(), adj->loss_part.get());
    cuda_check(cudaGetLastError(), "flow_loss_kernel launch");
    std::vector<double> part(blocks);
    cuda_check(cudaMemcpyAsync(part.data(), adj->loss_part.get(), sizeof(double) * blocks, cudaMemcpyDeviceToHost, s),
               "download loss");
    if (flows)
      cuda_check(cudaMemcpyAsync(flows, adj->flows.get(), sizeof(double) * total, cudaMemcpyDeviceToHost, s),
                 "download flows");
    cuda_check(cudaStreamSynchronize(s), "adjoint forward");
    double sum = 0.0;
    for (double v : part) sum += v;
    *loss = sum;
    adj->forward_done = true;
    return YB_OK;
  });
}

extern "C" int32_t yb_dc_adjoint_backward(yb_dc_adjoint *adj, double *grad_injections, double *grad_susceptance) {
  return guard([&] {
    require(adj != nullptr, "null adjoint");
    require(adj->forward_done, "backward needs a forward first");
    yb_dc_network *net = adj->net;
    const int64_t n = net->n, nl = net->n_branch, count = adj->count;
    cuda_check(cudaSetDevice(net->gpu->device), "cudaSetDevice");
    cudaStream_t s = net->gpu->stream;
    AdjointIO io{adj->g.get(), nl, adj->inc_ptr.get(), adj->inc_branch.get(), adj->inc_value.get(),
                 net->factor->in_slot.get(), adj->lambda.get(), n, net->factor->out_slot.get()};
    launch_domain_fp64(net->factor, count, io, s);
    const int64_t chunks = (count + kGradChunk - 1) / kGradChunk;
    const dim3 grid((unsigned)((nl + 255) / 256), (unsigned)chunks);
    grad_b_kernel<<<grid, 256, 0, s>>>(adj->theta.get(), adj->lambda.get(), n, adj->g.get(), (int32_t)nl,
                                       net->br_u_f.get(), net->br_u_t.get(), count, adj->gb_part.get());
    cuda_check(cudaGetLastError(), "grad_b_kernel launch");
    grad_b_reduce_kernel<<<(unsigned)((nl + 255) / 256), 256, 0, s>>>(adj->gb_part.get(), (int32_t)nl, chunks,
                                                                      adj->grad_b.get());
    cuda_check(cudaGetLastError(), "grad_b_reduce_kernel launch");
    if (grad_injections) {
      // dL/dp in bus order on the device, then one copy into the caller's array
      const int64_t total = net->n_bus * count;
      adj->grad_p.reserve((size_t)total);
      grad_p_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(adj->lambda.get(), n, adj->unknown.get(), net->n_bus,
                                                                   total, adj->grad_p.get());
      cuda_check(cudaGetLastError(), "grad_p_kernel launch");
      cuda_check(cudaMemcpyAsync(grad_injections, adj->grad_p.get(), sizeof(double) * total, cudaMemcpyDeviceToHost, s),
                 "download dL/dp");
    }
    if (grad_susceptance)
      cuda_check(cudaMemcpyAsync(grad_susceptance, adj->grad_b.get(), sizeof(double) * nl, cudaMemcpyDeviceToHost, s),
                 "download dL/db");
    cuda_check(cudaStreamSynchronize(s), "adjoint backward");
    return YB_OK;
  });
}
