// C ABI of complex LU factors on the GPU and their multi-network batched solve (no ybus
// counterpart: ybus_cuda is real FP64 only, ybus_cuda/src/sparse.rs:106-118). A complex128 LU
// factor of a Ybus, P A Q = L U made by ybus_sparse's generic Gilbert-Peierls LU
// (ybus_sparse/src/compressed_matrix/lu.rs:268-417), is uploaded in complex128 and complex64; many
// such factors of uneven orders solve their right-hand sides in one launch, in complex128 or in
// complex64 with complex128 refinement against the attached matrices (the stopping rules of
// `refine_normwise`, accuracy.rs:83-122, applied to the whole batch).
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "../../include/ybgpu.h"
#include "batch_solve.cuh"
#include "capi_common.hpp"
#include "device.cuh"
#include "factor_state.cuh"

using namespace yb;
using host::c128;

namespace {

host::Compressed<c128> csc_complex(int64_t n, const int64_t *ptr, const int64_t *idx, const double *val) {
  require(ptr != nullptr, "null pointer array");
  host::Compressed<c128> m;
  m.rows = m.cols = n;
  m.by_rows = false;
  m.ptr.assign(ptr, ptr + n + 1);
  require(m.ptr[0] == 0, "pointers must start at 0");
  for (int64_t i = 0; i < n; ++i) require(m.ptr[i + 1] >= m.ptr[i], "pointers must not decrease");
  const int64_t nnz = m.ptr[n];
  require(nnz == 0 || (idx && val), "null index or value array");
  m.idx.assign(idx, idx + nnz);
  m.val.resize(nnz);
  for (int64_t k = 0; k < nnz; ++k) {
    require(idx[k] >= 0 && idx[k] < n, "an index is out of range");
    m.val[k] = c128(val[2 * k], val[2 * k + 1]);
  }
  return m;
}

template <class R> void upload_complex_sweep(DeviceSweep<cplx<R>> &d, const Sweep<c128> &s, int32_t n, cudaStream_t st) {
  d.levels = s.levels, d.widest = s.widest, d.n = n, d.entries = s.entries();
  d.host_level_ptr = s.level_ptr;
  d.level_ptr.upload(s.level_ptr, st);
  d.row.upload(s.row, st);
  d.ptr.upload(s.ptr, st);
  d.col.upload(s.col.empty() ? std::vector<int32_t>{0} : s.col, st);
  std::vector<cplx<R>> v(std::max<size_t>(s.val.size(), 1)), di(s.dinv.size());
  for (size_t i = 0; i < s.val.size(); ++i) v[i] = from_std<R>(s.val[i]);
  for (size_t i = 0; i < s.dinv.size(); ++i) di[i] = from_std<R>(s.dinv[i]);
  d.val.upload(v, st);
  d.dinv.upload(di, st);
}

constexpr int kBatchWidth = 4;  // right-hand sides per tile

template <class R> DeviceSweep<cplx<R>> &sweep_of(yb_factor *f, bool fwd);
template <> DeviceSweep<cplx<double>> &sweep_of<double>(yb_factor *f, bool fwd) { return fwd ? f->fwdz : f->bwdz; }
template <> DeviceSweep<cplx<float>> &sweep_of<float>(yb_factor *f, bool fwd) { return fwd ? f->fwdc : f->bwdc; }

template <class R>
void launch_batch(const std::vector<yb_factor *> &fs, const std::vector<const cplx<double> *> &b,
                  const std::vector<int64_t> &ldb, const std::vector<cplx<double> *> &x, const std::vector<int64_t> &counts,
                  bool accumulate, cudaStream_t s, DeviceArray<uint8_t> &net_buf, DeviceArray<BatchItem> &item_buf,
                  DeviceArray<cplx<R>> &scratch, int sm_count) {
  using T = cplx<R>;
  const size_t k = fs.size();
  std::vector<BatchNet<T>> nets(k);
  int64_t max_n = 1;
  std::vector<std::pair<int64_t, BatchItem>> order;
  for (size_t i = 0; i < k; ++i) {
    yb_factor *f = fs[i];
    nets[i].n = (int32_t)f->n;
    nets[i].fwd = view(sweep_of<R>(f, true));
    nets[i].bwd = view(sweep_of<R>(f, false));
    nets[i].in_slot = f->in_slot.get();
    nets[i].out_slot = f->out_slot.get();
    nets[i].b = b[i], nets[i].ldb = ldb[i], nets[i].x = x[i], nets[i].ldx = f->n, nets[i].count = counts[i];
    max_n = std::max<int64_t>(max_n, f->n);
    const int64_t tiles = (counts[i] + kBatchWidth - 1) / kBatchWidth;
    for (int64_t t = 0; t < tiles; ++t) order.push_back({f->n, BatchItem{(int32_t)i, (int32_t)t}});
  }
  if (order.empty()) return;
  // largest networks first, so the long items start early
  std::stable_sort(order.begin(), order.end(), [](const auto &a, const auto &c) { return a.first > c.first; });
  std::vector<BatchItem> items(order.size());
  for (size_t i = 0; i < order.size(); ++i) items[i] = order[i].second;
  const int64_t grid = std::min<int64_t>((int64_t)items.size(), 2 * (int64_t)sm_count);
  const int64_t slice = max_n * kBatchWidth;
  net_buf.reserve(sizeof(BatchNet<T>) * k);
  item_buf.reserve(items.size());
  scratch.reserve((size_t)(grid * slice));
  cuda_check(cudaMemcpyAsync(net_buf.get(), nets.data(), sizeof(BatchNet<T>) * k, cudaMemcpyHostToDevice, s), "upload nets");
  cuda_check(cudaMemcpyAsync(item_buf.get(), items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice, s),
             "upload items");
  const auto *d_nets = reinterpret_cast<const BatchNet<T> *>(net_buf.get());
  if (accumulate)
    batch_solve_kernel<T, kBatchWidth, true><<<(unsigned)grid, 512, 0, s>>>(d_nets, item_buf.get(), (int64_t)items.size(),
                                                                           scratch.get(), slice);
  else
    batch_solve_kernel<T, kBatchWidth, false><<<(unsigned)grid, 512, 0, s>>>(d_nets, item_buf.get(), (int64_t)items.size(),
                                                                            scratch.get(), slice);
  cuda_check(cudaGetLastError(), "batch_solve_kernel launch");
}

// The batch's device workspace, kept between calls (one set per GPU of the first factor)
struct BatchWork {
  DeviceArray<uint8_t> nets, rnets;
  DeviceArray<BatchItem> items, columns;
  DeviceArray<cplx<double>> scratch128, residual;
  DeviceArray<cplx<float>> scratch64;
  DeviceArray<double> ratio;
};

}  // namespace

extern "C" int32_t yb_factor_from_lu_complex(yb_gpu *gpu, int64_t n, const int64_t *l_ptr, const int64_t *l_idx,
                                             const double *l_val, const int64_t *u_ptr, const int64_t *u_idx,
                                             const double *u_val, const int64_t *row_perm, const int64_t *col_perm,
                                             yb_factor **out) {
  return guard([&] {
    require(gpu && out, "null argument");
    require(n >= 1, "the order must be positive");
    require(row_perm && col_perm, "null permutation");
    auto lower = host::reorient(csc_complex(n, l_ptr, l_idx, l_val));
    auto upper = host::reorient(csc_complex(n, u_ptr, u_idx, u_val));
    std::vector<int64_t> p(row_perm, row_perm + n), q(col_perm, col_perm + n);
    auto f = std::make_unique<yb_factor>();
    f->gpu = gpu;
    f->n = n;
    f->kind = YB_LU;
    f->is_complex = true;
    cuda_check(cudaSetDevice(gpu->device), "cudaSetDevice");
    f->cplan = build_plan<c128>(n, lower, true, upper, p, q);
    cudaStream_t s = gpu->stream;
    f->in_slot.upload(f->cplan.in_slot, s);
    f->out_slot.upload(f->cplan.out_slot, s);
    upload_complex_sweep(f->fwdz, f->cplan.fwd, (int32_t)n, s);
    upload_complex_sweep(f->bwdz, f->cplan.bwd, (int32_t)n, s);
    upload_complex_sweep(f->fwdc, f->cplan.fwd, (int32_t)n, s);
    upload_complex_sweep(f->bwdc, f->cplan.bwd, (int32_t)n, s);
    f->error.resize(1);
    cuda_check(cudaMemsetAsync(f->error.get(), 0, sizeof(int32_t), s), "cudaMemsetAsync");
    cuda_check(cudaStreamSynchronize(s), "upload");
    f->width = 1024;
    *out = f.release();
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_attach_matrix_complex(yb_factor *f, const int64_t *a_ptr, const int64_t *a_idx,
                                                   const double *a_val) {
  return guard([&] {
    require(f && a_ptr, "null argument");
    require(f->is_complex, "a real factor attaches with yb_factor_attach_matrix");
    const int64_t n = f->n;
    require(a_ptr[0] == 0, "pointers must start at 0");
    for (int64_t i = 0; i < n; ++i) require(a_ptr[i + 1] >= a_ptr[i], "pointers must not decrease");
    const int64_t nnz = a_ptr[n];
    require(nnz < INT32_MAX, "the matrix has too many entries for 32-bit indices", host::kTooLarge);
    require(nnz == 0 || (a_idx && a_val), "null index or value array");
    std::vector<int32_t> p(n + 1), idx(std::max<int64_t>(nnz, 1), 0);
    std::vector<cplx<double>> val(std::max<int64_t>(nnz, 1));
    for (int64_t i = 0; i <= n; ++i) p[i] = (int32_t)a_ptr[i];
    for (int64_t k = 0; k < nnz; ++k) {
      require(a_idx[k] >= 0 && a_idx[k] < n, "a column index is out of range");
      idx[k] = (int32_t)a_idx[k];
      val[k] = cplx<double>(a_val[2 * k], a_val[2 * k + 1]);
    }
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = f->gpu->stream;
    f->za_ptr.upload(p, s), f->za_idx.upload(idx, s), f->za_val.upload(val, s);
    cuda_check(cudaStreamSynchronize(s), "matrix upload");
    f->za_rows = n;
    return YB_OK;
  });
}

extern "C" int32_t yb_solve_batch_complex(int64_t networks, yb_factor *const *factors, const double *const *d_rhs,
                                          double *const *d_out, const int64_t *counts, int32_t precision,
                                          int32_t max_steps, double tolerance, double *const *d_ratio, int32_t *steps,
                                          void *stream) {
  return guard([&] {
    require(networks >= 1 && factors && d_rhs && d_out && counts, "null argument");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(max_steps >= 0 && max_steps <= 64, "max_steps must be 0 to 64");
    yb_gpu *gpu = nullptr;
    std::vector<yb_factor *> fs(factors, factors + networks);
    std::vector<const cplx<double> *> b(networks);
    std::vector<cplx<double> *> x(networks);
    std::vector<int64_t> cnt(counts, counts + networks), ldb(networks);
    bool refine_possible = true;
    for (int64_t i = 0; i < networks; ++i) {
      require(fs[i] && fs[i]->is_complex, "every factor must be a complex LU factor");
      if (!gpu) gpu = fs[i]->gpu;
      require(fs[i]->gpu->device == gpu->device, "every factor must be on the same GPU");
      require(cnt[i] >= 0 && (cnt[i] == 0 || (d_rhs[i] && d_out[i])), "null device array");
      b[i] = reinterpret_cast<const cplx<double> *>(d_rhs[i]);
      x[i] = reinterpret_cast<cplx<double> *>(d_out[i]);
      ldb[i] = fs[i]->n;
      refine_possible = refine_possible && fs[i]->za_rows == fs[i]->n;
    }
    const bool need_residual = precision == YB_FP32 || d_ratio != nullptr;
    require(!need_residual || refine_possible, "refinement and ratios need the matrices: yb_factor_attach_matrix_complex");
    cuda_check(cudaSetDevice(gpu->device), "cudaSetDevice");
    cudaStream_t s = stream ? (cudaStream_t)stream : gpu->stream;
    if (!gpu->zwork) gpu->zwork = std::make_shared<BatchWork>();
    BatchWork &w = *static_cast<BatchWork *>(gpu->zwork.get());
    // the residual's per-network descriptors and the (network, column) list
    std::vector<ResidualNet> rn(networks);
    std::vector<BatchItem> cols;
    int64_t total = 0, max_total = 0;
    for (int64_t i = 0; i < networks; ++i) total += cnt[i] * fs[i]->n;
    if (need_residual) {
      w.residual.reserve((size_t)std::max<int64_t>(total, 1));
      int64_t off = 0, ratio_off = 0;
      int64_t all_cols = 0;
      for (int64_t i = 0; i < networks; ++i) all_cols += cnt[i];
      w.ratio.reserve((size_t)std::max<int64_t>(all_cols, 1));
      for (int64_t i = 0; i < networks; ++i) {
        yb_factor *f = fs[i];
        rn[i] = ResidualNet{(int32_t)f->n, f->za_ptr.get(), f->za_idx.get(), f->za_val.get(), b[i], f->n, x[i], f->n,
                            w.residual.get() + off, f->n, w.ratio.get() + ratio_off};
        for (int64_t c = 0; c < cnt[i]; ++c) cols.push_back(BatchItem{(int32_t)i, (int32_t)c});
        off += cnt[i] * f->n;
        ratio_off += cnt[i];
      }
      max_total = all_cols;
      w.rnets.reserve(sizeof(ResidualNet) * networks);
      w.columns.reserve(std::max<size_t>(cols.size(), 1));
      cuda_check(cudaMemcpyAsync(w.rnets.get(), rn.data(), sizeof(ResidualNet) * networks, cudaMemcpyHostToDevice, s),
                 "upload residual descriptors");
      if (!cols.empty())
        cuda_check(cudaMemcpyAsync(w.columns.get(), cols.data(), sizeof(BatchItem) * cols.size(), cudaMemcpyHostToDevice, s),
                   "upload columns");
    }
    auto residual = [&]() -> std::vector<double> {
      std::vector<double> ratios(max_total);
      if (max_total == 0) return ratios;
      batch_residual_kernel<<<(unsigned)max_total, 256, 0, s>>>(reinterpret_cast<const ResidualNet *>(w.rnets.get()),
                                                                w.columns.get());
      cuda_check(cudaGetLastError(), "batch_residual_kernel launch");
      cuda_check(cudaMemcpyAsync(ratios.data(), w.ratio.get(), sizeof(double) * max_total, cudaMemcpyDeviceToHost, s),
                 "download ratios");
      cuda_check(cudaStreamSynchronize(s), "residual");
      return ratios;
    };
    int32_t taken = 0;
    if (precision == YB_FP64) {
      launch_batch<double>(fs, b, ldb, x, cnt, false, s, w.nets, w.items, w.scratch128, gpu->sm_count);
    } else {
      launch_batch<float>(fs, b, ldb, x, cnt, false, s, w.nets, w.items, w.scratch64, gpu->sm_count);
      // refinement: solve the residual in complex64 and add the correction, while any column is
      // above the tolerance and the worst one at least halves
      std::vector<const cplx<double> *> r(networks);
      for (int64_t i = 0; i < networks; ++i) r[i] = rn[i].r;
      double previous = INFINITY;
      for (; taken < max_steps; ++taken) {
        const auto ratios = residual();
        double worst = 0.0;
        bool nan = false;
        for (double v : ratios) nan = nan || std::isnan(v), worst = std::max(worst, v);
        if (nan || worst <= tolerance || worst > 0.5 * previous) break;
        previous = worst;
        launch_batch<float>(fs, r, ldb, x, cnt, true, s, w.nets, w.items, w.scratch64, gpu->sm_count);
      }
    }
    if (d_ratio) {
      const auto ratios = residual();
      int64_t off = 0;
      for (int64_t i = 0; i < networks; ++i) {
        if (cnt[i] && d_ratio[i])
          cuda_check(cudaMemcpyAsync(d_ratio[i], w.ratio.get() + off, sizeof(double) * cnt[i], cudaMemcpyDeviceToDevice, s),
                     "copy ratios");
        off += cnt[i];
      }
      (void)ratios;
    }
    if (steps)
      for (int64_t i = 0; i < networks; ++i) steps[i] = taken;
    return YB_OK;
  });
}
