// C ABI of the GPU path: the device (`Gpu`), an uploaded factorization (`GpuFactor`) and its
// block solves, mirroring ybus_cuda (ybus_cuda/src/lib.rs:168-219, ybus_cuda/src/factor.rs).
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/ybgpu.h"
#include "capi_common.hpp"
#include "device.cuh"
#include "factor_state.cuh"
#include "domain_solve.cuh"
#include "lane_solve.cuh"
#include "lane_refine.cuh"
#include "smem_solve.cuh"
#include "stream_solve.cuh"
#include "solve.cuh"

using namespace yb;

namespace yb {
void noalloc_prepare(int device);  // noalloc.cu
}

// ---------------------------------------------------------------------------------------------
// Gpu
// ---------------------------------------------------------------------------------------------

extern "C" int32_t yb_gpu_new(int32_t device, yb_gpu **out) {
  return guard([&] {
    require(out != nullptr, "out is null");
    *out = nullptr;
    int count = 0;
    const cudaError_t err = cudaGetDeviceCount(&count);
    if (err == cudaErrorNoDevice || err == cudaErrorInsufficientDriver || count == 0) {
      cudaGetLastError();
      set_last_error("no CUDA device");
      return YB_NO_DEVICE;
    }
    cuda_check(err, "cudaGetDeviceCount");
    require(device >= 0 && device < count, "no such device");
    auto g = std::make_unique<yb_gpu>();
    g->device = device;
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    g->name = prop.name;
    g->sm_count = prop.multiProcessorCount;
    g->major = prop.major;
    g->minor = prop.minor;
    g->l2_bytes = prop.l2CacheSize;
    g->smem_optin = prop.sharedMemPerBlockOptin;
    g->smem_per_sm = prop.sharedMemPerMultiprocessor;
    cuda_check(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    noalloc_prepare(device);  // the allocation-free solve's fixed array, placed now rather than at its first call
    *out = g.release();
    return YB_OK;
  });
}

extern "C" void yb_gpu_free(yb_gpu *gpu) {
  if (!gpu) return;
  cudaSetDevice(gpu->device);
  if (gpu->stream) cudaStreamDestroy(gpu->stream);
  delete gpu;
}

extern "C" int32_t yb_gpu_name(const yb_gpu *gpu, char *buffer, size_t length) {
  return guard([&] {
    require(gpu && buffer && length, "null argument");
    const size_t copy = std::min(length - 1, gpu->name.size());
    std::memcpy(buffer, gpu->name.data(), copy);
    buffer[copy] = '\0';
    return YB_OK;
  });
}

extern "C" int32_t yb_gpu_memory(const yb_gpu *gpu, uint64_t *free_bytes, uint64_t *total_bytes) {
  return guard([&] {
    require(gpu != nullptr, "null gpu");
    cuda_check(cudaSetDevice(gpu->device), "cudaSetDevice");
    size_t f = 0, t = 0;
    cuda_check(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return YB_OK;
  });
}

extern "C" int32_t yb_gpu_properties(const yb_gpu *gpu, int32_t *sm_count, int32_t *major, int32_t *minor,
                                     int64_t *l2_bytes) {
  return guard([&] {
    require(gpu != nullptr, "null gpu");
    if (sm_count) *sm_count = gpu->sm_count;
    if (major) *major = gpu->major;
    if (minor) *minor = gpu->minor;
    if (l2_bytes) *l2_bytes = gpu->l2_bytes;
    return YB_OK;
  });
}

extern "C" void *yb_gpu_stream(const yb_gpu *gpu) { return gpu ? (void *)gpu->stream : nullptr; }

extern "C" int32_t yb_gpu_synchronize(const yb_gpu *gpu, void *stream) {
  return guard([&] {
    require(gpu != nullptr, "null gpu");
    cuda_check(cudaSetDevice(gpu->device), "cudaSetDevice");
    cuda_check(cudaStreamSynchronize(stream ? (cudaStream_t)stream : gpu->stream), "cudaStreamSynchronize");
    return YB_OK;
  });
}

// ---------------------------------------------------------------------------------------------
// GpuFactor
// ---------------------------------------------------------------------------------------------

namespace {

host::Compressed<double> csr_from_arrays(int64_t n, const int64_t *ptr, const int64_t *idx, const double *val,
                                         bool by_rows) {
  require(ptr != nullptr, "null pointer array");
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

// The transpose of a square CSR matrix, in CSR form: its CSC arrays read by rows.
host::Compressed<double> transpose_as_csr(const host::Compressed<double> &m) {
  host::Compressed<double> t = host::reorient(m);
  t.by_rows = true;
  return t;
}

yb_factor *make_factor(yb_gpu *gpu, int64_t n, host::Compressed<double> lower, bool unit_lower,
                       host::Compressed<double> upper, std::vector<int64_t> in_perm, std::vector<int64_t> out_perm,
                       int kind) {
  auto f = std::make_unique<yb_factor>();
  f->gpu = gpu;
  f->n = n;
  f->kind = kind;
  cuda_check(cudaSetDevice(gpu->device), "cudaSetDevice");
  f->plan = build_plan<double>(n, lower, unit_lower, upper, in_perm, out_perm);
  if (n == 1) {
    // ybus_cuda solves a single-row factor on the host (ybus_cuda/src/factor.rs:244-248): the
    // two triangles' diagonals, divided in the CPU's order
    f->single = true;
    f->single_lower = unit_lower ? 1.0 : lower.val[lower.ptr[1] - 1];
    for (int64_t p = upper.ptr[0]; p < upper.ptr[1]; ++p)
      if (upper.idx[p] == 0) f->single_upper = upper.val[p];
  }
  cudaStream_t s = gpu->stream;
  f->in_slot.upload(f->plan.in_slot, s);
  f->out_slot.upload(f->plan.out_slot, s);
  upload_sweep(f->fwd64, f->plan.fwd, f->plan.n, s);
  upload_sweep(f->bwd64, f->plan.bwd, f->plan.n, s);
  upload_sweep(f->fwd32, f->plan.fwd, f->plan.n, s);
  upload_sweep(f->bwd32, f->plan.bwd, f->plan.n, s);
  f->error.resize(1);
  cuda_check(cudaMemsetAsync(f->error.get(), 0, sizeof(int32_t), s), "cudaMemsetAsync");
  cuda_check(cudaStreamSynchronize(s), "upload");
  // Default block width as ybus_cuda chooses it: two n-column blocks of doubles per right-hand
  // side in a quarter of the free memory (ybus_cuda/src/factor.rs:157-160), capped higher here
  // because a block is one launch over all SMs rather than one SpSM call
  size_t free_bytes = 0, total = 0;
  cuda_check(cudaMemGetInfo(&free_bytes, &total), "cudaMemGetInfo");
  const int64_t width = (int64_t)(free_bytes / 4 / (2 * 8 * (size_t)std::max<int64_t>(n, 1)));
  f->width = std::max<int64_t>(1, std::min<int64_t>(width, kMaxDefaultWidth));
  if (n == 1) f->width = std::min<int64_t>(f->width, kSingleRowWidth);
  return f.release();
}

}  // namespace

extern "C" int32_t yb_factor_from_cholesky(yb_gpu *gpu, int64_t n, const int64_t *l_ptr, const int64_t *l_idx,
                                           const double *l_val, const int64_t *perm, yb_factor **out) {
  return guard([&] {
    require(gpu && out, "null argument");
    require(n >= 0, "negative order");
    require(n == 0 || perm, "null permutation");
    auto lower = csr_from_arrays(n, l_ptr, l_idx, l_val, true);
    auto upper = transpose_as_csr(lower);  // Lᵀ in CSR, each row's diagonal first
    std::vector<int64_t> p(perm, perm + n);
    *out = make_factor(gpu, n, std::move(lower), false, std::move(upper), p, p, YB_CHOLESKY);
    return YB_OK;
  });
}

namespace {
// Keeps an LU factor's arrays in the factor, for yb_solve_many_transpose.
void keep_lu_arrays(yb_factor *f, int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                    const int64_t *u_ptr, const int64_t *u_idx, const double *u_val, const int64_t *row_perm,
                    const int64_t *col_perm, bool transposed) {
  if (n == 0) return;
  const int64_t ln = l_ptr[n], un = u_ptr[n];
  f->lu_l_ptr.assign(l_ptr, l_ptr + n + 1), f->lu_l_idx.assign(l_idx, l_idx + ln), f->lu_l_val.assign(l_val, l_val + ln);
  f->lu_u_ptr.assign(u_ptr, u_ptr + n + 1), f->lu_u_idx.assign(u_idx, u_idx + un), f->lu_u_val.assign(u_val, u_val + un);
  f->lu_p.assign(row_perm, row_perm + n), f->lu_q.assign(col_perm, col_perm + n);
  f->has_lu_arrays = true, f->lu_transposed = transposed;
}
}  // namespace

extern "C" int32_t yb_factor_from_lu(yb_gpu *gpu, int64_t n, const int64_t *l_ptr, const int64_t *l_idx,
                                     const double *l_val, const int64_t *u_ptr, const int64_t *u_idx,
                                     const double *u_val, const int64_t *row_perm, const int64_t *col_perm,
                                     yb_factor **out) {
  return guard([&] {
    require(gpu && out, "null argument");
    require(n >= 0, "negative order");
    require(n == 0 || (row_perm && col_perm), "null permutation");
    auto l_csc = csr_from_arrays(n, l_ptr, l_idx, l_val, false);
    auto u_csc = csr_from_arrays(n, u_ptr, u_idx, u_val, false);
    auto lower = host::reorient(l_csc);
    auto upper = host::reorient(u_csc);
    std::vector<int64_t> p(row_perm, row_perm + n), q(col_perm, col_perm + n);
    yb_factor *f = make_factor(gpu, n, std::move(lower), true, std::move(upper), p, q, YB_LU);
    keep_lu_arrays(f, n, l_ptr, l_idx, l_val, u_ptr, u_idx, u_val, row_perm, col_perm, false);
    *out = f;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_from_lu_transposed(yb_gpu *gpu, int64_t n, const int64_t *l_ptr, const int64_t *l_idx,
                                                const double *l_val, const int64_t *u_ptr, const int64_t *u_idx,
                                                const double *u_val, const int64_t *row_perm, const int64_t *col_perm,
                                                yb_factor **out) {
  return guard([&] {
    require(gpu && out, "null argument");
    require(n >= 0, "negative order");
    require(n == 0 || (row_perm && col_perm), "null permutation");
    // A' = Q U' L' P: forward with U' (U's columns read as rows: CSC of U is CSR of U'), backward
    // with L' (unit diagonal stored first in L's columns, so first in L''s rows); b's slot i takes
    // row Q[i], x's row P[i] comes from slot i (Lu::solve_transpose, lu.rs:506-533)
    auto lower = csr_from_arrays(n, u_ptr, u_idx, u_val, true);
    auto upper = csr_from_arrays(n, l_ptr, l_idx, l_val, true);
    std::vector<int64_t> p(row_perm, row_perm + n), q(col_perm, col_perm + n);
    yb_factor *f = make_factor(gpu, n, std::move(lower), false, std::move(upper), q, p, YB_LU);
    keep_lu_arrays(f, n, l_ptr, l_idx, l_val, u_ptr, u_idx, u_val, row_perm, col_perm, true);
    *out = f;
    return YB_OK;
  });
}

extern "C" void yb_factor_free(yb_factor *f) {
  if (!f) return;
  cudaSetDevice(f->gpu->device);
  cudaStreamSynchronize(f->gpu->stream);
  delete f;
}

extern "C" int64_t yb_factor_dim(const yb_factor *f) { return f ? f->n : -1; }
extern "C" int64_t yb_factor_block_width(const yb_factor *f) { return f ? f->width : -1; }

extern "C" int32_t yb_factor_set_block_width(yb_factor *f, int64_t width) {
  return guard([&] {
    require(f != nullptr, "null factor");
    const int64_t most = f->n == 1 ? kSingleRowWidth : INT64_MAX;
    f->width = std::max<int64_t>(1, std::min<int64_t>(width, most));
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_timings(const yb_factor *f, double *upload_s, double *solve_s, double *download_s,
                                     int64_t *blocks) {
  return guard([&] {
    require(f != nullptr, "null factor");
    if (upload_s) *upload_s = f->timings.upload;
    if (solve_s) *solve_s = f->timings.solve;
    if (download_s) *download_s = f->timings.download;
    if (blocks) *blocks = f->timings.blocks;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_time_lane(yb_factor *f, int32_t on) {
  return guard([&] {
    require(f != nullptr, "null factor");
    f->lane_timing.on = on != 0;
    f->lane_timing.used = 0;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_lane_times(yb_factor *f, double *gather_ms, double *solve_ms, double *scatter_ms,
                                        int64_t *launches) {
  return guard([&] {
    require(f != nullptr, "null factor");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    LaneTiming &t = f->lane_timing;
    double ms[3] = {0, 0, 0};
    if (t.used > 0) cuda_check(cudaEventSynchronize(t.ev[t.used - 1][3]), "cudaEventSynchronize");
    for (size_t k = 0; k < t.used; ++k)
      for (int p = 0; p < 3; ++p) {
        float e = 0;
        cuda_check(cudaEventElapsedTime(&e, t.ev[k][p], t.ev[k][p + 1]), "cudaEventElapsedTime");
        ms[p] += e;
      }
    if (gather_ms) *gather_ms = ms[0];
    if (solve_ms) *solve_ms = ms[1];
    if (scatter_ms) *scatter_ms = ms[2];
    if (launches) *launches = (int64_t)t.used;
    t.used = 0;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_reset_timings(yb_factor *f) {
  return guard([&] {
    require(f != nullptr, "null factor");
    f->timings = Timings{};
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_plan_info(const yb_factor *f, int32_t *fwd_levels, int32_t *bwd_levels,
                                       int64_t *fwd_entries, int64_t *bwd_entries, int32_t *fwd_widest,
                                       int32_t *bwd_widest) {
  return guard([&] {
    require(f != nullptr, "null factor");
    if (fwd_levels) *fwd_levels = f->plan.fwd.levels;
    if (bwd_levels) *bwd_levels = f->plan.bwd.levels;
    if (fwd_entries) *fwd_entries = f->plan.fwd.entries();
    if (bwd_entries) *bwd_entries = f->plan.bwd.entries();
    if (fwd_widest) *fwd_widest = f->plan.fwd.widest;
    if (bwd_widest) *bwd_widest = f->plan.bwd.widest;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_tile(yb_factor *f, int32_t precision, int32_t tile_width, int32_t threads,
                                      int32_t blocks_per_sm) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(tile_width == 1 || tile_width == 2 || tile_width == 4 || tile_width == 8 || tile_width == 16 ||
                tile_width == 32,
            "the tile width must be a power of two up to 32");
    require(threads >= 32 && threads <= 512 && threads % 32 == 0, "threads must be a multiple of 32 up to 512");
    require(blocks_per_sm >= 1 && blocks_per_sm <= 8, "blocks per SM must be 1 to 8");
    TileConfig &t = precision == YB_FP64 ? f->tile64 : f->tile32;
    t.width = tile_width;
    t.threads = threads;
    t.blocks_per_sm = blocks_per_sm;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_tile_kind(yb_factor *f, int32_t precision, int32_t kind) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(kind >= kTileAuto && kind <= kTileLane, "unknown tile kind");
    (precision == YB_FP64 ? f->tile64 : f->tile32).kind = kind;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_stream(yb_factor *f, int32_t precision, int32_t warps, int32_t ring,
                                        int32_t page_bytes, int32_t narrow_rows) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(warps >= 1 && warps <= 16, "warps must be 1 to 16");
    require(ring >= 2 && ring <= 16, "the ring holds 2 to 16 pages");
    require(page_bytes >= 512 && page_bytes <= 16384 && page_bytes % 16 == 0,
            "page bytes must be a multiple of 16 from 512 to 16384");
    require(narrow_rows >= 0, "narrow rows must not be negative");
    TileConfig &t = precision == YB_FP64 ? f->tile64 : f->tile32;
    t.stream_warps = warps, t.ring = ring, t.page_bytes = page_bytes, t.narrow_rows = narrow_rows;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_tail_level(yb_factor *f, int32_t precision, int32_t tail_level) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(tail_level >= -1, "the tail level is -1 (chosen), 0 (none) or a forward level");
    (precision == YB_FP64 ? f->tile64 : f->tile32).tail_level = tail_level;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_phase_clock(yb_factor *f, void *d_clock) {
  return guard([&] {
    require(f != nullptr, "null factor");
    f->phase_clock = (long long *)d_clock;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_check_error(yb_factor *f) {
  return guard([&] {
    require(f != nullptr, "null factor");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    int32_t word = 0;
    cuda_check(cudaMemcpy(&word, f->error.get(), sizeof word, cudaMemcpyDeviceToHost), "read error word");
    if (word != 0) {
      cuda_check(cudaMemset(f->error.get(), 0, sizeof word), "clear error word");
      throw host::Error(host::kDeviceTimeout, "a bounded device wait ran out in a solve of this factor");
    }
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_withhold_lane_page(yb_factor *f, int32_t page) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(page >= -1, "page must be -1 or a page index");
    f->lane_withhold = page;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_get_tile(const yb_factor *f, int32_t precision, int32_t *tile_width, int32_t *threads,
                                      int32_t *blocks_per_sm) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    const TileConfig &t = precision == YB_FP64 ? f->tile64 : f->tile32;
    if (tile_width) *tile_width = t.width;
    if (threads) *threads = t.threads;
    if (blocks_per_sm) *blocks_per_sm = t.blocks_per_sm;
    return YB_OK;
  });
}

// ---------------------------------------------------------------------------------------------
// Launches
// ---------------------------------------------------------------------------------------------

namespace yb {

template <class T, int W, Load LOAD, Store STORE>
void launch_tiles_w(yb_factor *f, TileArgs<T> a, const TileConfig &cfg, cudaStream_t stream, DeviceArray<T> &scratch) {
  if (a.count <= 0) return;
  a.tiles = (a.count + W - 1) / W;
  const int64_t grid = std::min<int64_t>(a.tiles, (int64_t)f->gpu->sm_count * cfg.blocks_per_sm);
  scratch.reserve((size_t)grid * a.n * W);
  a.scratch = scratch.get();
  tile_solve_kernel<T, W, LOAD, STORE><<<(unsigned)grid, cfg.threads, 0, stream>>>(a);
  cuda_check(cudaGetLastError(), "tile_solve_kernel launch");
}

template <class T, Load LOAD, Store STORE>
void launch_tiles(yb_factor *f, TileArgs<T> a, const TileConfig &cfg, cudaStream_t stream, DeviceArray<T> &scratch) {
  switch (cfg.width) {
    case 1: return launch_tiles_w<T, 1, LOAD, STORE>(f, a, cfg, stream, scratch);
    case 2: return launch_tiles_w<T, 2, LOAD, STORE>(f, a, cfg, stream, scratch);
    case 4: return launch_tiles_w<T, 4, LOAD, STORE>(f, a, cfg, stream, scratch);
    case 8: return launch_tiles_w<T, 8, LOAD, STORE>(f, a, cfg, stream, scratch);
    case 16: return launch_tiles_w<T, 16, LOAD, STORE>(f, a, cfg, stream, scratch);
    case 32: return launch_tiles_w<T, 32, LOAD, STORE>(f, a, cfg, stream, scratch);
    default: throw host::Error(host::kInvalidArgument, "unsupported tile width");
  }
}

template <class T> void upload_slices(DeviceSlices<T> &d, const SliceSweep<double> &s, cudaStream_t stream) {
  d.levels = s.levels;
  d.slices = s.slices();
  d.entries = (int64_t)s.col.size();
  d.level_slice.upload(s.level_slice, stream);
  std::vector<int2> span(s.offset.size());
  for (size_t i = 0; i < span.size(); ++i) span[i] = make_int2(s.offset[i], s.length[i]);
  d.span.upload(span, stream);
  d.row.upload(s.row, stream);
  d.col.upload(s.col, stream);
  d.dinv.upload(convert<T>(s.dinv), stream);
  d.val.upload(convert<T>(s.val), stream);
}

template <class T>
DeviceSlices<T> *slices_for(yb_factor *f, std::map<int, std::unique_ptr<DeviceSlices<T>[]>> &cache, int W,
                            cudaStream_t stream) {
  auto it = cache.find(W);
  if (it != cache.end()) return it->second.get();
  std::unique_ptr<DeviceSlices<T>[]> pair(new DeviceSlices<T>[2]);
  upload_slices(pair[0], slice_sweep(f->plan.fwd, f->plan.n, 32 / W), stream);
  upload_slices(pair[1], slice_sweep(f->plan.bwd, f->plan.n, 32 / W), stream);
  auto *out = pair.get();
  cache.emplace(W, std::move(pair));
  return out;
}

template <class T> SliceView<T> slice_view(const DeviceSlices<T> &d) {
  return SliceView<T>{d.levels, d.level_slice.get(), d.span.get(), d.row.get(), d.dinv.get(), d.col.get(), d.val.get()};
}

template <class T> size_t smem_bytes(const yb_factor *f, int W) { return (size_t)(f->n + 2) * W * sizeof(T); }

template <class T> bool smem_fits(const yb_factor *f, const TileConfig &cfg) {
  return smem_bytes<T>(f, cfg.width) <= (size_t)f->gpu->smem_optin &&
         smem_bytes<T>(f, cfg.width) * cfg.blocks_per_sm <= (size_t)f->gpu->smem_per_sm;
}

template <class T, int W>
void launch_smem_w(yb_factor *f, SmemArgs<T> a, const TileConfig &cfg, cudaStream_t stream,
                   std::map<int, std::unique_ptr<DeviceSlices<T>[]>> &cache) {
  // entries prefetched per slice: as many as keep the kernel within 128 registers
  constexpr int CH = sizeof(T) == 8 ? 4 : 8;
  DeviceSlices<T> *sl = slices_for<T>(f, cache, W, stream);
  a.fwd = slice_view(sl[0]);
  a.bwd = slice_view(sl[1]);
  a.tiles = (a.count + W - 1) / W;
  const size_t smem = smem_bytes<T>(f, W);
  cuda_check(cudaFuncSetAttribute(smem_tile_kernel<T, W, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute");
  const int64_t grid = std::min<int64_t>(a.tiles, (int64_t)f->gpu->sm_count * cfg.blocks_per_sm);
  smem_tile_kernel<T, W, CH><<<(unsigned)grid, cfg.threads, smem, stream>>>(a);
  cuda_check(cudaGetLastError(), "smem_tile_kernel launch");
}

template <class T>
void launch_smem(yb_factor *f, SmemArgs<T> a, const TileConfig &cfg, cudaStream_t stream,
                 std::map<int, std::unique_ptr<DeviceSlices<T>[]>> &cache) {
  switch (cfg.width) {
    case 1: return launch_smem_w<T, 1>(f, a, cfg, stream, cache);
    case 2: return launch_smem_w<T, 2>(f, a, cfg, stream, cache);
    case 4: return launch_smem_w<T, 4>(f, a, cfg, stream, cache);
    case 8: return launch_smem_w<T, 8>(f, a, cfg, stream, cache);
    case 16: return launch_smem_w<T, 16>(f, a, cfg, stream, cache);
    case 32: return launch_smem_w<T, 32>(f, a, cfg, stream, cache);
    default: throw host::Error(host::kInvalidArgument, "unsupported tile width");
  }
}

// The dense tail's first level: the shallowest forward level whose rows and above number at most
// kTailRows (dense inverse entries grow as the square), or 0 for none.
constexpr int kTailRows = 400;
int32_t tail_level_for(const yb_factor *f, const TileConfig &cfg) {
  if (cfg.tail_level >= 0) return cfg.tail_level;
  const auto &F = f->plan.fwd;
  int32_t level = F.levels, rows = 0;
  while (level > 1 && rows + (F.level_ptr[level] - F.level_ptr[level - 1]) <= kTailRows) {
    rows += F.level_ptr[level] - F.level_ptr[level - 1];
    --level;
  }
  // worth it only when it removes a good number of levels
  return (F.levels - level >= 8) ? level : 0;
}

int32_t tail_rows_for(const yb_factor *f, int32_t level) {
  if (level <= 0 || level >= f->plan.fwd.levels) return 0;
  return f->plan.fwd.level_ptr[f->plan.fwd.levels] - f->plan.fwd.level_ptr[level];
}

template <class T> size_t stream_smem_bytes(const yb_factor *f, const TileConfig &cfg, int W) {
  const size_t y = (((size_t)(f->n + 2) * W * sizeof(T)) + 127) & ~(size_t)127;
  const int m = tail_rows_for(f, tail_level_for(f, cfg));
  const size_t tb = (((size_t)(m + 1) * W * sizeof(T)) + 15) & ~(size_t)15;
  const size_t ts = (((size_t)(m + 1) * 4) + 127) & ~(size_t)127;
  return y + tb + ts + (size_t)cfg.stream_warps * cfg.ring * cfg.page_bytes + (size_t)cfg.stream_warps * cfg.ring * 8;
}

template <class T> bool stream_fits(const yb_factor *f, const TileConfig &cfg, int W) {
  return stream_smem_bytes<T>(f, cfg, W) <= (size_t)f->gpu->smem_optin;
}

template <class T> DeviceStream *stream_for(yb_factor *f, const TileConfig &cfg, int W, cudaStream_t stream) {
  const int narrow = cfg.narrow_rows > 0 ? cfg.narrow_rows : 2 * (32 / W);
  const int tail_level = tail_level_for(f, cfg);
  const auto key = std::make_tuple((int)sizeof(T), W, cfg.stream_warps, cfg.page_bytes, narrow, tail_level);
  auto it = f->streams.find(key);
  if (it != f->streams.end()) return it->second.get();
  const StreamLayout lay =
      stream_layout(f->plan, W, (int)sizeof(T), cfg.stream_warps, cfg.page_bytes, narrow, tail_level);
  auto d = std::make_unique<DeviceStream>();
  d->stages = lay.stages;
  d->G = lay.G;
  d->records = lay.records;
  d->bytes = (int64_t)lay.blob.size();
  d->fwd_wide = lay.fwd_wide, d->bwd_wide = lay.bwd_wide;
  d->fwd_narrow_rows = lay.fwd_narrow_rows, d->bwd_narrow_rows = lay.bwd_narrow_rows;
  d->blob.upload(lay.blob, stream);
  d->warp_page.upload(lay.warp_page, stream);
  std::vector<uint8_t> scale(lay.load_scale.size() * sizeof(T));
  for (size_t i = 0; i < lay.load_scale.size(); ++i) {
    const T v = (T)lay.load_scale[i];
    std::memcpy(scale.data() + i * sizeof(T), &v, sizeof(T));
  }
  d->load_scale.upload(scale, stream);
  d->tail = lay.tail;
  d->tail_slot.upload(lay.tail_slot.empty() ? std::vector<int32_t>{0} : lay.tail_slot, stream);
  cuda_check(cudaStreamSynchronize(stream), "stream layout upload");
  auto *out = d.get();
  f->streams.emplace(key, std::move(d));
  return out;
}

template <class T, int W>
void launch_stream_w(yb_factor *f, StreamArgs a, const TileConfig &cfg, cudaStream_t stream) {
  DeviceStream *d = stream_for<T>(f, cfg, W, stream);
  a.tiles = (a.count + W - 1) / W;
  a.blob = d->blob.get();
  a.warp_page = d->warp_page.get();
  a.load_scale = d->load_scale.get();
  a.page_bytes = cfg.page_bytes;
  a.ring = cfg.ring;
  a.stages = d->stages;
  a.tail = d->tail;
  a.tail_slot = d->tail_slot.get();
  a.error = f->error.get();
  a.phase_clock = f->phase_clock;
  const size_t smem = stream_smem_bytes<T>(f, cfg, W);
  cuda_check(cudaFuncSetAttribute(stream_tile_kernel<T, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
             "cudaFuncSetAttribute");
  const int64_t grid = std::min<int64_t>(a.tiles, (int64_t)f->gpu->sm_count * cfg.blocks_per_sm);
  stream_tile_kernel<T, W><<<(unsigned)grid, cfg.stream_warps * 32, smem, stream>>>(a);
  cuda_check(cudaGetLastError(), "stream_tile_kernel launch");
}

template <class T> void launch_stream(yb_factor *f, StreamArgs a, const TileConfig &cfg, cudaStream_t stream) {
  switch (cfg.width) {
    case 1: return launch_stream_w<T, 1>(f, a, cfg, stream);
    case 2: return launch_stream_w<T, 2>(f, a, cfg, stream);
    case 4: return launch_stream_w<T, 4>(f, a, cfg, stream);
    case 8: return launch_stream_w<T, 8>(f, a, cfg, stream);
    case 16: return launch_stream_w<T, 16>(f, a, cfg, stream);
    case 32: return launch_stream_w<T, 32>(f, a, cfg, stream);
    default: throw host::Error(host::kInvalidArgument, "unsupported tile width");
  }
}

// The domain layout of a shape, built and uploaded on first use; null if the factor admits none
// (an upper-triangle entry of a top row reaching below the cut, as an LU factor may have).
template <class T> DeviceDomain *domain_for(yb_factor *f, const TileConfig &cfg, cudaStream_t stream) {
  const auto key = std::make_tuple((int)sizeof(T), cfg.domain_warps, cfg.domain_page, cfg.domain_cut);
  auto it = f->domains.find(key);
  if (it != f->domains.end()) return it->second.get();
  std::unique_ptr<DeviceDomain> d;
  try {
    const DomainLayout lay = domain_layout(f->plan, (int)sizeof(T), cfg.domain_warps, cfg.domain_page, cfg.domain_cut);
    d = std::make_unique<DeviceDomain>();
    d->K = lay.K, d->tail = lay.tail, d->stages = lay.stages, d->warps = lay.warps, d->page_bytes = lay.page_bytes;
    d->records = lay.records, d->bytes = (int64_t)lay.blob.size(), d->entries = lay.entries;
    d->dense_entries = lay.dense_entries, d->cost = lay.cost;
    d->blob.upload(lay.blob, stream);
    d->warp_page.upload(lay.warp_page, stream);
    d->tail_slot.upload(lay.tail_slot.empty() ? std::vector<int32_t>{0} : lay.tail_slot, stream);
    cuda_check(cudaStreamSynchronize(stream), "domain layout upload");
  } catch (const host::Error &e) {
    if (e.status != host::kInvalidArgument && e.status != host::kTooLarge) throw;
    d.reset();
  }
  auto *out = d.get();
  f->domains.emplace(key, std::move(d));
  return out;
}

template <class T> size_t domain_smem(const yb_factor *f, const TileConfig &cfg, const DeviceDomain *d, int W) {
  return domain_smem_bytes((int32_t)f->n, W, (int32_t)sizeof(T), d->tail, cfg.domain_warps, cfg.domain_ring,
                           cfg.domain_page);
}

template <class T, int W, class IO>
void launch_domain_w(yb_factor *f, const TileConfig &cfg, int64_t count, const IO &io, cudaStream_t stream) {
  DeviceDomain *d = domain_for<T>(f, cfg, stream);
  if (!d) throw host::Error(host::kInvalidArgument, "the factor admits no domain layout");
  const size_t smem = domain_smem<T>(f, cfg, d, W);
  if (smem > (size_t)f->gpu->smem_optin) throw host::Error(host::kInvalidArgument, "the tile does not fit in shared memory");
  DomainArgs a{};
  a.n = (int32_t)f->n;
  a.count = count;
  a.tiles = (count + W - 1) / W;
  a.blob = d->blob.get();
  a.warp_page = d->warp_page.get();
  a.page_bytes = cfg.domain_page;
  a.ring = cfg.domain_ring;
  a.stages = d->stages;
  a.tail = d->tail;
  a.tail_slot = d->tail_slot.get();
  a.error = f->error.get();
  a.phase_clock = f->phase_clock;
  // the footprint keeps kIoStaticSmem for the IO policy's static shared memory (its reductions,
  // which grow with W); a policy that needs more at this width runs at half the width
  cudaFuncAttributes attr{};
  cuda_check(cudaFuncGetAttributes(&attr, domain_tile_kernel<T, W, IO>), "cudaFuncGetAttributes");
  const size_t dynamic = smem - kIoStaticSmem;
  if (dynamic + attr.sharedSizeBytes > (size_t)f->gpu->smem_optin) {
    if constexpr (W > 1) {
      TileConfig half = cfg;
      half.width = W / 2;
      return launch_domain_w<T, W / 2, IO>(f, half, count, io, stream);
    } else {
      throw host::Error(host::kInvalidArgument, "the tile does not fit in shared memory");
    }
  }
  cuda_check(cudaFuncSetAttribute(domain_tile_kernel<T, W, IO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dynamic),
             "cudaFuncSetAttribute");
  const int64_t grid = std::min<int64_t>(a.tiles, (int64_t)f->gpu->sm_count);
  domain_tile_kernel<T, W, IO><<<(unsigned)grid, cfg.domain_warps * 32, dynamic, stream>>>(a, io);
  cuda_check(cudaGetLastError(), "domain_tile_kernel launch");
}

template <class T, class IO>
void launch_domain(yb_factor *f, const TileConfig &cfg, int64_t count, const IO &io, cudaStream_t stream) {
  switch (cfg.width) {
    case 1: return launch_domain_w<T, 1>(f, cfg, count, io, stream);
    case 2: return launch_domain_w<T, 2>(f, cfg, count, io, stream);
    case 4: return launch_domain_w<T, 4>(f, cfg, count, io, stream);
    case 8: return launch_domain_w<T, 8>(f, cfg, count, io, stream);
    case 16: return launch_domain_w<T, 16>(f, cfg, count, io, stream);
    default: throw host::Error(host::kInvalidArgument, "unsupported tile width for the domain solve");
  }
}

// The shape the auto kind runs: the streamed solve at the widest tile whose working vector and
// page rings fit in shared memory (one block per SM), else the global-scratch kernel.
// The lane solve's page ring, the most slots a layout may take (the automatic choice takes the lane
// solve only up to kLaneAutoSlots, which leave room for several blocks per SM), and the largest
// work array one launch fills (larger solves run in several launches)
constexpr int32_t kLaneMaxSlots = 256, kLaneAutoSlots = 64;
constexpr size_t kLaneWorkBytes = size_t(2) << 30;

template <class T> DeviceLane *lane_for(yb_factor *f, int warps, int page_bytes, int rpl, cudaStream_t stream) {
  const auto key = std::make_tuple((int)sizeof(T), warps, page_bytes, rpl);
  auto it = f->lanes.find(key);
  if (it != f->lanes.end()) return it->second.get();
  std::unique_ptr<DeviceLane> d;
  try {
    const LaneLayout lay = lane_layout(f->plan, (int)sizeof(T), page_bytes, kLaneMaxSlots, warps, rpl);
    d = std::make_unique<DeviceLane>();
    d->rpl = lay.rpl;
    d->warps = lay.warps, d->slots = lay.slots, d->page_bytes = lay.page_bytes, d->domains = lay.domains;
    d->top = lay.top, d->partials = lay.partials, d->fwd_live = lay.fwd_live, d->bwd_live = lay.bwd_live;
    d->entries = lay.fwd_entries + lay.bwd_entries, d->pages = lay.warp_page.back();
    d->blob.upload(lay.blob, stream);
    d->warp_page.upload(lay.warp_page, stream);
    d->in_pos.upload(lay.in_pos, stream);
    d->out_pos.upload(lay.out_pos, stream);
    d->host_out_pos = lay.out_pos;
    cuda_check(cudaStreamSynchronize(stream), "lane layout upload");
  } catch (const host::Error &e) {
    if (e.status != host::kInvalidArgument && e.status != host::kTooLarge) throw;
    d.reset();
  }
  auto *out = d.get();
  f->lanes.emplace(key, std::move(d));
  return out;
}

template <class T> size_t lane_smem(const DeviceLane *d) {
  return (size_t)d->warps * lane_warp_bytes<T>(d->slots, kLaneRing, d->page_bytes, d->rpl);
}

// The lane solve of `count` right-hand sides: gather into the work array, solve in place, scatter.
// The events of the next timed lane launch, or null when timing is off or its slots are full.
cudaEvent_t *lane_timing_slot(yb_factor *f) {
  LaneTiming &t = f->lane_timing;
  if (!t.on || t.used >= (size_t)LaneTiming::kSlots) return nullptr;
  if (t.used == t.ev.size()) {
    std::array<cudaEvent_t, 4> slot{};
    for (auto &e : slot) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
    t.ev.push_back(slot);
  }
  return t.ev[t.used++].data();
}

// The lane shape a solve of `count` right-hand sides takes: the configured one, or, when no caller
// or autotuner set the warps and the groups of 32 fit one wave of one block an SM, blocks of
// kLaneMaxWarps warps (measured on the 10,000-bus B′ at 4,096 right-hand sides: 0.61 against
// 0.76 ms per solve; on the 10,000-bus Jacobian: 1.37 against 1.84 ms).
TileConfig lane_shape(const yb_factor *f, TileConfig cfg, int64_t count) {
  if (cfg.lane_warps_auto && cfg.lane_rpl == 1 && cfg.lane_page == 0 && (count + 31) / 32 <= f->gpu->sm_count)
    cfg.lane_warps = kLaneMaxWarps;
  return cfg;
}

// The lane kernel for a layout's warps per block (the three-per-SM instance up to 8 warps, the
// one-per-SM instance above), its dynamic shared memory allowed.
template <class T, int R> auto lane_kernel(const DeviceLane *d, size_t smem) {
  auto k = d->warps > kLaneNarrowWarps ? lane_solve_kernel<T, R, true> : lane_solve_kernel<T, R, false>;
  cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "cudaFuncSetAttribute");
  return k;
}

template <class T, int R>
void launch_lane_r(yb_factor *f, DeviceLane *d, const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count,
                   cudaStream_t stream) {
  constexpr int64_t G = 32 * R;  // right-hand sides per group (a block)
  const int64_t n = f->n;
  const size_t group_bytes = (size_t)n * G * sizeof(T);
  const int64_t groups_all = (count + G - 1) / G;
  const int64_t per_launch = std::max<int64_t>(1, std::min<int64_t>(groups_all, (int64_t)(kLaneWorkBytes / group_bytes)));
  f->lane_work.reserve((size_t)per_launch * group_bytes);
  f->lane_partial.reserve((size_t)per_launch * std::max(d->partials, 1) * G * sizeof(T));
  T *work = reinterpret_cast<T *>(f->lane_work.get());
  T *partial = reinterpret_cast<T *>(f->lane_partial.get());
  const size_t smem = lane_smem<T>(d);
  if (smem > (size_t)f->gpu->smem_optin) throw host::Error(host::kInvalidArgument, "the lane solve's block does not fit in shared memory");
  const auto kernel = lane_kernel<T, R>(d, smem);
  LaneArgs a{};
  a.n = (int32_t)n;
  a.slots = d->slots, a.page_bytes = d->page_bytes, a.partials = d->partials;
  a.blob = d->blob.get();
  a.warp_page = d->warp_page.get();
  a.error = f->error.get();
  a.withhold = f->lane_withhold;  // a test's withheld page: this call's first launch only
  f->lane_withhold = -1;
  for (int64_t g0 = 0; g0 < groups_all; g0 += per_launch) {
    const int64_t groups = std::min(per_launch, groups_all - g0);
    const int64_t cols = std::min(count - g0 * G, groups * G);
    const unsigned io_grid = (unsigned)lane_io_blocks(groups, n);
    cudaEvent_t *ev = lane_timing_slot(f);
    if (ev) cuda_check(cudaEventRecord(ev[0], stream), "cudaEventRecord");
    lane_in_kernel<T, R><<<io_grid, kLaneIoWarps * 32, 0, stream>>>(b + g0 * G * ldb, ldb, cols, (int32_t)n, groups,
                                                                     d->in_pos.get(), work, nullptr);
    cuda_check(cudaGetLastError(), "lane_in_kernel launch");
    if (ev) cuda_check(cudaEventRecord(ev[1], stream), "cudaEventRecord");
    kernel<<<(unsigned)groups, d->warps * 32, smem, stream>>>(a, work, partial);
    cuda_check(cudaGetLastError(), "lane_solve_kernel launch");
    a.withhold = -1;
    if (ev) cuda_check(cudaEventRecord(ev[2], stream), "cudaEventRecord");
    lane_out_kernel<T, R><<<io_grid, kLaneIoWarps * 32, 0, stream>>>(work, cols, (int32_t)n, groups, d->out_pos.get(),
                                                                      x + g0 * G * ldx, ldx);
    cuda_check(cudaGetLastError(), "lane_out_kernel launch");
    if (ev) cuda_check(cudaEventRecord(ev[3], stream), "cudaEventRecord");
  }
}

// The lane solve of `count` right-hand sides with the layout's right-hand sides per lane.
template <class T>
void launch_lane(yb_factor *f, DeviceLane *d, const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count,
                 cudaStream_t stream) {
  if (d->rpl == 2)
    launch_lane_r<T, 2>(f, d, b, ldb, x, ldx, count, stream);
  else
    launch_lane_r<T, 1>(f, d, b, ldb, x, ldx, count, stream);
}

// The lane layout a solve takes, with `rpl` right-hand sides per lane: the configured warps per
// block, or fewer when a block does not fit shared memory; with page bytes 0, the largest page of
// 2048, 1024, 768 or 512 bytes with which three blocks (two with two right-hand sides per lane) fit
// an SM (each block's rows are a long chain, so the grid should be one wave of as many warps as
// fit), else 512; with two per lane and no page that lets two blocks fit, fewer warps (down to
// four) before one block an SM. Null when the factor admits no lane layout.
template <class T> DeviceLane *lane_pick(yb_factor *f, const TileConfig &cfg, int rpl, cudaStream_t stream) {
  const size_t blocks = rpl == 1 ? 3 : 2;
  DeviceLane *fallback = nullptr;
  for (int warps = cfg.lane_warps; warps >= 1; --warps) {
    DeviceLane *d = nullptr;
    if (cfg.lane_page > 0) {
      d = lane_for<T>(f, warps, cfg.lane_page, rpl, stream);
    } else {
      for (int page : {2048, 1024, 768, 512}) {
        d = lane_for<T>(f, warps, page, rpl, stream);
        if (!d || blocks * (lane_smem<T>(d) + 1024) <= (size_t)f->gpu->smem_per_sm) break;
      }
    }
    if (!d) return nullptr;
    if (lane_smem<T>(d) > (size_t)f->gpu->smem_optin) continue;
    if (rpl == 1 || cfg.lane_page > 0 || blocks * (lane_smem<T>(d) + 1024) <= (size_t)f->gpu->smem_per_sm) return d;
    if (!fallback) fallback = d;
    if (warps <= 4) break;
  }
  return fallback;
}

template <class T> TileConfig resolve(yb_factor *f, TileConfig cfg) {
  if (cfg.kind == kTileLane) cfg.kind = kTileAuto;  // callers other than the plain solve
  if (cfg.kind == kTileGlobal) return cfg;
  if (cfg.kind == kTileDomain || cfg.kind == kTileAuto) {
    DeviceDomain *d = domain_for<T>(f, cfg, f->gpu->stream);
    if (cfg.kind == kTileDomain) {
      if (!d) throw host::Error(host::kInvalidArgument, "the factor admits no domain layout");
      if (domain_smem<T>(f, cfg, d, cfg.width) > (size_t)f->gpu->smem_optin)
        throw host::Error(host::kInvalidArgument, "the tile does not fit in shared memory");
      return cfg;
    }
    if (d)
      for (int w = 16; w >= 1; w /= 2)
        if (domain_smem<T>(f, cfg, d, w) <= (size_t)f->gpu->smem_optin) {
          TileConfig c = cfg;
          c.width = w;
          c.kind = kTileDomain;
          return c;
        }
  }
  if (cfg.kind == kTileStream) {
    if (!stream_fits<T>(f, cfg, cfg.width)) throw host::Error(host::kInvalidArgument, "the tile does not fit in shared memory");
    return cfg;
  }
  if (cfg.kind == kTileAuto) {
    for (int w = 32; w >= 1; w /= 2)
      if (stream_fits<T>(f, cfg, w)) {
        TileConfig c = cfg;
        c.width = w;
        c.blocks_per_sm = 1;
        c.kind = kTileStream;
        return c;
      }
    cfg.kind = kTileGlobal;
    return cfg;
  }
  if (cfg.kind == kTileShared) {
    if (!smem_fits<T>(f, cfg)) throw host::Error(host::kInvalidArgument, "the tile does not fit in shared memory");
    return cfg;
  }
  for (int w = 32; w >= 1; w /= 2) {
    TileConfig c = cfg;
    c.width = w;
    c.blocks_per_sm = 1;
    c.kind = kTileShared;
    if (smem_fits<T>(f, c)) return c;
  }
  cfg.kind = kTileGlobal;
  return cfg;
}

template <class T> TileArgs<T> base_args(yb_factor *f, const DeviceSweep<T> &fwd, const DeviceSweep<T> &bwd) {
  TileArgs<T> a{};
  a.n = (int32_t)f->n;
  a.in_slot = f->in_slot.get();
  a.out_slot = f->out_slot.get();
  a.fwd = view(fwd);
  a.bwd = view(bwd);
  return a;
}

// The count of right-hand sides from which the automatic choice takes the lane solve: the
// configured one, or by the domain solve's automatic tile. Where its tiles hold two or more columns
// the domain solve is the faster below about 1,500 (measured on the 10,000-bus B′, tiles of 2: 0.34
// against 0.45 ms at 1,024 right-hand sides, 0.50 against 0.47 at 1,536, 0.58 against 0.50 at
// 2,048); where they hold one column, or it has none, the lane solve is the faster from two groups
// of 32 (the 10,000-bus Jacobian: 1.01 against 0.98 ms at 64, 7.05 against 1.09 ms at 1,024).
template <class T> int64_t lane_threshold(yb_factor *f, const TileConfig &cfg) {
  if (cfg.lane_min_count >= 0) return cfg.lane_min_count;
  TileConfig automatic = cfg;
  automatic.kind = kTileAuto;
  const TileConfig d = resolve<T>(f, automatic);
  return d.kind == kTileDomain && d.width >= 2 ? 1536 : 64;
}

// Solves `count` right-hand sides already on the device, in `precision`, on `stream`.
void solve_device(yb_factor *f, const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count, int precision,
                  cudaStream_t stream) {
  if (count <= 0 || f->n == 0) return;
  auto run = [&](auto zero, const TileConfig &configured, auto &fwd, auto &bwd, auto &scratch, auto &cache) {
    using T = decltype(zero);
    if (configured.kind == kTileLane || (configured.kind == kTileAuto && count >= lane_threshold<T>(f, configured))) {
      DeviceLane *d = lane_pick<T>(f, lane_shape(f, configured, count), configured.lane_rpl, stream);
      if (d && (configured.kind == kTileLane || d->slots <= kLaneAutoSlots)) {
        launch_lane<T>(f, d, b, ldb, x, ldx, count, stream);
        return;
      }
      if (configured.kind == kTileLane) throw host::Error(host::kInvalidArgument, "the factor admits no lane layout");
    }
    const TileConfig cfg = resolve<T>(f, configured);
    if (cfg.kind == kTileDomain) {
      DenseIO io{b, ldb, x, ldx, f->in_slot.get(), f->out_slot.get()};
      launch_domain<T>(f, cfg, count, io, stream);
    } else if (cfg.kind == kTileStream) {
      StreamArgs a{};
      a.n = (int32_t)f->n;
      a.count = count;
      a.b = b, a.ldb = ldb, a.x = x, a.ldx = ldx;
      a.in_slot = f->in_slot.get();
      a.out_slot = f->out_slot.get();
      launch_stream<T>(f, a, cfg, stream);
    } else if (cfg.kind == kTileShared) {
      SmemArgs<T> a{};
      a.n = (int32_t)f->n;
      a.count = count;
      a.b = b, a.ldb = ldb, a.x = x, a.ldx = ldx;
      a.in_slot = f->in_slot.get();
      a.out_slot = f->out_slot.get();
      launch_smem<T>(f, a, cfg, stream, cache);
    } else {
      auto a = base_args<T>(f, fwd, bwd);
      a.b = b, a.ldb = ldb, a.x = x, a.ldx = ldx, a.count = count;
      launch_tiles<T, Load::Dense, Store::Dense>(f, a, cfg, stream, scratch);
    }
  };
  if (precision == YB_FP64)
    run(0.0, f->tile64, f->fwd64, f->bwd64, f->scratch64, f->slices64);
  else
    run(0.0f, f->tile32, f->fwd32, f->bwd32, f->scratch32, f->slices32);
}

// Solves the right-hand sides e_plus - e_minus of `count` pairs (natural rows, -1 for none) into
// `out` (n x count, natural order), with each column's rank-one update of `base` when `base` is
// given (then alpha, inverse_weight and singular too). The domain solve where the factor admits it,
// else the global-scratch solve.
void solve_pairs_device(yb_factor *f, int64_t count, const int32_t *plus, const int32_t *minus, const double *base,
                        const double *alpha, const double *inverse_weight, int32_t *singular, double *out, int64_t ldo,
                        cudaStream_t stream) {
  if (count <= 0 || f->n == 0) return;
  TileConfig cfg = resolve<double>(f, f->tile64);
  if (cfg.kind == kTileDomain) {
    if (base) {
      PairIO<true> io{plus, minus, out, ldo, f->in_slot.get(), f->out_slot.get(), base, alpha, inverse_weight, singular};
      launch_domain<double>(f, cfg, count, io, stream);
    } else {
      PairIO<false> io{plus, minus, out, ldo, f->in_slot.get(), f->out_slot.get(), nullptr, nullptr, nullptr, nullptr};
      launch_domain<double>(f, cfg, count, io, stream);
    }
    return;
  }
  cfg = f->tile64;
  cfg.kind = kTileGlobal;
  auto a = base_args<double>(f, f->fwd64, f->bwd64);
  a.x = out, a.ldx = ldo, a.count = count;
  a.plus = plus, a.minus = minus;
  a.base = base, a.alpha = alpha, a.inverse_weight = inverse_weight, a.singular = singular;
  if (base)
    launch_tiles<double, Load::Pairs, Store::PairUpdate>(f, a, cfg, stream, f->scratch64);
  else
    launch_tiles<double, Load::Pairs, Store::Dense>(f, a, cfg, stream, f->scratch64);
}

// The domain solve in FP64 with an IO policy of the callers' (capi_dc.cu): the batched screening,
// the adjoint's solves.
template <class IO> void launch_domain_fp64(yb_factor *f, int64_t count, const IO &io, cudaStream_t stream) {
  const TileConfig cfg = resolve<double>(f, f->tile64);
  if (cfg.kind != kTileDomain)
    throw host::Error(host::kInvalidArgument, "this solve needs the domain solve, which the factor does not admit");
  launch_domain<double>(f, cfg, count, io, stream);
}
template void launch_domain_fp64<OutageIO>(yb_factor *, int64_t, const OutageIO &, cudaStream_t);
template void launch_domain_fp64<BusIO>(yb_factor *, int64_t, const BusIO &, cudaStream_t);
template void launch_domain_fp64<AdjointIO>(yb_factor *, int64_t, const AdjointIO &, cudaStream_t);

}  // namespace yb

extern "C" int32_t yb_solve_many_transpose(yb_factor *f, const double *rhs, int64_t count, double *out) {
  return guard([&]() -> int32_t {
    require(f != nullptr, "null factor");
    require(!f->is_complex, "a complex factor solves with yb_solve_batch_complex");
    if (f->kind != YB_LU) return yb_solve_many(f, rhs, count, out);  // a Cholesky factor: A' = A
    require(f->has_lu_arrays || f->n <= 1, "the factor keeps no LU arrays to transpose");
    if (f->n <= 1) return yb_solve_many(f, rhs, count, out);  // a single row: its own transpose
    if (!f->transposed) {
      yb_factor *t = nullptr;
      auto make = f->lu_transposed ? yb_factor_from_lu : yb_factor_from_lu_transposed;
      const int32_t st = make(f->gpu, f->n, f->lu_l_ptr.data(), f->lu_l_idx.data(), f->lu_l_val.data(),
                              f->lu_u_ptr.data(), f->lu_u_idx.data(), f->lu_u_val.data(), f->lu_p.data(),
                              f->lu_q.data(), &t);
      if (st != YB_OK) throw host::Error(st, "making the transposed factor failed");
      f->transposed.reset(t);
    }
    f->transposed->width = f->width;
    const int32_t st = yb_solve_many(f->transposed.get(), rhs, count, out);
    if (st != YB_OK) throw host::Error(st, "the transposed solve failed");
    return YB_OK;
  });
}

extern "C" int32_t yb_solve_many_mixed(yb_factor *f, const double *rhs, int64_t count, double *out, int32_t max_steps,
                                       double tolerance, int32_t *steps, double *ratio) {
  return guard([&]() -> int32_t {
    require(f != nullptr, "null factor");
    require(count >= 0, "negative count");
    const int64_t n = f->n;
    if (n == 0 || count == 0) return YB_OK;
    require(rhs && out, "null array");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = f->gpu->stream;
    // blocks of at most the block width and of at most 1 GiB of right-hand sides
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>({count, f->width, (int64_t)((size_t(1) << 30) / (8 * n))}));
    f->mixed_b.reserve((size_t)(n * chunk)), f->mixed_x.reserve((size_t)(n * chunk));
    f->mixed_ratio.reserve((size_t)chunk), f->mixed_steps.reserve((size_t)chunk);
    for (int64_t k0 = 0; k0 < count; k0 += chunk) {
      const int64_t c = std::min(chunk, count - k0);
      cuda_check(cudaMemcpyAsync(f->mixed_b.get(), rhs + k0 * n, sizeof(double) * n * c, cudaMemcpyHostToDevice, s),
                 "upload");
      const int32_t st = yb_solve_many_refined_device(f, f->mixed_b.get(), n, f->mixed_x.get(), n, c, max_steps,
                                                      tolerance, f->mixed_ratio.get(), f->mixed_steps.get(), s);
      if (st != YB_OK) throw host::Error(st, "the refined solve failed");
      cuda_check(cudaMemcpyAsync(out + k0 * n, f->mixed_x.get(), sizeof(double) * n * c, cudaMemcpyDeviceToHost, s),
                 "download");
      if (ratio)
        cuda_check(cudaMemcpyAsync(ratio + k0, f->mixed_ratio.get(), sizeof(double) * c, cudaMemcpyDeviceToHost, s),
                   "download");
      if (steps)
        cuda_check(cudaMemcpyAsync(steps + k0, f->mixed_steps.get(), sizeof(int32_t) * c, cudaMemcpyDeviceToHost, s),
                   "download");
      cuda_check(cudaStreamSynchronize(s), "refined solve");
    }
    return yb_factor_check_error(f);
  });
}

extern "C" int32_t yb_solve_many_device(yb_factor *f, const double *d_rhs, int64_t ldb, double *d_out, int64_t ldx,
                                        int64_t count, int32_t precision, void *stream) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(!f->is_complex, "a complex factor solves with yb_solve_batch_complex");
    require(count >= 0, "negative count");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(count == 0 || (d_rhs && d_out), "null device array");
    require(ldb >= f->n && ldx >= f->n, "a leading dimension is below the factor's order");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = stream ? (cudaStream_t)stream : f->gpu->stream;
    if (f->single && count > 0) {
      // One row: x = b / lower / upper, elementwise
      solve_single_row_device(f, d_rhs, ldb, d_out, ldx, count, s);
      return YB_OK;
    }
    solve_device(f, d_rhs, ldb, d_out, ldx, count, precision, s);
    return YB_OK;
  });
}

// `solve_many` (ybus_cuda/src/factor.rs:234-289) with host arrays: right-hand sides column-major
// n x count in the caller's order, solutions likewise. Blocks of `block_width` columns go up,
// are solved and come down; pinned caller memory is copied directly, pageable memory through a
// pinned staging buffer.
extern "C" int32_t yb_solve_many(yb_factor *f, const double *rhs, int64_t count, double *out) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(!f->is_complex, "a complex factor solves with yb_solve_batch_complex");
    require(count >= 0, "negative count");
    const int64_t n = f->n;
    if (n == 0 || count == 0) return YB_OK;
    require(rhs && out, "null array");
    if (f->single) {
      for (int64_t k = 0; k < count; ++k) out[k] = rhs[k] / f->single_lower / f->single_upper;
      return YB_OK;
    }
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = f->gpu->stream;
    // Chunks of at most the block width, small enough that uploads, solves and downloads of
    // successive chunks overlap (at least 256 right-hand sides, so a solve still fills the GPU)
    const int64_t chunk = std::min<int64_t>(f->width, std::min<int64_t>(kPipelineChunk, std::max<int64_t>(256, (count + 7) / 8)));
    constexpr int S = CopyPipeline::kSlots;
    auto &pipe = f->pipe;
    pipe.ensure();
    const size_t slot_values = (size_t)(n * std::min(chunk, count));
    f->dev_b.reserve(slot_values * S);
    f->dev_x.reserve(slot_values * S);
    auto is_pinned = [](const void *p) {
      cudaPointerAttributes attr{};
      if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      return attr.type == cudaMemoryTypeHost;
    };
    const bool pinned_in = is_pinned(rhs), pinned_out = is_pinned(out);
    int64_t slot_k0[S], slot_cols[S];
    bool busy[S] = {};
    // Waits for the chunk in `slot` to come back, unstages it and adds its stages' times
    auto finish = [&](int slot) {
      if (!busy[slot]) return;
      busy[slot] = false;
      cudaEvent_t *e = pipe.ev[slot];
      cuda_check(cudaEventSynchronize(e[CopyPipeline::kOutDone]), "download");
      const size_t bytes = (size_t)(n * slot_cols[slot]) * sizeof(double);
      if (!pinned_out) std::memcpy(out + slot_k0[slot] * n, pipe.stage_out[slot].get(bytes), bytes);
      float up = 0, solve = 0, down = 0;
      cuda_check(cudaEventElapsedTime(&up, e[CopyPipeline::kInStart], e[CopyPipeline::kInDone]), "cudaEventElapsedTime");
      cuda_check(cudaEventElapsedTime(&solve, e[CopyPipeline::kSolveStart], e[CopyPipeline::kSolved]), "cudaEventElapsedTime");
      cuda_check(cudaEventElapsedTime(&down, e[CopyPipeline::kOutStart], e[CopyPipeline::kOutDone]), "cudaEventElapsedTime");
      f->timings.upload += up * 1e-3;
      f->timings.solve += solve * 1e-3;
      f->timings.download += down * 1e-3;
      f->timings.blocks += 1;
    };
    // The uploads are the pipeline's bottleneck (the host link), so a call costs every upload plus
    // the last chunk's solve and download: over the last two chunks' worth of columns the chunks
    // halve, down to 256 columns, so that tail is short.
    const int64_t tail_min = std::min<int64_t>(chunk, 256);
    auto next_cols = [&](int64_t left) -> int64_t {
      if (left > 2 * chunk || left <= tail_min) return std::min(chunk, left);
      return std::min(chunk, std::max(tail_min, (left / 2 + 31) / 32 * 32));
    };
    int64_t c = 0;
    try {
      for (int64_t k0 = 0, cols = next_cols(count); k0 < count; k0 += cols, cols = next_cols(count - k0), ++c) {
        const int slot = (int)(c % S);
        finish(slot);  // the slot's previous chunk is back: its buffers are free
        const size_t bytes = (size_t)(n * cols) * sizeof(double);
        double *db = f->dev_b.get() + slot * slot_values, *dx = f->dev_x.get() + slot * slot_values;
        cudaEvent_t *e = pipe.ev[slot];
        const double *src = rhs + k0 * n;
        if (!pinned_in) {
          auto *stage = (double *)pipe.stage_in[slot].get(bytes);
          std::memcpy(stage, src, bytes);
          src = stage;
        }
        double *dst = pinned_out ? out + k0 * n : (double *)pipe.stage_out[slot].get(bytes);
        cuda_check(cudaEventRecord(e[CopyPipeline::kInStart], pipe.in), "cudaEventRecord");
        cuda_check(cudaMemcpyAsync(db, src, bytes, cudaMemcpyHostToDevice, pipe.in), "upload");
        cuda_check(cudaEventRecord(e[CopyPipeline::kInDone], pipe.in), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(s, e[CopyPipeline::kInDone], 0), "cudaStreamWaitEvent");
        cuda_check(cudaEventRecord(e[CopyPipeline::kSolveStart], s), "cudaEventRecord");
        solve_device(f, db, n, dx, n, cols, YB_FP64, s);
        cuda_check(cudaEventRecord(e[CopyPipeline::kSolved], s), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(pipe.out, e[CopyPipeline::kSolved], 0), "cudaStreamWaitEvent");
        cuda_check(cudaEventRecord(e[CopyPipeline::kOutStart], pipe.out), "cudaEventRecord");
        cuda_check(cudaMemcpyAsync(dst, dx, bytes, cudaMemcpyDeviceToHost, pipe.out), "download");
        cuda_check(cudaEventRecord(e[CopyPipeline::kOutDone], pipe.out), "cudaEventRecord");
        slot_k0[slot] = k0, slot_cols[slot] = cols, busy[slot] = true;
      }
      for (int64_t i = 0; i < S; ++i) finish((int)((c + i) % S));
    } catch (...) {
      // leave no copy in flight into the caller's arrays or the staging
      cudaStreamSynchronize(pipe.in);
      cudaStreamSynchronize(s);
      cudaStreamSynchronize(pipe.out);
      throw;
    }
    int32_t word = 0;
    cuda_check(cudaMemcpy(&word, f->error.get(), sizeof word, cudaMemcpyDeviceToHost), "read error word");
    if (word != 0) {
      cuda_check(cudaMemset(f->error.get(), 0, sizeof word), "clear error word");
      throw host::Error(host::kDeviceTimeout, "a bounded device wait ran out in the solve");
    }
    return YB_OK;
  });
}

namespace yb {

namespace {
__global__ void single_row_kernel(const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count, double lower,
                                  double upper) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count) x[k * ldx] = b[k * ldb] / lower / upper;
}
}  // namespace

void solve_single_row_device(yb_factor *f, const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count,
                             cudaStream_t stream) {
  const int threads = 256;
  const int64_t blocks = (count + threads - 1) / threads;
  single_row_kernel<<<(unsigned)blocks, threads, 0, stream>>>(b, ldb, x, ldx, count, f->single_lower, f->single_upper);
  cuda_check(cudaGetLastError(), "single_row_kernel launch");
}

}  // namespace yb

extern "C" int32_t yb_factor_stream_info(yb_factor *f, int32_t precision, int32_t *tile_width, int32_t *stages,
                                         int64_t *records, int64_t *bytes, int32_t *fwd_wide, int32_t *bwd_wide,
                                         int32_t *narrow_rows) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    const TileConfig &configured = precision == YB_FP64 ? f->tile64 : f->tile32;
    TileConfig cfg;
    DeviceStream *d = nullptr;
    if (precision == YB_FP64) {
      cfg = resolve<double>(f, configured);
      if (cfg.kind == kTileStream) d = stream_for<double>(f, cfg, cfg.width, f->gpu->stream);
    } else {
      cfg = resolve<float>(f, configured);
      if (cfg.kind == kTileStream) d = stream_for<float>(f, cfg, cfg.width, f->gpu->stream);
    }
    if (tile_width) *tile_width = cfg.width;
    if (stages) *stages = d ? d->stages : 0;
    if (records) *records = d ? d->records : 0;
    if (bytes) *bytes = d ? d->bytes : 0;
    if (fwd_wide) *fwd_wide = d ? d->fwd_wide : 0;
    if (bwd_wide) *bwd_wide = d ? d->bwd_wide : 0;
    if (narrow_rows) *narrow_rows = d ? d->fwd_narrow_rows + d->bwd_narrow_rows : 0;
    return d ? (int32_t)YB_OK : (int32_t)YB_ERROR_INVALID_ARGUMENT;
  });
}


extern "C" int32_t yb_factor_set_domain(yb_factor *f, int32_t precision, int32_t warps, int32_t ring, int32_t page_bytes,
                                        int32_t cut) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(warps >= 1 && warps <= 16, "warps must be 1 to 16");
    require(ring >= 2 && ring <= 8, "the ring holds 2 to 8 pages");
    require(page_bytes >= 512 && page_bytes <= 16384 && page_bytes % 16 == 0,
            "page bytes must be a multiple of 16 from 512 to 16384");
    require(cut >= -1, "the cut is -1 (chosen) or a forward level");
    TileConfig &t = precision == YB_FP64 ? f->tile64 : f->tile32;
    t.domain_warps = warps, t.domain_ring = ring, t.domain_page = page_bytes, t.domain_cut = cut;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_domain_info(yb_factor *f, int32_t precision, int32_t *tile_width, int32_t *cut,
                                         int32_t *top_rows, int64_t *records, int64_t *bytes, int64_t *smem_bytes,
                                         double *model_cycles) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    const TileConfig &configured = precision == YB_FP64 ? f->tile64 : f->tile32;
    TileConfig cfg = precision == YB_FP64 ? resolve<double>(f, configured) : resolve<float>(f, configured);
    if (cfg.kind != kTileDomain) throw host::Error(host::kInvalidArgument, "the solve this precision runs is not the domain solve");
    DeviceDomain *d = precision == YB_FP64 ? domain_for<double>(f, cfg, f->gpu->stream) : domain_for<float>(f, cfg, f->gpu->stream);
    if (tile_width) *tile_width = cfg.width;
    if (cut) *cut = d->K;
    if (top_rows) *top_rows = d->tail;
    if (records) *records = d->records;
    if (bytes) *bytes = d->bytes;
    if (smem_bytes)
      *smem_bytes = (int64_t)(precision == YB_FP64 ? domain_smem<double>(f, cfg, d, cfg.width) : domain_smem<float>(f, cfg, d, cfg.width));
    if (model_cycles) *model_cycles = d->cost;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_lane_info(yb_factor *f, int32_t precision, int64_t *info) {
  return guard([&] {
    require(f != nullptr && info != nullptr, "null argument");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(!f->is_complex, "a complex factor has no lane solve");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    const TileConfig &t = precision == YB_FP64 ? f->tile64 : f->tile32;
    DeviceLane *d = precision == YB_FP64 ? lane_pick<double>(f, t, t.lane_rpl, f->gpu->stream)
                                         : lane_pick<float>(f, t, t.lane_rpl, f->gpu->stream);
    if (!d) throw host::Error(host::kInvalidArgument, "the factor admits no lane layout");
    const size_t smem = precision == YB_FP64 ? lane_smem<double>(d) : lane_smem<float>(d);
    const int64_t v[12] = {d->slots, d->pages, d->page_bytes, d->fwd_live, d->bwd_live, d->entries, (int64_t)smem,
                           d->warps, d->domains, d->top, d->partials, d->rpl};
    std::copy(v, v + 12, info);
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_lane(yb_factor *f, int32_t precision, int32_t warps, int32_t page_bytes) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(warps >= 1 && warps <= kLaneMaxWarps, "1 to 16 warps per block");
    require(page_bytes == 0 || (page_bytes >= 256 && page_bytes <= 16384 && page_bytes % 16 == 0),
            "pages of 256 to 16384 bytes, a multiple of 16, or 0 for the automatic choice");
    TileConfig &t = precision == YB_FP64 ? f->tile64 : f->tile32;
    t.lane_warps = warps, t.lane_page = page_bytes, t.lane_warps_auto = false;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_lane_rhs_per_lane(yb_factor *f, int32_t precision, int32_t rhs_per_lane) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(rhs_per_lane == 1 || rhs_per_lane == 2, "1 or 2 right-hand sides per lane");
    (precision == YB_FP64 ? f->tile64 : f->tile32).lane_rpl = rhs_per_lane;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_lane_min_count(yb_factor *f, int32_t precision, int64_t min_count) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(min_count >= -1, "a count, or -1 for the automatic threshold");
    (precision == YB_FP64 ? f->tile64 : f->tile32).lane_min_count = min_count;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_set_refine_lane_min_count(yb_factor *f, int64_t min_count) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(min_count >= 0, "negative count");
    f->tile32.refine_lane_min_count = min_count;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_lane_min_counts(const yb_factor *f, int32_t precision, int64_t *lane_min_count,
                                             int64_t *refine_lane_min_count) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    yb_factor *g = const_cast<yb_factor *>(f);  // the automatic threshold may build the domain layout
    if (lane_min_count)
      *lane_min_count = precision == YB_FP64 ? lane_threshold<double>(g, g->tile64) : lane_threshold<float>(g, g->tile32);
    if (refine_lane_min_count) *refine_lane_min_count = f->tile32.refine_lane_min_count;
    return YB_OK;
  });
}

extern "C" int32_t yb_factor_attach_matrix(yb_factor *f, const int64_t *a_ptr, const int64_t *a_idx,
                                           const double *a_val) {
  return guard([&] {
    require(f != nullptr && a_ptr != nullptr, "null argument");
    const int64_t n = f->n;
    require(a_ptr[0] == 0, "pointers must start at 0");
    for (int64_t i = 0; i < n; ++i) require(a_ptr[i + 1] >= a_ptr[i], "pointers must not decrease");
    const int64_t nnz = a_ptr[n];
    require(nnz == 0 || (a_idx && a_val), "null index or value array");
    require(nnz < INT32_MAX, "the matrix has too many entries for 32-bit indices", host::kTooLarge);
    for (int64_t k = 0; k < nnz; ++k) require(a_idx[k] >= 0 && a_idx[k] < n, "a column index is out of range");
    // rows in natural order, 32 to a slice (sliced ELL: entry q of row 32g + l at ptr[g] + 32q + l),
    // columns mapped to solution slots (x's row c comes from slot out_slot[c]); padding entries
    // read the always-zero slot n with value 0
    const int64_t slices = (n + 31) / 32;
    std::vector<int32_t> p(slices + 1, 0), idx;
    std::vector<double> val;
    for (int64_t g = 0; g < slices; ++g) {
      int64_t width = 0;
      for (int64_t r = 32 * g; r < std::min<int64_t>(n, 32 * g + 32); ++r) width = std::max<int64_t>(width, a_ptr[r + 1] - a_ptr[r]);
      const size_t o = idx.size();
      idx.resize(o + 32 * width, (int32_t)n);
      val.resize(o + 32 * width, 0.0);
      for (int64_t r = 32 * g; r < std::min<int64_t>(n, 32 * g + 32); ++r)
        for (int64_t k = a_ptr[r]; k < a_ptr[r + 1]; ++k) {
          const size_t at = o + 32 * (size_t)(k - a_ptr[r]) + (size_t)(r - 32 * g);
          idx[at] = f->plan.out_slot[a_idx[k]];
          val[at] = a_val[k];
        }
      require(idx.size() < (size_t)INT32_MAX, "the matrix is too large for 32-bit offsets", host::kTooLarge);
      p[g + 1] = (int32_t)idx.size();
    }
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = f->gpu->stream;
    f->a_ptr.upload(p, s);
    f->a_idx.upload(idx.empty() ? std::vector<int32_t>{0} : idx, s);
    f->a_val.upload(val.empty() ? std::vector<double>{0.0} : val, s);
    // and A as given (CSR, natural order), for the lane refinement's residual
    std::vector<int32_t> csr_ptr(n + 1), csr_idx(nnz ? nnz : 1, 0);
    std::vector<double> csr_val(nnz ? nnz : 1, 0.0);
    for (int64_t i = 0; i <= n; ++i) csr_ptr[i] = (int32_t)a_ptr[i];
    for (int64_t k = 0; k < nnz; ++k) csr_idx[k] = (int32_t)a_idx[k], csr_val[k] = a_val[k];
    f->a_csr_ptr.upload(csr_ptr, s);
    f->a_csr_idx.upload(csr_idx, s);
    f->a_csr_val.upload(csr_val, s);
    cuda_check(cudaStreamSynchronize(s), "matrix upload");
    f->a_host_ptr.assign(a_ptr, a_ptr + n + 1);
    f->a_host_idx.assign(a_idx, a_idx + nnz);
    f->a_host_val.assign(a_val, a_val + nnz);
    f->a_attached += 1;
    f->a_rows = n;
    return YB_OK;
  });
}

namespace yb {
// The refined solve's copy of A for a lane layout (LaneRefineArgs' res_*): rows in natural order,
// 32 to a slice, entry q of row 32 s + l at ptr[s] + 32 q + l, each column as the work row that
// holds its unknown (out_pos).
void lane_residual_matrix(yb_factor *f, DeviceLane *d, cudaStream_t stream) {
  if (d->res_matrix == f->a_attached) return;
  const int64_t n = f->n, slices = (n + 31) / 32;
  std::vector<int32_t> ptr(slices + 1, 0), len(n), col;
  std::vector<double> val;
  for (int64_t s = 0; s < slices; ++s) {
    int64_t width = 0;
    for (int64_t r = 32 * s; r < std::min<int64_t>(n, 32 * s + 32); ++r)
      width = std::max<int64_t>(width, f->a_host_ptr[r + 1] - f->a_host_ptr[r]);
    const size_t o = col.size();
    require(o + 32 * (size_t)width < (size_t)INT32_MAX, "the matrix is too large for 32-bit offsets", host::kTooLarge);
    col.resize(o + 32 * width, 0);
    val.resize(o + 32 * width, 0.0);
    for (int64_t r = 32 * s; r < std::min<int64_t>(n, 32 * s + 32); ++r) {
      len[r] = (int32_t)(f->a_host_ptr[r + 1] - f->a_host_ptr[r]);
      for (int64_t k = f->a_host_ptr[r]; k < f->a_host_ptr[r + 1]; ++k) {
        const size_t at = o + 32 * (size_t)(k - f->a_host_ptr[r]) + (size_t)(r - 32 * s);
        col[at] = d->host_out_pos[f->a_host_idx[k]];
        val[at] = f->a_host_val[k];
      }
    }
    ptr[s + 1] = (int32_t)col.size();
  }
  d->res_ptr.upload(ptr, stream);
  d->res_len.upload(len.empty() ? std::vector<int32_t>{0} : len, stream);
  d->res_col.upload(col.empty() ? std::vector<int32_t>{0} : col, stream);
  d->res_val.upload(val.empty() ? std::vector<double>{0.0} : val, stream);
  cuda_check(cudaStreamSynchronize(stream), "residual matrix upload");
  d->res_matrix = f->a_attached;
}

// The refined solve through the lane solve (lane_refine.cuh), per launch's run of groups: b
// gathered once into the FP32 work array; per pass the FP32 lane solve (its correction into its
// own array), the FP64 residual of the iterate it completes (which also writes that iterate into
// the caller's x for the columns still refining), each column's decision, the restore of the best
// iterate where a pass made it no better, and, while another pass may follow, the iterate carried
// in FP64. Every kernel of a pass skips the groups that have stopped.
void launch_lane_refined(yb_factor *f, DeviceLane *d, const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count,
                         int32_t max_steps, double tolerance, double *ratio_out, int32_t *steps_out, cudaStream_t stream) {
  using T = float;
  const int64_t n = f->n;
  const size_t group_vals = (size_t)n * 32;
  const int64_t groups_all = (count + 31) / 32;
  const int64_t per_launch = std::max<int64_t>(1, std::min<int64_t>(groups_all, (int64_t)(kLaneWorkBytes / (group_vals * sizeof(T)))));
  const int64_t cols_most = per_launch * 32;
  lane_residual_matrix(f, d, stream);
  f->lane_work.reserve((size_t)per_launch * group_vals * sizeof(T));
  f->lane_partial.reserve((size_t)per_launch * std::max(d->partials, 1) * 32 * sizeof(T));
  f->refine_parts.reserve(2 * (size_t)per_launch * group_vals);
  if (max_steps >= 2) f->refine_scratch.reserve((size_t)per_launch * group_vals);
  // per column: rmax, bmax, cur, best (8 bytes each), best_steps (4); per group: col_active,
  // write_mask, restore_mask (4 each), active (1)
  const size_t state_bytes = (size_t)cols_most * 36 + (size_t)per_launch * 13 + 64;
  f->refine_state.reserve(state_bytes);
  T *work = reinterpret_cast<T *>(f->lane_work.get());
  T *partial = reinterpret_cast<T *>(f->lane_partial.get());
  T *dA = f->refine_parts.get(), *dB = dA + (size_t)per_launch * group_vals;
  double *X = f->refine_scratch.get();
  uint8_t *st = f->refine_state.get();
  LaneRefineArgs r{};
  r.n = (int32_t)n;
  r.rmax = reinterpret_cast<unsigned long long *>(st);
  r.bmax = r.rmax + cols_most;
  r.cur = reinterpret_cast<double *>(r.bmax + cols_most);
  r.best = r.cur + cols_most;
  r.best_steps = reinterpret_cast<int32_t *>(r.best + cols_most);
  r.col_active = reinterpret_cast<uint32_t *>(r.best_steps + cols_most);
  r.write_mask = r.col_active + per_launch;
  r.restore_mask = r.write_mask + per_launch;
  r.active = reinterpret_cast<uint8_t *>(r.restore_mask + per_launch);
  r.in_pos = d->in_pos.get(), r.out_pos = d->out_pos.get();
  r.res_ptr = d->res_ptr.get(), r.res_len = d->res_len.get(), r.res_col = d->res_col.get(), r.res_val = d->res_val.get();
  r.work = work;
  r.ldb = ldb, r.ldx = ldx;
  const size_t smem = lane_smem<T>(d);
  if (smem > (size_t)f->gpu->smem_optin) throw host::Error(host::kInvalidArgument, "the lane solve's block does not fit in shared memory");
  const auto kernel = lane_kernel<T, 1>(d, smem);
  LaneArgs a{};
  a.n = (int32_t)n;
  a.slots = d->slots, a.page_bytes = d->page_bytes, a.partials = d->partials;
  a.blob = d->blob.get();
  a.warp_page = d->warp_page.get();
  a.error = f->error.get();
  a.group_active = r.active;
  a.withhold = -1;
  auto check = [](const char *what) { cuda_check(cudaGetLastError(), what); };
  for (int64_t g0 = 0; g0 < groups_all; g0 += per_launch) {
    const int64_t groups = std::min(per_launch, groups_all - g0);
    r.groups = groups;
    r.count = std::min(count - g0 * 32, groups * 32);
    r.b = b + g0 * 32 * ldb, r.x = x + g0 * 32 * ldx;
    r.ratio_out = ratio_out ? ratio_out + g0 * 32 : nullptr;
    r.steps_out = steps_out ? steps_out + g0 * 32 : nullptr;
    const unsigned rows_grid = (unsigned)(groups * res_parts(n));  // blocks of kResRows rows of one group
    const unsigned group_grid = (unsigned)((groups * 32 + 127) / 128);  // a warp per group
    const int64_t init_n = std::max(r.count, groups);
    lane_refine_init_kernel<<<(unsigned)((init_n + 255) / 256), 256, 0, stream>>>(r);
    check("lane_refine_init_kernel launch");
    lane_in_kernel<T><<<(unsigned)lane_io_blocks(groups, n), kLaneIoWarps * 32, 0, stream>>>(r.b, ldb, r.count, (int32_t)n,
                                                                                           groups, d->in_pos.get(), work,
                                                                                           nullptr);
    check("lane_in_kernel launch");
    const int64_t carry_parts = std::max<int64_t>(1, (int64_t)((group_vals + 8191) / 8192));  // 8,192 values a block
    const unsigned carry_grid = (unsigned)(groups * carry_parts);
    for (int32_t pass = 0; pass <= max_steps; ++pass) {
      T *dk = pass == 1 ? dB : dA;  // this pass's correction
      a.xout = dk;
      kernel<<<(unsigned)groups, d->warps * 32, smem, stream>>>(a, work, partial);
      check("lane_solve_kernel launch");
      if (pass == 0)
        lane_residual_kernel<0><<<rows_grid, kResWarps * 32, 0, stream>>>(r, dk, nullptr, nullptr, true);
      else if (pass == 1)
        lane_residual_kernel<1><<<rows_grid, kResWarps * 32, 0, stream>>>(r, dk, dA, nullptr, false);
      else
        lane_residual_kernel<2><<<rows_grid, kResWarps * 32, 0, stream>>>(r, dk, nullptr, X, false);
      check("lane_residual_kernel launch");
      lane_refine_decide_kernel<<<group_grid, 128, 0, stream>>>(r, pass, max_steps, tolerance);
      check("lane_refine_decide_kernel launch");
      // the best iterate back where this pass made no better (x_{pass-1}), or x0 where pass 0 ends
      if (pass <= 1)
        lane_restore_kernel<T><<<rows_grid, kResWarps * 32, 0, stream>>>(r, dA);
      else
        lane_restore_kernel<double><<<rows_grid, kResWarps * 32, 0, stream>>>(r, X);
      check("lane_restore_kernel launch");
      if (pass >= 1 && pass < max_steps) {  // x_pass in FP64 for the next pass's residual
        if (pass == 1)
          lane_carry_kernel<T><<<carry_grid, 256, 0, stream>>>(r, dA, dB, X, carry_parts);
        else
          lane_carry_kernel<double><<<carry_grid, 256, 0, stream>>>(r, X, dA, X, carry_parts);
        check("lane_carry_kernel launch");
      }
    }
  }
}
}  // namespace yb

extern "C" int32_t yb_solve_many_refined_device(yb_factor *f, const double *d_rhs, int64_t ldb, double *d_out,
                                                int64_t ldx, int64_t count, int32_t max_steps, double tolerance,
                                                double *d_ratio, int32_t *d_steps, void *stream) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(count >= 0, "negative count");
    require(max_steps >= 0 && max_steps <= 64, "max_steps must be 0 to 64");
    require(tolerance >= 0.0, "the tolerance must not be negative");
    require(count == 0 || (d_rhs && d_out), "null device array");
    require(ldb >= f->n && ldx >= f->n, "a leading dimension is below the factor's order");
    require(!f->is_complex, "a complex factor solves with yb_solve_batch_complex");
    require(f->a_rows == f->n, "no matrix attached: call yb_factor_attach_matrix first");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    if (count == 0 || f->n == 0) return YB_OK;
    require(!f->single, "a single-row factor needs no refinement: use yb_solve_many_device");
    cudaStream_t s = stream ? (cudaStream_t)stream : f->gpu->stream;
    const TileConfig &t32 = f->tile32;
    if (t32.kind == kTileLane ||
        (t32.kind == kTileAuto && count >= std::max(lane_threshold<float>(f, t32), t32.refine_lane_min_count))) {
      DeviceLane *d = lane_pick<float>(f, lane_shape(f, t32, count), 1, s);  // its kernels take groups of 32 columns
      if (d && (t32.kind == kTileLane || d->slots <= kLaneAutoSlots)) {
        launch_lane_refined(f, d, d_rhs, ldb, d_out, ldx, count, max_steps, tolerance, d_ratio, d_steps, s);
        return YB_OK;
      }
      if (t32.kind == kTileLane) throw host::Error(host::kInvalidArgument, "the factor admits no lane layout");
    }
    TileConfig cfg = resolve<float>(f, f->tile32);
    if (cfg.kind != kTileDomain)
      throw host::Error(host::kInvalidArgument, "the refined solve needs the domain solve, which this factor does not admit");
    const int64_t tiles = (count + cfg.width - 1) / cfg.width;
    const int64_t grid = std::min<int64_t>(tiles, (int64_t)f->gpu->sm_count);
    f->refine_scratch.reserve((size_t)(2 * grid * f->n * cfg.width));  // each block's R and previous x
    RefineIO io{};
    io.scratch = f->refine_scratch.get();
    io.b = d_rhs, io.ldb = ldb, io.x = d_out, io.ldx = ldx;
    io.in_slot = f->in_slot.get(), io.out_slot = f->out_slot.get();
    io.a_ptr = f->a_ptr.get(), io.a_idx = f->a_idx.get(), io.a_val = f->a_val.get();
    io.max_steps = max_steps, io.tolerance = tolerance;
    io.ratio_out = d_ratio, io.steps_out = d_steps;
    launch_domain<float>(f, cfg, count, io, s);
    return YB_OK;
  });
}

namespace yb {
namespace {
// Deterministic right-hand sides for timing: values in [-1, 1] from a multiplicative hash of the index
__global__ void autotune_fill_kernel(double *b, int64_t total) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) b[i] = (double)((i * 2654435761LL) % 2001) / 1000.0 - 1.0;
}
}  // namespace
}  // namespace yb

extern "C" int32_t yb_factor_autotune(yb_factor *f, int32_t precision, int64_t count, int32_t *config, double *best_ms) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(!f->is_complex, "a complex factor has no domain solve to tune");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(count >= 1, "at least one right-hand side");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = f->gpu->stream;
    const int64_t n = f->n;
    DeviceArray<double> b((size_t)(n * count)), x((size_t)(n * count));
    autotune_fill_kernel<<<(unsigned)((n * count + 255) / 256), 256, 0, s>>>(b.get(), n * count);
    cuda_check(cudaGetLastError(), "autotune_fill_kernel launch");
    TileConfig &t = precision == YB_FP64 ? f->tile64 : f->tile32;
    const TileConfig saved = t;
    TileConfig best = saved;
    double best_time = INFINITY;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
    cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
    // times one configuration (a warm-up, then the mean of three solves) and keeps the fastest
    auto time_config = [&](const TileConfig &run) {
      t = run;
      solve_device(f, b.get(), n, x.get(), n, count, precision, s);
      cuda_check(cudaEventRecord(e0, s), "cudaEventRecord");
      for (int rep = 0; rep < 3; ++rep) solve_device(f, b.get(), n, x.get(), n, count, precision, s);
      cuda_check(cudaEventRecord(e1, s), "cudaEventRecord");
      cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
      float ms = 0;
      cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
      if (ms / 3 < best_time) best_time = ms / 3, best = run;
    };
    const int warps_list[] = {8, 12, 16}, page_list[] = {1536, 2048}, ring_list[] = {2, 3};
    for (int warps : warps_list)
      for (int page : page_list)
        for (int ring : ring_list) {
          TileConfig c = saved;
          c.kind = kTileAuto;
          c.domain_warps = warps, c.domain_page = page, c.domain_ring = ring;
          TileConfig r;
          try {
            r = precision == YB_FP64 ? resolve<double>(f, c) : resolve<float>(f, c);
          } catch (const host::Error &) {
            continue;
          }
          if (r.kind != kTileDomain) continue;
          for (int w = r.width; w >= 1 && w >= r.width / 2; w /= 2) {
            TileConfig run = r;
            run.width = w;
            time_config(run);
          }
        }
    // the global-scratch solve (every factor admits it: working vectors in global memory, the
    // fallback for factors whose tiles do not fit shared memory) at each tile width and two block
    // sizes
    for (int w : {1, 2, 4, 8, 16, 32})
      for (int threads : {256, 512}) {
        TileConfig run = saved;
        run.kind = kTileGlobal, run.width = w, run.threads = threads, run.blocks_per_sm = 2;
        try {
          time_config(run);
        } catch (const host::Error &) {
          continue;
        }
      }
    // the lane solve, when the factor admits it, at 4, 6 and 8 warps per block, with one and with
    // two right-hand sides per lane, and with one at 12 and 16 (one block an SM: for fewer groups
    // than SMs)
    for (int rpl : {1, 2})
      for (int warps : {4, 6, 8, 12, 16}) {
        if (rpl == 2 && warps > kLaneNarrowWarps) continue;
        TileConfig run = saved;
        run.kind = kTileLane, run.lane_warps = warps, run.lane_page = 0, run.lane_rpl = rpl, run.lane_warps_auto = false;
        DeviceLane *d = precision == YB_FP64 ? lane_pick<double>(f, run, rpl, s) : lane_pick<float>(f, run, rpl, s);
        if (!d || d->warps != warps) continue;  // none, or the block took fewer warps (timed on its own)
        time_config(run);
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    t = std::isfinite(best_time) ? best : saved;
    if (config) {
      if (t.kind == kTileGlobal) {
        config[0] = t.kind, config[1] = t.width, config[2] = t.threads / 32, config[3] = t.blocks_per_sm, config[4] = 0;
      } else if (t.kind == kTileLane) {
        DeviceLane *d = precision == YB_FP64 ? lane_pick<double>(f, t, t.lane_rpl, s) : lane_pick<float>(f, t, t.lane_rpl, s);
        config[0] = t.kind, config[1] = 0, config[2] = t.lane_warps, config[3] = kLaneRing, config[4] = d->page_bytes;
      } else {
        config[0] = t.kind, config[1] = t.width, config[2] = t.domain_warps, config[3] = t.domain_ring,
        config[4] = t.domain_page;
      }
    }
    if (best_ms) *best_ms = best_time;
    return YB_OK;
  });
}
