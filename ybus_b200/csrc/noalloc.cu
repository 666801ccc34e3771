// A solve entry point that allocates nothing on the device.
//
// Some callers cannot let a library call cudaMalloc during a solve: a host program that has
// handed all of a GPU's memory to its own pool allocator (a caching allocator that reserved the
// device up front, so a cudaMalloc from the library could fail or fragment it), or a real-time
// loop where a device allocation's implicit synchronisation and unbounded latency are not
// acceptable. For them, yb_solve_many_device_noalloc runs the level-scheduled tile solve
// (solve.cuh) with its per-block working vectors in a fixed array compiled into this library,
// instead of the scratch buffer the ordinary entry points grow on demand.
//
// The array is kNoAllocScratchBytes (16 MiB) of device memory that every GPU which loads the
// library holds until the process exits. yb_gpu_new looks the array's device address up
// (cudaGetSymbolAddress, with that device current) and keeps it, which also makes the driver load
// this file's module and place the array then: with lazy module loading (the default since CUDA
// 12.2) that would otherwise happen at the first solve of this entry point, which would then
// allocate after all. All calls share the one array and it keeps whatever the last call
// left there: nothing in it needs to start at zero (each tile's load overwrites every slot it
// uses), but calls whose kernels overlap on the GPU, on two streams or two host threads, race on
// it and must be serialised by the caller.
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "../../include/ybgpu.h"
#include "capi_common.hpp"
#include "device.cuh"
#include "factor_state.cuh"
#include "solve.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_lock;
void *g_noalloc_address[kMaxDevices] = {};

// The array's device address on `device` (the current device), looked up once.
void *scratch_address(int device) {
  if (device < 0 || device >= kMaxDevices) throw yb::host::Error(yb::host::kInvalidArgument, "device index out of range");
  std::lock_guard<std::mutex> hold(g_noalloc_lock);
  if (!g_noalloc_address[device]) {
    void *p = nullptr;
    yb::cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress of the fixed scratch array");
    g_noalloc_address[device] = p;
  }
  return g_noalloc_address[device];
}

template <class T, int W>
void launch(yb_factor *f, const yb::DeviceSweep<T> &fwd, const yb::DeviceSweep<T> &bwd, const yb::TileConfig &cfg,
            const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count, cudaStream_t stream) {
  const size_t slice = (size_t)f->n * W * sizeof(T);
  if (slice > kNoAllocScratchBytes)
    throw yb::host::Error(yb::host::kTooLarge,
                          "one block's working vectors (order x tile width x value size) exceed the 16 MiB fixed "
                          "scratch array of yb_solve_many_device_noalloc; use a narrower tile or yb_solve_many_device");
  yb::TileArgs<T> a{};
  a.n = (int32_t)f->n;
  a.count = count;
  a.tiles = (count + W - 1) / W;
  a.b = b, a.ldb = ldb, a.x = x, a.ldx = ldx;
  a.in_slot = f->in_slot.get();
  a.out_slot = f->out_slot.get();
  a.fwd = yb::view(fwd);
  a.bwd = yb::view(bwd);
  const int64_t fit = (int64_t)(kNoAllocScratchBytes / slice);
  const int64_t grid = std::min<int64_t>(std::min<int64_t>(a.tiles, (int64_t)f->gpu->sm_count * cfg.blocks_per_sm), fit);
  a.scratch = reinterpret_cast<T *>(scratch_address(f->gpu->device));
  yb::tile_solve_kernel<T, W, yb::Load::Dense, yb::Store::Dense><<<(unsigned)grid, cfg.threads, 0, stream>>>(a);
  yb::cuda_check(cudaGetLastError(), "tile_solve_kernel launch");
}

template <class T>
void dispatch(yb_factor *f, const yb::DeviceSweep<T> &fwd, const yb::DeviceSweep<T> &bwd, const yb::TileConfig &cfg,
              const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count, cudaStream_t stream) {
  switch (cfg.width) {
    case 1: return launch<T, 1>(f, fwd, bwd, cfg, b, ldb, x, ldx, count, stream);
    case 2: return launch<T, 2>(f, fwd, bwd, cfg, b, ldb, x, ldx, count, stream);
    case 4: return launch<T, 4>(f, fwd, bwd, cfg, b, ldb, x, ldx, count, stream);
    case 8: return launch<T, 8>(f, fwd, bwd, cfg, b, ldb, x, ldx, count, stream);
    case 16: return launch<T, 16>(f, fwd, bwd, cfg, b, ldb, x, ldx, count, stream);
    case 32: return launch<T, 32>(f, fwd, bwd, cfg, b, ldb, x, ldx, count, stream);
    default: throw yb::host::Error(yb::host::kInvalidArgument, "unsupported tile width");
  }
}

// Loads every kernel the entry point may launch (a function's code is placed in device memory when
// it is first used, under lazy loading)
template <class T, int W> void load_kernel() {
  cudaFuncAttributes attr{};
  yb::cuda_check(cudaFuncGetAttributes(&attr, yb::tile_solve_kernel<T, W, yb::Load::Dense, yb::Store::Dense>),
                 "loading the allocation-free solve's kernels");
}
template <class T> void load_kernels() {
  load_kernel<T, 1>(), load_kernel<T, 2>(), load_kernel<T, 4>(), load_kernel<T, 8>(), load_kernel<T, 16>(),
      load_kernel<T, 32>();
}

}  // namespace

namespace yb {
// Called by yb_gpu_new with `device` current: the fixed array is placed, its address kept and the
// entry point's kernels loaded now, so that no later call of yb_solve_many_device_noalloc loads a
// module or allocates.
void noalloc_prepare(int device) {
  scratch_address(device);
  load_kernels<double>();
  load_kernels<float>();
}
}  // namespace yb

extern "C" int32_t yb_solve_many_device_noalloc(yb_factor *f, const double *d_rhs, int64_t ldb, double *d_out,
                                                int64_t ldx, int64_t count, int32_t precision, void *stream) {
  using namespace yb;
  return guard([&] {
    require(f != nullptr, "null factor");
    require(!f->is_complex, "a complex factor solves with yb_solve_batch_complex");
    require(count >= 0, "negative count");
    require(precision == YB_FP64 || precision == YB_FP32, "unknown precision");
    require(count == 0 || (d_rhs && d_out), "null device array");
    require(ldb >= f->n && ldx >= f->n, "a leading dimension is below the factor's order");
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    if (count == 0 || f->n == 0) return YB_OK;
    cudaStream_t s = stream ? (cudaStream_t)stream : f->gpu->stream;
    if (f->single) {
      solve_single_row_device(f, d_rhs, ldb, d_out, ldx, count, s);
      return YB_OK;
    }
    if (precision == YB_FP64)
      dispatch<double>(f, f->fwd64, f->bwd64, f->tile64, d_rhs, ldb, d_out, ldx, count, s);
    else
      dispatch<float>(f, f->fwd32, f->bwd32, f->tile32, d_rhs, ldb, d_out, ldx, count, s);
    return YB_OK;
  });
}
