// The state behind the C ABI's opaque handles `yb_gpu` and `yb_factor`.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <map>
#include <memory>
#include <string>
#include <tuple>

#include "../../include/ybgpu.h"
#include "cplx.cuh"
#include "device.cuh"
#include "plan.hpp"

// The widest block `yb_factor` chooses by itself. ybus_cuda caps its default at 1,024 because each
// block is one cuSPARSE SpSM call (ybus_cuda/src/factor.rs:12); here a block is one persistent
// launch that needs at least one tile per SM to fill the GPU, so the cap is higher.
constexpr int64_t kMaxDefaultWidth = 65536;
// The largest chunk of right-hand sides the host-array solve moves through its copy pipeline
constexpr int64_t kPipelineChunk = 1024;
// The widest block a single-row factor uses (ybus_cuda/src/factor.rs:14-16): kept for API parity.
constexpr int64_t kSingleRowWidth = 64;

struct yb_gpu {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0, major = 0, minor = 0;
  int64_t l2_bytes = 0;
  int64_t smem_optin = 0;       // largest dynamic shared memory a block may opt into
  int64_t smem_per_sm = 0;
  std::string name;
  std::shared_ptr<void> zwork;  // the complex batch's device workspace (capi_complex.cu), kept between calls
};

namespace yb {

// Seconds spent in `yb_solve_many`'s stages (ybus_cuda/src/factor.rs:22-31).
struct Timings {
  double upload = 0, solve = 0, download = 0;
  int64_t blocks = 0;
};

// Per-launch times of the lane solve, when switched on: events before the gather and after the
// gather, the solve and the scatter of every launch, kept for up to kSlots launches between reads.
struct LaneTiming {
  static constexpr int kSlots = 4096;
  bool on = false;
  int device = -1;
  std::vector<std::array<cudaEvent_t, 4>> ev;
  size_t used = 0;
  LaneTiming() = default;
  LaneTiming(const LaneTiming &) = delete;
  LaneTiming &operator=(const LaneTiming &) = delete;
  ~LaneTiming() {
    for (auto &slot : ev)
      for (auto &e : slot)
        if (e) cudaEventDestroy(e);
  }
};

// The host-array solve's overlap: chunks of right-hand sides pass through an upload stream, the
// solve stream and a download stream, so the two copy engines and the SMs work on successive
// chunks at once. Each of kSlots slots holds one chunk's device buffers (and, for pageable host
// arrays, pinned staging) and the events that time its three stages.
struct CopyPipeline {
  static constexpr int kSlots = 4;
  enum { kInStart, kInDone, kSolveStart, kSolved, kOutStart, kOutDone, kEvents };
  int device = -1;
  cudaStream_t in = nullptr, out = nullptr;
  cudaEvent_t ev[kSlots][kEvents] = {};
  PinnedBuffer stage_in[kSlots], stage_out[kSlots];
  CopyPipeline() = default;
  CopyPipeline(const CopyPipeline &) = delete;
  CopyPipeline &operator=(const CopyPipeline &) = delete;
  ~CopyPipeline() {
    for (auto &slot : ev)
      for (auto &e : slot)
        if (e) cudaEventDestroy(e);
    if (in) cudaStreamDestroy(in);
    if (out) cudaStreamDestroy(out);
  }
  void ensure() {
    if (in) return;
    cuda_check(cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking), "cudaStreamCreate");
    for (auto &slot : ev)
      for (auto &e : slot) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
  }
};

// Which tile solve runs: the shared-memory one (the tile's working vector in shared memory) when
// it fits, or the one whose working vectors live in a global scratch buffer.
enum TileKind : int { kTileAuto = 0, kTileShared = 1, kTileGlobal = 2, kTileStream = 3, kTileDomain = 4, kTileLane = 5 };

// The launch shape of the tile solve for one precision.
struct TileConfig {
  int width = 8;          // right-hand sides per tile
  int threads = 512;      // threads per block
  int blocks_per_sm = 1;  // resident blocks per SM the grid is sized for
  int kind = kTileAuto;
  // the streamed solve's shape: warps per block, pages in flight per warp, page bytes, and the
  // row count under which a level goes to warp 0 (0: twice the rows of a slice)
  int stream_warps = 8, ring = 4, page_bytes = 2048, narrow_rows = 0;
  int tail_level = -1;  // forward level from which rows form the dense tail (0: none, -1: chosen)
  // the domain solve's shape: warps per block, pages in flight per warp, page bytes, and the cut
  // (first forward level of the top block; -1: chosen by the layout's cost model)
  int domain_warps = 16, domain_ring = 2, domain_page = 2048, domain_cut = -1;
  // the automatic choice takes the lane solve from this many right-hand sides on (one warp per 32:
  // fewer leave SMs idle, where the domain solve's tiles spread over all of them); -1: by the
  // factor's domain tiles (lane_threshold in capi_gpu.cu)
  int64_t lane_min_count = -1;
  int lane_warps = 8, lane_page = 0;  // the lane solve's warps per block (one group of 32 right-hand sides), page bytes
  int lane_rpl = 1;                   // right-hand sides per lane of the plain lane solve (1 or 2)
  // lane_warps not set by a caller or the autotuner: a solve of no more groups of 32 than SMs then
  // takes blocks of kLaneMaxWarps (one an SM, each warp's chain of rows shorter)
  bool lane_warps_auto = true;
  // the refined solve takes the lane solve from this many right-hand sides on (its passes cost more
  // launches than the plain solve's, so its crossover with the fused domain refinement lies higher:
  // 2,048 on the 10,000-bus B′ with blocks of 16 warps up to one wave)
  int64_t refine_lane_min_count = 2048;
};

// A lane layout on the device (LaneLayout in plan.hpp).
struct DeviceLane {
  int32_t warps = 0, slots = 0, page_bytes = 0, domains = 0, top = 0, partials = 0, fwd_live = 0, bwd_live = 0;
  int32_t rpl = 1;  // right-hand sides per lane the layout's offsets count
  int64_t entries = 0, pages = 0;
  DeviceArray<uint8_t> blob;
  DeviceArray<int32_t> warp_page, in_pos, out_pos;
  std::vector<int32_t> host_out_pos;
  // the refined solve's copy of the attached A (LaneRefineArgs' res_*): natural rows in slices of
  // 32, columns as work rows; built at its first use, for the matrix attached then
  int64_t res_matrix = -1;  // the attach count it was built for
  DeviceArray<int32_t> res_ptr, res_len, res_col;
  DeviceArray<double> res_val;
};

// A domain layout on the device (DomainLayout in plan.hpp).
struct DeviceDomain {
  int32_t K = 0, tail = 0, stages = 0, warps = 0, page_bytes = 0;
  int64_t records = 0, bytes = 0, entries = 0, dense_entries = 0;
  double cost = 0;
  DeviceArray<uint8_t> blob;
  DeviceArray<int32_t> warp_page, tail_slot;
};

// A streamed layout on the device (StreamLayout in plan.hpp).
struct DeviceStream {
  int32_t stages = 0, G = 0;
  int64_t records = 0, bytes = 0;
  int32_t fwd_wide = 0, bwd_wide = 0, fwd_narrow_rows = 0, bwd_narrow_rows = 0;
  DeviceArray<uint8_t> blob;
  DeviceArray<int32_t> warp_page;
  DeviceArray<uint8_t> load_scale;
  int32_t tail = 0;
  DeviceArray<int32_t> tail_slot;
};

// A sliced sweep on the device (SliceSweep in plan.hpp), at value type T.
template <class T> struct DeviceSlices {
  int32_t levels = 0;
  int64_t slices = 0, entries = 0;
  DeviceArray<int32_t> level_slice, row, col;
  DeviceArray<int2> span;
  DeviceArray<T> dinv, val;
};

}  // namespace yb

struct yb_factor {
  yb_gpu *gpu = nullptr;
  int64_t n = 0;
  int kind = 0;
  yb::Plan<double> plan;
  yb::DeviceArray<int32_t> in_slot, out_slot;
  yb::DeviceSweep<double> fwd64, bwd64;
  yb::DeviceSweep<float> fwd32, bwd32;
  yb::TileConfig tile64{8, 512, 1}, tile32{8, 512, 1};
  // sliced sweeps per tile width (built on first use): [width] -> {forward, backward}
  std::map<int, std::unique_ptr<yb::DeviceSlices<double>[]>> slices64;
  std::map<int, std::unique_ptr<yb::DeviceSlices<float>[]>> slices32;
  // streamed layouts by shape (precision, width, warps, page bytes, narrow rows)
  std::map<std::tuple<int, int, int, int, int, int>, std::unique_ptr<yb::DeviceStream>> streams;
  // domain layouts by shape (value bytes, warps, page bytes, cut); a null entry: the factor admits none
  std::map<std::tuple<int, int, int, int>, std::unique_ptr<yb::DeviceDomain>> domains;
  // lane layouts by (value bytes, warps, page bytes); a null entry: the factor admits none
  std::map<std::tuple<int, int, int, int>, std::unique_ptr<yb::DeviceLane>> lanes;
  yb::DeviceArray<uint8_t> lane_work, lane_partial;  // the lane solve's work and partial arrays
  yb::LaneTiming lane_timing;
  yb::DeviceArray<int32_t> error;  // the device error word (a bounded wait that ran out)
  int32_t lane_withhold = -1;      // a test's page to withhold in the next plain lane solve, or -1
  long long *phase_clock = nullptr;  // diagnostics buffer of the caller's, or null
  yb::DeviceArray<double> scratch64;
  yb::DeviceArray<float> scratch32;
  yb::DeviceArray<double> dev_b, dev_x;
  // the matrix A the factor factors, for refinement: rows in natural order, columns mapped to
  // the solution slots, FP64
  int64_t a_rows = -1;
  yb::DeviceArray<int32_t> a_ptr, a_idx;
  yb::DeviceArray<int32_t> a_csr_ptr, a_csr_idx;  // A as attached (CSR, natural order)
  yb::DeviceArray<double> a_csr_val;
  yb::DeviceArray<uint8_t> refine_state;  // the lane refinement's per-column and per-group state
  yb::DeviceArray<double> a_val;
  yb::DeviceArray<double> refine_scratch;  // per block n * W residuals; the lane refinement's FP64 iterate
  yb::DeviceArray<float> refine_parts;     // the lane refinement's FP32 corrections (two work arrays)
  std::vector<int64_t> a_host_ptr, a_host_idx;  // A as attached (CSR, natural order), on the host
  std::vector<double> a_host_val;
  int64_t a_attached = 0;                  // how many times a matrix was attached
  // a complex LU factor (yb_factor_from_lu_complex): its plan, its sweeps in complex128 and
  // complex64, and the complex matrix attached for refinement (CSR, natural order)
  bool is_complex = false;
  yb::Plan<yb::host::c128> cplan;
  yb::DeviceSweep<yb::cplx<double>> fwdz, bwdz;
  yb::DeviceSweep<yb::cplx<float>> fwdc, bwdc;
  int64_t za_rows = -1;
  yb::DeviceArray<int32_t> za_ptr, za_idx;
  yb::DeviceArray<yb::cplx<double>> za_val;
  yb::PinnedBuffer staging;
  yb::CopyPipeline pipe;
  // an LU factor's arrays as given (yb_factor_from_lu or _transposed), from which the transposed
  // solve makes the factor of the transposed matrix at its first use
  bool has_lu_arrays = false, lu_transposed = false;
  std::vector<int64_t> lu_l_ptr, lu_l_idx, lu_u_ptr, lu_u_idx, lu_p, lu_q;
  std::vector<double> lu_l_val, lu_u_val;
  std::unique_ptr<yb_factor> transposed;
  // the host-array refined solve's device arrays
  yb::DeviceArray<double> mixed_b, mixed_x, mixed_ratio;
  yb::DeviceArray<int32_t> mixed_steps;
  int64_t width = 1;
  yb::Timings timings;
  bool single = false;
  double single_lower = 1.0, single_upper = 1.0;
};

namespace yb {
void solve_pairs_device(yb_factor *f, int64_t count, const int32_t *plus, const int32_t *minus, const double *base,
                        const double *alpha, const double *inverse_weight, int32_t *singular, double *out, int64_t ldo,
                        cudaStream_t stream);
void solve_single_row_device(yb_factor *f, const double *b, int64_t ldb, double *x, int64_t ldx, int64_t count,
                             cudaStream_t stream);
}
