// C ABI of the blocks solved on the device (ybus_cuda/src/pairs.rs): right-hand sides
// e_plus - e_minus built on the device, optional rank-one Sherman-Morrison updates, and operators
// applied to the solutions (M theta + offset, one entry per column zeroed) downloaded whole or
// reduced to each column's largest |value| * weight, so only what a caller asks for leaves the GPU.
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/ybgpu.h"
#include "capi_common.hpp"
#include "device.cuh"
#include "factor_state.cuh"

using namespace yb;

// A block of solutions on the device: n x columns, column-major, natural (unknown) order
// (ybus_cuda `GpuBlock`, pairs.rs:90-110).
struct yb_block {
  yb_factor *factor = nullptr;
  int64_t columns = 0;
  DeviceArray<double> data;
  std::vector<int32_t> singular;
};

// A sparse matrix over a factor's unknowns (ybus_cuda `GpuOperator`, pairs.rs:55-86), rows x n CSR.
// The solutions here are in natural order, so its columns need no renumbering.
struct yb_operator {
  yb_factor *factor = nullptr;
  int64_t rows = 0;
  DeviceArray<int32_t> ptr, idx;
  DeviceArray<double> val, offset, weight;
};

namespace {

// One entry of M theta + offset for a column theta, entries summed in stored order, with the
// column's zeroed row set to 0 (ybus_cuda/src/kernels.cu:61-74 and the SpMM of pairs.rs:318-366)
__device__ __forceinline__ double product_entry(const int32_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                                                const double *__restrict__ val, const double *__restrict__ offset,
                                                const double *__restrict__ theta, int i, int zero_row) {
  if (i == zero_row) return 0.0;
  double s = offset[i];
  for (int p = ptr[i]; p < ptr[i + 1]; ++p) s = __dadd_rn(s, __dmul_rn(val[p], theta[idx[p]]));
  return s;
}

__global__ void product_kernel(const int32_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                               const double *__restrict__ val, const double *__restrict__ offset, int rows,
                               const double *__restrict__ theta, int64_t ldt, const int32_t *__restrict__ zero,
                               double *__restrict__ out, int64_t ldo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t k = blockIdx.y;
  if (i < rows) out[k * ldo + i] = product_entry(ptr, idx, val, offset, theta + k * ldt, i, zero[k]);
}

// Keeps the larger (value, row): the larger value, the smaller row on a tie, row -1 never winning
__device__ __forceinline__ void better(double &v, int &r, double v2, int r2) {
  if (r2 >= 0 && (v2 > v || (v2 == v && (r < 0 || r2 < r)))) v = v2, r = r2;
}

// One block of 256 threads per column: the largest |value| * weight and its row (the smallest on a
// tie; -1 and 0.0 if every product is zero), non-finite values taking no part but flagging the
// column (ybus_cuda/src/kernels.cu:78-128). With an operator (ptr non-null) the values are its
// products, computed as product_kernel computes them; otherwise the block's own entries.
__global__ void column_max_kernel(const double *__restrict__ block, int64_t ld, int rows,
                                  const double *__restrict__ weight, const int32_t *__restrict__ ptr,
                                  const int32_t *__restrict__ idx, const double *__restrict__ val,
                                  const double *__restrict__ offset, const int32_t *__restrict__ zero,
                                  double *__restrict__ best, int32_t *__restrict__ best_row,
                                  int32_t *__restrict__ not_finite) {
  __shared__ double sv[8];
  __shared__ int sr[8], sb[8];
  const int64_t k = blockIdx.x;
  const double *column = block + k * ld;
  double v = 0.0;
  int r = -1, bad = 0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const double x = ptr ? product_entry(ptr, idx, val, offset, column, i, zero[k]) : column[i];
    if (!isfinite(x)) {
      bad = 1;
      continue;
    }
    const double product = fabs(x) * (weight ? weight[i] : 1.0);
    if (product > v) v = product, r = i;  // rows increase, so a strictly larger product wins
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const double v2 = __shfl_xor_sync(0xffffffffu, v, off);
    const int r2 = __shfl_xor_sync(0xffffffffu, r, off);
    bad |= __shfl_xor_sync(0xffffffffu, bad, off);
    better(v, r, v2, r2);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sv[warp] = v, sr[warp] = r, sb[warp] = bad;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      better(v, r, sv[w], sr[w]);
      bad |= sb[w];
    }
    best[k] = r >= 0 ? v : 0.0;
    best_row[k] = r;
    not_finite[k] = bad;
  }
}

std::vector<int32_t> rows32(const int64_t *rows, int64_t count, int64_t limit, bool allow_none, const char *what) {
  std::vector<int32_t> out(count);
  for (int64_t k = 0; k < count; ++k) {
    const int64_t r = rows ? rows[k] : -1;
    require((allow_none && r == -1) || (r >= 0 && r < limit), what);
    out[k] = (int32_t)r;
  }
  return out;
}

yb_block *make_block(yb_factor *f, int64_t count, const int64_t *plus, const int64_t *minus, const double *base,
                     const double *alpha, const double *inverse_weight) {
  require(f != nullptr, "null factor");
  require(!f->is_complex, "pair solves take a real factor");
  require(count >= 0, "negative count");
  require(count <= f->width, "at most block_width() pairs");
  require(count == 0 || (plus && minus), "null pair arrays");
  const int64_t n = f->n;
  auto p = rows32(plus, count, n, true, "unknowns below dim()");
  auto m = rows32(minus, count, n, true, "unknowns below dim()");
  for (int64_t k = 0; k < count; ++k) require(p[k] < 0 || p[k] != m[k], "a pair's two unknowns must differ");
  if (base) require(count == 0 || (alpha && inverse_weight), "null update arrays");
  cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
  cudaStream_t s = f->gpu->stream;
  auto b = std::make_unique<yb_block>();
  b->factor = f;
  b->columns = count;
  b->singular.assign(count, 0);
  b->data.resize((size_t)std::max<int64_t>(1, n * count));
  if (count == 0 || n == 0) return b.release();
  DeviceArray<int32_t> dp, dm, dsing;
  dp.upload(p, s);
  dm.upload(m, s);
  DeviceArray<double> dbase, dalpha, dinv;
  if (base) {
    dbase.upload(std::vector<double>(base, base + n), s);
    dalpha.upload(std::vector<double>(alpha, alpha + count), s);
    dinv.upload(std::vector<double>(inverse_weight, inverse_weight + count), s);
    dsing.resize((size_t)count);
  }
  solve_pairs_device(f, count, dp.get(), dm.get(), base ? dbase.get() : nullptr, base ? dalpha.get() : nullptr,
                     base ? dinv.get() : nullptr, base ? dsing.get() : nullptr, b->data.get(), n, s);
  if (base)
    cuda_check(cudaMemcpyAsync(b->singular.data(), dsing.get(), sizeof(int32_t) * count, cudaMemcpyDeviceToHost, s),
               "download singular flags");
  cuda_check(cudaStreamSynchronize(s), "pair solves");
  return b.release();
}

void maxima(yb_block *b, yb_operator *op, const int64_t *zero_rows, int64_t *row, double *value, int32_t *not_finite) {
  yb_factor *f = b->factor;
  const int64_t count = b->columns;
  if (count == 0) return;
  cudaStream_t s = f->gpu->stream;
  DeviceArray<double> best((size_t)count);
  DeviceArray<int32_t> best_row((size_t)count), bad((size_t)count), zero;
  if (op) zero.upload(rows32(zero_rows, count, op->rows, true, "rows to zero below the operator's rows"), s);
  const int rows = (int)(op ? op->rows : f->n);
  column_max_kernel<<<(unsigned)count, 256, 0, s>>>(
      b->data.get(), f->n, rows, op ? op->weight.get() : nullptr, op ? op->ptr.get() : nullptr,
      op ? op->idx.get() : nullptr, op ? op->val.get() : nullptr, op ? op->offset.get() : nullptr,
      op ? zero.get() : nullptr, best.get(), best_row.get(), bad.get());
  cuda_check(cudaGetLastError(), "column_max_kernel launch");
  std::vector<double> v(count);
  std::vector<int32_t> r(count), nf(count);
  cuda_check(cudaMemcpyAsync(v.data(), best.get(), sizeof(double) * count, cudaMemcpyDeviceToHost, s), "download");
  cuda_check(cudaMemcpyAsync(r.data(), best_row.get(), sizeof(int32_t) * count, cudaMemcpyDeviceToHost, s), "download");
  cuda_check(cudaMemcpyAsync(nf.data(), bad.get(), sizeof(int32_t) * count, cudaMemcpyDeviceToHost, s), "download");
  cuda_check(cudaStreamSynchronize(s), "column maxima");
  for (int64_t k = 0; k < count; ++k) {
    if (row) row[k] = r[k];
    if (value) value[k] = v[k];
    if (not_finite) not_finite[k] = nf[k];
  }
}

void check_operator(const yb_block *b, const yb_operator *op) {
  require(b && op, "null argument");
  require(op->factor == b->factor, "an operator of this factorization");
}

}  // namespace

extern "C" int32_t yb_pair_solves(yb_factor *f, int64_t count, const int64_t *plus, const int64_t *minus,
                                  yb_block **out) {
  return guard([&] {
    require(out != nullptr, "null out");
    *out = make_block(f, count, plus, minus, nullptr, nullptr, nullptr);
    return YB_OK;
  });
}

extern "C" int32_t yb_pair_updates(yb_factor *f, const double *base, int64_t count, const int64_t *plus,
                                   const int64_t *minus, const double *alpha, const double *inverse_weight,
                                   yb_block **out) {
  return guard([&] {
    require(out != nullptr, "null out");
    require(f != nullptr && (base != nullptr || f->n == 0), "one base value per unknown");
    *out = make_block(f, count, plus, minus, base, alpha, inverse_weight);
    return YB_OK;
  });
}

extern "C" int64_t yb_block_columns(const yb_block *b) { return b ? b->columns : -1; }

extern "C" int32_t yb_block_singular(const yb_block *b, int32_t *singular) {
  return guard([&] {
    require(b && (singular || b->columns == 0), "null argument");
    std::copy(b->singular.begin(), b->singular.end(), singular);
    return YB_OK;
  });
}

extern "C" int32_t yb_block_solutions(yb_block *b, double *out) {
  return guard([&] {
    require(b != nullptr, "null block");
    const int64_t total = b->factor->n * b->columns;
    if (total == 0) return YB_OK;
    require(out != nullptr, "null output");
    cuda_check(cudaSetDevice(b->factor->gpu->device), "cudaSetDevice");
    cuda_check(cudaMemcpy(out, b->data.get(), sizeof(double) * total, cudaMemcpyDeviceToHost), "download solutions");
    return YB_OK;
  });
}

extern "C" int32_t yb_block_maxima(yb_block *b, int64_t *row, double *value, int32_t *not_finite) {
  return guard([&] {
    require(b != nullptr, "null block");
    cuda_check(cudaSetDevice(b->factor->gpu->device), "cudaSetDevice");
    maxima(b, nullptr, nullptr, row, value, not_finite);
    return YB_OK;
  });
}

extern "C" int32_t yb_block_product(yb_block *b, yb_operator *op, const int64_t *zero_rows, double *out) {
  return guard([&] {
    check_operator(b, op);
    const int64_t count = b->columns, rows = op->rows;
    if (count == 0 || rows == 0) return YB_OK;
    require(out != nullptr, "null output");
    yb_factor *f = b->factor;
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = f->gpu->stream;
    DeviceArray<int32_t> zero;
    zero.upload(rows32(zero_rows, count, rows, true, "rows to zero below the operator's rows"), s);
    DeviceArray<double> dout((size_t)(rows * count));
    require(count < 65536, "at most 65,535 columns a product");
    const dim3 grid((unsigned)((rows + 255) / 256), (unsigned)count);
    product_kernel<<<grid, 256, 0, s>>>(op->ptr.get(), op->idx.get(), op->val.get(), op->offset.get(), (int)rows,
                                        b->data.get(), f->n, zero.get(), dout.get(), rows);
    cuda_check(cudaGetLastError(), "product_kernel launch");
    cuda_check(cudaMemcpyAsync(out, dout.get(), sizeof(double) * rows * count, cudaMemcpyDeviceToHost, s),
               "download products");
    cuda_check(cudaStreamSynchronize(s), "products");
    return YB_OK;
  });
}

extern "C" int32_t yb_block_product_maxima(yb_block *b, yb_operator *op, const int64_t *zero_rows, int64_t *row,
                                           double *value, int32_t *not_finite) {
  return guard([&] {
    check_operator(b, op);
    cuda_check(cudaSetDevice(b->factor->gpu->device), "cudaSetDevice");
    maxima(b, op, zero_rows, row, value, not_finite);
    return YB_OK;
  });
}

extern "C" void yb_block_free(yb_block *b) {
  if (!b) return;
  cudaSetDevice(b->factor->gpu->device);
  delete b;
}

extern "C" int32_t yb_operator_new(yb_factor *f, int64_t rows, const int64_t *ptr, const int64_t *idx,
                                   const double *val, yb_operator **out) {
  return guard([&] {
    require(f && out && ptr, "null argument");
    require(rows >= 0 && rows < INT32_MAX, "bad row count");
    const int64_t n = f->n;
    require(ptr[0] == 0, "pointers must start at 0");
    for (int64_t i = 0; i < rows; ++i) require(ptr[i + 1] >= ptr[i], "pointers must not decrease");
    const int64_t nnz = ptr[rows];
    require(nnz < INT32_MAX, "too many entries for 32-bit indices", host::kTooLarge);
    require(nnz == 0 || (idx && val), "null index or value array");
    std::vector<int32_t> p(rows + 1), c(std::max<int64_t>(nnz, 1), 0);
    for (int64_t i = 0; i <= rows; ++i) p[i] = (int32_t)ptr[i];
    for (int64_t k = 0; k < nnz; ++k) {
      require(idx[k] >= 0 && idx[k] < n, "one column per unknown");
      c[k] = (int32_t)idx[k];
    }
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = f->gpu->stream;
    auto op = std::make_unique<yb_operator>();
    op->factor = f;
    op->rows = rows;
    op->ptr.upload(p, s);
    op->idx.upload(c, s);
    op->val.upload(nnz ? std::vector<double>(val, val + nnz) : std::vector<double>{0.0}, s);
    op->offset.upload(std::vector<double>(std::max<int64_t>(rows, 1), 0.0), s);
    op->weight.upload(std::vector<double>(std::max<int64_t>(rows, 1), 1.0), s);
    cuda_check(cudaStreamSynchronize(s), "operator upload");
    *out = op.release();
    return YB_OK;
  });
}

extern "C" int64_t yb_operator_rows(const yb_operator *op) { return op ? op->rows : -1; }

extern "C" int32_t yb_operator_set_offset(yb_operator *op, const double *offset) {
  return guard([&] {
    require(op && (offset || op->rows == 0), "one offset per row");
    if (op->rows == 0) return YB_OK;
    cuda_check(cudaSetDevice(op->factor->gpu->device), "cudaSetDevice");
    cuda_check(cudaMemcpy(op->offset.get(), offset, sizeof(double) * op->rows, cudaMemcpyHostToDevice), "upload offset");
    return YB_OK;
  });
}

extern "C" int32_t yb_operator_set_weights(yb_operator *op, const double *weights) {
  return guard([&] {
    require(op && (weights || op->rows == 0), "one weight per row");
    if (op->rows == 0) return YB_OK;
    cuda_check(cudaSetDevice(op->factor->gpu->device), "cudaSetDevice");
    cuda_check(cudaMemcpy(op->weight.get(), weights, sizeof(double) * op->rows, cudaMemcpyHostToDevice), "upload weights");
    return YB_OK;
  });
}

extern "C" void yb_operator_free(yb_operator *op) {
  if (!op) return;
  cudaSetDevice(op->factor->gpu->device);
  delete op;
}
