// For comparison only: ybus_cuda's own route to the same solve (ybus_cuda/src/sparse.rs:371-420,
// factor.rs:234-289: the two triangles as CSR matrices, cuSPARSE SpSM lower then upper on blocks of
// `width` right-hand sides), run on the same factor and device arrays as the library's solves so
// that a bench can time the two side by side on one GPU. No solve of this library calls it.
// cuSPARSE is opened with dlopen on the first call, so the library itself does not depend on it.
#include <cuda_runtime.h>
#include <cusparse.h>
#include <dlfcn.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/ybgpu.h"
#include "capi_common.hpp"
#include "device.cuh"
#include "factor_state.cuh"

using namespace yb;

namespace {

struct Sparse {
  decltype(&cusparseCreate) create;
  decltype(&cusparseDestroy) destroy;
  decltype(&cusparseSetStream) set_stream;
  decltype(&cusparseCreateCsr) create_csr;
  decltype(&cusparseDestroySpMat) destroy_sp;
  decltype(&cusparseSpMatSetAttribute) set_attr;
  decltype(&cusparseCreateDnMat) create_dn;
  decltype(&cusparseDestroyDnMat) destroy_dn;
  decltype(&cusparseSpSM_createDescr) spsm_create;
  decltype(&cusparseSpSM_destroyDescr) spsm_destroy;
  decltype(&cusparseSpSM_bufferSize) spsm_buffer;
  decltype(&cusparseSpSM_analysis) spsm_analysis;
  decltype(&cusparseSpSM_solve) spsm_solve;
};

const Sparse &sparse() {
  static Sparse s{};
  static bool ok = false;
  static std::once_flag once;
  std::call_once(once, [] {
    void *h = dlopen("libcusparse.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libcusparse.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) return;
    auto get = [&](auto &fn, const char *name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
      return fn != nullptr;
    };
    ok = get(s.create, "cusparseCreate") && get(s.destroy, "cusparseDestroy") && get(s.set_stream, "cusparseSetStream") &&
         get(s.create_csr, "cusparseCreateCsr") && get(s.destroy_sp, "cusparseDestroySpMat") &&
         get(s.set_attr, "cusparseSpMatSetAttribute") && get(s.create_dn, "cusparseCreateDnMat") &&
         get(s.destroy_dn, "cusparseDestroyDnMat") && get(s.spsm_create, "cusparseSpSM_createDescr") &&
         get(s.spsm_destroy, "cusparseSpSM_destroyDescr") && get(s.spsm_buffer, "cusparseSpSM_bufferSize") &&
         get(s.spsm_analysis, "cusparseSpSM_analysis") && get(s.spsm_solve, "cusparseSpSM_solve");
  });
  if (!ok) throw host::Error(host::kInvalidArgument, "cuSPARSE could not be opened");
  return s;
}

void sp_check(cusparseStatus_t st, const char *what) {
  if (st != CUSPARSE_STATUS_SUCCESS)
    throw host::Error(host::kCuda, std::string(what) + ": cuSPARSE status " + std::to_string((int)st));
}

// One sweep of the plan as a CSR matrix in slot order (each row's columns ascending, its diagonal
// 1 / dinv included).
void sweep_csr(const Sweep<double> &sw, int32_t n, std::vector<int32_t> &ptr, std::vector<int32_t> &idx,
               std::vector<double> &val) {
  std::vector<std::vector<std::pair<int32_t, double>>> rows(n);
  for (int32_t p = 0; p < n; ++p) {
    const int32_t r = sw.row[p];
    for (int32_t q = sw.ptr[p]; q < sw.ptr[p + 1]; ++q) rows[r].push_back({sw.col[q], sw.val[q]});
    rows[r].push_back({r, 1.0 / sw.dinv[p]});
  }
  ptr.assign(1, 0);
  idx.clear(), val.clear();
  for (auto &row : rows) {
    std::sort(row.begin(), row.end());
    for (auto [c, v] : row) idx.push_back(c), val.push_back(v);
    ptr.push_back((int32_t)idx.size());
  }
}

// b's columns into slot order, zero past `cols`; and back into x
__global__ void spsm_gather_kernel(const double *__restrict__ b, int64_t ldb, int64_t cols, int32_t n,
                                   const int32_t *__restrict__ in_slot, int64_t width, double *__restrict__ out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)n * width) return;
  const int64_t c = k / n, i = k - c * n;
  out[c * n + in_slot[i]] = c < cols ? b[c * ldb + i] : 0.0;
}
__global__ void spsm_scatter_kernel(const double *__restrict__ y, int64_t cols, int32_t n,
                                    const int32_t *__restrict__ out_slot, double *__restrict__ x, int64_t ldx) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)n * cols) return;
  const int64_t c = k / n, i = k - c * n;
  x[c * ldx + i] = y[c * n + out_slot[i]];
}

}  // namespace

extern "C" int32_t yb_reference_spsm_solve(yb_factor *f, const double *d_rhs, int64_t ldb, double *d_out, int64_t ldx,
                                           int64_t count, int64_t width, double *solve_ms) {
  return guard([&] {
    require(f != nullptr, "null factor");
    require(!f->is_complex && f->kind == YB_CHOLESKY, "the comparison takes a real Cholesky factor");
    require(count >= 1 && width >= 1 && d_rhs && d_out, "bad argument");
    require(ldb >= f->n && ldx >= f->n, "a leading dimension is below the factor's order");
    const Sparse &sp = sparse();
    const int32_t n = (int32_t)f->n;
    cuda_check(cudaSetDevice(f->gpu->device), "cudaSetDevice");
    cudaStream_t s = f->gpu->stream;
    std::vector<int32_t> lp, li, up, ui;
    std::vector<double> lv, uv;
    sweep_csr(f->plan.fwd, n, lp, li, lv);
    sweep_csr(f->plan.bwd, n, up, ui, uv);
    DeviceArray<int32_t> d_lp, d_li, d_up, d_ui;
    DeviceArray<double> d_lv, d_uv, d_b((size_t)n * width), d_t((size_t)n * width), d_y((size_t)n * width);
    d_lp.upload(lp, s), d_li.upload(li, s), d_lv.upload(lv, s);
    d_up.upload(up, s), d_ui.upload(ui, s), d_uv.upload(uv, s);
    cusparseHandle_t handle = nullptr;
    sp_check(sp.create(&handle), "cusparseCreate");
    cusparseSpMatDescr_t L = nullptr, U = nullptr;
    cusparseDnMatDescr_t B = nullptr, T = nullptr, Y = nullptr;
    cusparseSpSMDescr_t dl = nullptr, du = nullptr;
    DeviceArray<uint8_t> buf_l, buf_u;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto release = [&] {
      if (dl) sp.spsm_destroy(dl);
      if (du) sp.spsm_destroy(du);
      if (B) sp.destroy_dn(B);
      if (T) sp.destroy_dn(T);
      if (Y) sp.destroy_dn(Y);
      if (L) sp.destroy_sp(L);
      if (U) sp.destroy_sp(U);
      if (handle) sp.destroy(handle);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    };
    try {
      sp_check(sp.set_stream(handle, s), "cusparseSetStream");
      sp_check(sp.create_csr(&L, n, n, (int64_t)lv.size(), d_lp.get(), d_li.get(), d_lv.get(), CUSPARSE_INDEX_32I,
                             CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F),
               "cusparseCreateCsr");
      sp_check(sp.create_csr(&U, n, n, (int64_t)uv.size(), d_up.get(), d_ui.get(), d_uv.get(), CUSPARSE_INDEX_32I,
                             CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F),
               "cusparseCreateCsr");
      cusparseFillMode_t lower = CUSPARSE_FILL_MODE_LOWER, upper = CUSPARSE_FILL_MODE_UPPER;
      cusparseDiagType_t non_unit = CUSPARSE_DIAG_TYPE_NON_UNIT;
      sp_check(sp.set_attr(L, CUSPARSE_SPMAT_FILL_MODE, &lower, sizeof lower), "fill mode");
      sp_check(sp.set_attr(L, CUSPARSE_SPMAT_DIAG_TYPE, &non_unit, sizeof non_unit), "diag type");
      sp_check(sp.set_attr(U, CUSPARSE_SPMAT_FILL_MODE, &upper, sizeof upper), "fill mode");
      sp_check(sp.set_attr(U, CUSPARSE_SPMAT_DIAG_TYPE, &non_unit, sizeof non_unit), "diag type");
      sp_check(sp.create_dn(&B, n, width, n, d_b.get(), CUDA_R_64F, CUSPARSE_ORDER_COL), "cusparseCreateDnMat");
      sp_check(sp.create_dn(&T, n, width, n, d_t.get(), CUDA_R_64F, CUSPARSE_ORDER_COL), "cusparseCreateDnMat");
      sp_check(sp.create_dn(&Y, n, width, n, d_y.get(), CUDA_R_64F, CUSPARSE_ORDER_COL), "cusparseCreateDnMat");
      sp_check(sp.spsm_create(&dl), "cusparseSpSM_createDescr");
      sp_check(sp.spsm_create(&du), "cusparseSpSM_createDescr");
      const double one = 1.0;
      const auto op = CUSPARSE_OPERATION_NON_TRANSPOSE;
      size_t bl = 0, bu = 0;
      sp_check(sp.spsm_buffer(handle, op, op, &one, L, B, T, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, dl, &bl), "bufferSize");
      sp_check(sp.spsm_buffer(handle, op, op, &one, U, T, Y, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, du, &bu), "bufferSize");
      buf_l.reserve(std::max<size_t>(bl, 1)), buf_u.reserve(std::max<size_t>(bu, 1));
      sp_check(sp.spsm_analysis(handle, op, op, &one, L, B, T, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, dl, buf_l.get()),
               "analysis");
      sp_check(sp.spsm_analysis(handle, op, op, &one, U, T, Y, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, du, buf_u.get()),
               "analysis");
      cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
      cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
      cuda_check(cudaEventRecord(e0, s), "cudaEventRecord");
      const int64_t gb = ((int64_t)n * width + 255) / 256;
      for (int64_t c0 = 0; c0 < count; c0 += width) {
        const int64_t cols = std::min(width, count - c0);
        spsm_gather_kernel<<<(unsigned)gb, 256, 0, s>>>(d_rhs + c0 * ldb, ldb, cols, n, f->in_slot.get(), width, d_b.get());
        cuda_check(cudaGetLastError(), "spsm_gather_kernel launch");
        sp_check(sp.spsm_solve(handle, op, op, &one, L, B, T, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, dl), "SpSM lower");
        sp_check(sp.spsm_solve(handle, op, op, &one, U, T, Y, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, du), "SpSM upper");
        const int64_t gs = ((int64_t)n * cols + 255) / 256;
        spsm_scatter_kernel<<<(unsigned)gs, 256, 0, s>>>(d_y.get(), cols, n, f->out_slot.get(), d_out + c0 * ldx, ldx);
        cuda_check(cudaGetLastError(), "spsm_scatter_kernel launch");
      }
      cuda_check(cudaEventRecord(e1, s), "cudaEventRecord");
      cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
      float ms = 0;
      cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
      if (solve_ms) *solve_ms = ms;
    } catch (...) {
      cudaStreamSynchronize(s);
      release();
      throw;
    }
    release();
    return YB_OK;
  });
}
