// For comparison only, built as its own library (libybcompare.so) that no solve of libybgpu.so
// loads: ybus_cuda's own route to the solve (ybus_cuda/src/sparse.rs:371-420, factor.rs:234-289:
// the two triangles of a Cholesky factor as CSR matrices, cuSPARSE SpSM lower then upper on blocks
// of `width` right-hand sides, the last block padded with zeros), on device arrays as
// yb_solve_many_device takes them, so a bench can time it beside the library's solves on one GPU.
// cuSPARSE is opened with dlopen on the first call.
//
//   int32_t ybc_spsm_solve(int64_t n, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
//                          const int64_t *lt_ptr, const int64_t *lt_idx, const double *lt_val,
//                          const int64_t *perm, const double *d_rhs, int64_t ldb, double *d_out, int64_t ldx,
//                          int64_t count, int64_t width, double *solve_ms, char *message, size_t length);
//
// L (CSR, each row's diagonal last) and L' (CSR, diagonal first) of P A P' = L L', perm = P (row i
// of P A P' is row perm[i] of A), host arrays; right-hand sides and solutions column-major in A's
// order on the device. solve_ms receives the time of the solves, their analysis excluded. Returns
// 0, or 1 with a message.
#include <cuda_runtime.h>
#include <cusparse.h>
#include <dlfcn.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

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
  if (!ok) throw std::runtime_error("cuSPARSE could not be opened");
  return s;
}

void sp_check(cusparseStatus_t st, const char *what) {
  if (st != CUSPARSE_STATUS_SUCCESS) throw std::runtime_error(std::string(what) + ": cuSPARSE status " + std::to_string((int)st));
}
void cu_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// A device array freed on scope exit.
template <class T> struct Buffer {
  T *p = nullptr;
  explicit Buffer(size_t count) { cu_check(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)), "cudaMalloc"); }
  Buffer(const std::vector<T> &v, cudaStream_t s) : Buffer(v.size()) {
    cu_check(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
  }
  ~Buffer() { cudaFree(p); }
  Buffer(const Buffer &) = delete;
  Buffer &operator=(const Buffer &) = delete;
};

// b's columns permuted (row i of P b is b's row perm[i]), zero past `cols`; and y back into x
__global__ void gather_kernel(const double *__restrict__ b, int64_t ldb, int64_t cols, int32_t n,
                              const int32_t *__restrict__ perm, int64_t width, double *__restrict__ out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)n * width) return;
  const int64_t c = k / n, i = k - c * n;
  out[c * n + i] = c < cols ? b[c * ldb + perm[i]] : 0.0;
}
__global__ void scatter_kernel(const double *__restrict__ y, int64_t cols, int32_t n, const int32_t *__restrict__ perm,
                               double *__restrict__ x, int64_t ldx) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (int64_t)n * cols) return;
  const int64_t c = k / n, i = k - c * n;
  x[c * ldx + perm[i]] = y[c * n + i];
}

std::vector<int32_t> narrow(const int64_t *v, size_t count) {
  std::vector<int32_t> out(count);
  for (size_t i = 0; i < count; ++i) {
    if (v[i] < 0 || v[i] > INT32_MAX) throw std::runtime_error("an index does not fit 32 bits");
    out[i] = (int32_t)v[i];
  }
  return out;
}

}  // namespace

extern "C" int32_t ybc_spsm_solve(int64_t n64, const int64_t *l_ptr, const int64_t *l_idx, const double *l_val,
                                  const int64_t *lt_ptr, const int64_t *lt_idx, const double *lt_val,
                                  const int64_t *perm, const double *d_rhs, int64_t ldb, double *d_out, int64_t ldx,
                                  int64_t count, int64_t width, double *solve_ms, char *message, size_t length) {
  cusparseHandle_t handle = nullptr;
  cusparseSpMatDescr_t L = nullptr, U = nullptr;
  cusparseDnMatDescr_t B = nullptr, T = nullptr, Y = nullptr;
  cusparseSpSMDescr_t dl = nullptr, du = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStream_t s = nullptr;
  const Sparse *sp = nullptr;
  auto release = [&] {
    if (sp) {
      if (dl) sp->spsm_destroy(dl);
      if (du) sp->spsm_destroy(du);
      if (B) sp->destroy_dn(B);
      if (T) sp->destroy_dn(T);
      if (Y) sp->destroy_dn(Y);
      if (L) sp->destroy_sp(L);
      if (U) sp->destroy_sp(U);
      if (handle) sp->destroy(handle);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
  };
  try {
    if (n64 < 1 || n64 > INT32_MAX || count < 1 || width < 1 || !l_ptr || !lt_ptr || !perm || !d_rhs || !d_out ||
        ldb < n64 || ldx < n64)
      throw std::runtime_error("bad argument");
    const int32_t n = (int32_t)n64;
    sp = &sparse();
    cu_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    const std::vector<int32_t> lp = narrow(l_ptr, n + 1), li = narrow(l_idx, l_ptr[n]);
    const std::vector<int32_t> up = narrow(lt_ptr, n + 1), ui = narrow(lt_idx, lt_ptr[n]);
    const std::vector<double> lv(l_val, l_val + l_ptr[n]), uv(lt_val, lt_val + lt_ptr[n]);
    const std::vector<int32_t> pm = narrow(perm, n);
    Buffer<int32_t> d_lp(lp, s), d_li(li, s), d_up(up, s), d_ui(ui, s), d_perm(pm, s);
    Buffer<double> d_lv(lv, s), d_uv(uv, s), d_b((size_t)n * width), d_t((size_t)n * width), d_y((size_t)n * width);
    sp_check(sp->create(&handle), "cusparseCreate");
    sp_check(sp->set_stream(handle, s), "cusparseSetStream");
    sp_check(sp->create_csr(&L, n, n, (int64_t)lv.size(), d_lp.p, d_li.p, d_lv.p, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                            CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F),
             "cusparseCreateCsr");
    sp_check(sp->create_csr(&U, n, n, (int64_t)uv.size(), d_up.p, d_ui.p, d_uv.p, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                            CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F),
             "cusparseCreateCsr");
    cusparseFillMode_t lower = CUSPARSE_FILL_MODE_LOWER, upper = CUSPARSE_FILL_MODE_UPPER;
    cusparseDiagType_t non_unit = CUSPARSE_DIAG_TYPE_NON_UNIT;
    sp_check(sp->set_attr(L, CUSPARSE_SPMAT_FILL_MODE, &lower, sizeof lower), "fill mode");
    sp_check(sp->set_attr(L, CUSPARSE_SPMAT_DIAG_TYPE, &non_unit, sizeof non_unit), "diag type");
    sp_check(sp->set_attr(U, CUSPARSE_SPMAT_FILL_MODE, &upper, sizeof upper), "fill mode");
    sp_check(sp->set_attr(U, CUSPARSE_SPMAT_DIAG_TYPE, &non_unit, sizeof non_unit), "diag type");
    sp_check(sp->create_dn(&B, n, width, n, d_b.p, CUDA_R_64F, CUSPARSE_ORDER_COL), "cusparseCreateDnMat");
    sp_check(sp->create_dn(&T, n, width, n, d_t.p, CUDA_R_64F, CUSPARSE_ORDER_COL), "cusparseCreateDnMat");
    sp_check(sp->create_dn(&Y, n, width, n, d_y.p, CUDA_R_64F, CUSPARSE_ORDER_COL), "cusparseCreateDnMat");
    sp_check(sp->spsm_create(&dl), "cusparseSpSM_createDescr");
    sp_check(sp->spsm_create(&du), "cusparseSpSM_createDescr");
    const double one = 1.0;
    const auto op = CUSPARSE_OPERATION_NON_TRANSPOSE;
    size_t bl = 0, bu = 0;
    sp_check(sp->spsm_buffer(handle, op, op, &one, L, B, T, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, dl, &bl), "bufferSize");
    sp_check(sp->spsm_buffer(handle, op, op, &one, U, T, Y, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, du, &bu), "bufferSize");
    Buffer<uint8_t> buf_l(bl), buf_u(bu);
    sp_check(sp->spsm_analysis(handle, op, op, &one, L, B, T, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, dl, buf_l.p), "analysis");
    sp_check(sp->spsm_analysis(handle, op, op, &one, U, T, Y, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, du, buf_u.p), "analysis");
    cu_check(cudaEventCreate(&e0), "cudaEventCreate");
    cu_check(cudaEventCreate(&e1), "cudaEventCreate");
    cu_check(cudaEventRecord(e0, s), "cudaEventRecord");
    const int64_t gb = ((int64_t)n * width + 255) / 256;
    for (int64_t c0 = 0; c0 < count; c0 += width) {
      const int64_t cols = std::min(width, count - c0);
      gather_kernel<<<(unsigned)gb, 256, 0, s>>>(d_rhs + c0 * ldb, ldb, cols, n, d_perm.p, width, d_b.p);
      cu_check(cudaGetLastError(), "gather launch");
      sp_check(sp->spsm_solve(handle, op, op, &one, L, B, T, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, dl), "SpSM lower");
      sp_check(sp->spsm_solve(handle, op, op, &one, U, T, Y, CUDA_R_64F, CUSPARSE_SPSM_ALG_DEFAULT, du), "SpSM upper");
      const int64_t gs = ((int64_t)n * cols + 255) / 256;
      scatter_kernel<<<(unsigned)gs, 256, 0, s>>>(d_y.p, cols, n, d_perm.p, d_out + c0 * ldx, ldx);
      cu_check(cudaGetLastError(), "scatter launch");
    }
    cu_check(cudaEventRecord(e1, s), "cudaEventRecord");
    cu_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0;
    cu_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    if (solve_ms) *solve_ms = ms;
    cu_check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  } catch (const std::exception &e) {
    if (s) cudaStreamSynchronize(s);
    release();
    if (message && length) {
      const size_t c = std::min(length - 1, std::strlen(e.what()));
      std::memcpy(message, e.what(), c);
      message[c] = '\0';
    }
    return 1;
  }
  release();
  return 0;
}
