// Device memory, error checking and the per-factor device state shared by the CUDA translation
// units of libybgpu.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "host/sparse.hpp"
#include "plan.hpp"

namespace yb {

inline void cuda_check(cudaError_t err, const char *what) {
  if (err != cudaSuccess)
    throw host::Error(host::kCuda, std::string(what) + ": " + cudaGetErrorString(err));
}

// Owns a device allocation of `count` elements of T.
template <class T> class DeviceArray {
 public:
  DeviceArray() = default;
  explicit DeviceArray(size_t count) { resize(count); }
  ~DeviceArray() { release(); }
  DeviceArray(const DeviceArray &) = delete;
  DeviceArray &operator=(const DeviceArray &) = delete;
  DeviceArray(DeviceArray &&o) noexcept : ptr_(o.ptr_), count_(o.count_) { o.ptr_ = nullptr, o.count_ = 0; }
  DeviceArray &operator=(DeviceArray &&o) noexcept {
    if (this != &o) {
      release();
      ptr_ = o.ptr_, count_ = o.count_;
      o.ptr_ = nullptr, o.count_ = 0;
    }
    return *this;
  }
  void resize(size_t count) {
    if (count == count_) return;
    release();
    if (count) cuda_check(cudaMalloc(&ptr_, count * sizeof(T)), "cudaMalloc");
    count_ = count;
  }
  // Grows (never shrinks) to at least `count` elements; the contents are not kept.
  void reserve(size_t count) {
    if (count > count_) resize(count);
  }
  void upload(const std::vector<T> &host, cudaStream_t stream) {
    resize(host.size());
    if (!host.empty())
      cuda_check(cudaMemcpyAsync(ptr_, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, stream),
                 "cudaMemcpyAsync upload");
  }
  T *get() const { return ptr_; }
  size_t size() const { return count_; }

 private:
  void release() {
    if (ptr_) cudaFree(ptr_);
    ptr_ = nullptr;
    count_ = 0;
  }
  T *ptr_ = nullptr;
  size_t count_ = 0;
};

// Page-locked host memory, grown as needed (ybus_cuda/src/factor.rs:63-89 keeps the same kind of
// staging for its copies).
class PinnedBuffer {
 public:
  ~PinnedBuffer() {
    if (ptr_) cudaFreeHost(ptr_);
  }
  void *get(size_t bytes) {
    if (bytes > bytes_) {
      if (ptr_) cudaFreeHost(ptr_);
      ptr_ = nullptr;
      bytes_ = 0;
      cuda_check(cudaHostAlloc(&ptr_, bytes, cudaHostAllocDefault), "cudaHostAlloc");
      bytes_ = bytes;
    }
    return ptr_;
  }

 private:
  void *ptr_ = nullptr;
  size_t bytes_ = 0;
};

// One sweep of a factor on the device, at value type T.
template <class T> struct DeviceSweep {
  int32_t levels = 0, widest = 0, n = 0;
  int64_t entries = 0;
  DeviceArray<int32_t> level_ptr, row, ptr, col;
  DeviceArray<T> val, dinv;
  std::vector<int32_t> host_level_ptr;
};

// The view of a sweep a kernel takes by value.
template <class T> struct SweepView {
  int32_t levels;
  const int32_t *__restrict__ level_ptr;
  const int32_t *__restrict__ row;
  const int32_t *__restrict__ ptr;
  const int32_t *__restrict__ col;
  const T *__restrict__ val;
  const T *__restrict__ dinv;
};

template <class T> SweepView<T> view(const DeviceSweep<T> &s) {
  return SweepView<T>{s.levels, s.level_ptr.get(), s.row.get(), s.ptr.get(), s.col.get(), s.val.get(), s.dinv.get()};
}

template <class Dst, class Src> std::vector<Dst> convert(const std::vector<Src> &v) {
  std::vector<Dst> out(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = (Dst)v[i];
  return out;
}

template <class T, class S> void upload_sweep(DeviceSweep<T> &d, const Sweep<S> &s, int32_t n, cudaStream_t stream) {
  d.levels = s.levels;
  d.widest = s.widest;
  d.n = n;
  d.entries = s.entries();
  d.host_level_ptr = s.level_ptr;
  d.level_ptr.upload(s.level_ptr, stream);
  d.row.upload(s.row, stream);
  d.ptr.upload(s.ptr, stream);
  d.col.upload(s.col, stream);
  d.val.upload(convert<T>(s.val), stream);
  d.dinv.upload(convert<T>(s.dinv), stream);
}

}  // namespace yb
