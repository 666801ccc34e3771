// A complex number for the kernels: re and im of type R (float for complex64, double for
// complex128), with the textbook multiply (no fused multiply-add across the real and imaginary
// parts is implied by the type; the compiler may contract each part's products and sums).
#pragma once

#include <cuda_runtime.h>

#include <complex>

namespace yb {

template <class R> struct cplx {
  R re, im;
  __host__ __device__ constexpr cplx() : re(0), im(0) {}
  __host__ __device__ constexpr cplx(R r) : re(r), im(0) {}
  __host__ __device__ constexpr cplx(R r, R i) : re(r), im(i) {}
  template <class S> __host__ __device__ explicit constexpr cplx(const cplx<S> &o) : re((R)o.re), im((R)o.im) {}
  __host__ __device__ cplx &operator+=(const cplx &o) {
    re += o.re, im += o.im;
    return *this;
  }
  __host__ __device__ cplx &operator-=(const cplx &o) {
    re -= o.re, im -= o.im;
    return *this;
  }
  __host__ __device__ cplx &operator*=(const cplx &o) {
    const R r = re * o.re - im * o.im, i = re * o.im + im * o.re;
    re = r, im = i;
    return *this;
  }
};

template <class R> __host__ __device__ inline cplx<R> operator+(cplx<R> a, const cplx<R> &b) { return a += b; }
template <class R> __host__ __device__ inline cplx<R> operator-(cplx<R> a, const cplx<R> &b) { return a -= b; }
template <class R> __host__ __device__ inline cplx<R> operator*(cplx<R> a, const cplx<R> &b) { return a *= b; }
template <class R> __host__ __device__ inline bool operator==(const cplx<R> &a, const cplx<R> &b) {
  return a.re == b.re && a.im == b.im;
}
template <class R> __host__ __device__ inline bool operator!=(const cplx<R> &a, const cplx<R> &b) { return !(a == b); }

// |z| without overflow for the magnitudes a residual takes
template <class R> __device__ inline double magnitude(const cplx<R> &z) { return hypot((double)z.re, (double)z.im); }

template <class R> inline cplx<R> from_std(const std::complex<double> &z) { return cplx<R>((R)z.real(), (R)z.imag()); }

}  // namespace yb
