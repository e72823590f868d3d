// Shared device types for the FDTD kernels: real/complex field scalars, launch helpers, error checks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lsfdtd {

// A complex field value laid out as (re, im), the layout of torch.complex64 / complex128 and of
// std::complex, so field tensors are passed straight through. Aligned to its size (as those tensors are),
// so that a value moves in one 8- or 16-byte access instead of two.
template <typename R>
struct alignas(2 * sizeof(R)) cplx {
  R re, im;
};

template <typename F> struct real_of { using type = F; };
template <typename R> struct real_of<cplx<R>> { using type = R; };
template <typename F> struct is_cplx { static constexpr bool value = false; };
template <typename R> struct is_cplx<cplx<R>> { static constexpr bool value = true; };

template <typename R> __host__ __device__ __forceinline__ cplx<R> operator+(cplx<R> a, cplx<R> b) {
  return {a.re + b.re, a.im + b.im};
}
template <typename R> __host__ __device__ __forceinline__ cplx<R> operator-(cplx<R> a, cplx<R> b) {
  return {a.re - b.re, a.im - b.im};
}
template <typename R> __host__ __device__ __forceinline__ cplx<R> operator*(cplx<R> a, R s) {
  return {a.re * s, a.im * s};
}
template <typename R> __host__ __device__ __forceinline__ cplx<R> operator*(R s, cplx<R> a) {
  return {s * a.re, s * a.im};
}
template <typename R> __host__ __device__ __forceinline__ cplx<R> operator*(cplx<R> a, cplx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R> __host__ __device__ __forceinline__ cplx<R>& operator+=(cplx<R>& a, cplx<R> b) {
  a = a + b;
  return a;
}
template <typename R> __host__ __device__ __forceinline__ cplx<R>& operator-=(cplx<R>& a, cplx<R> b) {
  a = a - b;
  return a;
}

template <typename F> __host__ __device__ __forceinline__ F zero() { return F(0); }
template <> __host__ __device__ __forceinline__ cplx<float> zero<cplx<float>>() { return {0.f, 0.f}; }
template <> __host__ __device__ __forceinline__ cplx<double> zero<cplx<double>>() { return {0.0, 0.0}; }

// |v|^2 in double, for the monitor energy
__device__ __forceinline__ double norm2(float v) { return (double)v * (double)v; }
__device__ __forceinline__ double norm2(double v) { return v * v; }
template <typename R> __device__ __forceinline__ double norm2(cplx<R> v) {
  return (double)v.re * (double)v.re + (double)v.im * (double)v.im;
}

// field value as complex<double> (DFT accumulation is in double)
__device__ __forceinline__ cplx<double> to_c64(float v) { return {(double)v, 0.0}; }
__device__ __forceinline__ cplx<double> to_c64(double v) { return {v, 0.0}; }
template <typename R> __device__ __forceinline__ cplx<double> to_c64(cplx<R> v) {
  return {(double)v.re, (double)v.im};
}

// a complex phase (re, im) stored in double, applied to a field value (real fields never see a phase)
template <typename F> __device__ __forceinline__ F apply_phase(F v, double re, double im);
template <> __device__ __forceinline__ float apply_phase<float>(float v, double, double) { return v; }
template <> __device__ __forceinline__ double apply_phase<double>(double v, double, double) { return v; }
template <> __device__ __forceinline__ cplx<float> apply_phase<cplx<float>>(cplx<float> v, double re, double im) {
  return v * cplx<float>{(float)re, (float)im};
}
template <> __device__ __forceinline__ cplx<double> apply_phase<cplx<double>>(cplx<double> v, double re, double im) {
  return v * cplx<double>{re, im};
}

// Loads through the read-only data path, for arrays no thread writes during the kernel (lets the compiler
// issue them ahead of the kernel's stores), and stores marked global (no false dependence on shared memory)
__device__ __forceinline__ float ro(const float* p) { return __ldg(p); }
__device__ __forceinline__ double ro(const double* p) { return __ldg(p); }
__device__ __forceinline__ cplx<float> ro(const cplx<float>* p) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  return {v.x, v.y};
}
__device__ __forceinline__ cplx<double> ro(const cplx<double>* p) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return {v.x, v.y};
}
__device__ __forceinline__ void st_global(float* p, float v) { __stcg(p, v); }
__device__ __forceinline__ void st_global(double* p, double v) { __stcg(p, v); }
__device__ __forceinline__ void st_global(cplx<float>* p, cplx<float> v) {
  __stcg(reinterpret_cast<float2*>(p), make_float2(v.re, v.im));
}
__device__ __forceinline__ void st_global(cplx<double>* p, cplx<double> v) {
  __stcg(reinterpret_cast<double2*>(p), make_double2(v.re, v.im));
}

inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace lsfdtd
