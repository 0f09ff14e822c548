// Shared device/host helpers for the QSM CUDA library: complex arithmetic,
// compile-time trigonometry for codelet twiddles, and error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace qsm {

// ---------------------------------------------------------------------------
// Complex types: float2 / double2 carry (re, im).
// ---------------------------------------------------------------------------
template <typename T> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename T> using cplx_t = typename CplxOf<T>::type;

template <typename C> __host__ __device__ __forceinline__ C mk(decltype(C::x) re, decltype(C::x) im) {
  C c; c.x = re; c.y = im; return c;
}
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
  return mk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __host__ __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mk<C>(a.x * s, a.y * s); }
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
// multiply by +i / -i
template <typename C> __host__ __device__ __forceinline__ C cmul_i(C a) { return mk<C>(-a.y, a.x); }
template <typename C> __host__ __device__ __forceinline__ C cmul_mi(C a) { return mk<C>(a.y, -a.x); }

// ---------------------------------------------------------------------------
// Compile-time sin/cos of 2*pi*p/q (Taylor series on an octant-reduced angle).
// Used for codelet constants and, evaluated at run time on the host, for the
// per-length twiddle tables.
// ---------------------------------------------------------------------------
constexpr double kPi = 3.141592653589793238462643383279502884;

__host__ __device__ constexpr double taylor_sin(double x) {
  double x2 = x * x, term = x, sum = x;
  for (int k = 1; k < 14; ++k) {
    term *= -x2 / (double)((2 * k) * (2 * k + 1));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double taylor_cos(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int k = 1; k < 14; ++k) {
    term *= -x2 / (double)((2 * k - 1) * (2 * k));
    sum += term;
  }
  return sum;
}
// cos(2*pi*p/q)
__host__ __device__ constexpr double cos2pi(long long p, long long q) {
  p %= q; if (p < 0) p += q;
  long long p8 = 8 * p, o = p8 / q, r = p8 - o * q;
  // angle = (pi/4)*(o + r/q); map to quadrant m and signed residual psi
  long long m = 0; double psi = 0.0;
  if ((o & 1) == 0) { m = o / 2; psi = (kPi / 4.0) * (double)r / (double)q; }
  else { m = (o + 1) / 2; psi = -(kPi / 4.0) * (double)(q - r) / (double)q; }
  double c = taylor_cos(psi), s = taylor_sin(psi);
  switch (m & 3) {
    case 0: return c;
    case 1: return -s;
    case 2: return -c;
    default: return s;
  }
}
// sin(2*pi*p/q)
__host__ __device__ constexpr double sin2pi(long long p, long long q) {
  p %= q; if (p < 0) p += q;
  long long p8 = 8 * p, o = p8 / q, r = p8 - o * q;
  long long m = 0; double psi = 0.0;
  if ((o & 1) == 0) { m = o / 2; psi = (kPi / 4.0) * (double)r / (double)q; }
  else { m = (o + 1) / 2; psi = -(kPi / 4.0) * (double)(q - r) / (double)q; }
  double c = taylor_cos(psi), s = taylor_sin(psi);
  switch (m & 3) {
    case 0: return s;
    case 1: return c;
    case 2: return -s;
    default: return -c;
  }
}

// soft threshold, src/utils/mod.rs:44-56
template <typename T> __host__ __device__ __forceinline__ T shrink(T x, T t) {
  return x > t ? x - t : (x < -t ? x + t : T(0));
}

__host__ __device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }

}  // namespace qsm
