// Scalar field abstraction shared by every kernel of the LDL^T path: real
// f64/f32 and complex-symmetric c64/c32 (A = A^T, no conjugation in the
// factor).  Semantics follow the reference Scalar trait (src/scalar.rs:25-251):
// pivot magnitudes are compared in f64, |z| = hypot(re, im), 1/z =
// conj(z)/|z|^2, and complex products are the plain 4-multiply form.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rsd {

template <typename R>
struct cplx {
  R re, im;
};

using c64 = cplx<double>;
using c32 = cplx<float>;

template <typename T> struct Field;

template <>
struct Field<double> {
  using Real = double;
  using Lo = float;
  static constexpr bool complex = false;
  __host__ __device__ static double zero() { return 0.0; }
  __host__ __device__ static double one() { return 1.0; }
  __host__ __device__ static double from_real(double r) { return r; }
  __host__ __device__ static double mag(double x) { return fabs(x); }
  __host__ __device__ static double mag2(double x) { return x * x; }
  __host__ __device__ static double real(double x) { return x; }
  __host__ __device__ static double add(double a, double b) { return a + b; }
  __host__ __device__ static double sub(double a, double b) { return a - b; }
  __host__ __device__ static double mul(double a, double b) { return a * b; }
  __host__ __device__ static double neg(double a) { return -a; }
  __host__ __device__ static double recip(double a) { return 1.0 / a; }
  __host__ __device__ static bool is_zero(double a) { return a == 0.0; }
  __host__ __device__ static double conj(double a) { return a; }
  __host__ __device__ static double scale(double a, double s) { return a * s; }
  // c - a*b
  __device__ static double fnma(double a, double b, double c) { return fma(-a, b, c); }
  __device__ static double fma_(double a, double b, double c) { return fma(a, b, c); }
};

template <>
struct Field<float> {
  using Real = float;
  using Lo = float;
  static constexpr bool complex = false;
  __host__ __device__ static float zero() { return 0.0f; }
  __host__ __device__ static float one() { return 1.0f; }
  __host__ __device__ static float from_real(double r) { return (float)r; }
  __host__ __device__ static double mag(float x) { return (double)fabsf(x); }
  __host__ __device__ static double mag2(float x) { return (double)x * (double)x; }
  __host__ __device__ static double real(float x) { return x; }
  __host__ __device__ static float add(float a, float b) { return a + b; }
  __host__ __device__ static float sub(float a, float b) { return a - b; }
  __host__ __device__ static float mul(float a, float b) { return a * b; }
  __host__ __device__ static float neg(float a) { return -a; }
  __host__ __device__ static float recip(float a) { return 1.0f / a; }
  __host__ __device__ static bool is_zero(float a) { return a == 0.0f; }
  __host__ __device__ static float conj(float a) { return a; }
  __host__ __device__ static float scale(float a, double s) { return a * (float)s; }
  __device__ static float fnma(float a, float b, float c) { return fmaf(-a, b, c); }
  __device__ static float fma_(float a, float b, float c) { return fmaf(a, b, c); }
};

template <typename R>
struct FieldC {
  using T = cplx<R>;
  using Real = R;
  static constexpr bool complex = true;
  __host__ __device__ static T zero() { return T{0, 0}; }
  __host__ __device__ static T one() { return T{1, 0}; }
  __host__ __device__ static T from_real(double r) { return T{(R)r, 0}; }
  __host__ __device__ static double mag(T x) { return (double)hypot((double)x.re, (double)x.im); }
  __host__ __device__ static double mag2(T x) { return (double)x.re * (double)x.re + (double)x.im * (double)x.im; }
  __host__ __device__ static double real(T x) { return (double)x.re; }
  __host__ __device__ static T add(T a, T b) { return T{a.re + b.re, a.im + b.im}; }
  __host__ __device__ static T sub(T a, T b) { return T{a.re - b.re, a.im - b.im}; }
  __host__ __device__ static T mul(T a, T b) { return T{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
  __host__ __device__ static T neg(T a) { return T{-a.re, -a.im}; }
  __host__ __device__ static T recip(T a) {
    R ns = a.re * a.re + a.im * a.im;
    return T{a.re / ns, -a.im / ns};
  }
  __host__ __device__ static bool is_zero(T a) { return a.re == 0 && a.im == 0; }
  __host__ __device__ static T conj(T a) { return T{a.re, -a.im}; }
  __host__ __device__ static T scale(T a, double s) { return T{a.re * (R)s, a.im * (R)s}; }
  __device__ static T fnma(T a, T b, T c) {
    return T{c.re - a.re * b.re + a.im * b.im, c.im - a.re * b.im - a.im * b.re};
  }
  __device__ static T fma_(T a, T b, T c) {
    return T{c.re + a.re * b.re - a.im * b.im, c.im + a.re * b.im + a.im * b.re};
  }
};

template <> struct Field<c64> : FieldC<double> { using Lo = c32; };
template <> struct Field<c32> : FieldC<float> { using Lo = c32; };

// Magnitude of the f32 magnitude types follows the reference: computed in
// the field's own precision, compared in f64.
template <typename T>
__device__ __forceinline__ T ld_global(const T* p) {
  return *p;
}

}  // namespace rsd
