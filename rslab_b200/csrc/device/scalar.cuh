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
  __device__ static double mag2(double x) { return __dmul_rn(x, x); }
  __host__ __device__ static double real(double x) { return x; }
  __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
  __device__ static double sub(double a, double b) { return __dsub_rn(a, b); }
  __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
  __host__ __device__ static double neg(double a) { return -a; }
  __device__ static double recip(double a) { return __ddiv_rn(1.0, a); }
  __host__ __device__ static bool is_zero(double a) { return a == 0.0; }
  __host__ __device__ static double conj(double a) { return a; }
  __device__ static double scale(double a, double s) { return __dmul_rn(a, s); }
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
  __device__ static double mag2(float x) { return __dmul_rn((double)x, (double)x); }
  __host__ __device__ static double real(float x) { return x; }
  __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
  __device__ static float sub(float a, float b) { return __fsub_rn(a, b); }
  __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
  __host__ __device__ static float neg(float a) { return -a; }
  __device__ static float recip(float a) { return __fdiv_rn(1.0f, a); }
  __host__ __device__ static bool is_zero(float a) { return a == 0.0f; }
  __host__ __device__ static float conj(float a) { return a; }
  __device__ static float scale(float a, double s) { return __fmul_rn(a, (float)s); }
  __device__ static float fnma(float a, float b, float c) { return fmaf(-a, b, c); }
  __device__ static float fma_(float a, float b, float c) { return fmaf(a, b, c); }
};

// Non-contracting real ops for the complex field (identical rounding to a
// host build with -ffp-contract=off).
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }

// |z| = m sqrt(1 + (s/m)^2), m = max(|re|,|im|), s = min: the scaled modulus,
// evaluated identically by the oracle so pivot comparisons agree bit for bit.
__device__ __forceinline__ double cmag(double re, double im) {
  double a = fabs(re), b = fabs(im);
  double m = fmax(a, b), s = fmin(a, b);
  if (m == 0.0) return 0.0;
  double r = __ddiv_rn(s, m);
  return __dmul_rn(m, sqrt(__dadd_rn(1.0, __dmul_rn(r, r))));
}

template <typename R>
struct FieldC {
  using T = cplx<R>;
  using Real = R;
  static constexpr bool complex = true;
  __host__ __device__ static T zero() { return T{0, 0}; }
  __host__ __device__ static T one() { return T{1, 0}; }
  __host__ __device__ static T from_real(double r) { return T{(R)r, 0}; }
  __device__ static double mag(T x) { return cmag((double)x.re, (double)x.im); }
  __device__ static double mag2(T x) {
    return __dadd_rn(__dmul_rn((double)x.re, (double)x.re), __dmul_rn((double)x.im, (double)x.im));
  }
  __host__ __device__ static double real(T x) { return (double)x.re; }
  __device__ static T add(T a, T b) { return T{radd(a.re, b.re), radd(a.im, b.im)}; }
  __device__ static T sub(T a, T b) { return T{rsub(a.re, b.re), rsub(a.im, b.im)}; }
  __device__ static T mul(T a, T b) {
    return T{rsub(rmul(a.re, b.re), rmul(a.im, b.im)), radd(rmul(a.re, b.im), rmul(a.im, b.re))};
  }
  __host__ __device__ static T neg(T a) { return T{-a.re, -a.im}; }
  __device__ static T recip(T a) {
    R ns = radd(rmul(a.re, a.re), rmul(a.im, a.im));
    return T{rdiv(a.re, ns), rdiv(-a.im, ns)};
  }
  __host__ __device__ static bool is_zero(T a) { return a.re == 0 && a.im == 0; }
  __host__ __device__ static T conj(T a) { return T{a.re, -a.im}; }
  __device__ static T scale(T a, double s) { return T{rmul(a.re, (R)s), rmul(a.im, (R)s)}; }
  // c - a*b and c + a*b with the fused form of the reference's complex
  // mul_add (src/scalar.rs:235-241): re = fma(a.re, b.re, fma(-a.im, b.im, c.re)).
  __device__ static T fnma(T a, T b, T c) { return fma_(T{-a.re, -a.im}, b, c); }
  __device__ static T fma_(T a, T b, T c) {
    return T{fma(a.re, b.re, fma(-a.im, b.im, c.re)), fma(a.re, b.im, fma(a.im, b.re, c.im))};
  }
};

template <> struct Field<c64> : FieldC<double> { using Lo = c32; };
template <> struct Field<c32> : FieldC<float> { using Lo = c32; };

}  // namespace rsd
