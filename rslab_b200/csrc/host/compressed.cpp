// CompressedLdltFactors (src/dense/ldlt_generic.rs:434-536): the factor in
// the reference LdltFactors layout with its CSC index arrays and pivot
// permutation stored as uint32 (half the index bytes of the int64 export),
// built from a device factor through rslab_export_factors, plus its
// single-right-hand-side solve on the host.  The solve uses the reference's
// expressions: forward y_i = fmadd(l, -y_j, y_i), the 1x1 / 2x2 D solve with
// det and recip, backward acc = acc - l * y_i (no fused multiply-add there),
// so it is bit-identical to the reference's solve_ldlt on the same factors.
// Like the reference container it solves with the factors of the
// equilibrated matrix (the scaling belongs to the solver object).
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/rslab_b200.h"
#include "host.hpp"

namespace rslab {
void set_last_error(const std::string& msg);
int64_t factor_dimension(const rslab_fac_handle* fac);
}

struct rslab_cfac_handle {
  int dtype = RSLAB_F64;
  int64_t n = 0;
  std::vector<uint32_t> col_ptr, row_idx, perm;
  std::vector<unsigned char> values, d, dsub;  // dtype elements
  std::vector<uint8_t> two;
};

namespace {

using rslab::RslabError;
using rslab::Status;

template <typename R>
struct Cx {
  R re, im;
};

// The reference's Scalar operations (src/scalar.rs): fmadd is the fused
// mul_add (complex: re = fma(a.re, b.re, fma(-a.im, b.im, c.re)), im =
// fma(a.re, b.im, fma(a.im, b.re, c.im))); every other product and sum is
// rounded on its own (the host sources are built with -ffp-contract=off).
template <typename R>
struct Ops {
  static R zero() { return R(0); }
  static R fmadd(R a, R b, R c) { return std::fma(a, b, c); }
  static R mul(R a, R b) { return a * b; }
  static R sub(R a, R b) { return a - b; }
  static R neg(R a) { return -a; }
  static bool is_zero(R a) { return a == R(0); }
  static R recip(R a) { return R(1) / a; }
};
template <typename R>
struct Ops<Cx<R>> {
  using T = Cx<R>;
  static T zero() { return {0, 0}; }
  static T fmadd(T a, T b, T c) {
    return {std::fma(a.re, b.re, std::fma(-a.im, b.im, c.re)), std::fma(a.re, b.im, std::fma(a.im, b.re, c.im))};
  }
  static T mul(T a, T b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
  static T sub(T a, T b) { return {a.re - b.re, a.im - b.im}; }
  static T neg(T a) { return {-a.re, -a.im}; }
  static bool is_zero(T a) { return a.re == 0 && a.im == 0; }
  static T recip(T a) {
    const R ns = a.re * a.re + a.im * a.im;
    return {a.re / ns, -a.im / ns};
  }
};

template <typename T>
int solve_compressed(const rslab_cfac_handle& C, const T* rhs, T* x) {
  using O = Ops<T>;
  const int64_t n = C.n;
  const T* lv = reinterpret_cast<const T*>(C.values.data());
  const T* dd = reinterpret_cast<const T*>(C.d.data());
  const T* ds = reinterpret_cast<const T*>(C.dsub.data());
  std::vector<T> y(n);
  for (int64_t i = 0; i < n; ++i) y[i] = rhs[C.perm[i]];
  for (int64_t j = 0; j < n; ++j) {
    const T nzj = O::sub(O::zero(), y[j]);
    for (uint32_t k = C.col_ptr[j] + 1; k < C.col_ptr[j + 1]; ++k) {
      const uint32_t i = C.row_idx[k];
      y[i] = O::fmadd(lv[k], nzj, y[i]);
    }
  }
  int64_t k = 0;
  while (k < n) {
    if (C.two[k]) {
      const T d11 = dd[k], d21 = ds[k], d22 = dd[k + 1];
      const T det = O::sub(O::mul(d11, d22), O::mul(d21, d21));
      if (O::is_zero(det)) return (int)Status::NumericallyRankDeficient;
      const T detinv = O::recip(det);
      const T z0 = y[k], z1 = y[k + 1];
      y[k] = O::mul(O::sub(O::mul(d22, z0), O::mul(d21, z1)), detinv);
      y[k + 1] = O::mul(O::sub(O::mul(d11, z1), O::mul(d21, z0)), detinv);
      k += 2;
    } else {
      if (O::is_zero(dd[k])) return (int)Status::NumericallyRankDeficient;
      y[k] = O::mul(y[k], O::recip(dd[k]));
      k += 1;
    }
  }
  for (int64_t j = n - 1; j >= 0; --j) {
    T acc = y[j];
    for (uint32_t q = C.col_ptr[j] + 1; q < C.col_ptr[j + 1]; ++q) acc = O::sub(acc, O::mul(lv[q], y[C.row_idx[q]]));
    y[j] = acc;
  }
  for (int64_t i = 0; i < n; ++i) x[C.perm[i]] = y[i];
  return 0;
}

size_t field_bytes(int dtype) { return dtype == RSLAB_C64 ? 16 : (dtype == RSLAB_F64 || dtype == RSLAB_C32) ? 8 : 4; }

int fail_c(const RslabError& e) {
  rslab::set_last_error(e.what());
  return (int)e.status;
}

}  // namespace

extern "C" {

int rslab_compress_factors(const rslab_fac_handle* fac, rslab_cfac_handle** out) {
  try {
    if (!fac || !out) throw RslabError(Status::InvalidInput, "null argument");
    *out = nullptr;
    rslab_factor_info_t info{};
    if (int rc = rslab_factor_info(fac, &info)) return rc;
    int64_t nnz = 0;
    if (int rc = rslab_export_factors(fac, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                      &nnz))
      return rc;
    auto C = std::make_unique<rslab_cfac_handle>();
    C->dtype = info.dtype;
    const size_t es = field_bytes(C->dtype);
    const int64_t n = rslab::factor_dimension(fac);
    if (n < 0) throw RslabError(Status::InvalidInput, "bad factor handle");
    if ((uint64_t)n > 0xffffffffull || (uint64_t)nnz > 0xffffffffull)
      throw RslabError(Status::InvalidInput,
                       "indices do not fit 32 bits (n = " + std::to_string(n) + ", nnz(L) = " + std::to_string(nnz) +
                           "): 32-bit compression does not apply");
    std::vector<int64_t> cp(n + 1), ri(std::max<int64_t>(nnz, 1)), pm(std::max<int64_t>(n, 1));
    C->n = n;
    C->values.resize(std::max<int64_t>(nnz, 1) * es);
    C->d.resize(std::max<int64_t>(n, 1) * es);
    C->dsub.resize(std::max<int64_t>(n, 1) * es);
    C->two.resize(std::max<int64_t>(n, 1));
    if (int rc = rslab_export_factors(fac, cp.data(), ri.data(), C->values.data(), C->d.data(), C->dsub.data(),
                                      C->two.data(), pm.data(), nullptr, nullptr))
      return rc;
    C->col_ptr.assign(cp.begin(), cp.end());
    C->row_idx.assign(ri.begin(), ri.begin() + nnz);
    C->perm.assign(pm.begin(), pm.begin() + n);
    C->values.resize(nnz * es);
    *out = C.release();
    return 0;
  } catch (const RslabError& e) {
    return fail_c(e);
  } catch (const std::exception& e) {
    return fail_c(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_cfac_info(const rslab_cfac_handle* c, int64_t* n, int64_t* nnz, int64_t* index_bytes, int32_t* dtype) {
  if (!c) return fail_c(RslabError(Status::InvalidInput, "null handle"));
  if (n) *n = c->n;
  if (nnz) *nnz = (int64_t)c->row_idx.size();
  if (index_bytes) *index_bytes = 4 * (int64_t)(c->col_ptr.size() + c->row_idx.size() + c->perm.size());
  if (dtype) *dtype = c->dtype;
  return 0;
}

int rslab_cfac_export(const rslab_cfac_handle* c, uint32_t* l_col_ptr, uint32_t* l_row_idx, void* l_values,
                      void* d_diag, void* d_subdiag, uint8_t* two_by_two, uint32_t* perm) {
  if (!c) return fail_c(RslabError(Status::InvalidInput, "null handle"));
  const size_t es = field_bytes(c->dtype);
  if (l_col_ptr) std::memcpy(l_col_ptr, c->col_ptr.data(), c->col_ptr.size() * 4);
  if (l_row_idx) std::memcpy(l_row_idx, c->row_idx.data(), c->row_idx.size() * 4);
  if (l_values) std::memcpy(l_values, c->values.data(), c->row_idx.size() * es);
  if (d_diag) std::memcpy(d_diag, c->d.data(), c->n * es);
  if (d_subdiag) std::memcpy(d_subdiag, c->dsub.data(), c->n * es);
  if (two_by_two) std::memcpy(two_by_two, c->two.data(), c->n);
  if (perm) std::memcpy(perm, c->perm.data(), c->perm.size() * 4);
  return 0;
}

int rslab_cfac_solve(const rslab_cfac_handle* c, const void* rhs, void* x) {
  if (!c || !rhs || !x) return fail_c(RslabError(Status::InvalidInput, "null argument"));
  int rc = 0;
  switch (c->dtype) {
    case RSLAB_F64: rc = solve_compressed<double>(*c, (const double*)rhs, (double*)x); break;
    case RSLAB_C64: rc = solve_compressed<Cx<double>>(*c, (const Cx<double>*)rhs, (Cx<double>*)x); break;
    case RSLAB_F32: rc = solve_compressed<float>(*c, (const float*)rhs, (float*)x); break;
    case RSLAB_C32: rc = solve_compressed<Cx<float>>(*c, (const Cx<float>*)rhs, (Cx<float>*)x); break;
    default: return fail_c(RslabError(Status::InvalidInput, "bad field"));
  }
  if (rc) rslab::set_last_error("numerically rank deficient pivot block");
  return rc;
}

void rslab_free_cfac(rslab_cfac_handle* c) { delete c; }

}  // extern "C"
