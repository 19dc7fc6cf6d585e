// ORACLE — test infrastructure only.  Never linked into, or called by, the
// rslab_b200 product; only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load it, as the checker / reported CPU baseline.
//
// A plain C++ restatement of the reference CPU numeric path (Rust, not
// buildable here: no cargo/rustc in the image), function by function:
//   onepass_scale / apply_symmetric_scaling   src/numeric/sparse_solver.rs:380-421
//   inv_sqrt_scale_guarded                    src/scaling/mod.rs:85-96
//   factor_left_looking (A_perm, row structures, update lists)
//                                             src/numeric/multifrontal_ldlt.rs:3346-3401, 2121-2152
//   ll_factor_node (assembly + cmod)          src/numeric/multifrontal_ldlt.rs:2400-2728
//   ll_cdiv_emit (blocked panel-bounded BK)   src/numeric/multifrontal_ldlt.rs:2759-3256
//   apply_bk_panel_trailing (deep-row replay) src/numeric/multifrontal_ldlt.rs:1347-1408
//   swap_sym_lower_bounded / bk_alpha         src/dense/ldlt_generic.rs:70-110
//   ldlt_emit_and_free + final concatenation  src/numeric/multifrontal_ldlt.rs:2328-2388, 3535-3575
//   solve_ldlt_block / LdltSolver::solve_many src/dense/ldlt_generic.rs:618-714, sparse_solver.rs:302-325
//   CscMatrix::symv                           src/sparse/csc.rs:294-308
//   sym_norm_inf, refine_ladder, MixedLdltSolver::solve_to
//                                             src/numeric/mixed.rs:140-221, 258-291, 358-371
//   gmres (FGMRES, MGS + DGKS, Givens)        src/numeric/iterative.rs:587-666, 822-1037
// The symbolic structure (sym.perm, supernode ranges, children) is an input:
// it comes from the product's host analysis, whose ordering is pinned by the
// reference's AMD golden permutations; the oracle rebuilds A_perm, the row
// structures and the update lists itself.
//
// Complex arithmetic follows num-complex 0.4.6 (plain mul, inv = conj/|z|^2,
// norm = hypot).  The reference's Schur GEMMs run in the `gemm` crate 0.18.2
// whose per-element rounding is shape dependent; the oracle computes the same
// products with plain loops, so GEMM-level results agree to rounding only.
// Timing mode (oracle_set_parallel): the same factor with the two Schur
// products (cmod and the deferred in-panel update) computed by a BLAS GEMM
// (OpenBLAS, loaded at run time) and the assembly forest scheduled level by
// level with independent supernodes on different threads, as the reference
// runs sibling subtrees concurrently on rayon and its GEMMs in the gemm crate
// (multifrontal_ldlt.rs:847-866, 3264-3297).  Its results equal the exact
// mode's to rounding (the GEMM summation order differs); it is the timed CPU
// baseline, the exact mode is the checker.
// Build: oracle/build_oracle.sh (g++ -O2 -ffp-contract=off -fopenmp).
#include <dlfcn.h>
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

namespace orc {

template <typename R>
struct Cx {
  R re, im;
  Cx() : re(0), im(0) {}
  Cx(R r, R i = 0) : re(r), im(i) {}
};
template <typename R> inline Cx<R> operator+(Cx<R> a, Cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R> inline Cx<R> operator-(Cx<R> a, Cx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R> inline Cx<R> operator-(Cx<R> a) { return {-a.re, -a.im}; }
template <typename R> inline Cx<R> operator*(Cx<R> a, Cx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R> inline bool operator==(Cx<R> a, Cx<R> b) { return a.re == b.re && a.im == b.im; }
template <typename R> inline bool operator!=(Cx<R> a, Cx<R> b) { return !(a == b); }

// Scalar traits (src/scalar.rs:25-251).
template <typename T> struct S;
template <> struct S<double> {
  using Lo = float;
  static constexpr double EPS = 2.220446049250313e-16;
  static double zero() { return 0; }
  static double one() { return 1; }
  static double from_real(double r) { return r; }
  static double mag(double x) { return std::fabs(x); }
  static double mag2(double x) { return x * x; }
  static double real(double x) { return x; }
  static double conj(double x) { return x; }
  static double recip(double x) { return 1.0 / x; }
  static double fmadd(double a, double b, double c) { return std::fma(a, b, c); }
  static float demote(double x) { return (float)x; }
};
template <> struct S<float> {
  using Lo = float;
  static constexpr double EPS = 1.1920928955078125e-07;
  static float zero() { return 0; }
  static float one() { return 1; }
  static float from_real(double r) { return (float)r; }
  static double mag(float x) { return std::fabs((double)x); }
  static double mag2(float x) { return (double)x * (double)x; }
  static double real(float x) { return x; }
  static float conj(float x) { return x; }
  static float recip(float x) { return 1.0f / x; }
  static float fmadd(float a, float b, float c) { return std::fma(a, b, c); }
  static float demote(float x) { return x; }
};
template <typename R> struct SC {
  using T = Cx<R>;
  static T zero() { return T(0, 0); }
  static T one() { return T(1, 0); }
  static T from_real(double r) { return T((R)r, 0); }
  // |z| = m sqrt(1 + (s/m)^2) with m = max(|re|,|im|), s = min: the scaled
  // modulus (the reference's hypot, up to its last-ulp rounding).
  static double mag(T x) {
    double a = std::fabs((double)x.re), b = std::fabs((double)x.im);
    double m = std::max(a, b), s = std::min(a, b);
    if (m == 0.0) return 0.0;
    double r = s / m;
    return m * std::sqrt(1.0 + r * r);
  }
  static double mag2(T x) { return (double)x.re * (double)x.re + (double)x.im * (double)x.im; }
  static double real(T x) { return x.re; }
  static T conj(T x) { return T(x.re, -x.im); }
  static T recip(T x) {
    R ns = x.re * x.re + x.im * x.im;
    return T(x.re / ns, -x.im / ns);
  }
  static T fmadd(T a, T b, T c) {
    R re = std::fma(a.re, b.re, std::fma(-a.im, b.im, c.re));
    R im = std::fma(a.re, b.im, std::fma(a.im, b.re, c.im));
    return T(re, im);
  }
};
template <> struct S<Cx<double>> : SC<double> {
  using Lo = Cx<float>;
  static constexpr double EPS = 2.220446049250313e-16;
  static Cx<float> demote(Cx<double> x) { return Cx<float>((float)x.re, (float)x.im); }
};
template <> struct S<Cx<float>> : SC<float> {
  using Lo = Cx<float>;
  static constexpr double EPS = 1.1920928955078125e-07;
  static Cx<float> demote(Cx<float> x) { return x; }
};
inline double promote_v(float x) { return x; }
inline Cx<double> promote_v(Cx<float> x) { return Cx<double>(x.re, x.im); }

enum Status { OK = 0, RANK_DEFICIENT = 1, INVALID = 2, DIMENSION = 3 };

// Lower-triangle CSC, sorted rows, duplicates summed (src/sparse/csc.rs:41-155).
template <typename T>
struct Csc {
  int64_t n = 0;
  std::vector<int64_t> cp, ri;
  std::vector<T> v;
};

template <typename T>
Csc<T> from_triplets(int64_t n, const std::vector<int64_t>& r, const std::vector<int64_t>& c,
                     const std::vector<T>& val) {
  Csc<T> a;
  a.n = n;
  std::vector<int64_t> cnt(n, 0);
  for (int64_t x : c) cnt[x]++;
  std::vector<int64_t> cp(n + 1, 0);
  for (int64_t j = 0; j < n; ++j) cp[j + 1] = cp[j] + cnt[j];
  std::vector<int64_t> ri(cp[n]);
  std::vector<T> vv(cp[n]);
  std::vector<int64_t> off(cp.begin(), cp.end() - 1);
  for (size_t k = 0; k < r.size(); ++k) {
    int64_t pos = off[c[k]]++;
    ri[pos] = r[k];
    vv[pos] = val[k];
  }
  a.cp.assign(n + 1, 0);
  for (int64_t j = 0; j < n; ++j) {
    std::vector<std::pair<int64_t, T>> pr;
    for (int64_t k = cp[j]; k < cp[j + 1]; ++k) pr.push_back({ri[k], vv[k]});
    std::stable_sort(pr.begin(), pr.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    for (size_t q = 0; q < pr.size(); ++q) {
      if (q > 0 && pr[q].first == a.ri.back()) {
        a.v.back() = a.v.back() + pr[q].second;
      } else {
        a.ri.push_back(pr[q].first);
        a.v.push_back(pr[q].second);
      }
    }
    a.cp[j + 1] = (int64_t)a.ri.size();
  }
  return a;
}

inline double inv_sqrt_scale_guarded(double m) {
  if (m > 0.0) {
    double cand = 1.0 / std::sqrt(m);
    if (std::isfinite(cand) && cand > 0.0) return cand;
    return 1.0;
  }
  return 1.0;
}

template <typename T>
std::vector<double> onepass_scale(const Csc<T>& a) {
  std::vector<double> rm(a.n, 0.0);
  for (int64_t j = 0; j < a.n; ++j)
    for (int64_t k = a.cp[j]; k < a.cp[j + 1]; ++k) {
      int64_t i = a.ri[k];
      double m = S<T>::mag(a.v[k]);
      if (m > rm[i]) rm[i] = m;
      if (i != j && m > rm[j]) rm[j] = m;
    }
  std::vector<double> s(a.n);
  for (int64_t i = 0; i < a.n; ++i) s[i] = inv_sqrt_scale_guarded(rm[i]);
  return s;
}

template <typename T>
void symv(const Csc<T>& a, const T* x, T* y) {
  for (int64_t i = 0; i < a.n; ++i) y[i] = S<T>::zero();
  for (int64_t j = 0; j < a.n; ++j)
    for (int64_t k = a.cp[j]; k < a.cp[j + 1]; ++k) {
      int64_t i = a.ri[k];
      T v = a.v[k];
      y[i] = y[i] + v * x[j];
      if (i != j) y[j] = y[j] + v * x[i];
    }
}

template <typename T>
double sym_norm_inf(const Csc<T>& a) {
  std::vector<double> rs(a.n, 0.0);
  for (int64_t c = 0; c < a.n; ++c)
    for (int64_t k = a.cp[c]; k < a.cp[c + 1]; ++k) {
      int64_t r = a.ri[k];
      double m = S<T>::mag(a.v[k]);
      rs[r] += m;
      if (r != c) rs[c] += m;
    }
  double mx = 0;
  for (double x : rs) mx = std::max(mx, x);
  return mx;
}

// Reference factor container (src/dense/ldlt_generic.rs:31-66).
template <typename T>
struct Factors {
  int64_t n = 0;
  std::vector<int64_t> lcp, lri;
  std::vector<T> lv, d, dsub;
  std::vector<uint8_t> two;
  std::vector<int64_t> perm;
  int64_t n_perturbed = 0;
  int64_t ipos = 0, ineg = 0, izero = 0;
};

struct SymIn {
  int64_t n = 0;
  std::vector<int64_t> perm, perm_inv;
  int64_t ns = 0;
  std::vector<int64_t> first, ncol;
  std::vector<std::vector<int64_t>> children;
};

constexpr double GROWTH_EPS = 1e-14;
inline double bk_alpha() { return (1.0 + std::sqrt(17.0)) / 8.0; }

template <typename T>
T perturb_pivot(T d, double floor_) {
  double m = S<T>::mag(d);
  if (m >= floor_) return d;
  if (m == 0.0) return S<T>::from_real(floor_);
  return d * S<T>::from_real(floor_ / m);
}

template <typename T>
void swap_sym_lower_bounded(T* a, int64_t n, int64_t p, int64_t q, int64_t row_limit) {
  for (int64_t i = q + 1; i < row_limit; ++i) std::swap(a[p * n + i], a[q * n + i]);
  for (int64_t i = p + 1; i < q; ++i) std::swap(a[p * n + i], a[i * n + q]);
  std::swap(a[p * n + p], a[q * n + q]);
  for (int64_t j = 0; j < p; ++j) std::swap(a[j * n + p], a[j * n + q]);
}

template <typename T>
void apply_bk_panel_trailing(T* base, int64_t nrow, int64_t kb, int64_t ke, const std::vector<T>& dd,
                             const std::vector<T>& dsub, const std::vector<uint8_t>& two,
                             const std::vector<int64_t>& deep_swaps, const std::vector<T>& snap, int64_t nb,
                             int64_t r0, int64_t r1) {
  int64_t k = kb;
  while (k < ke) {
    int64_t kp = deep_swaps[k - kb];
    if (kp >= 0) {
      int64_t src = two[k] ? k + 1 : k;
      for (int64_t i = r0; i < r1; ++i) std::swap(base[src * nrow + i], base[kp * nrow + i]);
    }
    if (two[k]) {
      T d11 = dd[k], d21 = dsub[k], d22 = dd[k + 1];
      T det = d11 * d22 - d21 * d21;
      T detinv = S<T>::recip(det);
      for (int64_t j = k + 2; j < ke; ++j) {
        T l1j = snap[(k - kb) * nb + (j - kb)];
        T l2j = snap[(k + 1 - kb) * nb + (j - kb)];
        for (int64_t i = r0; i < r1; ++i)
          base[j * nrow + i] = base[j * nrow + i] - base[k * nrow + i] * l1j - base[(k + 1) * nrow + i] * l2j;
      }
      for (int64_t i = r0; i < r1; ++i) {
        T wik = base[k * nrow + i], wik1 = base[(k + 1) * nrow + i];
        base[k * nrow + i] = (d22 * wik - d21 * wik1) * detinv;
        base[(k + 1) * nrow + i] = (d11 * wik1 - d21 * wik) * detinv;
      }
      k += 2;
    } else {
      T dinv = S<T>::recip(dd[k]);
      for (int64_t j = k + 1; j < ke; ++j) {
        T w = snap[(k - kb) * nb + (j - kb)];
        if (w != S<T>::zero())
          for (int64_t i = r0; i < r1; ++i) base[j * nrow + i] = base[j * nrow + i] - base[k * nrow + i] * w;
      }
      for (int64_t i = r0; i < r1; ++i) base[k * nrow + i] = base[k * nrow + i] * dinv;
      k += 1;
    }
  }
}

struct FactorOpts {
  bool perturb = false;
  double floor_ = 0;
  bool drop = false;
  double drop_tol = 0;
  int64_t panel_nb = 64;
  bool fast = false;  // timing mode: BLAS products + level-parallel schedule
};

// CBLAS of an ILP64 OpenBLAS (64-bit dimensions), resolved by name from the
// library path given to oracle_set_parallel.
struct Blas {
  using real_gemm_d = void (*)(int, int, int, int64_t, int64_t, int64_t, double, const double*, int64_t,
                               const double*, int64_t, double, double*, int64_t);
  using real_gemm_s = void (*)(int, int, int, int64_t, int64_t, int64_t, float, const float*, int64_t,
                               const float*, int64_t, float, float*, int64_t);
  using cplx_gemm = void (*)(int, int, int, int64_t, int64_t, int64_t, const void*, const void*, int64_t,
                             const void*, int64_t, const void*, void*, int64_t);
  real_gemm_d dgemm = nullptr;
  real_gemm_s sgemm = nullptr;
  cplx_gemm zgemm = nullptr, cgemm = nullptr;
  void (*set_threads)(int) = nullptr;
  int threads = 1;
  bool ok() const { return dgemm && sgemm && zgemm && cgemm && set_threads; }
};
static Blas g_blas;
static bool g_fast = false;

constexpr int kColMajor = 102, kNoTrans = 111, kTrans = 112;

// C = A B^T, A m x k (lda), B n x k (ldb), C m x n (ldc), column-major.
inline void gemm_nt(int64_t m, int64_t n, int64_t k, const double* A, int64_t lda, const double* B, int64_t ldb,
                    double* C, int64_t ldc) {
  g_blas.dgemm(kColMajor, kNoTrans, kTrans, m, n, k, 1.0, A, lda, B, ldb, 0.0, C, ldc);
}
inline void gemm_nt(int64_t m, int64_t n, int64_t k, const float* A, int64_t lda, const float* B, int64_t ldb,
                    float* C, int64_t ldc) {
  g_blas.sgemm(kColMajor, kNoTrans, kTrans, m, n, k, 1.0f, A, lda, B, ldb, 0.0f, C, ldc);
}
inline void gemm_nt(int64_t m, int64_t n, int64_t k, const Cx<double>* A, int64_t lda, const Cx<double>* B,
                    int64_t ldb, Cx<double>* C, int64_t ldc) {
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  g_blas.zgemm(kColMajor, kNoTrans, kTrans, m, n, k, one, A, lda, B, ldb, zero, C, ldc);
}
inline void gemm_nt(int64_t m, int64_t n, int64_t k, const Cx<float>* A, int64_t lda, const Cx<float>* B,
                    int64_t ldb, Cx<float>* C, int64_t ldc) {
  const float one[2] = {1.0f, 0.0f}, zero[2] = {0.0f, 0.0f};
  g_blas.cgemm(kColMajor, kNoTrans, kTrans, m, n, k, one, A, lda, B, ldb, zero, C, ldc);
}

template <typename T>
struct Panel {
  std::vector<T> p, d, dsub;
  std::vector<uint8_t> two;
  std::vector<int64_t> lperm;
};

// Blocked panel-bounded BK on one assembled, cmod-updated panel.
template <typename T>
int cdiv(Panel<T>& P, int64_t nrow, int64_t ncol, const FactorOpts& o, int64_t& nperturbed) {
  std::vector<T>& panel = P.p;
  const int64_t nb = ncol >= 512 ? std::max<int64_t>(o.panel_nb, 128) : o.panel_nb;
  const double alpha = bk_alpha();
  P.d.assign(ncol, S<T>::zero());
  P.dsub.assign(ncol, S<T>::zero());
  P.two.assign(ncol, 0);
  P.lperm.resize(nrow);
  for (int64_t i = 0; i < nrow; ++i) P.lperm[i] = i;
  std::vector<T> l1(nrow), l2(nrow);
  std::vector<int64_t> deep(nb);
  std::vector<T> snap(nb * nb, S<T>::zero());
  auto& d = P.d;
  auto& dsub = P.dsub;
  auto& two = P.two;
  int64_t kb = 0;
  while (kb < ncol) {
    int64_t ke = std::min(kb + nb, ncol);
    std::fill(deep.begin(), deep.end(), -1);
    int64_t k = kb;
    while (k < ke) {
      double absakk = S<T>::mag(panel[k + k * nrow]);
      double colmax_sq = 0.0;
      int64_t imax = k;
      for (int64_t i = k + 1; i < ke; ++i) {
        double m = S<T>::mag2(panel[k * nrow + i]);
        if (m > colmax_sq) {
          colmax_sq = m;
          imax = i;
        }
      }
      double colmax = std::sqrt(colmax_sq);
      int kstep;
      int64_t kp;
      if (std::max(absakk, colmax) == 0.0) {
        if (!o.perturb) return RANK_DEFICIENT;
        kstep = 1;
        kp = k;
      } else if (absakk >= alpha * colmax) {
        kstep = 1;
        kp = k;
      } else {
        double rowmax_sq = 0.0;
        for (int64_t j = k; j < imax; ++j) rowmax_sq = std::max(rowmax_sq, S<T>::mag2(panel[j * nrow + imax]));
        for (int64_t i = imax + 1; i < ke; ++i) rowmax_sq = std::max(rowmax_sq, S<T>::mag2(panel[imax * nrow + i]));
        double rowmax = std::sqrt(rowmax_sq);
        if (absakk >= alpha * colmax * (colmax / rowmax)) {
          kstep = 1;
          kp = k;
        } else if (S<T>::mag(panel[imax * nrow + imax]) >= alpha * rowmax) {
          kstep = 1;
          kp = imax;
        } else {
          kstep = 2;
          kp = imax;
        }
      }
      if (kstep == 1) {
        if (kp != k) {
          swap_sym_lower_bounded(panel.data(), nrow, k, kp, ke);
          std::swap(P.lperm[k], P.lperm[kp]);
          deep[k - kb] = kp;
        }
        T dk = panel[k + k * nrow];
        if (o.perturb) {
          if (S<T>::mag(dk) < o.floor_) {
            dk = perturb_pivot(dk, o.floor_);
            panel[k + k * nrow] = dk;
            nperturbed++;
          }
        } else if (dk == S<T>::zero()) {
          return RANK_DEFICIENT;
        }
        d[k] = dk;
        T dinv = S<T>::recip(dk);
        for (int64_t j = k + 1; j < ke; ++j) {
          T w = panel[k * nrow + j] * dinv;
          snap[(k - kb) * nb + (j - kb)] = w;
          if (w != S<T>::zero())
            for (int64_t i = j; i < ke; ++i) panel[j * nrow + i] = panel[j * nrow + i] - panel[k * nrow + i] * w;
        }
        for (int64_t i = k + 1; i < ke; ++i) panel[k * nrow + i] = panel[k * nrow + i] * dinv;
        k += 1;
      } else {
        if (kp != k + 1) {
          swap_sym_lower_bounded(panel.data(), nrow, k + 1, kp, ke);
          std::swap(P.lperm[k + 1], P.lperm[kp]);
          deep[k - kb] = kp;
        }
        T d11 = panel[k + k * nrow];
        T d21 = panel[k * nrow + k + 1];
        T d22 = panel[(k + 1) + (k + 1) * nrow];
        T det = d11 * d22 - d21 * d21;
        double scale = std::max(std::max(S<T>::mag(d11), S<T>::mag(d22)), S<T>::mag(d21));
        double growth_floor = GROWTH_EPS * scale * scale;
        if (o.perturb) {
          double fl = std::max(o.floor_ * o.floor_, growth_floor);
          if (S<T>::mag(det) < fl) {
            double lift = std::max(o.floor_, scale * std::sqrt(GROWTH_EPS));
            d11 = d11 + S<T>::from_real(lift);
            d22 = d22 + S<T>::from_real(lift);
            det = d11 * d22 - d21 * d21;
            if (S<T>::mag(det) < fl) det = det + S<T>::from_real(fl);
            nperturbed++;
          }
        } else if (S<T>::mag(det) <= growth_floor) {
          return RANK_DEFICIENT;
        }
        T detinv = S<T>::recip(det);
        d[k] = d11;
        dsub[k] = d21;
        d[k + 1] = d22;
        two[k] = 1;
        for (int64_t i = k + 2; i < ke; ++i) {
          T wik = panel[k * nrow + i], wik1 = panel[(k + 1) * nrow + i];
          l1[i] = (d22 * wik - d21 * wik1) * detinv;
          l2[i] = (d11 * wik1 - d21 * wik) * detinv;
          snap[(k - kb) * nb + (i - kb)] = l1[i];
          snap[(k + 1 - kb) * nb + (i - kb)] = l2[i];
        }
        for (int64_t j = k + 2; j < ke; ++j) {
          T a = l1[j], b = l2[j];
          for (int64_t i = j; i < ke; ++i)
            panel[j * nrow + i] = panel[j * nrow + i] - panel[k * nrow + i] * a - panel[(k + 1) * nrow + i] * b;
        }
        for (int64_t i = k + 2; i < ke; ++i) {
          panel[k * nrow + i] = l1[i];
          panel[(k + 1) * nrow + i] = l2[i];
        }
        k += 2;
      }
    }
    if (nrow > ke) {
      // rows are replayed independently: as the reference does above
      // deep * pw^2 >= 8e6 (DEFAULT_PAR_CDIV, gemm_tuning.rs:22;
      // multifrontal_ldlt.rs:3022-3056), one contiguous chunk of rows per
      // thread gives the same values as one pass
      const int64_t deep_rows = nrow - ke, pw = ke - kb;
      const int64_t nth = omp_get_max_threads();
      const bool par = o.fast && deep_rows * pw * pw >= 8000000 && nth > 1 && !omp_in_parallel();
      const int64_t cs = par ? (deep_rows + nth - 1) / nth : deep_rows;
      const int64_t chunks = (deep_rows + cs - 1) / cs;
#pragma omp parallel for schedule(static, 1) if (par)
      for (int64_t c = 0; c < chunks; ++c) {
        const int64_t r0 = ke + c * cs, r1 = std::min<int64_t>(r0 + cs, nrow);
        apply_bk_panel_trailing(panel.data(), nrow, kb, ke, d, dsub, two, deep, snap, nb, r0, r1);
      }
    }
    // Deferred panel Schur: panel[ke.., ke..ncol] -= L21 D R^T (lower part).
    int64_t pw = ke - kb, cw = ncol - ke, mt = nrow - ke;
    if (pw > 0 && cw > 0 && mt > 0) {
      std::vector<T> l21(mt * pw), g(mt * pw);
      for (int64_t cc = 0; cc < pw; ++cc)
        for (int64_t rr = 0; rr < mt; ++rr) l21[rr + cc * mt] = panel[(ke + rr) + (kb + cc) * nrow];
      int64_t cc = 0;
      while (cc < pw) {
        int64_t c = kb + cc;
        if (two[c]) {
          T d11 = d[c], d21 = dsub[c], d22 = d[c + 1];
          for (int64_t rr = 0; rr < mt; ++rr) {
            T a = l21[rr + cc * mt], b = l21[rr + (cc + 1) * mt];
            g[rr + cc * mt] = a * d11 + b * d21;
            g[rr + (cc + 1) * mt] = a * d21 + b * d22;
          }
          cc += 2;
        } else {
          T dc = d[c];
          for (int64_t rr = 0; rr < mt; ++rr) g[rr + cc * mt] = l21[rr + cc * mt] * dc;
          cc += 1;
        }
      }
      // tmp = G L21^T (FMA accumulation in ascending q), then the lower part
      // of tmp is subtracted from the panel.
      if (o.fast) {
        std::vector<T> tmp(mt * cw);
        gemm_nt(mt, cw, pw, g.data(), mt, l21.data(), mt, tmp.data(), mt);
        for (int64_t c2 = 0; c2 < cw; ++c2) {
          T* col = panel.data() + (ke + c2) * nrow + ke;
          for (int64_t rr = c2; rr < mt; ++rr) col[rr] = col[rr] - tmp[rr + c2 * mt];
        }
        kb = ke;
        continue;
      }
#pragma omp parallel for schedule(dynamic, 16) if (mt * cw * pw > 4000000)
      for (int64_t c2 = 0; c2 < cw; ++c2) {
        T* col = panel.data() + (ke + c2) * nrow + ke;
        for (int64_t rr = c2; rr < mt; ++rr) {
          T acc = S<T>::zero();
          for (int64_t q = 0; q < pw; ++q) acc = S<T>::fmadd(g[rr + q * mt], l21[c2 + q * mt], acc);
          col[rr] = col[rr] - acc;
        }
      }
    }
    kb = ke;
  }
  return OK;
}

template <typename T>
struct OracleFactor {
  Factors<T> f;
  std::vector<double> scale;
  Csc<T> a;  // original matrix (for refinement)
  int status = OK;
};

// factor_left_looking on the equilibrated matrix `a` (already scaled).
template <typename T>
int factor_left_looking(const SymIn& sym, const Csc<T>& a, const FactorOpts& o, Factors<T>& out) {
  const int64_t n = sym.n;
  std::vector<int64_t> rows, cols;
  std::vector<T> vals;
  for (int64_t j = 0; j < n; ++j)
    for (int64_t k = a.cp[j]; k < a.cp[j + 1]; ++k) {
      int64_t gi = sym.perm_inv[a.ri[k]], gj = sym.perm_inv[j];
      if (gi >= gj) {
        rows.push_back(gi);
        cols.push_back(gj);
      } else {
        rows.push_back(gj);
        cols.push_back(gi);
      }
      vals.push_back(a.v[k]);
    }
  Csc<T> ap = from_triplets(n, rows, cols, vals);
  const int64_t ns = sym.ns;
  // Row structures.
  std::vector<std::vector<int64_t>> rs(ns);
  std::vector<uint8_t> mark;
  // Full symmetric pattern of A_perm's structure: the lower CSC plus its
  // transpose, which is what the symbolic permuted pattern holds.
  std::vector<std::vector<int64_t>> below(n);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t k = ap.cp[j]; k < ap.cp[j + 1]; ++k)
      if (ap.ri[k] > j) below[j].push_back(ap.ri[k]);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t f0 = sym.first[s], own_last = f0 + sym.ncol[s];
    std::vector<int64_t> tr;
    for (int64_t j = f0; j < own_last; ++j)
      for (int64_t r : below[j])
        if (r >= own_last) tr.push_back(r);
    for (int64_t ch : sym.children[s])
      for (size_t q = (size_t)sym.ncol[ch]; q < rs[ch].size(); ++q)
        if (rs[ch][q] >= own_last) tr.push_back(rs[ch][q]);
    std::sort(tr.begin(), tr.end());
    tr.erase(std::unique(tr.begin(), tr.end()), tr.end());
    for (int64_t j = f0; j < own_last; ++j) rs[s].push_back(j);
    rs[s].insert(rs[s].end(), tr.begin(), tr.end());
  }
  std::vector<int64_t> col2sn(n);
  for (int64_t s = 0; s < ns; ++s)
    for (int64_t c = 0; c < sym.ncol[s]; ++c) col2sn[sym.first[s] + c] = s;
  std::vector<std::vector<int64_t>> ul(ns);
  for (int64_t k = 0; k < ns; ++k) {
    int64_t last = -1;
    for (size_t q = (size_t)sym.ncol[k]; q < rs[k].size(); ++q) {
      int64_t s = col2sn[rs[k][q]];
      if (s != last) {
        ul[s].push_back(k);
        last = s;
      }
    }
  }
  std::vector<Panel<T>> store(ns);
  std::vector<int64_t> e_offset(ns, 0);
  {
    int64_t acc = 0;
    for (int64_t s = 0; s < ns; ++s) {
      e_offset[s] = acc;
      acc += sym.ncol[s];
    }
  }
  out.n = n;
  out.perm.assign(n, 0);
  out.d.assign(n, S<T>::zero());
  out.dsub.assign(n, S<T>::zero());
  out.two.assign(n, 0);
  std::vector<int64_t> e_of_g(n, -1);
  // per-supernode results, summed in supernode order at the end
  std::vector<int64_t> sn_pert(ns, 0), sn_ipos(ns, 0), sn_ineg(ns, 0), sn_izero(ns, 0);
  // One supernode: assembly, cmod from its updaters, cdiv, emit maps and
  // inertia.  `gloc` (global row -> panel row, -1 elsewhere) is the caller's
  // scratch; updaters are complete when this runs.
  auto process = [&](int64_t s, std::vector<int64_t>& gloc) -> int {
    const int64_t first = sym.first[s], ncol = sym.ncol[s], nrow = (int64_t)rs[s].size();
    Panel<T>& P = store[s];
    P.p.assign(nrow * ncol, S<T>::zero());
    for (int64_t li = 0; li < nrow; ++li) gloc[rs[s][li]] = li;
    for (int64_t p = 0; p < ncol; ++p) {
      int64_t c = first + p;
      for (int64_t k = ap.cp[c]; k < ap.cp[c + 1]; ++k) {
        int64_t li = gloc[ap.ri[k]];
        P.p[li + p * nrow] = P.p[li + p * nrow] + ap.v[k];
      }
    }
    // cmod: sequential per-update path.
    for (int64_t kk : ul[s]) {
      const Panel<T>& K = store[kk];
      const int64_t nck = sym.ncol[kk], nrk = (int64_t)rs[kk].size();
      const int64_t* ok = rs[kk].data() + nck;
      const int64_t nok = nrk - nck;
      int64_t p0 = std::lower_bound(ok, ok + nok, first) - ok;
      int64_t p1 = std::lower_bound(ok, ok + nok, first + ncol) - ok;
      int64_t npk = p1 - p0;
      if (npk == 0) continue;
      // G = rows [p0,p1) of k's off-diagonal block times D (column-major npk x nck).
      std::vector<T> vd(npk * nck);
      int64_t ck = 0;
      while (ck < nck) {
        if (K.two[ck]) {
          T d11 = K.d[ck], d21 = K.dsub[ck], d22 = K.d[ck + 1];
          for (int64_t i = 0; i < npk; ++i) {
            T x = K.p[(nck + p0 + i) + ck * nrk], y = K.p[(nck + p0 + i) + (ck + 1) * nrk];
            vd[i + ck * npk] = d11 * x + d21 * y;
            vd[i + (ck + 1) * npk] = d21 * x + d22 * y;
          }
          ck += 2;
        } else {
          T dk = K.d[ck];
          for (int64_t i = 0; i < npk; ++i) vd[i + ck * npk] = K.p[(nck + p0 + i) + ck * nrk] * dk;
          ck += 1;
        }
      }
      if (o.fast) {
        // W = L_k[p0 + c0 .., :] G[c0 .. c0 + cb, :]^T by BLAS, 512 target
        // columns at a time, then the rows r >= c are scattered.
        for (int64_t c0 = 0; c0 < npk; c0 += 512) {
          const int64_t cb = std::min<int64_t>(512, npk - c0), m = nok - p0 - c0;
          std::vector<T> W(m * cb);
          gemm_nt(m, cb, nck, K.p.data() + nck + p0 + c0, nrk, vd.data() + c0, npk, W.data(), m);
          for (int64_t c = 0; c < cb; ++c) {
            T* dst = P.p.data() + (ok[p0 + c0 + c] - first) * nrow;
            for (int64_t r = c; r < m; ++r) {
              const int64_t tr = gloc[ok[p0 + c0 + r]];
              dst[tr] = dst[tr] - W[r + c * m];
            }
          }
        }
        continue;
      }
      // U[r, c] = sum_q L_k[p0 + r, q] * G[c, q] (FMA accumulation in
      // ascending q, as the gemm crate's FMA kernels); rows r >= c only.
#pragma omp parallel for schedule(dynamic, 8) if ((nok - p0) * npk * nck > 4000000)
      for (int64_t c = 0; c < npk; ++c) {
        int64_t tcol = ok[p0 + c] - first;
        T* dst = P.p.data() + tcol * nrow;
        for (int64_t r = p0 + c; r < nok; ++r) {
          T acc = S<T>::zero();
          for (int64_t q = 0; q < nck; ++q) acc = S<T>::fmadd(K.p[(nck + r) + q * nrk], vd[c + q * npk], acc);
          int64_t tr = gloc[ok[r]];
          dst[tr] = dst[tr] - acc;
        }
      }
    }
    int st = cdiv(P, nrow, ncol, o, sn_pert[s]);
    for (int64_t li = 0; li < nrow; ++li) gloc[rs[s][li]] = -1;
    if (st != OK) return st;
    // Emit maps + inertia.
    int64_t eoff = e_offset[s];
    int64_t pp = 0;
    while (pp < ncol) {
      int64_t g = rs[s][P.lperm[pp]];
      int64_t e = eoff + pp;
      e_of_g[g] = e;
      out.perm[e] = sym.perm[g];
      out.d[e] = P.d[pp];
      if (P.two[pp]) {
        int64_t g2 = rs[s][P.lperm[pp + 1]];
        e_of_g[g2] = e + 1;
        out.perm[e + 1] = sym.perm[g2];
        out.d[e + 1] = P.d[pp + 1];
        out.dsub[e] = P.dsub[pp];
        out.two[e] = 1;
        double det_r = S<T>::real(P.d[pp] * P.d[pp + 1] - P.dsub[pp] * P.dsub[pp]);
        double tr_r = S<T>::real(P.d[pp] + P.d[pp + 1]);
        if (det_r < 0.0) {
          sn_ipos[s]++;
          sn_ineg[s]++;
        } else if (det_r > 0.0) {
          if (tr_r >= 0.0)
            sn_ipos[s] += 2;
          else
            sn_ineg[s] += 2;
        } else {
          sn_izero[s]++;
          if (tr_r >= 0.0)
            sn_ipos[s]++;
          else
            sn_ineg[s]++;
        }
        pp += 2;
      } else {
        double r = S<T>::real(P.d[pp]);
        if (r > 0.0)
          sn_ipos[s]++;
        else if (r < 0.0)
          sn_ineg[s]++;
        else
          sn_izero[s]++;
        pp += 1;
      }
    }
    return OK;
  };
  if (!o.fast) {
    // Supernodes are in postorder: sequential 0..ns is a valid schedule.
    std::vector<int64_t> gloc(n, -1);
    for (int64_t s = 0; s < ns; ++s) {
      const int st = process(s, gloc);
      if (st != OK) return st;
    }
  } else {
    // Assembly-tree levels (children before parents); a level's supernodes
    // are independent.  Wide levels: one supernode per thread, one-thread
    // BLAS; narrow levels: one supernode at a time, all threads in BLAS.
    std::vector<int64_t> level(ns, 0);
    int64_t nlev = 0;
    for (int64_t s = 0; s < ns; ++s) {
      for (int64_t c : sym.children[s]) level[s] = std::max(level[s], level[c] + 1);
      nlev = std::max(nlev, level[s] + 1);
    }
    std::vector<std::vector<int64_t>> by_level(nlev);
    for (int64_t s = 0; s < ns; ++s) by_level[level[s]].push_back(s);
    const int nth = omp_get_max_threads();
    std::vector<std::vector<int64_t>> glocs(nth, std::vector<int64_t>(n, -1));
    std::vector<int> sn_st(ns, OK);
    for (const auto& L : by_level) {
      if ((int64_t)L.size() >= nth && nth > 1) {
        g_blas.set_threads(1);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t i = 0; i < (int64_t)L.size(); ++i) sn_st[L[i]] = process(L[i], glocs[omp_get_thread_num()]);
      } else {
        g_blas.set_threads(g_blas.threads);
        for (int64_t s : L) sn_st[s] = process(s, glocs[0]);
      }
      for (int64_t s : L)
        if (sn_st[s] != OK) return sn_st[s];
    }
    g_blas.set_threads(g_blas.threads);
  }
  int64_t nperturbed = 0;
  for (int64_t s = 0; s < ns; ++s) {
    nperturbed += sn_pert[s];
    out.ipos += sn_ipos[s];
    out.ineg += sn_ineg[s];
    out.izero += sn_izero[s];
  }
  // Emit compact L (every row's e index is known once all panels are done):
  // each supernode's columns into its own buffer (in parallel in timing
  // mode), then concatenated in supernode order.
  std::vector<std::vector<int64_t>> sn_ri(ns), sn_cnt(ns);
  std::vector<std::vector<T>> sn_v(ns);
  auto emit = [&](int64_t s) {
    const Panel<T>& P = store[s];
    const int64_t ncol = sym.ncol[s], nrow = (int64_t)rs[s].size();
    std::vector<std::pair<int64_t, T>> col;
    for (int64_t p = 0; p < ncol; ++p) {
      col.clear();
      int64_t de = e_of_g[rs[s][P.lperm[p]]];
      col.push_back({de, S<T>::one()});
      int64_t i0 = P.two[p] ? p + 2 : p + 1;
      for (int64_t i = i0; i < nrow; ++i) {
        T v = P.p[i + p * nrow];
        if (v != S<T>::zero()) col.push_back({e_of_g[rs[s][P.lperm[i]]], v});
      }
      if (o.drop) {
        double cm = 0;
        for (auto& x : col)
          if (x.first != de) cm = std::max(cm, S<T>::mag(x.second));
        double th = o.drop_tol * cm;
        std::vector<std::pair<int64_t, T>> kept;
        for (auto& x : col)
          if (x.first == de || S<T>::mag(x.second) >= th) kept.push_back(x);
        col.swap(kept);
      }
      std::stable_sort(col.begin(), col.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      for (auto& x : col) {
        sn_ri[s].push_back(x.first);
        sn_v[s].push_back(x.second);
      }
      sn_cnt[s].push_back((int64_t)col.size());
    }
  };
#pragma omp parallel for schedule(dynamic, 4) if (o.fast)
  for (int64_t s = 0; s < ns; ++s) emit(s);
  out.lcp.assign(1, 0);
  int64_t total = 0;
  for (int64_t s = 0; s < ns; ++s) total += (int64_t)sn_ri[s].size();
  out.lri.reserve(total);
  out.lv.reserve(total);
  for (int64_t s = 0; s < ns; ++s) {
    out.lri.insert(out.lri.end(), sn_ri[s].begin(), sn_ri[s].end());
    out.lv.insert(out.lv.end(), sn_v[s].begin(), sn_v[s].end());
    for (int64_t c : sn_cnt[s]) out.lcp.push_back(out.lcp.back() + c);
    std::vector<int64_t>().swap(sn_ri[s]);
    std::vector<T>().swap(sn_v[s]);
  }
  out.n_perturbed = nperturbed;
  return OK;
}

// solve_ldlt_block (row-major n x nrhs, unscaled factors).
template <typename T>
int solve_block(const Factors<T>& f, const T* b, int64_t nrhs, T* x) {
  const int64_t n = f.n;
  std::vector<T> y(n * nrhs), row(nrhs);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t c = 0; c < nrhs; ++c) y[i * nrhs + c] = b[f.perm[i] * nrhs + c];
  for (int64_t j = 0; j < n; ++j) {
    for (int64_t c = 0; c < nrhs; ++c) row[c] = y[j * nrhs + c];
    for (int64_t k = f.lcp[j] + 1; k < f.lcp[j + 1]; ++k) {
      int64_t i = f.lri[k];
      T nl = S<T>::zero() - f.lv[k];
      for (int64_t c = 0; c < nrhs; ++c) y[i * nrhs + c] = S<T>::fmadd(nl, row[c], y[i * nrhs + c]);
    }
  }
  int64_t k = 0;
  while (k < n) {
    if (f.two[k]) {
      T d11 = f.d[k], d21 = f.dsub[k], d22 = f.d[k + 1];
      T det = d11 * d22 - d21 * d21;
      if (det == S<T>::zero()) return RANK_DEFICIENT;
      T di = S<T>::recip(det);
      for (int64_t c = 0; c < nrhs; ++c) {
        T z0 = y[k * nrhs + c], z1 = y[(k + 1) * nrhs + c];
        y[k * nrhs + c] = (d22 * z0 - d21 * z1) * di;
        y[(k + 1) * nrhs + c] = (d11 * z1 - d21 * z0) * di;
      }
      k += 2;
    } else {
      if (f.d[k] == S<T>::zero()) return RANK_DEFICIENT;
      T di = S<T>::recip(f.d[k]);
      for (int64_t c = 0; c < nrhs; ++c) y[k * nrhs + c] = y[k * nrhs + c] * di;
      k += 1;
    }
  }
  for (int64_t j = n - 1; j >= 0; --j) {
    for (int64_t c = 0; c < nrhs; ++c) row[c] = y[j * nrhs + c];
    for (int64_t kk = f.lcp[j] + 1; kk < f.lcp[j + 1]; ++kk) {
      int64_t i = f.lri[kk];
      T nl = S<T>::zero() - f.lv[kk];
      for (int64_t c = 0; c < nrhs; ++c) row[c] = S<T>::fmadd(nl, y[i * nrhs + c], row[c]);
    }
    for (int64_t c = 0; c < nrhs; ++c) y[j * nrhs + c] = row[c];
  }
  for (int64_t i = 0; i < n; ++i)
    for (int64_t c = 0; c < nrhs; ++c) x[f.perm[i] * nrhs + c] = y[i * nrhs + c];
  return OK;
}

// solve_ldlt_many (src/dense/ldlt_generic.rs:564-614): with >= 8 columns and
// n * nrhs >= 2^18 the columns are split into one contiguous chunk per
// thread, each solved by solve_block on a compact copy; every column sees the
// same operations as in one block solve, so the result is bit-identical.
template <typename T>
int solve_many(const Factors<T>& f, const T* b, int64_t nrhs, T* x) {
  const int64_t n = f.n;
  const int nth = omp_get_max_threads();
  if (nrhs < 8 || n * nrhs < (1 << 18) || nth < 2) return solve_block(f, b, nrhs, x);
  const int64_t nch = std::min<int64_t>(nth, nrhs), w0 = (nrhs + nch - 1) / nch;
  int bad = OK;
#pragma omp parallel for schedule(static, 1)
  for (int64_t t = 0; t < nch; ++t) {
    const int64_t c0 = t * w0, c1 = std::min(nrhs, c0 + w0), w = c1 - c0;
    if (w <= 0) continue;
    std::vector<T> sub(n * w), xs(n * w);
    for (int64_t i = 0; i < n; ++i)
      for (int64_t c = 0; c < w; ++c) sub[i * w + c] = b[i * nrhs + c0 + c];
    const int st = solve_block(f, sub.data(), w, xs.data());
    if (st != OK) {
#pragma omp critical
      bad = st;
    }
    for (int64_t i = 0; i < n; ++i)
      for (int64_t c = 0; c < w; ++c) x[i * nrhs + c0 + c] = xs[i * w + c];
  }
  return bad;
}

// LdltSolver::solve_many: scale, solve, scale back.
template <typename T>
int solver_solve(const OracleFactor<T>& F, const T* b, int64_t nrhs, T* x) {
  const int64_t n = F.f.n;
  std::vector<T> bh(b, b + n * nrhs);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t c = 0; c < nrhs; ++c) bh[i * nrhs + c] = bh[i * nrhs + c] * S<T>::from_real(F.scale[i]);
  int st = solve_many(F.f, bh.data(), nrhs, x);
  if (st != OK) return st;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t c = 0; c < nrhs; ++c) x[i * nrhs + c] = x[i * nrhs + c] * S<T>::from_real(F.scale[i]);
  return OK;
}

template <typename T>
double norm_inf(const std::vector<T>& v) {
  double m = 0;
  for (const T& x : v) m = std::max(m, S<T>::mag(x));
  return m;
}
template <typename T>
double norm2(const T* v, int64_t n) {
  double s = 0;
  for (int64_t i = 0; i < n; ++i) s += S<T>::mag2(v[i]);
  return std::sqrt(s);
}
template <typename T>
T dotc(const T* x, const T* y, int64_t n) {
  T s = S<T>::zero();
  for (int64_t i = 0; i < n; ++i) s = s + S<T>::conj(x[i]) * y[i];
  return s;
}
template <typename T>
void givens(T f, T g, T& c, T& s) {
  if (g == S<T>::zero()) {
    c = S<T>::one();
    s = S<T>::zero();
    return;
  }
  if (f == S<T>::zero()) {
    c = S<T>::zero();
    s = S<T>::one();
    return;
  }
  double r = std::sqrt(S<T>::mag2(f) + S<T>::mag2(g));
  T inv = S<T>::from_real(1.0 / r);
  c = f * inv;
  s = g * inv;
}

struct MixedInfo {
  int64_t ir_iters = 0, gmres_iters = 0;
  double backward_error = 0;
  int certified = 0;
};

// Low-precision preconditioner: z = promote(F_lo^{-1} demote(r)).
template <typename T>
struct LoPre {
  using L = typename S<T>::Lo;
  const OracleFactor<L>* lo;
  int apply(const T* r, T* z, int64_t n) const {
    std::vector<L> rl(n), zl(n);
    for (int64_t i = 0; i < n; ++i) rl[i] = S<T>::demote(r[i]);
    int st = solver_solve(*lo, rl.data(), 1, zl.data());
    if (st != OK) return st;
    for (int64_t i = 0; i < n; ++i) z[i] = promote_v(zl[i]);
    return OK;
  }
};

template <typename T>
int gmres(const Csc<T>& a, const T* b, const LoPre<T>& pre, double tol, int64_t max_iter, int64_t restart,
          std::vector<T>& x, int64_t& iters) {
  const int64_t n = a.n, m = std::max<int64_t>(restart, 1);
  const double eta = 0.7071067811865476;
  double bnorm = norm2(b, n);
  if (bnorm == 0.0) {
    std::fill(x.begin(), x.end(), S<T>::zero());
    iters = 0;
    return OK;
  }
  int64_t total = 0;
  std::vector<T> w(n), ax(n), r(n), v(n * (m + 1)), zb(n * m), h((m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
  for (;;) {
    symv(a, x.data(), ax.data());
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
    double beta = norm2(r.data(), n);
    double fr = beta / bnorm;
    if (fr <= tol || total >= max_iter) break;
    T ib = S<T>::from_real(1.0 / beta);
    for (int64_t k = 0; k < n; ++k) v[k] = r[k] * ib;
    std::fill(h.begin(), h.end(), S<T>::zero());
    std::fill(cs.begin(), cs.end(), S<T>::zero());
    std::fill(sn.begin(), sn.end(), S<T>::zero());
    std::fill(g.begin(), g.end(), S<T>::zero());
    g[0] = S<T>::from_real(beta);
    int64_t jdim = 0;
    for (int64_t j = 0; j < m; ++j) {
      if (total >= max_iter) break;
      int st = pre.apply(&v[j * n], &zb[j * n], n);
      if (st != OK) return st;
      symv(a, &zb[j * n], w.data());
      double w0 = norm2(w.data(), n);
      for (int64_t i = 0; i <= j; ++i) {
        T hij = dotc(&v[i * n], w.data(), n);
        h[i * m + j] = hij;
        for (int64_t k = 0; k < n; ++k) w[k] = w[k] - hij * v[i * n + k];
      }
      double hn = norm2(w.data(), n);
      if (hn < eta * w0) {
        for (int64_t i = 0; i <= j; ++i) {
          T s = dotc(&v[i * n], w.data(), n);
          h[i * m + j] = h[i * m + j] + s;
          for (int64_t k = 0; k < n; ++k) w[k] = w[k] - s * v[i * n + k];
        }
        hn = norm2(w.data(), n);
      }
      h[(j + 1) * m + j] = S<T>::from_real(hn);
      if (hn > 0.0) {
        T inv = S<T>::from_real(1.0 / hn);
        for (int64_t k = 0; k < n; ++k) v[(j + 1) * n + k] = w[k] * inv;
      } else {
        for (int64_t k = 0; k < n; ++k) v[(j + 1) * n + k] = S<T>::zero();
      }
      for (int64_t i = 0; i < j; ++i) {
        T t = S<T>::conj(cs[i]) * h[i * m + j] + S<T>::conj(sn[i]) * h[(i + 1) * m + j];
        h[(i + 1) * m + j] = -sn[i] * h[i * m + j] + cs[i] * h[(i + 1) * m + j];
        h[i * m + j] = t;
      }
      T c, s;
      givens(h[j * m + j], h[(j + 1) * m + j], c, s);
      cs[j] = c;
      sn[j] = s;
      h[j * m + j] = S<T>::conj(c) * h[j * m + j] + S<T>::conj(s) * h[(j + 1) * m + j];
      h[(j + 1) * m + j] = S<T>::zero();
      T gn = -s * g[j];
      g[j] = S<T>::conj(c) * g[j];
      g[j + 1] = gn;
      total++;
      jdim = j + 1;
      if (S<T>::mag(g[j + 1]) / bnorm <= tol) break;
    }
    int64_t jd = jdim;
    if (jd > 0) {
      double hmax = 0;
      for (int64_t i = 0; i < jdim; ++i) hmax = std::max(hmax, S<T>::mag(h[i * m + i]));
      double th = 2.220446049250313e-16 * hmax;
      for (int64_t i = 0; i < jdim; ++i)
        if (S<T>::mag(h[i * m + i]) <= th) {
          jd = i;
          break;
        }
    }
    for (int64_t i = jd - 1; i >= 0; --i) {
      T s = g[i];
      for (int64_t k = i + 1; k < jd; ++k) s = s - h[i * m + k] * y[k];
      y[i] = s * S<T>::recip(h[i * m + i]);
    }
    for (int64_t i = 0; i < jd; ++i)
      for (int64_t k = 0; k < n; ++k) x[k] = x[k] + zb[i * n + k] * y[i];
  }
  iters = total;
  return OK;
}

template <typename T>
int refine_ladder(const Csc<T>& a, const LoPre<T>& pre, const T* b, double anorm, double target,
                  std::vector<T>& x, MixedInfo& info) {
  const int64_t n = a.n;
  double bnorm = 0;
  for (int64_t i = 0; i < n; ++i) bnorm = std::max(bnorm, S<T>::mag(b[i]));
  std::vector<T> ax(n), r(n), dx(n);
  auto berr = [&](const std::vector<T>& xx, const std::vector<T>& rr) {
    double xn = norm_inf(xx), rn = norm_inf(rr);
    return rn / std::max(anorm * xn + bnorm, std::numeric_limits<double>::min());
  };
  int64_t ir = 0;
  std::vector<T> best = x;
  double best_be = std::numeric_limits<double>::infinity();
  double prev_rn = std::numeric_limits<double>::infinity();
  for (;;) {
    symv(a, x.data(), ax.data());
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
    double be = berr(x, r);
    if (be < best_be) {
      best_be = be;
      best = x;
    }
    if (be <= target) {
      x = best;
      info = {ir, 0, best_be, 1};
      return OK;
    }
    double rn = norm_inf(r);
    if (ir >= 8 || (ir > 0 && rn > prev_rn * 0.5)) break;
    prev_rn = rn;
    int st = pre.apply(r.data(), dx.data(), n);
    if (st != OK) return st;
    for (int64_t i = 0; i < n; ++i) x[i] = x[i] + dx[i];
    ir++;
  }
  std::vector<T> xg = best;
  int64_t gi = 0;
  int st = gmres(a, b, pre, target, 120, 30, xg, gi);
  if (st != OK) return st;
  symv(a, xg.data(), ax.data());
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
  double be2 = berr(xg, r);
  if (be2 < best_be) {
    x = xg;
    best_be = be2;
  } else {
    x = best;
  }
  info = {ir, gi, best_be, best_be <= target ? 1 : 0};
  return OK;
}

struct Handle {
  int dtype;  // 0 f64, 1 c64, 2 f32, 3 c32
  void* f;
};

template <typename T>
OracleFactor<T>* build(const SymIn& sym, int64_t n, const int64_t* cp, const int64_t* ri, const T* vals,
                       int scaling, const FactorOpts& o) {
  auto* F = new OracleFactor<T>();
  F->a.n = n;
  F->a.cp.assign(cp, cp + n + 1);
  F->a.ri.assign(ri, ri + cp[n]);
  F->a.v.assign(vals, vals + cp[n]);
  if (scaling)
    F->scale = onepass_scale(F->a);
  else
    F->scale.assign(n, 1.0);
  Csc<T> sc = F->a;
  for (int64_t j = 0; j < n; ++j)
    for (int64_t k = sc.cp[j]; k < sc.cp[j + 1]; ++k)
      sc.v[k] = sc.v[k] * S<T>::from_real(F->scale[sc.ri[k]] * F->scale[j]);
  F->status = factor_left_looking(sym, sc, o, F->f);
  return F;
}

}  // namespace orc

using namespace orc;

extern "C" {

// Timing mode on (fast = 1: BLAS products from the ILP64 OpenBLAS at
// blas_path, `threads` OpenMP threads and BLAS threads) or off (fast = 0:
// the exact plain-loop checker).  Returns 0, or -1 if the BLAS did not load.
int oracle_set_parallel(int fast, const char* blas_path, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  if (!fast) {
    g_fast = false;
    return 0;
  }
  if (!g_blas.ok()) {
    void* h = dlopen(blas_path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return -1;
    g_blas.dgemm = (Blas::real_gemm_d)dlsym(h, "scipy_cblas_dgemm64_");
    g_blas.sgemm = (Blas::real_gemm_s)dlsym(h, "scipy_cblas_sgemm64_");
    g_blas.zgemm = (Blas::cplx_gemm)dlsym(h, "scipy_cblas_zgemm64_");
    g_blas.cgemm = (Blas::cplx_gemm)dlsym(h, "scipy_cblas_cgemm64_");
    g_blas.set_threads = (void (*)(int))dlsym(h, "scipy_openblas_set_num_threads64_");
    if (!g_blas.ok()) return -1;
  }
  g_blas.threads = threads > 0 ? threads : omp_get_max_threads();
  g_blas.set_threads(g_blas.threads);
  g_fast = true;
  return 0;
}

// Factor `A` (lower CSC, values of dtype) with the given symbolic structure.
void* oracle_factor(int dtype, int64_t n, const int64_t* cp, const int64_t* ri, const void* vals, const int64_t* perm,
                    int64_t ns, const int64_t* sn_first, const int64_t* sn_ncol, const int64_t* ch_ptr,
                    const int64_t* ch_idx, int scaling, double perturb_floor, double drop_tol, int64_t panel_nb,
                    int* status) {
  SymIn sym;
  sym.n = n;
  sym.perm.assign(perm, perm + n);
  sym.perm_inv.assign(n, 0);
  for (int64_t k = 0; k < n; ++k) sym.perm_inv[perm[k]] = k;
  sym.ns = ns;
  sym.first.assign(sn_first, sn_first + ns);
  sym.ncol.assign(sn_ncol, sn_ncol + ns);
  sym.children.resize(ns);
  for (int64_t s = 0; s < ns; ++s) sym.children[s].assign(ch_idx + ch_ptr[s], ch_idx + ch_ptr[s + 1]);
  FactorOpts o;
  if (perturb_floor >= 0) {
    o.perturb = true;
    o.floor_ = perturb_floor;
  }
  if (drop_tol >= 0) {
    o.drop = true;
    o.drop_tol = drop_tol;
  }
  o.panel_nb = std::max<int64_t>(panel_nb, 8);
  o.fast = g_fast;
  auto* h = new Handle{dtype, nullptr};
  int st = OK;
  switch (dtype) {
    case 0: {
      auto* F = build<double>(sym, n, cp, ri, (const double*)vals, scaling, o);
      st = F->status;
      h->f = F;
      break;
    }
    case 1: {
      auto* F = build<Cx<double>>(sym, n, cp, ri, (const Cx<double>*)vals, scaling, o);
      st = F->status;
      h->f = F;
      break;
    }
    case 2: {
      auto* F = build<float>(sym, n, cp, ri, (const float*)vals, scaling, o);
      st = F->status;
      h->f = F;
      break;
    }
    case 3: {
      auto* F = build<Cx<float>>(sym, n, cp, ri, (const Cx<float>*)vals, scaling, o);
      st = F->status;
      h->f = F;
      break;
    }
    default:
      st = INVALID;
  }
  *status = st;
  return h;
}

#define ORC_DISPATCH(h, BODY)                                 \
  switch ((h)->dtype) {                                       \
    case 0: {                                                 \
      using T = double;                                       \
      auto* F = (OracleFactor<T>*)(h)->f;                     \
      BODY;                                                   \
      break;                                                  \
    }                                                         \
    case 1: {                                                 \
      using T = Cx<double>;                                   \
      auto* F = (OracleFactor<T>*)(h)->f;                     \
      BODY;                                                   \
      break;                                                  \
    }                                                         \
    case 2: {                                                 \
      using T = float;                                        \
      auto* F = (OracleFactor<T>*)(h)->f;                     \
      BODY;                                                   \
      break;                                                  \
    }                                                         \
    case 3: {                                                 \
      using T = Cx<float>;                                    \
      auto* F = (OracleFactor<T>*)(h)->f;                     \
      BODY;                                                   \
      break;                                                  \
    }                                                         \
  }

int64_t oracle_factor_nnz(void* hp) {
  auto* h = (Handle*)hp;
  int64_t r = 0;
  ORC_DISPATCH(h, r = (int64_t)F->f.lv.size());
  return r;
}

// Export the reference LdltFactors layout (+ the equilibration scale).
void oracle_export(void* hp, int64_t* lcp, int64_t* lri, void* lv, void* d, void* dsub, uint8_t* two, int64_t* perm,
                   double* scale, int64_t* info5) {
  auto* h = (Handle*)hp;
  ORC_DISPATCH(h, {
    const auto& f = F->f;
    std::memcpy(lcp, f.lcp.data(), f.lcp.size() * 8);
    std::memcpy(lri, f.lri.data(), f.lri.size() * 8);
    std::memcpy(lv, f.lv.data(), f.lv.size() * sizeof(T));
    std::memcpy(d, f.d.data(), f.d.size() * sizeof(T));
    std::memcpy(dsub, f.dsub.data(), f.dsub.size() * sizeof(T));
    std::memcpy(two, f.two.data(), f.two.size());
    std::memcpy(perm, f.perm.data(), f.perm.size() * 8);
    std::memcpy(scale, F->scale.data(), F->scale.size() * 8);
    info5[0] = f.ipos;
    info5[1] = f.ineg;
    info5[2] = f.izero;
    info5[3] = f.n_perturbed;
    info5[4] = F->status;
  });
}

// LdltSolver::solve_many on row-major n x nrhs.
int oracle_solve(void* hp, const void* b, int64_t nrhs, void* x) {
  auto* h = (Handle*)hp;
  int st = INVALID;
  ORC_DISPATCH(h, { st = F->status != OK ? F->status : solver_solve(*F, (const T*)b, nrhs, (T*)x); });
  return st;
}

// MixedLdltSolver::solve_to: `hlo` holds the low-precision factor of cast(A)
// (dtype 2 or 3); `a_*` is the original high-precision A (dtype 0 or 1).
int oracle_mixed_solve(void* hlo, int dtype_hi, int64_t n, const int64_t* cp, const int64_t* ri, const void* avals,
                       const void* b, double target, void* x, int64_t* iters2, double* be, int* certified) {
  auto* lo = (Handle*)hlo;
  MixedInfo info;
  int st = OK;
  if (dtype_hi == 0) {
    Csc<double> a;
    a.n = n;
    a.cp.assign(cp, cp + n + 1);
    a.ri.assign(ri, ri + cp[n]);
    a.v.assign((const double*)avals, (const double*)avals + cp[n]);
    LoPre<double> pre{(OracleFactor<float>*)lo->f};
    std::vector<double> xx(n);
    st = pre.apply((const double*)b, xx.data(), n);
    if (st == OK) st = refine_ladder(a, pre, (const double*)b, sym_norm_inf(a), target, xx, info);
    std::memcpy(x, xx.data(), n * sizeof(double));
  } else {
    using T = Cx<double>;
    Csc<T> a;
    a.n = n;
    a.cp.assign(cp, cp + n + 1);
    a.ri.assign(ri, ri + cp[n]);
    a.v.assign((const T*)avals, (const T*)avals + cp[n]);
    LoPre<T> pre{(OracleFactor<Cx<float>>*)lo->f};
    std::vector<T> xx(n);
    st = pre.apply((const T*)b, xx.data(), n);
    if (st == OK) st = refine_ladder(a, pre, (const T*)b, sym_norm_inf(a), target, xx, info);
    std::memcpy(x, xx.data(), n * sizeof(T));
  }
  iters2[0] = info.ir_iters;
  iters2[1] = info.gmres_iters;
  *be = info.backward_error;
  *certified = info.certified;
  return st;
}

// y = A x with the stored lower triangle (CscMatrix::symv), for residual checks.
void oracle_symv(int dtype, int64_t n, const int64_t* cp, const int64_t* ri, const void* vals, const void* x, void* y) {
  if (dtype == 0) {
    Csc<double> a;
    a.n = n;
    a.cp.assign(cp, cp + n + 1);
    a.ri.assign(ri, ri + cp[n]);
    a.v.assign((const double*)vals, (const double*)vals + cp[n]);
    symv(a, (const double*)x, (double*)y);
  } else {
    using T = Cx<double>;
    Csc<T> a;
    a.n = n;
    a.cp.assign(cp, cp + n + 1);
    a.ri.assign(ri, ri + cp[n]);
    a.v.assign((const T*)vals, (const T*)vals + cp[n]);
    symv(a, (const T*)x, (T*)y);
  }
}

void oracle_free(void* hp) {
  auto* h = (Handle*)hp;
  if (!h) return;
  ORC_DISPATCH(h, delete F);
  delete h;
}

}  // extern "C"
