// sm_100a kernels of the supernodal multi-RHS solve x = s . P L^-T D^-1 L^-1 P^T (s . b)
// straight from the device-resident panels, plus the FP64 residual / norm /
// Krylov vector kernels of the refinement driver.
//
// Vectors are row-major n x nrhs (the reference RHS layout,
// src/dense/ldlt_generic.rs:556-714).  Two index spaces are used:
//   g : the analysed (fill-reducing) order — panel row structures live here;
//   e : pivot order, e = first_col(s) + pivot position inside s.
// Forward:  per level, k_chain (wave_solve.cuh) pulls every descendant's
//           push U_k = L21_k z_k into the columns of s (update-list order,
//           no atomics) and solves the unit-lower
//           diagonal blocks in pivot order with their precomputed
//           inverses, and k_stream forms U_s; D^-1 follows the whole sweep
//           (k_dsolve).
// Backward: per level (root first), k_stream forms the off-diagonal dots
//           against the ancestors' x (read through the row structure),
//           then k_chain
//           back-substitutes the diagonal blocks.
// Reference: solve_ldlt_block (src/dense/ldlt_generic.rs:618-714).
#pragma once

#include "scalar.cuh"

namespace rsd {

constexpr int SOLVE_NT = 256;
constexpr int RHS_MAX = 16;  // right-hand sides per pass (larger counts loop)
constexpr int TB = 64;       // block edge of the diagonal-block solves

struct SolveArgs {
  const int* sn_first;
  const int* sn_ncol;
  const int* sn_nrow;
  const long long* sn_poff;
  const long long* sn_rsoff;
  const int* rs;
  const int* upd_ptr;
  const int* upd_k;
  const int* upd_p0;
  const int* upd_p1;
  const void* panel;
  const void* d;
  const void* dsub;
  const unsigned char* kind;
  const int* lperm;
  void* Yg;   // n x ld, g order
  void* Ze;   // n x ld, e order
  void* Xg;   // n x ld, g order
  void* U;    // sum_s (nrow_s - ncol_s) x ld: U_s = L21_s z_s
  void* Wb;   // n x ld, e order: backward off-diagonal dots
  const long long* uoff;  // row offset of U_s
  const int* pull_ptr;    // n + 1: pull list of column g (g order)
  const int* pull_src;    // U row of each push, update-list order per g
  const int2* dots_red;   // per supernode: (first partial-sum slot, row chunks) of its split backward dots
  const void* linv;       // inverses of the TB x TB diagonal blocks of wide supernodes
  const long long* linv_off;
  void* Wp;               // slots x 32 x ld partial sums of the split backward dots
  int* wstate;            // wavefront solves: status, abort word, ticket counters, block flags
  int ld;     // row stride (total rhs count)
  int c0;     // first rhs column of this pass
  int nrhs;   // rhs columns in this pass (<= RHS_MAX)
};

// Yg[g] = s[perm[g]] * b[perm[g]] (scaled, permuted in).
template <typename T>
__global__ void k_perm_in(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ s,
                          const T* __restrict__ b, T* __restrict__ Yg) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n * nrhs) return;
  int g = (int)(idx / nrhs), c = (int)(idx % nrhs);
  int i = perm[g];
  Yg[idx] = Field<T>::scale(b[(long long)i * nrhs + c], s[i]);
}

// x[perm[g]] = s[perm[g]] * Xg[g] (permuted out, scaled back).
template <typename T>
__global__ void k_perm_out(int n, int nrhs, const int* __restrict__ perm, const double* __restrict__ s,
                           const T* __restrict__ Xg, T* __restrict__ x) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n * nrhs) return;
  int g = (int)(idx / nrhs), c = (int)(idx % nrhs);
  int i = perm[g];
  x[(long long)i * nrhs + c] = Field<T>::scale(Xg[idx], s[i]);
}

template <typename T>
__device__ __forceinline__ T shfl_T(T v, int src) {
  if constexpr (Field<T>::complex) {
    T r;
    r.re = __shfl_sync(0xffffffffu, v.re, src);
    r.im = __shfl_sync(0xffffffffu, v.im, src);
    return r;
  } else {
    return __shfl_sync(0xffffffffu, v, src);
  }
}

// Inverse of the unit lower TB x TB diagonal block [j0, j0+nb) of a
// supernode's panel (task (s, j0)), column-major into its TB x TB slot, or
// an ncol x ncol slot for a single-block supernode (only the nb x nb corner
// is written; readers zero-fill the rest).  Row-step
// substitution: for i = 1 .. nb-1 in turn, X[i, j] = -sum_{k=j}^{i-1}
// L[i, k] X[k, j] for every j < i at once, four threads per column j
// splitting k (partials added in a fixed order), so each step is a short
// dot product instead of a column-long serial chain.  Runs once per factor,
// after the supernode's panel factorization.
constexpr int DI_NT = 4 * TB;

template <typename T>
__global__ void __launch_bounds__(DI_NT) k_diag_inv(const int2* __restrict__ tasks, const int* __restrict__ sn_ncol,
                                                    const int* __restrict__ sn_nrow,
                                                    const long long* __restrict__ sn_poff, const T* __restrict__ panel,
                                                    const int* __restrict__ status, T* __restrict__ linv,
                                                    const long long* __restrict__ linv_off) {
  using F = Field<T>;
  if (status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls = reinterpret_cast<T*>(smem_raw);  // Ls[i * (TB + 1) + k] = L[i, k], k < i
  T* Xs = Ls + TB * (TB + 1);               // Xs[k * (TB + 1) + j] = X[k, j]
  const int2 tk = tasks[blockIdx.x];
  const int s = tk.x, j0 = tk.y;
  const int ncol = sn_ncol[s], nrow = sn_nrow[s];
  const int nb = min(TB, ncol - j0);
  const T* L = panel + sn_poff[s];
  for (int e = threadIdx.x; e < TB * TB; e += DI_NT) {
    const int i = e % TB, k = e / TB;
    Ls[i * (TB + 1) + k] = (i < nb && k < i) ? L[(j0 + i) + (long long)(j0 + k) * nrow] : F::zero();
    Xs[k * (TB + 1) + i] = (k == i && i < nb) ? F::one() : F::zero();
  }
  __syncthreads();
  const int j = threadIdx.x >> 2, q = threadIdx.x & 3;
  for (int i = 1; i < nb; ++i) {
    T acc = F::zero();
    if (j < i)
      for (int k = j + q; k < i; k += 4) acc = F::fma_(Ls[i * (TB + 1) + k], Xs[k * (TB + 1) + j], acc);
    // fixed-order sum of the four partials: ((p0 + p1) + (p2 + p3))
    T o = shfl_T(acc, (threadIdx.x & 31) ^ 1);
    T pair = (q & 1) ? F::add(o, acc) : F::add(acc, o);
    T o2 = shfl_T(pair, (threadIdx.x & 31) ^ 2);
    T tot = (q & 2) ? F::add(o2, pair) : F::add(pair, o2);
    if (j < i && q == 0) Xs[i * (TB + 1) + j] = F::sub(F::zero(), tot);
    __syncthreads();
  }
  // single-block supernodes store ncol x ncol (leading dimension ncol)
  const int ldo = ncol <= TB ? ncol : TB;
  T* out = linv + linv_off[s] + (long long)(j0 / TB) * TB * TB;
  for (int e = threadIdx.x; e < nb * nb; e += DI_NT) {
    const int i = e % nb, jj = e / nb;
    out[i + (long long)jj * ldo] = Xs[i * (TB + 1) + jj];
  }
}

// D^-1 on the e-indexed forward solution, after the whole forward sweep
// (ancestors' gathers need z, not D^-1 z).  1x1 and 2x2 blocks.
template <typename T>
__global__ void k_dsolve(int n, SolveArgs a) {
  using F = Field<T>;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n * a.nrhs) return;
  const int e = (int)(idx / a.nrhs), c = (int)(idx % a.nrhs);
  const T* d = reinterpret_cast<const T*>(a.d);
  const T* ds = reinterpret_cast<const T*>(a.dsub);
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0;
  const unsigned char kd = a.kind[e];
  if (kd == 0) {
    T* z = Z + (long long)e * a.ld + c;
    *z = F::mul(*z, F::recip(d[e]));
  } else if (kd == 1) {
    T d11 = d[e], d21 = ds[e], d22 = d[e + 1];
    T det = F::sub(F::mul(d11, d22), F::mul(d21, d21));
    T di = F::recip(det);
    T* z0 = Z + (long long)e * a.ld + c;
    T* z1 = Z + (long long)(e + 1) * a.ld + c;
    T a0 = *z0, a1 = *z1;
    *z0 = F::mul(F::sub(F::mul(d22, a0), F::mul(d21, a1)), di);
    *z1 = F::mul(F::sub(F::mul(d11, a1), F::mul(d21, a0)), di);
  }
}

// ---------------------------------------------------------------------------
// FP64 refinement kernels.
// ---------------------------------------------------------------------------

// r = b - A x (row-major n x nrhs) with the full symmetric CSR of A whose
// values are gathered from the stored lower triangle through `vmap`.
template <typename T>
__global__ void k_residual(int n, int nrhs, const long long* __restrict__ rp, const int* __restrict__ ci,
                           const long long* __restrict__ vmap, const T* __restrict__ val, const T* __restrict__ x,
                           const T* __restrict__ b, T* __restrict__ r) {
  using F = Field<T>;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n * nrhs) return;
  int i = (int)(idx / nrhs), c = (int)(idx % nrhs);
  T acc = F::zero();
  for (long long p = rp[i]; p < rp[i + 1]; ++p) acc = F::fma_(val[vmap[p]], x[(long long)ci[p] * nrhs + c], acc);
  r[idx] = F::sub(b[idx], acc);
}

// y = A x (same layout).
template <typename T>
__global__ void k_spmv(int n, int nrhs, const long long* __restrict__ rp, const int* __restrict__ ci,
                       const long long* __restrict__ vmap, const T* __restrict__ val, const T* __restrict__ x,
                       T* __restrict__ y) {
  using F = Field<T>;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)n * nrhs) return;
  int i = (int)(idx / nrhs), c = (int)(idx % nrhs);
  T acc = F::zero();
  for (long long p = rp[i]; p < rp[i + 1]; ++p) acc = F::fma_(val[vmap[p]], x[(long long)ci[p] * nrhs + c], acc);
  y[idx] = acc;
}

// Per-column max |v| (column c of a row-major n x nrhs) into out[c] as bits.
template <typename T>
__global__ void k_colmax(long long n, int nrhs, const T* __restrict__ v, unsigned long long* __restrict__ out) {
  __shared__ double sm[256];
  const int c = blockIdx.y;
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, Field<T>::mag(v[i * nrhs + c]));
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMax(&out[c], __double_as_longlong(sm[0]));
}

// x += dx (elementwise).
template <typename T>
__global__ void k_axpy1(long long m, const T* __restrict__ dx, T* __restrict__ x) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < m) x[i] = Field<T>::add(x[i], dx[i]);
}

// Low <-> high precision vector casts.
template <typename Hi, typename Lo>
__global__ void k_cast_down(long long m, const Hi* __restrict__ a, Lo* __restrict__ b);
template <>
__global__ void k_cast_down<double, float>(long long m, const double* __restrict__ a, float* __restrict__ b) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < m) b[i] = (float)a[i];
}
template <>
__global__ void k_cast_down<c64, c32>(long long m, const c64* __restrict__ a, c32* __restrict__ b) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < m) b[i] = c32{(float)a[i].re, (float)a[i].im};
}
template <typename Lo, typename Hi>
__global__ void k_cast_up(long long m, const Lo* __restrict__ a, Hi* __restrict__ b);
template <>
__global__ void k_cast_up<float, double>(long long m, const float* __restrict__ a, double* __restrict__ b) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < m) b[i] = (double)a[i];
}
template <>
__global__ void k_cast_up<c32, c64>(long long m, const c32* __restrict__ a, c64* __restrict__ b) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < m) b[i] = c64{(double)a[i].re, (double)a[i].im};
}

// Inertia of the factored D (per-pivot rules, multifrontal_ldlt.rs:3220-3249).
template <typename T>
__global__ void k_inertia(int n, const T* __restrict__ d, const T* __restrict__ dsub,
                          const unsigned char* __restrict__ kind, unsigned long long* __restrict__ cnt) {
  using F = Field<T>;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long pos = 0, neg = 0, zer = 0;
  if (e < n) {
    unsigned char kd = kind[e];
    if (kd == 0) {
      double r = F::real(d[e]);
      if (r > 0) pos = 1;
      else if (r < 0) neg = 1;
      else zer = 1;
    } else if (kd == 1) {
      double det_r = F::real(F::sub(F::mul(d[e], d[e + 1]), F::mul(dsub[e], dsub[e])));
      double tr_r = F::real(F::add(d[e], d[e + 1]));
      if (det_r < 0) {
        pos = 1;
        neg = 1;
      } else if (det_r > 0) {
        if (tr_r >= 0) pos = 2;
        else neg = 2;
      } else {
        zer = 1;
        if (tr_r >= 0) pos = 1;
        else neg = 1;
      }
    }
  }
  if (pos) atomicAdd(&cnt[0], pos);
  if (neg) atomicAdd(&cnt[1], neg);
  if (zer) atomicAdd(&cnt[2], zer);
}

}  // namespace rsd
