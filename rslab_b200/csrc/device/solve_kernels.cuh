// sm_100a kernels of the supernodal multi-RHS solve x = s . P L^-T D^-1 L^-1 P^T (s . b)
// straight from the device-resident panels, plus the FP64 residual / norm /
// Krylov vector kernels of the refinement driver.
//
// Vectors are row-major n x nrhs (the reference RHS layout,
// src/dense/ldlt_generic.rs:556-714).  Two index spaces are used:
//   g : the analysed (fill-reducing) order — panel row structures live here;
//   e : pivot order, e = first_col(s) + pivot position inside s.
// Forward:  per level, k_fwd_gather pulls every descendant's push
//           U_k = L21_k z_k into the columns of s (update-list order, no
//           atomics), k_fwd_diag (narrow) or k_chain (wide, wave_solve.cuh)
//           solve the unit-lower diagonal block in pivot order, and
//           k_stream forms U_s; D^-1 follows the whole sweep (k_dsolve).
// Backward: per level (root first), k_bwd_gather / k_stream form the
//           off-diagonal dots against the ancestors' x, then k_bwd (narrow)
//           or k_chain (wide) back-substitute the diagonal block.
// Reference: solve_ldlt_block (src/dense/ldlt_generic.rs:618-714).
#pragma once

#include "scalar.cuh"

namespace rsd {

constexpr int SOLVE_NT = 256;
constexpr int RHS_MAX = 16;  // right-hand sides per pass (larger counts loop)
constexpr int SB = 32;       // diagonal-block edge of the in-CTA substitutions
constexpr int SOLVE_BIG = 128;  // wider supernodes use the multi-CTA blocked diagonal solves
constexpr int TB = 64;          // block edge of the multi-CTA diagonal solves

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

// acc[c] += sum_{q in [q_begin, q_end)} L[r, q] * V[q][c]: one lane per row r,
// warps split q (stride NW); the partial sums are reduced through smem.
template <typename T>
__device__ __forceinline__ void lane_row_dot(T (&acc)[RHS_MAX], const T* __restrict__ Lrow, long long ld,
                                             int q_begin, int q_end, const T* __restrict__ V, int vld, int nrhs,
                                             bool row_ok) {
  using F = Field<T>;
  const int warp = threadIdx.x >> 5;
  constexpr int NW = SOLVE_NT / 32;
  for (int q = q_begin + warp; q < q_end; q += NW) {
    T l = row_ok ? Lrow[(long long)q * ld] : F::zero();
    const T* v = V + (long long)q * vld;
#pragma unroll
    for (int c = 0; c < RHS_MAX; ++c)
      if (c < nrhs) acc[c] = F::fma_(l, v[c], acc[c]);
  }
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

// Ls[i * 33 + j] = L[j0 + i, j0 + j] for j < i < nb (strict lower part of the
// nb x nb diagonal block), zero elsewhere.  Loads coalesced along i.
template <typename T>
__device__ __forceinline__ void stage_diag_block(const T* __restrict__ L, int nrow, int j0, int nb, T* Ls) {
#pragma unroll
  for (int e = threadIdx.x; e < SB * SB; e += SOLVE_NT) {
    const int i = e & (SB - 1), j = e / SB;
    Ls[i * (SB + 1) + j] = (i < nb && j < i) ? L[(j0 + i) + (long long)(j0 + j) * nrow] : Field<T>::zero();
  }
}

// Pivot-order unit-lower substitution of columns [j_begin, j_end) of a panel
// in 32-column blocks (one CTA), in place on Z (pivot order, holding y):
//   z[p] = y[p] - sum_{q in [q_begin, p)} L[p,q] z[q].
// Per block: the left part [q_begin, j0) is a warp-split dot whose partial
// sums are added in warp order; the diagonal block is staged in shared memory
// and every warp substitutes its own right-hand sides (c = warp, warp + NW, ..)
// with one lane per row, so no warp waits on a global load inside the
// 32-step dependency chain.  Per (p, c) the operation sequence is fixed:
// z = y - left; then z -= L[p,q] z[q] for q ascending.
template <typename T>
__device__ void fwd_block_range(const SolveArgs& a, const T* __restrict__ L, int nrow, T* Z, int j_begin, int j_end,
                                int q_begin, T* red, T* Ls, T* zb) {
  using F = Field<T>;
  constexpr int NW = SOLVE_NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j0 = j_begin; j0 < j_end; j0 += SB) {
    const int nb = min(SB, j_end - j0);
    const bool left = j0 > q_begin;
    if (left) {
      T acc[RHS_MAX];
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c) acc[c] = F::zero();
      lane_row_dot<T>(acc, L + j0 + lane, nrow, q_begin, j0, Z, a.ld, a.nrhs, lane < nb);
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c)
        if (c < a.nrhs) red[(warp * 32 + lane) * RHS_MAX + c] = acc[c];
    }
    stage_diag_block<T>(L, nrow, j0, nb, Ls);
    __syncthreads();
    for (int e = threadIdx.x; e < SB * RHS_MAX; e += SOLVE_NT) {
      const int i = e & (SB - 1), c = e / SB;
      if (c >= a.nrhs) continue;
      T v = F::zero();
      if (i < nb) {
        v = Z[(long long)(j0 + i) * a.ld + c];
        if (left) {
          T s = F::zero();
          for (int w = 0; w < NW; ++w) s = F::add(s, red[(w * 32 + i) * RHS_MAX + c]);
          v = F::sub(v, s);
        }
      }
      zb[i * RHS_MAX + c] = v;
    }
    __syncthreads();
    for (int c = warp; c < a.nrhs; c += NW) {
      T z = zb[lane * RHS_MAX + c];
#pragma unroll
      for (int q = 0; q < SB; ++q) {
        if (q < nb) {
          const T zq = shfl_T(z, q);
          z = F::fnma(Ls[lane * (SB + 1) + q], zq, z);
        }
      }
      if (lane < nb) Z[(long long)(j0 + lane) * a.ld + c] = z;
    }
    __syncthreads();
  }
}

// Forward gather of supernode s, pivot positions [p0, p0 + 16) (thread =
// position x right-hand side): Z[p] = Y[g] minus every push U_k[r] that lands
// on g = first + lperm[p], in update-list order (the pull list of g, built
// at analysis).  No atomics and no block-wide barrier per updater.
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_fwd_gather(SolveArgs a, const int2* __restrict__ tasks) {
  using F = Field<T>;
  const int2 tk = tasks[blockIdx.x];
  const int s = tk.x, p = tk.y + (int)(threadIdx.x / RHS_MAX), c = (int)(threadIdx.x % RHS_MAX);
  const int first = a.sn_first[s], ncol = a.sn_ncol[s];
  if (p >= ncol || c >= a.nrhs) return;
  const int g = first + a.lperm[first + p];
  const T* U = reinterpret_cast<const T*>(a.U) + a.c0 + c;
  T y = reinterpret_cast<const T*>(a.Yg)[a.c0 + (long long)g * a.ld + c];
  const int t0 = a.pull_ptr[g], t1 = a.pull_ptr[g + 1];
#pragma unroll 4
  for (int t = t0; t < t1; ++t) y = F::sub(y, U[(long long)a.pull_src[t] * a.ld]);
  reinterpret_cast<T*>(a.Ze)[a.c0 + (long long)(first + p) * a.ld + c] = y;
}

// Forward diagonal block of a narrow supernode s (ncol <= SOLVE_BIG, one
// CTA): Z already holds the gathered y in pivot order; solve in place.
// Wider supernodes use the block chain (k_chain).
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_fwd_diag(SolveArgs a, const int* __restrict__ tasks) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);        // NW x 32 x RHS_MAX
  T* Ls = red + (SOLVE_NT / 32) * 32 * RHS_MAX;  // 32 x 33
  T* zb = Ls + SB * (SB + 1);                    // 32 x RHS_MAX
  const int s = tasks[blockIdx.x];
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  fwd_block_range<T>(a, L, nrow, Z, 0, ncol, 0, red, Ls, zb);
}

// Inverse of the unit lower TB x TB diagonal block [j0, j0+nb) of a wide
// supernode's panel (task (s, j0)), column-major into its TB x TB slot;
// thread j forms column j by forward substitution, x_i = -sum_k L_ik x_k.
// Runs once per factor, after the supernode's panel factorization.
template <typename T>
__global__ void __launch_bounds__(TB) k_diag_inv(const int2* __restrict__ tasks, const int* __restrict__ sn_ncol,
                                                 const int* __restrict__ sn_nrow, const long long* __restrict__ sn_poff,
                                                 const T* __restrict__ panel, const int* __restrict__ status,
                                                 T* __restrict__ linv, const long long* __restrict__ linv_off) {
  using F = Field<T>;
  if (status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls = reinterpret_cast<T*>(smem_raw);  // TB x (TB + 1), row i at i * (TB + 1)
  T* Xs = Ls + TB * (TB + 1);               // TB x (TB + 1)
  const int2 tk = tasks[blockIdx.x];
  const int s = tk.x, j0 = tk.y;
  const int ncol = sn_ncol[s], nrow = sn_nrow[s];
  const int nb = min(TB, ncol - j0);
  const T* L = panel + sn_poff[s];
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
    const int i = e % TB, j = e / TB;
    Ls[i * (TB + 1) + j] = (i < nb && j < i) ? L[(j0 + i) + (long long)(j0 + j) * nrow] : F::zero();
  }
  __syncthreads();
  const int j = threadIdx.x;
  if (j < TB) {
    for (int i = 0; i < TB; ++i) Xs[i * (TB + 1) + j] = (i == j && j < nb) ? F::one() : F::zero();
    if (j < nb)
      for (int i = j + 1; i < nb; ++i) {
        T acc = F::zero();
        for (int k = j; k < i; ++k) acc = F::fma_(Ls[i * (TB + 1) + k], Xs[k * (TB + 1) + j], acc);
        Xs[i * (TB + 1) + j] = F::sub(F::zero(), acc);
      }
  }
  __syncthreads();
  T* out = linv + linv_off[s] + (long long)(j0 / TB) * TB * TB;
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
    const int i = e % TB, jj = e / TB;
    out[i + (long long)jj * TB] = Xs[i * (TB + 1) + jj];
  }
}

// Backward substitution of pivot columns [jb, je) of a panel in 32-column
// blocks from the last (one CTA), in place on Z; final values also go to X
// (g order).  Per block: v[p] -= sum_{r in [j1, r_end)} L[r, p] v[r] over
// the solved rows below it (warp per column, lanes over r, shuffle tree),
// then the transposed in-block substitution from a shared-memory copy of
// the diagonal block, warps over right-hand sides, lanes over rows.
// Per (p, c): v = Z[p] (- Wb[p] when given) - below; then v -= L[q,p] v[q]
// for q descending.
template <typename T>
__device__ void bwd_block_range(const SolveArgs& a, const T* __restrict__ L, int nrow, T* Z, const T* Wb, T* Xw,
                                const int* __restrict__ lp, int first, int jb, int je, int r_end, T* vb, T* Ls) {
  using F = Field<T>;
  constexpr int NW = SOLVE_NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nblk = (je - jb + SB - 1) / SB;
  for (int b = nblk - 1; b >= 0; --b) {
    const int j0 = jb + b * SB, nb = min(SB, je - j0), j1 = j0 + nb;
    for (int pc = warp; pc < nb; pc += NW) {
      const int p = j0 + pc;
      T acc[RHS_MAX];
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c) acc[c] = F::zero();
      const T* Lc = L + (long long)p * nrow;
      for (int r = j1 + lane; r < r_end; r += 32) {
        T l = Lc[r];
        const T* v = Z + (long long)r * a.ld;
#pragma unroll
        for (int c = 0; c < RHS_MAX; ++c)
          if (c < a.nrhs) acc[c] = F::fma_(l, v[c], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c) {
        if (c >= a.nrhs) continue;
        T x = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          if constexpr (Field<T>::complex) {
            x.re += __shfl_down_sync(0xffffffffu, x.re, o);
            x.im += __shfl_down_sync(0xffffffffu, x.im, o);
          } else {
            x += __shfl_down_sync(0xffffffffu, x, o);
          }
        }
        if (lane == 0) vb[pc * RHS_MAX + c] = x;
      }
    }
    stage_diag_block<T>(L, nrow, j0, nb, Ls);
    __syncthreads();
    const int p = j0 + lane;
    const bool ok = lane < nb;
    for (int c = warp; c < a.nrhs; c += NW) {
      T v = F::zero();
      if (ok) {
        v = Z[(long long)p * a.ld + c];
        if (Wb) v = F::sub(v, Wb[(long long)p * a.ld + c]);
        v = F::sub(v, vb[lane * RHS_MAX + c]);
      }
#pragma unroll
      for (int q = SB - 1; q >= 1; --q) {
        if (q < nb) {
          const T vq = shfl_T(v, q);
          v = F::fnma(Ls[q * (SB + 1) + lane], vq, v);
        }
      }
      if (ok) {
        Z[(long long)p * a.ld + c] = v;
        Xw[(long long)(first + lp[p]) * a.ld + c] = v;
      }
    }
    __syncthreads();
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

// Backward solve of a narrow supernode s (one CTA): blocks of 32 pivots
// from the last; the off-diagonal dots (Wb, k_stream) come first.
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_bwd(SolveArgs a, const int* __restrict__ tasks) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls = reinterpret_cast<T*>(smem_raw);  // 32 x 33
  T* vb = Ls + SB * (SB + 1);              // 32 x RHS_MAX
  const int s = tasks[blockIdx.x];
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  // Wb is written by the dots only when the supernode has off-diagonal rows
  const T* Wb = nrow > ncol ? reinterpret_cast<const T*>(a.Wb) + a.c0 + (long long)first * a.ld : nullptr;
  bwd_block_range<T>(a, L, nrow, Z, Wb, reinterpret_cast<T*>(a.Xg) + a.c0, a.lperm + first, first, 0, ncol, ncol,
                     vb, Ls);
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
