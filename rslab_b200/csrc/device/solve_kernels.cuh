// sm_100a kernels of the supernodal multi-RHS solve x = s . P L^-T D^-1 L^-1 P^T (s . b)
// straight from the device-resident panels, plus the FP64 residual / norm /
// Krylov vector kernels of the refinement driver.
//
// Vectors are row-major n x nrhs (the reference RHS layout,
// src/dense/ldlt_generic.rs:556-714).  Two index spaces are used:
//   g : the analysed (fill-reducing) order — panel row structures live here;
//   e : pivot order, e = first_col(s) + pivot position inside s.
// Forward:  per level, k_fwd_gather pulls every descendant's L_k * z_k into
//           the columns of s (update-list order, no atomics), then
//           k_fwd_diag solves the unit-lower diagonal block in pivot order and
//           applies D^-1.
// Backward: per level (root first), k_bwd dots each column of s against the
//           already-solved rows (own pivots in e order, ancestors in g order)
//           and back-substitutes the diagonal block.
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
// warps split q; result reduced through smem `red` (NW x 32 x RHS_MAX).
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
__device__ __forceinline__ void reduce_warps(T (&acc)[RHS_MAX], T* red, int nrhs) {
  using F = Field<T>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NW = SOLVE_NT / 32;
#pragma unroll
  for (int c = 0; c < RHS_MAX; ++c)
    if (c < nrhs) red[(warp * 32 + lane) * RHS_MAX + c] = acc[c];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int c = 0; c < RHS_MAX; ++c) {
      if (c >= nrhs) continue;
      T s = F::zero();
      for (int w = 0; w < NW; ++w) s = F::add(s, red[(w * 32 + lane) * RHS_MAX + c]);
      acc[c] = s;
    }
  }
  __syncthreads();
}

// Pivot-order unit-lower substitution of columns [j_begin, j_end) of a panel
// in 32-column blocks (one CTA): z[p] = y[p] - sum_{q in [q_begin, p)} L[p,q] z[q].
// y comes from the g-ordered RHS through lperm (from_y) or already sits in Z.
template <typename T>
__device__ void fwd_block_range(const SolveArgs& a, const T* __restrict__ L, int nrow, T* Z, const T* Yfirst,
                                const int* __restrict__ lp, int j_begin, int j_end, int q_begin, bool from_y, T* red) {
  using F = Field<T>;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j0 = j_begin; j0 < j_end; j0 += SB) {
    const int nb = min(SB, j_end - j0);
    T acc[RHS_MAX];
#pragma unroll
    for (int c = 0; c < RHS_MAX; ++c) acc[c] = F::zero();
    lane_row_dot<T>(acc, L + j0 + lane, nrow, q_begin, j0, Z, a.ld, a.nrhs, lane < nb);
    reduce_warps<T>(acc, red, a.nrhs);
    if (warp == 0) {
      T z[RHS_MAX];
      const int p = j0 + lane;
      const bool ok = lane < nb;
      const T* yrow = from_y ? Yfirst + (long long)((ok ? lp[p] : 0)) * a.ld : Z + (long long)(ok ? p : 0) * a.ld;
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c) z[c] = (ok && c < a.nrhs) ? F::sub(yrow[c], acc[c]) : F::zero();
      for (int q = 0; q < nb; ++q) {
        const int qq = j0 + q;
        T l = F::zero();
        if (ok && lane > q) l = L[p + (long long)qq * nrow];
#pragma unroll
        for (int c = 0; c < RHS_MAX; ++c) {
          if (c >= a.nrhs) continue;
          T zq;
          if constexpr (Field<T>::complex) {
            zq.re = __shfl_sync(0xffffffffu, z[c].re, q);
            zq.im = __shfl_sync(0xffffffffu, z[c].im, q);
          } else {
            zq = __shfl_sync(0xffffffffu, z[c], q);
          }
          z[c] = F::fnma(l, zq, z[c]);
        }
      }
      if (ok)
#pragma unroll
        for (int c = 0; c < RHS_MAX; ++c)
          if (c < a.nrhs) Z[(long long)p * a.ld + c] = z[c];
    }
    __syncthreads();
  }
}

// Forward step of supernode s (one CTA):
//  1. pull the descendants' pushes: y[g] -= U_k[r] for every updater k (in
//     update-list order) and its off-diagonal rows r landing in s's columns;
//  2. pivot-order unit-lower substitution of the diagonal block in 32-column
//     blocks (left-looking inside the panel) -> z_s (e order); supernodes
//     wider than SOLVE_BIG only stage y here and are solved by the blocked
//     multi-CTA kernels k_ftrsv_blk / k_ftrsv_upd.
// The push U_s = L21_s z_s (k_fwd_push) follows as a separate launch.
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_fwd_diag(SolveArgs a, const int* __restrict__ tasks) {
  using F = Field<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);
  const int s = tasks[blockIdx.x];
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  const int* lp = a.lperm + first;
  T* Y = reinterpret_cast<T*>(a.Yg) + a.c0;
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  T* Uall = reinterpret_cast<T*>(a.U) + a.c0;
  // 1. gather the pushes of the updaters (distinct rows within one updater).
  for (int u = a.upd_ptr[s]; u < a.upd_ptr[s + 1]; ++u) {
    const int k = a.upd_k[u], p0 = a.upd_p0[u], p1 = a.upd_p1[u];
    const int* ok = a.rs + a.sn_rsoff[k] + a.sn_ncol[k];
    const T* Uk = Uall + a.uoff[k] * a.ld;
    const int cnt = (p1 - p0) * a.nrhs;
    for (int e = threadIdx.x; e < cnt; e += SOLVE_NT) {
      const int r = p0 + e / a.nrhs, c = e % a.nrhs;
      T* y = Y + (long long)ok[r] * a.ld + c;
      *y = F::sub(*y, Uk[(long long)r * a.ld + c]);
    }
    __syncthreads();
  }
  // 2. diagonal block: in this CTA for narrow supernodes; wide ones only
  //    stage y in pivot order into Z for the blocked multi-CTA solve.
  if (ncol > SOLVE_BIG) {
    for (int e = threadIdx.x; e < ncol * a.nrhs; e += SOLVE_NT) {
      const int p = e / a.nrhs, c = e % a.nrhs;
      Z[(long long)p * a.ld + c] = Y[(long long)(first + lp[p]) * a.ld + c];
    }
    return;
  }
  fwd_block_range<T>(a, L, nrow, Z, Y + (long long)first * a.ld, lp, 0, ncol, 0, true, red);
}

// Forward push of supernode s, rows [ncol + r0, ncol + r0 + 64):
// U_s = L21_s z_s.  Two 32-row lane groups x four q-splits (warps); the
// q-split partial sums are added in a fixed order (deterministic).
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_fwd_push(SolveArgs a, const int2* __restrict__ tasks) {
  using F = Field<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);  // [4 splits][64 rows][RHS_MAX]
  const int2 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = tk.y;
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  const T* Z = reinterpret_cast<const T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  T* Us = reinterpret_cast<T*>(a.U) + a.c0 + a.uoff[s] * a.ld;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rg = warp & 1, qs = warp >> 1;  // row group, q split
  const int rl = rg * 32 + lane;            // local row 0..63
  const int r = ncol + r0 + rl;
  const bool ok = r < nrow;
  T acc[RHS_MAX];
#pragma unroll
  for (int c = 0; c < RHS_MAX; ++c) acc[c] = F::zero();
  for (int q = qs; q < ncol; q += 4) {
    T l = ok ? L[r + (long long)q * nrow] : F::zero();
    const T* zq = Z + (long long)q * a.ld;
#pragma unroll
    for (int c = 0; c < RHS_MAX; ++c)
      if (c < a.nrhs) acc[c] = F::fma_(l, zq[c], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < RHS_MAX; ++c)
    if (c < a.nrhs) red[(qs * 64 + rl) * RHS_MAX + c] = acc[c];
  __syncthreads();
  for (int e = threadIdx.x; e < 64 * a.nrhs; e += SOLVE_NT) {
    const int row = e / a.nrhs, c = e % a.nrhs;
    const int rr = ncol + r0 + row;
    if (rr >= nrow) continue;
    T v = red[(0 * 64 + row) * RHS_MAX + c];
    v = F::add(v, red[(1 * 64 + row) * RHS_MAX + c]);
    v = F::add(v, red[(2 * 64 + row) * RHS_MAX + c]);
    v = F::add(v, red[(3 * 64 + row) * RHS_MAX + c]);
    Us[(long long)(rr - ncol) * a.ld + c] = v;
  }
}

// out[p][c] = sum_{r in [r_begin, r_end)} L[r, p] * V(r)[c] for the 32
// columns p in [p0, p0+32) of a panel, V(r) = the RHS row of panel row r
// (gathered through rs for ancestor rows).  32-row chunks of V and of the
// L tile are staged in shared memory and reused by all 32 columns; thread t
// owns column t % 32 and right-hand sides t / 32 + 8 i; fixed summation order.
template <typename T, bool GATHER>
__device__ void dot_cols_tile(const T* __restrict__ L, int nrow, int p0, int ncols, int r_begin, int r_end,
                              const T* __restrict__ V, const int* __restrict__ rss, int ld, int nrhs,
                              T (&acc)[RHS_MAX / 8], T* Ls, T* Vs) {
  using F = Field<T>;
  constexpr int NRC = RHS_MAX / 8;
  const int tid = threadIdx.x, pc = tid & 31, cg = tid >> 5;
#pragma unroll
  for (int q = 0; q < NRC; ++q) acc[q] = F::zero();
  for (int r0 = r_begin; r0 < r_end; r0 += 32) {
    const int rows = min(32, r_end - r0);
    for (int e = tid; e < 32 * 32; e += SOLVE_NT) {
      const int c = e >> 5, r = e & 31;  // column c, row r: coalesced along r
      Ls[r * 33 + c] = (r < rows && c < ncols) ? L[(r0 + r) + (long long)(p0 + c) * nrow] : F::zero();
    }
    for (int e = tid; e < 32 * nrhs; e += SOLVE_NT) {
      const int r = e / nrhs, c = e % nrhs;
      T v = F::zero();
      if (r < rows) {
        const long long row = GATHER ? (long long)rss[r0 + r] : (long long)(r0 + r);
        v = V[row * ld + c];
      }
      Vs[r * RHS_MAX + c] = v;
    }
    __syncthreads();
    for (int r = 0; r < rows; ++r) {
      const T l = Ls[r * 33 + pc];
#pragma unroll
      for (int q = 0; q < NRC; ++q) {
        const int c = cg + 8 * q;
        if (c < nrhs) acc[q] = F::fma_(l, Vs[r * RHS_MAX + c], acc[q]);
      }
    }
    __syncthreads();
  }
}

// Backward off-diagonal dots of supernode s, pivot columns [c0, c0+32):
// sum_{r >= ncol} L[r, p] x[g_r] -> Wb (narrow supernodes) or subtracted from
// Z directly (wide supernodes, solved by the blocked kernels).
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_bwd_off(SolveArgs a, const int2* __restrict__ tasks) {
  using F = Field<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls = reinterpret_cast<T*>(smem_raw);  // 32 x 33
  T* Vs = Ls + 32 * 33;                    // 32 x RHS_MAX
  const int2 tk = tasks[blockIdx.x];
  const int s = tk.x, c0 = tk.y;
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  const int* rss = a.rs + a.sn_rsoff[s];
  const T* X = reinterpret_cast<const T*>(a.Xg) + a.c0;
  T* Wb = reinterpret_cast<T*>(a.Wb) + a.c0 + (long long)first * a.ld;
  T* Zs = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  const int cols_here = min(32, ncol - c0);
  T acc[RHS_MAX / 8];
  dot_cols_tile<T, true>(L, nrow, c0, cols_here, ncol, nrow, X, rss, a.ld, a.nrhs, acc, Ls, Vs);
  const int pc = threadIdx.x & 31, cg = threadIdx.x >> 5;
  if (pc < cols_here) {
    const int p = c0 + pc;
#pragma unroll
    for (int q = 0; q < RHS_MAX / 8; ++q) {
      const int c = cg + 8 * q;
      if (c >= a.nrhs) continue;
      if (ncol > SOLVE_BIG) {
        T* z = Zs + (long long)p * a.ld + c;
        *z = F::sub(*z, acc[q]);
      } else {
        Wb[(long long)p * a.ld + c] = acc[q];
      }
    }
  }
}

// Blocked forward solve of a wide supernode, block [j0, j0+64): in-block
// substitution on Z (which already holds y minus the earlier blocks).
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_ftrsv_blk(SolveArgs a, const int4* __restrict__ tasks) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, j0 = tk.y;
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  fwd_block_range<T>(a, L, nrow, Z, nullptr, nullptr, j0, min(j0 + TB, ncol), j0, false, red);
}

// Right-looking update after forward block [j0, j0+64) of a wide supernode:
// Z[r] -= sum_{q in block} L[r, q] z[q] for own rows r in [r0, r0+64).
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_ftrsv_upd(SolveArgs a, const int4* __restrict__ tasks) {
  using F = Field<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);  // [4 splits][64 rows][RHS_MAX]
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, j0 = tk.y, r0 = tk.z;
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const int j1 = min(j0 + TB, ncol);
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int rg = warp & 1, qs = warp >> 1;
  const int rl = rg * 32 + lane;
  const int r = r0 + rl;
  const bool ok = r < ncol;
  T acc[RHS_MAX];
#pragma unroll
  for (int c = 0; c < RHS_MAX; ++c) acc[c] = F::zero();
  for (int q = j0 + qs; q < j1; q += 4) {
    T l = ok ? L[r + (long long)q * nrow] : F::zero();
    const T* zq = Z + (long long)q * a.ld;
#pragma unroll
    for (int c = 0; c < RHS_MAX; ++c)
      if (c < a.nrhs) acc[c] = F::fma_(l, zq[c], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < RHS_MAX; ++c)
    if (c < a.nrhs) red[(qs * 64 + rl) * RHS_MAX + c] = acc[c];
  __syncthreads();
  for (int e = threadIdx.x; e < 64 * a.nrhs; e += SOLVE_NT) {
    const int row = e / a.nrhs, c = e % a.nrhs;
    const int rr = r0 + row;
    if (rr >= ncol) continue;
    T v = red[(0 * 64 + row) * RHS_MAX + c];
    v = F::add(v, red[(1 * 64 + row) * RHS_MAX + c]);
    v = F::add(v, red[(2 * 64 + row) * RHS_MAX + c]);
    v = F::add(v, red[(3 * 64 + row) * RHS_MAX + c]);
    T* z = Z + (long long)rr * a.ld + c;
    *z = F::sub(*z, v);
  }
}

// Blocked backward solve of a wide supernode, block [j0, j0+64): in-block
// substitution with L^T (v already holds w - L21^T x - later blocks), then
// the block's final values go to X in g order.
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_btrsv_blk(SolveArgs a, const int4* __restrict__ tasks) {
  using F = Field<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);
  T* vb = red + (SOLVE_NT / 32) * 32 * RHS_MAX;
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, jb = tk.y;
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const int je = min(jb + TB, ncol);
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  const int* lp = a.lperm + first;
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  T* Xw = reinterpret_cast<T*>(a.Xg) + a.c0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = SOLVE_NT / 32;
  const int nblk = (je - jb + SB - 1) / SB;
  for (int b = nblk - 1; b >= 0; --b) {
    const int j0 = jb + b * SB, nb = min(SB, je - j0), j1 = j0 + nb;
    for (int pc = warp; pc < nb; pc += NW) {
      const int p = j0 + pc;
      T acc[RHS_MAX];
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c) acc[c] = F::zero();
      const T* Lc = L + (long long)p * nrow;
      for (int r = j1 + lane; r < je; r += 32) {
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
    __syncthreads();
    if (warp == 0) {
      const int p = j0 + lane;
      const bool ok = lane < nb;
      T v[RHS_MAX];
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c)
        v[c] = (ok && c < a.nrhs) ? F::sub(Z[(long long)p * a.ld + c], vb[lane * RHS_MAX + c]) : F::zero();
      for (int q = nb - 1; q >= 1; --q) {
        const int qq = j0 + q;
        T l = F::zero();
        if (ok && lane < q) l = L[qq + (long long)p * nrow];
#pragma unroll
        for (int c = 0; c < RHS_MAX; ++c) {
          if (c >= a.nrhs) continue;
          T vq;
          if constexpr (Field<T>::complex) {
            vq.re = __shfl_sync(0xffffffffu, v[c].re, q);
            vq.im = __shfl_sync(0xffffffffu, v[c].im, q);
          } else {
            vq = __shfl_sync(0xffffffffu, v[c], q);
          }
          v[c] = F::fnma(l, vq, v[c]);
        }
      }
      if (ok) {
        T* xo = Xw + (long long)(first + lp[p]) * a.ld;
#pragma unroll
        for (int c = 0; c < RHS_MAX; ++c)
          if (c < a.nrhs) {
            Z[(long long)p * a.ld + c] = v[c];
            xo[c] = v[c];
          }
      }
    }
    __syncthreads();
  }
}

// Right-looking backward update after block [jb, jb+64) of a wide supernode:
// v[p] -= sum_{r in block} L[r, p] v[r] for columns p in [c0, c0+32) < jb.
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_btrsv_upd(SolveArgs a, const int4* __restrict__ tasks) {
  using F = Field<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls = reinterpret_cast<T*>(smem_raw);
  T* Vs = Ls + 32 * 33;
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, jb = tk.y, c0 = tk.z;
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const int je = min(jb + TB, ncol);
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  const int cols_here = min(32, jb - c0);
  T acc[RHS_MAX / 8];
  dot_cols_tile<T, false>(L, nrow, c0, cols_here, jb, je, Z, nullptr, a.ld, a.nrhs, acc, Ls, Vs);
  const int pc = threadIdx.x & 31, cg = threadIdx.x >> 5;
  if (pc < cols_here) {
    const int p = c0 + pc;
#pragma unroll
    for (int q = 0; q < RHS_MAX / 8; ++q) {
      const int c = cg + 8 * q;
      if (c >= a.nrhs) continue;
      T* z = Z + (long long)p * a.ld + c;
      *z = F::sub(*z, acc[q]);
    }
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

// Backward solve of supernode s (one CTA): blocks of 32 pivots from the
// last; each column dotted against the solved rows below it.
template <typename T>
__global__ void __launch_bounds__(SOLVE_NT) k_bwd(SolveArgs a, const int* __restrict__ tasks) {
  using F = Field<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* red = reinterpret_cast<T*>(smem_raw);
  T* vb = red + (SOLVE_NT / 32) * 32 * RHS_MAX;  // [32 rows of the block] x RHS_MAX
  const int s = tasks[blockIdx.x];
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  const int* lp = a.lperm + first;
  T* Z = reinterpret_cast<T*>(a.Ze) + a.c0 + (long long)first * a.ld;
  const T* Wb = reinterpret_cast<const T*>(a.Wb) + a.c0 + (long long)first * a.ld;
  T* Xw = reinterpret_cast<T*>(a.Xg) + a.c0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = SOLVE_NT / 32;
  const int nblk = (ncol + SB - 1) / SB;
  const bool has_off = nrow > ncol;  // Wb is written by k_bwd_off only then
  for (int b = nblk - 1; b >= 0; --b) {
    const int j0 = b * SB, nb = min(SB, ncol - j0), j1 = j0 + nb;
    // acc[p][c] = sum_{r >= j1} L[r, p] * v(r): warp per column p, lanes over r.
    for (int pc = warp; pc < nb; pc += NW) {
      const int p = j0 + pc;
      T acc[RHS_MAX];
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c) acc[c] = F::zero();
      const T* Lc = L + (long long)p * nrow;
      for (int r = j1 + lane; r < ncol; r += 32) {
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
    __syncthreads();
    if (warp == 0) {
      const int p = j0 + lane;
      const bool ok = lane < nb;
      T v[RHS_MAX];
#pragma unroll
      for (int c = 0; c < RHS_MAX; ++c)
        v[c] = (ok && c < a.nrhs)
                   ? F::sub(has_off ? F::sub(Z[(long long)p * a.ld + c], Wb[(long long)p * a.ld + c])
                                    : Z[(long long)p * a.ld + c],
                            vb[lane * RHS_MAX + c])
                   : F::zero();
      // Backward inside the block: v[p] -= L[q, p] v[q] for q > p.
      for (int q = nb - 1; q >= 1; --q) {
        const int qq = j0 + q;
        T l = F::zero();
        if (ok && lane < q) l = L[qq + (long long)p * nrow];
#pragma unroll
        for (int c = 0; c < RHS_MAX; ++c) {
          if (c >= a.nrhs) continue;
          T vq;
          if constexpr (Field<T>::complex) {
            vq.re = __shfl_sync(0xffffffffu, v[c].re, q);
            vq.im = __shfl_sync(0xffffffffu, v[c].im, q);
          } else {
            vq = __shfl_sync(0xffffffffu, v[c], q);
          }
          v[c] = F::fnma(l, vq, v[c]);
        }
      }
      if (ok) {
        T* xo = Xw + (long long)(first + lp[p]) * a.ld;
#pragma unroll
        for (int c = 0; c < RHS_MAX; ++c)
          if (c < a.nrhs) {
            Z[(long long)p * a.ld + c] = v[c];
            xo[c] = v[c];
          }
      }
    }
    __syncthreads();
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
