// sm_100a kernels of the supernodal left-looking Bunch-Kaufman LDL^T factor.
//
// Data layout in HBM (one pool per factor handle, offsets fixed at analysis):
//   panel[s]  : nrow_s x ncol_s column-major (stride nrow_s) at poff[s]; after
//               the factor rows/cols are in the panel's pivot order, the
//               strictly-lower part holds L (2x2 coupling entry = d21, never
//               read as L), the diagonal holds D.
//   e-indexed : d[n], dsub[n], kind[n] (0 = 1x1, 1/2 = first/second column of
//               a 2x2 block), lperm[n] (pivot position -> pre-pivot local
//               column) — e = first_col(s) + pivot position.
// Kernels (one level of the assembly tree per launch group):
//   k_assemble      scatter-add of the equilibrated A (precomputed targets)
//   k_cmod          tile-owner gather of every descendant update (deterministic
//                   updater order, no atomics) — ll_factor_node cmod
//   k_getf2         panel-bounded BK on one nb-wide block — ll_cdiv_emit getf2
//   k_deep          deep-row replay of a block's swaps/transforms —
//                   apply_bk_panel_trailing
//   k_schur         deferred in-panel Schur update of the remaining columns
// Reference: src/numeric/multifrontal_ldlt.rs:2400-3256, 1347-1408.
#pragma once

#include "async_copy.cuh"
#include "scalar.cuh"

namespace rsd {

constexpr int TILE = 64;      // output tile edge of the GEMM-class kernels
constexpr int TPB = 256;      // threads per CTA of the GEMM-class kernels
constexpr int FUSE_DEEP_ROWS = 192;  // getf2 replays this many deep rows itself
constexpr int EA_ROWS = 1024;        // front rows per extend-add task
// Blocks of at most this many columns with at most this many deep rows run
// on the 128-thread getf2 (registers capped so several CTAs share an SM).
constexpr int GETF2_NARROW_PW = 32, GETF2_NARROW_DEEP = 96;
__host__ __device__ constexpr int getf2_narrow_minb(size_t es) { return es >= 16 ? 4 : 8; }
// CTAs per SM the 512-thread getf2 is compiled for (64 registers a thread
// for 4- and 8-byte fields)
__host__ __device__ constexpr int getf2_wide_minb(size_t es) { return es >= 16 ? 1 : 2; }
// ... and the 256-thread one, used for launches of many blocks
__host__ __device__ constexpr int getf2_mid_minb(size_t es) { return es >= 16 ? 2 : 4; }
// Tensor engine of the single-precision fields: getf2 launches of at least
// this many blocks use the right-looking kernel (two CTAs per SM) rather
// than the left-looking one (one CTA per SM, shorter steps).
constexpr int GETF2_LL_MAX_TASKS = 2 * 148;

struct FactorArgs {
  // structure (device)
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
  // numeric state
  void* panel;
  void* d;
  void* dsub;
  unsigned char* kind;
  int* lperm;
  void* scratch;        // per getf2 slot: snap[nb*nb] T + swaps[nb] int, then the block transform M[nb*nb] T
  long long scratch_stride;  // bytes per slot
  int* status;          // [0] = error code, [1] = first failing supernode, [2] = n_perturbed
  double perturb_floor; // < 0: exact mode
  void* gpool;          // G_k = L21_k D_k, (nrow_k - ncol_k) x ncol_k at goff[k] (tensor-core cmod)
  const long long* goff;
  const double* floor_dev;  // non-null: static-pivot floor computed on the device (force-accept)
  int deep_mm;              // tall panels: getf2 forms the block transform M, k_deep_mm applies it
  // Multifrontal variant: the contribution blocks of the fronts, supernode
  // s's (nrow - ncol)^2 column-major block at cb_off[s].
  void* cbpool;
  const long long* cb_off;
  // Pivot record (e-indexed, block-local): kp for a 1x1 step at e, -(kp + 1)
  // for a 2x2 step starting at e.  Written by every factor that searches; when
  // *pivot_reuse is set, getf2 replays the recorded steps instead of searching
  // (static pivot reuse across a value sweep of one pattern).
  int* pivrec;
  const int* pivot_reuse;
};

// Byte offset of the block transform M in a getf2 scratch slot, and the slot
// size, for panel width nb and element size es.
__host__ __device__ constexpr long long replay_mm_off(long long nb, long long es) {
  return (nb * nb * es + 3 * nb * 4 + 255) / 256 * 256;
}
__host__ __device__ constexpr long long getf2_scratch_stride(long long nb, long long es) {
  return (replay_mm_off(nb, es) + nb * nb * es + 255) / 256 * 256;
}

// ---------------------------------------------------------------------------
// Equilibration + assembly.
// ---------------------------------------------------------------------------

// Row maxima of |A| over the stored lower triangle, both triangles counted
// (onepass_scale, src/numeric/sparse_solver.rs:399-421).  Non-negative
// doubles order like their bit patterns, so atomicMax on the bits is exact
// and order independent.
template <typename T>
__global__ void k_rowmax(long long nnz, const int* __restrict__ row, const int* __restrict__ col,
                         const T* __restrict__ val, unsigned long long* __restrict__ rmax) {
  long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  double m = Field<T>::mag(val[k]);
  unsigned long long b = __double_as_longlong(m);
  int i = row[k], j = col[k];
  atomicMax(&rmax[i], b);
  if (i != j) atomicMax(&rmax[j], b);
}

// s_i = 1/sqrt(rowmax_i), guarded (src/scaling/mod.rs:85-96).
__global__ void k_scale_from_rowmax(int n, const unsigned long long* __restrict__ rmax, double* __restrict__ s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double m = __longlong_as_double(rmax[i]);
  double r = 1.0;
  if (m > 0.0) {
    double c = 1.0 / sqrt(m);
    if (isfinite(c) && c > 0.0) r = c;
  }
  s[i] = r;
}

// panel[dst[k]] = A_k * s_i * s_j.  Every stored entry has its own target
// (the permutation is a bijection), so this is a plain scatter.
template <typename T>
__global__ void k_assemble(long long nnz, const int* __restrict__ row, const int* __restrict__ col,
                           const T* __restrict__ val, const double* __restrict__ s,
                           const long long* __restrict__ dst, T* __restrict__ panel) {
  long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  int i = row[k], j = col[k];
  panel[dst[k]] = Field<T>::scale(val[k], s[i] * s[j]);
}

// Demote a high-precision value array to the low-precision field.
template <typename Hi, typename Lo>
__global__ void k_demote(long long nnz, const Hi* __restrict__ a, Lo* __restrict__ b);

template <>
__global__ void k_demote<double, float>(long long nnz, const double* __restrict__ a, float* __restrict__ b) {
  long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k < nnz) b[k] = (float)a[k];
}
template <>
__global__ void k_demote<c64, c32>(long long nnz, const c64* __restrict__ a, c32* __restrict__ b) {
  long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k < nnz) b[k] = c32{(float)a[k].re, (float)a[k].im};
}

// ---------------------------------------------------------------------------
// Shared GEMM-class tile engine: acc[i][j] = sum_t A(i,t) * G(j,t), G = L*D,
// i, j < 64, computed by 256 threads as 4x4 register micro-tiles
// (rows ty + 16*ii, cols tx + 16*jj).
// ---------------------------------------------------------------------------

// Inner-dimension chunk of the tile engine (elements of T per A/B row).
template <typename T> struct KChunk { static constexpr int v = 32; };
template <> struct KChunk<c64> { static constexpr int v = 16; };

// G(j, t) for column t of a factored panel with block-diagonal D.
template <typename T>
__device__ __forceinline__ T ld_G(const T* __restrict__ L, long long ld, int j, int t, const T* __restrict__ d,
                                  const T* __restrict__ dsub, const unsigned char* __restrict__ kind) {
  using F = Field<T>;
  unsigned char kd = kind[t];
  T a = L[j + (long long)t * ld];
  if (kd == 0) return F::mul(a, d[t]);
  if (kd == 1) {
    T b = L[j + (long long)(t + 1) * ld];
    return F::add(F::mul(d[t], a), F::mul(dsub[t], b));
  }
  T p = L[j + (long long)(t - 1) * ld];
  return F::add(F::mul(dsub[t - 1], p), F::mul(d[t], a));
}

// acc[i][j] = sum_t A(i,t) * B(j,t) over t in [0, kdim) for i, j < 64.
// A rows  : L_A + i (i < arows), column t at stride lda
// B rows  : L_B + j (j < brows), column t at stride ldb
// D (indexed by t) multiplies the B operand (D_ON_A = false: the cmod form
// U = L_k G^T, G = L_k D) or the A operand (D_ON_A = true: the deferred
// panel Schur tmp = (L21 D) L21^T).  Accumulation is one explicit FMA per t in
// ascending t, the same order as the oracle.  256 threads, 4x4 register
// micro-tiles (rows ty + 16*ii, cols tx + 16*jj); the next chunk is fetched
// into registers while the current one is multiplied out of shared memory.
template <typename T, bool D_ON_A = false>
__device__ void tile_product(T (&acc)[4][4], const T* __restrict__ LA, long long lda, int arows,
                             const T* __restrict__ LB, long long ldb, int brows, int kdim,
                             const T* __restrict__ d, const T* __restrict__ dsub,
                             const unsigned char* __restrict__ kind, T* As, T* Bs) {
  using F = Field<T>;
  constexpr int KT = KChunk<T>::v;
  constexpr int PER = KT * TILE / TPB;  // elements of each operand staged per thread
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = F::zero();
  T ra[PER], rb[PER];
  auto fetch = [&](int t0) {
    const int kt = min(KT, kdim - t0);
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = tid + q * TPB;
      const int t = e / TILE, r = e % TILE;
      T av = F::zero(), bv = F::zero();
      if (t < kt) {
        if constexpr (D_ON_A) {
          if (r < arows) av = ld_G(LA, lda, r, t0 + t, d, dsub, kind);
          if (r < brows) bv = LB[r + (long long)(t0 + t) * ldb];
        } else {
          if (r < arows) av = LA[r + (long long)(t0 + t) * lda];
          if (r < brows) bv = ld_G(LB, ldb, r, t0 + t, d, dsub, kind);
        }
      }
      ra[q] = av;
      rb[q] = bv;
    }
  };
  if (kdim > 0) fetch(0);
  for (int t0 = 0; t0 < kdim; t0 += KT) {
    const int kt = min(KT, kdim - t0);
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = tid + q * TPB;
      As[e] = ra[q];
      Bs[e] = rb[q];
    }
    __syncthreads();
    if (t0 + KT < kdim) fetch(t0 + KT);
    if (kt == KT) {
#pragma unroll 8
      for (int t = 0; t < KT; ++t) {
        T a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[t * TILE + ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[t * TILE + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = F::fma_(a[i], b[j], acc[i][j]);
      }
    } else {
      for (int t = 0; t < kt; ++t) {
        T a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[t * TILE + ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[t * TILE + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = F::fma_(a[i], b[j], acc[i][j]);
      }
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int lower_bound_i(const int* __restrict__ a, int lo, int hi, int key) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// cmod: task = (s, (r0/64) << 16 | (c0/64), pair_begin, pair_end): tile rows
// [r0, r0+64) x cols [c0, c0+64) of s's panel.  The pairs, precomputed at
// analysis, list in update-list order every descendant k whose update lands
// in the tile: (k, a, q0, nr << 16 | nc) = k's off-diagonal rows [a, a+nr)
// times its rows [q0, q0+nc) (the tile's columns).  No searches at run time
// beyond the tile-local row positions.
//
// Per pair the product U = L_k[a.., :] G_k[q0.., :]^T (G_k = L21_k D_k,
// formed once per updater by k_make_g with ld_G's arithmetic) runs in the
// updater's row space: operands are contiguous column runs of k's panel and
// of G_k, staged by cp.async into two shared-memory stages (the next chunk,
// possibly of the next pair, loads while the current one is multiplied).
// 128 threads, warp w owns rows 16w..16w+15 of the pair, each thread an 8 x 4
// register micro-tile (8 consecutive rows, columns cx + 16 j: conflict-free
// shared-memory reads); warps whose rows lie past nr skip the arithmetic.
// Every product is one explicit FMA per column t in ascending t, then
// subtracted from the tile held in shared memory through the pair's row /
// column maps (rows r >= column c in k's ordering only): the same operations
// in the same order as the oracle, so the result is bit-identical to it.
// ---------------------------------------------------------------------------
constexpr int CM_NT = 128;
template <typename T> struct CmChunk { static constexpr int v = 16; };
template <> struct CmChunk<c64> { static constexpr int v = 8; };

// Shared memory of k_cmod: the tile, two operand stages, two row / column
// maps and the tile's row structure.
template <typename T>
__host__ __device__ constexpr size_t smem_cmod_bytes() {
  return (size_t)TILE * TILE * sizeof(T) + 2 * 2 * (size_t)CmChunk<T>::v * TILE * sizeof(T) + 5 * TILE * 4 + 16;
}

template <typename T>
__global__ void __launch_bounds__(CM_NT, 2) k_cmod(FactorArgs fa, const int4* __restrict__ tasks,
                                                   const int4* __restrict__ pairs) {
  using F = Field<T>;
  constexpr int KC = CmChunk<T>::v;
  constexpr int STAGE = 2 * KC * TILE;  // A chunk [t][64 rows] then B chunk [t][64 cols]
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* acc_s = reinterpret_cast<T*>(smem_raw);  // [64 cols][64 rows]
  T* stg = acc_s + TILE * TILE;               // 2 stages
  int* rs_tile = reinterpret_cast<int*>(stg + 2 * STAGE);  // 64
  int* rowmap = rs_tile + TILE;                            // 2 x 64 (pair parity)
  int* colmap = rowmap + 2 * TILE;                         // 2 x 64

  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = (tk.y >> 16) * TILE, c0 = (tk.y & 0xffff) * TILE;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int rows_here = min(TILE, nrow - r0), cols_here = min(TILE, ncol - c0);
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  const int* rss = fa.rs + fa.sn_rsoff[s];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int e = tid; e < TILE * TILE; e += CM_NT) {
    const int c = e / TILE, r = e % TILE;
    T v = F::zero();
    if (r < rows_here && c < cols_here) v = panel[(r0 + r) + (long long)(c0 + c) * nrow];
    acc_s[e] = v;
  }
  if (tid < TILE) rs_tile[tid] = tid < rows_here ? rss[r0 + tid] : INT_MAX;
  const T* pall = reinterpret_cast<const T*>(fa.panel);
  const T* gall = reinterpret_cast<const T*>(fa.gpool);

  // chunk stream over (pair u, columns [t0, t0 + KC) of its updater)
  struct Cur {
    int u, t0;
  };
  auto issue = [&](Cur x, int st) {
    const int4 pr = pairs[x.u];
    const int k = pr.x, a = pr.y, q0 = pr.z, nr = pr.w >> 16, nc = pr.w & 0xffff;
    const int nck = fa.sn_ncol[k], nrk = fa.sn_nrow[k];
    const T* A = pall + fa.sn_poff[k] + nck + a;
    const T* B = gall + fa.goff[k] + q0;
    const long long ldb = nrk - nck;
    T* As = stg + st * STAGE;
    T* Bs = As + KC * TILE;
    for (int e = tid; e < KC * TILE; e += CM_NT) {
      const int t = e / TILE, r = e % TILE, tt = x.t0 + t;
      const bool in_t = tt < nck;
      cp_async_zfill<(int)sizeof(T)>(As + e, in_t && r < nr ? A + r + (long long)tt * nrk : A, in_t && r < nr);
      cp_async_zfill<(int)sizeof(T)>(Bs + e, in_t && r < nc ? B + r + (long long)tt * ldb : B, in_t && r < nc);
    }
    cp_async_commit();
  };
  auto advance = [&](Cur x) -> Cur {
    const int nck = fa.sn_ncol[pairs[x.u].x];
    x.t0 += KC;
    if (x.t0 >= nck) {
      x.u += 1;
      x.t0 = 0;
    }
    return x;
  };

  const int ry = lane >> 4, cx = lane & 15;
  const int rb = 16 * warp + 8 * ry;  // this thread's rows rb..rb+7, columns cx + 16 j
  T acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = F::zero();

  Cur cur{tk.z, 0};
  if (tk.z < tk.w) issue(cur, 0);
  int st = 0, parity = 0;
  while (cur.u < tk.w) {
    const int4 pr = pairs[cur.u];
    const int k = pr.x, a = pr.y, q0 = pr.z, nr = pr.w >> 16, nc = pr.w & 0xffff;
    const int nck = fa.sn_ncol[k];
    if (cur.t0 == 0) {
      // the tile positions of this pair's rows and columns (read only at the
      // pair's scatter, after at least one block barrier)
      __syncthreads();  // rs_tile written / the map slot's previous reader done
      const int* ok = fa.rs + fa.sn_rsoff[k] + nck;
      if (tid < nr) rowmap[parity * TILE + tid] = lower_bound_i(rs_tile, 0, rows_here, ok[a + tid]);
      if (tid >= TILE && tid - TILE < nc) colmap[parity * TILE + tid - TILE] = ok[q0 + tid - TILE] - first - c0;
    }
    const Cur nx = advance(cur);
    if (nx.u < tk.w) {
      issue(nx, st ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const T* As = stg + st * STAGE;
    const T* Bs = As + KC * TILE;
    const int kt = min(KC, nck - cur.t0);
    if (rb - 8 * ry < nr) {  // the warp has rows of this pair
      if (kt == KC) {
#pragma unroll 2
        for (int t = 0; t < KC; ++t) {
          T av[8], bv[4];
          lds_row<T, 8>(As + t * TILE + rb, av);
#pragma unroll
          for (int j = 0; j < 4; ++j) bv[j] = Bs[t * TILE + cx + 16 * j];
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = F::fma_(av[i], bv[j], acc[i][j]);
        }
      } else {
        for (int t = 0; t < kt; ++t) {
          T av[8], bv[4];
          lds_row<T, 8>(As + t * TILE + rb, av);
#pragma unroll
          for (int j = 0; j < 4; ++j) bv[j] = Bs[t * TILE + cx + 16 * j];
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = F::fma_(av[i], bv[j], acc[i][j]);
        }
      }
    }
    if (nx.u != cur.u) {
      // the pair is complete: subtract it from the tile, reset the registers
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int ri = rb + i;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cj = cx + 16 * j;
          if (ri < nr && cj < nc && a + ri >= q0 + cj) {
            const int e = colmap[parity * TILE + cj] * TILE + rowmap[parity * TILE + ri];
            acc_s[e] = F::sub(acc_s[e], acc[i][j]);
          }
          acc[i][j] = F::zero();
        }
      }
      parity ^= 1;
    }
    __syncthreads();  // the stage is free for the load after next
    st ^= 1;
    cur = nx;
  }
  __syncthreads();
  for (int e = tid; e < TILE * TILE; e += CM_NT) {
    const int c = e / TILE, r = e % TILE;
    if (r < rows_here && c < cols_here && r0 + r >= c0 + c) panel[(r0 + r) + (long long)(c0 + c) * nrow] = acc_s[e];
  }
}

// ---------------------------------------------------------------------------
// Deferred in-panel Schur: task = (s, kb, r0, c0) with tile rows [ke+r0, ...)
// and cols [ke+c0, ...): panel -= L21 D L21^T on rows >= cols.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(TPB) k_schur(FactorArgs fa, const int4* __restrict__ tasks, int nb_small,
                                               int nb_big) {
  using F = Field<T>;
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);
  T* Bs = As + KChunk<T>::v * TILE;
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, kb = tk.y, r0 = tk.z, c0 = tk.w;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int nb = ncol >= 512 ? nb_big : nb_small;
  const int ke = min(kb + nb, ncol);
  const int pw = ke - kb, mt = nrow - ke, cw = ncol - ke;
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  const int rows_here = min(TILE, mt - r0), cols_here = min(TILE, cw - c0);
  const T* L21 = panel + ke + (long long)kb * nrow;
  T acc[4][4];
  tile_product<T, true>(acc, L21 + r0, nrow, rows_here, L21 + c0, nrow, cols_here, pw,
                  reinterpret_cast<const T*>(fa.d) + first + kb, reinterpret_cast<const T*>(fa.dsub) + first + kb,
                  fa.kind + first + kb, As, Bs);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // every load before the first store (distinct targets)
  T old[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int rr = r0 + ty + 16 * i, cc = c0 + tx + 16 * j;
      const bool in = ty + 16 * i < rows_here && tx + 16 * j < cols_here && rr >= cc;
      old[i][j] = in ? panel[(ke + rr) + (long long)(ke + cc) * nrow] : F::zero();
    }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int rr = r0 + ty + 16 * i, cc = c0 + tx + 16 * j;
      if (ty + 16 * i < rows_here && tx + 16 * j < cols_here && rr >= cc)
        panel[(ke + rr) + (long long)(ke + cc) * nrow] = F::sub(old[i][j], acc[i][j]);
    }
}

// ---------------------------------------------------------------------------
// Multifrontal variant (factor_front + extend-add, multifrontal_ldlt.rs:901,
// 1494-1510).  A front of supernode s is its panel (nrow x ncol, the
// fully-summed columns) plus its contribution block CB_s (m x m, m = nrow -
// ncol, the trailing rows and columns, lower part).
//
// k_extend_add: task (s, ct, pair_begin, pair_end): front columns [64 ct,
// 64 ct + 64) of s, front rows of one chunk of EA_ROWS; pair (c, ja, jb):
// child c's contribution-block columns [ja, jb) land there, its rows
// [i0, i1) (the pair's row range) in the chunk.  Children are added in order (a block barrier between
// them), each entry (i, j), i >= j, of a child's block into the front entry
// (map[i], map[j]) (the child's rows' positions in the front): the panel
// when map[j] < ncol, CB_s otherwise.  Deterministic; no atomics.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_extend_add(FactorArgs fa, const int4* __restrict__ tasks,
                                                    const int4* __restrict__ pairs, const int2* __restrict__ prow,
                                                    const int* __restrict__ emap,
                                                    const long long* __restrict__ emoff) {
  using F = Field<T>;
  if (fa.status[0] != 0) return;
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s], ms = nrow - ncol;
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  T* cbs = reinterpret_cast<T*>(fa.cbpool) + fa.cb_off[s];
  constexpr int EB = 8;  // entries per thread per batch: every load of a batch before its stores
  for (int u = tk.z; u < tk.w; ++u) {
    const int4 pr = pairs[u];
    const int c = pr.x, mc = fa.sn_nrow[c] - fa.sn_ncol[c];
    const T* cbc = reinterpret_cast<const T*>(fa.cbpool) + fa.cb_off[c];
    const int* map = emap + emoff[c];
    // the child's columns [ja, jb) x rows [i0, i1) (the rows landing in this
    // task's row chunk) as one index space (rows fastest: coalesced reads of
    // the child's block), entries above the diagonal skipped; the targets of
    // one child are distinct
    const int2 rr = prow[u];
    const int len = rr.y - rr.x;
    const int tot = (pr.z - pr.y) * len;  // at most 64 columns x EA_ROWS rows
    for (int e0 = 0; e0 < tot; e0 += EB * 256) {
      T* tp[EB];
      T v[EB], old[EB];
#pragma unroll
      for (int q = 0; q < EB; ++q) {
        const int e = e0 + (int)threadIdx.x + q * 256;
        tp[q] = nullptr;
        if (e < tot) {
          const int j = pr.y + e / len, i = rr.x + e % len;
          if (i >= j) {
            const int li = map[i], lj = map[j];
            tp[q] = lj < ncol ? panel + li + (long long)lj * nrow : cbs + (li - ncol) + (long long)(lj - ncol) * ms;
            v[q] = cbc[i + (long long)j * mc];
          }
        }
      }
#pragma unroll
      for (int q = 0; q < EB; ++q) old[q] = tp[q] ? *tp[q] : F::zero();
#pragma unroll
      for (int q = 0; q < EB; ++q)
        if (tp[q]) *tp[q] = F::add(old[q], v[q]);
    }
    __syncthreads();  // the next child's additions follow this one's
  }
}

// k_front_cb: task (s, r0, c0, 0): CB_s rows [r0, r0 + 64) x columns [c0,
// c0 + 64), r0 >= c0, minus (L21 D L21^T) over all of s's columns (the
// tile engine with D on the row operand, as the in-panel Schur update), on
// its lower part.
template <typename T>
__global__ void __launch_bounds__(TPB) k_front_cb(FactorArgs fa, const int4* __restrict__ tasks) {
  using F = Field<T>;
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);
  T* Bs = As + KChunk<T>::v * TILE;
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = tk.y, c0 = tk.z;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s], m = nrow - ncol;
  const T* L21 = reinterpret_cast<const T*>(fa.panel) + fa.sn_poff[s] + ncol;
  T* cb = reinterpret_cast<T*>(fa.cbpool) + fa.cb_off[s];
  const int rows_here = min(TILE, m - r0), cols_here = min(TILE, m - c0);
  T acc[4][4];
  tile_product<T, true>(acc, L21 + r0, nrow, rows_here, L21 + c0, nrow, cols_here, ncol,
                        reinterpret_cast<const T*>(fa.d) + first, reinterpret_cast<const T*>(fa.dsub) + first,
                        fa.kind + first, As, Bs);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // every load before the first store (distinct targets)
  T old[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int rr = r0 + ty + 16 * i, cc = c0 + tx + 16 * j;
      const bool in = ty + 16 * i < rows_here && tx + 16 * j < cols_here && rr >= cc;
      old[i][j] = in ? cb[rr + (long long)cc * m] : F::zero();
    }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int rr = r0 + ty + 16 * i, cc = c0 + tx + 16 * j;
      if (ty + 16 * i < rows_here && tx + 16 * j < cols_here && rr >= cc)
        cb[rr + (long long)cc * m] = F::sub(old[i][j], acc[i][j]);
    }
}

// ---------------------------------------------------------------------------
// Block reductions for the pivot search: max of a non-negative double with
// the lowest index on ties (the reference's strict `>` scan).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void argmax_combine(double& v, int& i, double v2, int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// Warp-wide argmax_combine of every lane's (v, i), v >= 0 or -1 (none): the
// same result (largest v, then smallest i) from three warp reductions on an
// order-preserving key (bits of v + 1; 0 for none), instead of a shuffle tree.
__device__ __forceinline__ void warp_argmax(double& v, int& i) {
  const unsigned long long key = v >= 0.0 ? (unsigned long long)__double_as_longlong(v) + 1ull : 0ull;
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool win = hi == mhi && lo == mlo;
  const int mi = (int)__reduce_min_sync(0xffffffffu, win ? (unsigned)i : 0xffffffffu);
  const unsigned long long mk = ((unsigned long long)mhi << 32) | mlo;
  v = mk == 0ull ? -1.0 : __longlong_as_double((long long)(mk - 1ull));
  i = mk == 0ull ? INT_MAX : mi;
}

template <int NT>
__device__ void block_argmax(double& v, int& idx, double* red_v, int* red_i) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double v2 = __shfl_down_sync(0xffffffffu, v, o);
    int i2 = __shfl_down_sync(0xffffffffu, idx, o);
    argmax_combine(v, idx, v2, i2);
  }
  if (lane == 0) {
    red_v[wid] = v;
    red_i[wid] = idx;
  }
  __syncthreads();
  if (wid == 0) {
    v = lane < NT / 32 ? red_v[lane] : -1.0;
    idx = lane < NT / 32 ? red_i[lane] : INT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double v2 = __shfl_down_sync(0xffffffffu, v, o);
      int i2 = __shfl_down_sync(0xffffffffu, idx, o);
      argmax_combine(v, idx, v2, i2);
    }
    if (lane == 0) {
      red_v[0] = v;
      red_i[0] = idx;
    }
  }
  __syncthreads();
  v = red_v[0];
  idx = red_i[0];
  __syncthreads();
}

// Packed lower-triangle index of (i, j), i >= j, in a pw x pw block.
__device__ __forceinline__ int pk(int i, int j, int pw) { return j * pw - (j * (j - 1)) / 2 + (i - j); }

// Warp-per-row replay: lane l holds columns l + 32*j (j < NS) of one deep
// row in registers; every pivot step's broadcast / interchange goes through
// shuffles, so a warp replays a whole row with no block barrier.  The
// per-element op sequence is exactly apply_bk_panel_trailing's.
template <typename T>
__device__ __forceinline__ T shfl_t(T v, int src) {
  if constexpr (Field<T>::complex) {
    T r;
    r.re = __shfl_sync(0xffffffffu, v.re, src);
    r.im = __shfl_sync(0xffffffffu, v.im, src);
    return r;
  } else {
    return __shfl_sync(0xffffffffu, v, src);
  }
}

template <typename T, int NS>
__device__ __forceinline__ T pick(const T (&x)[NS], int slot) {
  T v = x[0];
#pragma unroll
  for (int j = 1; j < NS; ++j)
    if (j == slot) v = x[j];
  return v;
}

template <typename T, int NS>
__device__ __forceinline__ void put(T (&x)[NS], int slot, T v) {
#pragma unroll
  for (int j = 0; j < NS; ++j)
    if (j == slot) x[j] = v;
}

// Per-block replay program in shared memory, filled once per CTA: for pivot
// step k the swap target, the pivot kind and the inverse of the pivot block
// (1x1: 1/d; 2x2: 1/det with det = d11 d22 - d21^2), plus d and dsub.
template <typename T>
struct ReplayProg {
  int* sw;
  unsigned char* kd;
  T* inv;
  T* dd;
  T* ds;
};

template <typename T>
__host__ __device__ constexpr size_t replay_prog_bytes(int nb) {
  return (size_t)nb * (3 * sizeof(T) + sizeof(int) + 1) + 16;
}

// Carve the program out of `mem` (16-byte aligned) and fill it (all threads).
template <typename T, int NT>
__device__ ReplayProg<T> load_replay_prog(unsigned char* mem, int pw, int nb, const int* __restrict__ swaps,
                                          const T* __restrict__ d, const T* __restrict__ dsub,
                                          const unsigned char* __restrict__ kind) {
  using F = Field<T>;
  ReplayProg<T> P;
  P.inv = reinterpret_cast<T*>(mem);
  P.dd = P.inv + nb;
  P.ds = P.dd + nb;
  P.sw = reinterpret_cast<int*>(P.ds + nb);
  P.kd = reinterpret_cast<unsigned char*>(P.sw + nb);
  for (int k = threadIdx.x; k < pw; k += NT) {
    const unsigned char kk = kind[k];
    P.sw[k] = swaps[k];
    P.kd[k] = kk;
    P.dd[k] = d[k];
    P.ds[k] = dsub[k];
    T inv = F::zero();
    if (kk == 0) {
      inv = F::recip(d[k]);
    } else if (kk == 1) {
      const T d11 = d[k], d21 = dsub[k], d22 = d[k + 1];
      inv = F::recip(F::sub(F::mul(d11, d22), F::mul(d21, d21)));
    }
    P.inv[k] = inv;
  }
  return P;
}

// Replay pivot steps [k_begin, k_end) of a block on NR rows held by one warp
// (x[row][slot], column = lane + 32 slot): the swaps, then per pivot the
// elimination of the later columns with the snapshot multipliers and the
// scaling by the inverse pivot block.  S holds snapshot rows k_begin ..
// k_end - 1 (row stride `lds`).  The rows are independent, so the NR
// dependency chains interleave; each row sees the same operation sequence as
// a lone row.
template <typename T, int NS, int NR>
__device__ void replay_rows_warp(T (&x)[NR][NS], int pw, const T* S, int lds, int k_begin, int k_end, int kb,
                                 const ReplayProg<T>& P) {
  using F = Field<T>;
  const int lane = threadIdx.x & 31;
  int k = k_begin;
  // the next step's program words are read one step ahead, so a step's
  // branches do not wait on shared memory
  int kp_n = k < k_end ? P.sw[k] : -1;
  bool two_n = k < k_end && P.kd[k] == 1;
  while (k < k_end) {
    const int kp = kp_n;
    const bool two = two_n;
    const int kn = k + (two ? 2 : 1);
    if (kn < k_end) {
      kp_n = P.sw[kn];
      two_n = P.kd[kn] == 1;
    }
    if (kp >= 0) {
      const int src = two ? k + 1 : k, dst = kp - kb;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const T vs = shfl_t(pick(x[r], src >> 5), src & 31);
        const T vd = shfl_t(pick(x[r], dst >> 5), dst & 31);
        if (lane == (src & 31)) put(x[r], src >> 5, vd);
        if (lane == (dst & 31)) put(x[r], dst >> 5, vs);
      }
    }
    if (two) {
      const T d11 = P.dd[k], d21 = P.ds[k], d22 = P.dd[k + 1], detinv = P.inv[k];
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const T xk = shfl_t(pick(x[r], k >> 5), k & 31);
        const T xk1 = shfl_t(pick(x[r], (k + 1) >> 5), (k + 1) & 31);
#pragma unroll
        for (int j = 0; j < NS; ++j) {
          const int col = lane + 32 * j;
          if (col >= k + 2 && col < pw) {
            const T l1 = S[(k - k_begin) * lds + col], l2 = S[(k + 1 - k_begin) * lds + col];
            T v = F::sub(x[r][j], F::mul(xk, l1));
            x[r][j] = F::sub(v, F::mul(xk1, l2));
          }
        }
        if (lane == (k & 31)) put(x[r], k >> 5, F::mul(F::sub(F::mul(d22, xk), F::mul(d21, xk1)), detinv));
        if (lane == ((k + 1) & 31))
          put(x[r], (k + 1) >> 5, F::mul(F::sub(F::mul(d11, xk1), F::mul(d21, xk)), detinv));
      }
    } else {
      const T dinv = P.inv[k];
      T w[NS];  // the step's multipliers, loaded before the broadcast they do not depend on
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        const int col = lane + 32 * j;
        w[j] = (col > k && col < pw) ? S[(k - k_begin) * lds + col] : F::zero();
      }
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const T xk = shfl_t(pick(x[r], k >> 5), k & 31);
#pragma unroll
        for (int j = 0; j < NS; ++j)
          if (!F::is_zero(w[j])) x[r][j] = F::sub(x[r][j], F::mul(xk, w[j]));
        if (lane == (k & 31)) put(x[r], k >> 5, F::mul(xk, dinv));
      }
    }
    k = kn;
  }
}

// Snapshot rows staged per slice of pivot steps (one more when a 2x2 pivot
// straddles the slice end).
constexpr int REPLAY_SL = 16;

// All of a block's pivot steps on the warp's rows, the snapshot multipliers
// read from shared memory: per slice of REPLAY_SL steps the CTA copies the
// slice's snapshot rows (all columns < pw, stride nb) into S, then every warp
// replays those steps.  S holds (REPLAY_SL + 1) x nb elements; every thread
// of the CTA calls this (it synchronises the block).
template <typename T, int NT, int NS, int NR, int SL = REPLAY_SL>
__device__ void replay_rows_sliced(T (&x)[NR][NS], int pw, int nb, const T* __restrict__ snap, int kb,
                                   const ReplayProg<T>& P, T* S) {
  for (int k0 = 0; k0 < pw;) {
    int k1 = min(k0 + SL, pw);
    if (k1 < pw && P.kd[k1 - 1] == 1) ++k1;
    __syncthreads();
    const int cnt = (k1 - k0) * pw;
    for (int e = threadIdx.x; e < cnt; e += NT) {
      const int r = e / pw, c = e - r * pw;
      cp_async_zfill<sizeof(T)>(S + r * nb + c, snap + (long long)(k0 + r) * nb + c, true);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    replay_rows_warp<T, NS, NR>(x, pw, S, nb, k0, k1, kb, P);
    k0 = k1;
  }
  __syncthreads();
}

// Replay a block's pivot steps on deep rows [r_begin, r_end) of a panel:
// rows staged through shared memory (32 rows x pw, padded stride) so both
// the global loads / stores and the per-row register fills are conflict-free;
// each warp replays its 32 / NW rows together.  `P` holds the program.  While
// the rows sit in registers the staging buffer X carries the snapshot slices.
//
// IDENT: the rows are those of the pw x pw identity instead (rows
// [r_begin, r_end) of it), and the results go to M (row-major, stride nb):
// the replay is linear in the row, so M is the block's transform and every
// deep row x becomes x M.
// R rows per pass (a multiple of the warp count).  The snapshot slices of SL
// steps use S (default: X, free while the rows sit in registers; it must
// hold (SL + 1) x nb elements, or pw x nb when SL >= pw).
template <typename T, int NT, bool IDENT = false, int R = 32, int SL = REPLAY_SL>
__device__ void replay_deep_rows(T* panel, long long nrow, int kb, int pw, int nb, int r_begin, int r_end,
                                 const T* __restrict__ snap, const ReplayProg<T>& P, T* X, T* M = nullptr,
                                 T* S = nullptr) {
  constexpr int LDX = R + 1;
  if (!S) S = X;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NW = NT / 32;
  constexpr int NR = R / NW;
  for (int rs0 = r_begin; rs0 < r_end; rs0 += R) {
    const int rows = min(R, r_end - rs0);
    // fixed trip count (panel blocks are at most 128 wide): all loads in flight
#pragma unroll 16
    for (int e = threadIdx.x; e < R * 128; e += NT) {
      const int c = e / R, r = e % R;
      if (r < rows && c < pw) {
        if constexpr (IDENT)
          X[c * LDX + r] = c == rs0 + r ? Field<T>::one() : Field<T>::zero();
        else
          X[c * LDX + r] = panel[(rs0 + r) + (long long)(kb + c) * nrow];
      }
    }
    __syncthreads();
    // rows warp + NW i; rows past `rows` replay zeros and are not stored
    if (pw <= 64) {
      T x[NR][2];
#pragma unroll
      for (int i = 0; i < NR; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int col = lane + 32 * j, r = warp + NW * i;
          x[i][j] = (col < pw && r < rows) ? X[col * LDX + r] : Field<T>::zero();
        }
      replay_rows_sliced<T, NT, 2, NR, SL>(x, pw, nb, snap, kb, P, S);
#pragma unroll
      for (int i = 0; i < NR; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int col = lane + 32 * j, r = warp + NW * i;
          if (col < pw && r < rows) X[col * LDX + r] = x[i][j];
        }
    } else {
      T x[NR][4];
#pragma unroll
      for (int i = 0; i < NR; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int col = lane + 32 * j, r = warp + NW * i;
          x[i][j] = (col < pw && r < rows) ? X[col * LDX + r] : Field<T>::zero();
        }
      replay_rows_sliced<T, NT, 4, NR, SL>(x, pw, nb, snap, kb, P, S);
#pragma unroll
      for (int i = 0; i < NR; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int col = lane + 32 * j, r = warp + NW * i;
          if (col < pw && r < rows) X[col * LDX + r] = x[i][j];
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < R * pw; e += NT) {
      if constexpr (IDENT) {
        const int r = e / pw, c = e % pw;  // row-major M: coalesced along c
        if (r < rows) M[(long long)(rs0 + r) * nb + c] = X[c * LDX + r];
      } else {
        const int c = e / R, r = e % R;
        if (r < rows) panel[(rs0 + r) + (long long)(kb + c) * nrow] = X[c * LDX + r];
      }
    }
    __syncthreads();
  }
}

constexpr int DEEP_R = 32;  // deep rows per replay chunk

// The lower pw x pw block of panel columns [kb, kb + pw) into packed
// storage: a fixed-count loop over the smallest W x W square (W = 32, 64 or
// 128) that holds the block, so every load of a thread is in flight at once
// and a narrow block does not walk the 128 x 128 index space.
template <typename T, int NT, int W>
__device__ __forceinline__ void load_packed_block_w(T* A, const T* panel, long long nrow, int kb, int pw) {
#pragma unroll 8
  for (int e = threadIdx.x; e < W * W; e += NT) {
    const int i = e % W, j = e / W;
    if (i < pw && j <= i) A[pk(i, j, pw)] = panel[(kb + i) + (long long)(kb + j) * nrow];
  }
}
template <typename T, int NT>
__device__ __forceinline__ void load_packed_block(T* A, const T* panel, long long nrow, int kb, int pw) {
  if (pw > 64)
    load_packed_block_w<T, NT, 128>(A, panel, nrow, kb, pw);
  else if (pw > 32)
    load_packed_block_w<T, NT, 64>(A, panel, nrow, kb, pw);
  else
    load_packed_block_w<T, NT, 32>(A, panel, nrow, kb, pw);
}

// The end of a BK panel block, shared by both getf2 kernels: the block's
// local pivot order into lperm, the status word (first failing supernode,
// perturbation count), the packed block back into the panel (the 2x2
// coupling entry lives in dsub only: its panel slot is stored as an exact
// zero), the block's interchanges applied to the rows' left segments
// (columns [0, kb)), and for a short panel the replay of the block's pivot
// steps on its deep rows.  Every thread of the CTA calls it; `src_row` has
// room for pw ints.
template <typename T, int NT>
__device__ void getf2_finish(const FactorArgs& fa, int s, int kb, int pw, int nb, int nrow, int ke, int fuse,
                             T* panel, T* A, int* lp_s, int* lpermG, int* ctl, int* swp_p, int* swp_q, int* supp,
                             int* src_row, unsigned char* kindG, T* dG, T* dsG, T* snap, int* swaps, int nperturbed,
                             unsigned char* smem_raw) {
  using F = Field<T>;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int NW = NT / 32;
  for (int i = tid; i < pw; i += NT) lpermG[kb + i] = lp_s[i];
  if (ctl[3]) {
    if (tid == 0) {
      if (atomicCAS(&fa.status[0], 0, 1) == 0) fa.status[1] = s;
    }
    return;
  }
  if (tid == 0 && nperturbed) atomicAdd(&fa.status[2], nperturbed);
  // Write the block back; the 2x2 coupling entry (i = j + 1 of a 2x2) lives
  // in dsub only, so its panel slot is stored as an exact zero (it is never
  // an L multiplier).
  __syncthreads();
  for (int j = warp; j < pw; j += NW) {
    const bool two = kindG[j] == 1;
    for (int i = j + lane; i < pw; i += 32)
      panel[(kb + i) + (long long)(kb + j) * nrow] = (two && i == j + 1) ? F::zero() : A[pk(i, j, pw)];
  }
  // Left row segments of the interchanges (columns [0, kb), rows of this
  // block): the swap sequence composes to one row permutation of the block;
  // only the rows it moves are copied, in column chunks whose loads are all
  // in flight before the barrier that precedes the stores (same final values).
  const int nsw = ctl[2];
  if (nsw > 0 && kb > 0) {
    __syncthreads();
    if (tid == 0) {
      for (int r = 0; r < pw; ++r) src_row[r] = r;
      for (int t = 0; t < nsw; ++t) {
        const int p = swp_p[t] - kb, q = swp_q[t] - kb;
        const int x = src_row[p];
        src_row[p] = src_row[q];
        src_row[q] = x;
      }
      int m = 0;
      for (int r = 0; r < pw; ++r)
        if (src_row[r] != r) supp[m++] = r;
      ctl[1] = m;
    }
    __syncthreads();
    const int ns = ctl[1];
    if (ns > 0) {
      constexpr int PER = 8;  // elements per thread per chunk
      const int cols = max(1, (NT * PER) / ns);
      for (int j0 = 0; j0 < kb; j0 += cols) {
        const int jn = min(cols, kb - j0);
        T v[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const int idx = tid + u * NT;
          if (idx < ns * jn) {
            const int r = supp[idx % ns], j = j0 + idx / ns;
            v[u] = panel[(kb + src_row[r]) + (long long)j * nrow];
          }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const int idx = tid + u * NT;
          if (idx < ns * jn) {
            const int r = supp[idx % ns], j = j0 + idx / ns;
            panel[(kb + r) + (long long)j * nrow] = v[u];
          }
        }
        __syncthreads();
      }
    }
  }
  // kind/d written by tid 0 are read by the replay below.
  __syncthreads();
  if (fuse && nrow > ke) {
    // Replay this block's pivot steps on the deep rows [ke, nrow).
    unsigned char* pmem = smem_raw + (((size_t)(DEEP_R + 1) * nb * sizeof(T) + 15) & ~size_t(15));
    const ReplayProg<T> P = load_replay_prog<T, NT>(pmem, pw, nb, swaps, dG, dsG, kindG);
    __syncthreads();
    // rows per pass: 32 with 8 or more warps, 8 with 4 (two rows a warp)
    replay_deep_rows<T, NT, false, (NT >= 256 ? 32 : 8)>(panel, nrow, kb, pw, nb, ke, nrow, snap, P, A);
  }
}

// ---------------------------------------------------------------------------
// getf2: task = (s, kb, slot, fuse) — unblocked BK over panel columns [kb, ke)
// with every pivot candidate, update and interchange bounded to rows < ke.
// ---------------------------------------------------------------------------
template <typename T, int NT, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) k_getf2(FactorArgs fa, const int4* __restrict__ tasks, int nb_small,
                                              int nb_big) {
  using F = Field<T>;
  if (fa.status[0] != 0) return;
  const double pfloor = fa.floor_dev ? *fa.floor_dev : fa.perturb_floor;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, kb = tk.y, slot = tk.z, fuse = tk.w;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int nb = ncol >= 512 ? nb_big : nb_small;
  const int ke = min(kb + nb, ncol), pw = ke - kb;
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  T* dG = reinterpret_cast<T*>(fa.d) + first + kb;
  T* dsG = reinterpret_cast<T*>(fa.dsub) + first + kb;
  unsigned char* kindG = fa.kind + first + kb;
  int* lpermG = fa.lperm + first;
  unsigned char* sc = reinterpret_cast<unsigned char*>(fa.scratch) + (long long)slot * fa.scratch_stride;
  T* snap = reinterpret_cast<T*>(sc);                      // nb x nb
  int* swaps = reinterpret_cast<int*>(snap + (long long)nb * nb);  // nb

  T* A = reinterpret_cast<T*>(smem_raw);              // packed lower pw x pw
  const int npk = pw * (pw + 1) / 2;
  // Two sets (by step parity) of the step's multipliers l1 / l2 (column k /
  // k+1) and the same columns before scaling u1 / u2 (read by the update).
  T* l1 = A + npk;
  // 16-byte aligned reduction scratch after the (possibly 4-byte) field arrays.
  double* red_v = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(l1 + 8 * pw) + 15) & ~uintptr_t(15));
  int* red_i = reinterpret_cast<int*>(red_v + 32);
  int* ctl = red_i + 32;  // [0] kstep [1] kp [2] nswaps [3] error
  int* lp_s = ctl + 16;   // the block's slice of lperm
  int* swp_p = lp_s + nb; // swap log of this block (row pairs for the left segments)
  int* swp_q = swp_p + nb;
  int* supp = swp_q + nb; // rows moved by the composed permutation

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  constexpr int NW = NT / 32;
  // flat fixed-count load of the lower block (at most 128 x 128): loads in flight
  load_packed_block<T, NT>(A, panel, nrow, kb, pw);
  if (kb == 0)
    for (int p = tid; p < ncol; p += NT) lpermG[p] = p;
  for (int e = tid; e < pw; e += NT) {
    dG[e] = F::zero();
    dsG[e] = F::zero();
    kindG[e] = 0;
    swaps[e] = -1;
  }
  for (int e = tid; e < pw * nb; e += NT) snap[e] = F::zero();
  if (tid == 0) {
    ctl[2] = 0;
    ctl[3] = 0;
  }
  __syncthreads();
  for (int i = tid; i < pw; i += NT) lp_s[i] = lpermG[kb + i];
  __syncthreads();
  const double alpha = (1.0 + sqrt(17.0)) / 8.0;
  int nperturbed = 0;
  // Pipelined pivot steps.  Warp 0 decides step k (arg-max / max
  // reductions, BK test, interchange, multipliers, the finished column(s) k)
  // into the multiplier set of the step's parity; then warps 1.. apply the
  // rank-1 / rank-2 trailing update of step k to the columns beyond the next
  // pivot column kn = k + kstep, while warp 0 updates column kn itself and
  // already decides step kn.  That early decision completes when the BK test
  // needs no row maximum (so no interchange either: both would read or move
  // entries other warps are still updating); otherwise it is redone in full
  // after the step's barrier.  One block barrier per step on the fast path;
  // per element the operation sequence, and every decision, are unchanged.
  // Control slots by iteration parity: {k, kstep, pending}.
  int* cslot = ctl + 4;
  auto bufs = [&](int par, T*& L1, T*& L2, T*& U1, T*& U2) {
    L1 = l1 + 4 * par * pw;
    L2 = L1 + pw;
    U1 = L2 + pw;
    U2 = U1 + pw;
  };
  // Warp 0: decide step k into multiplier set / control slot `par`.  With
  // `full` false, returns false (writing nothing) when the row-maximum test
  // is needed.
  const bool reuse = fa.pivot_reuse && fa.pivrec && *fa.pivot_reuse != 0;
  int* prec = fa.pivrec ? fa.pivrec + first + kb : nullptr;  // no record without a handle
  auto decide = [&](int k, int par, bool full) -> bool {
    T *L1, *L2, *U1, *U2;
    bufs(par, L1, L2, U1, U2);
    int kstep = 1, kp = k;
    bool err = false;
    if (reuse) {
      // the recorded step: no search (a zero pivot is still caught below).
      // An early decision (other warps still updating) may only take a 1x1
      // step without interchange, as in the search below: defer the rest.
      const int code = prec[k];
      kstep = code < 0 ? 2 : 1;
      kp = code < 0 ? -code - 1 : code;
      if (!full && (kstep != 1 || kp != k)) return false;
    } else {
    // |a_kk| first: independent of the column scan, its latency overlaps it
    const double absakk = F::mag(A[pk(k, k, pw)]);
    double v = -1.0;
    int idx = INT_MAX;
    // blocks are at most 128 wide: four predicated lanes-strided slots
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int i = k + 1 + lane + 32 * t;
      if (i < pw) argmax_combine(v, idx, F::mag2(A[pk(i, k, pw)]), i);
    }
    warp_argmax(v, idx);
    const double colmax = sqrt(v > 0.0 ? v : 0.0);
    const int imax = v > 0.0 ? idx : k;
    if (fmax(absakk, colmax) == 0.0) {
      err = pfloor < 0.0;
    } else if (absakk >= alpha * colmax) {
    } else {
      if (!full) return false;
      double rmx = 0.0;
      for (int jj = k + lane; jj < imax; jj += 32) rmx = fmax(rmx, F::mag2(A[pk(imax, jj, pw)]));
      for (int ii = imax + 1 + lane; ii < pw; ii += 32) rmx = fmax(rmx, F::mag2(A[pk(ii, imax, pw)]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) rmx = fmax(rmx, __shfl_xor_sync(0xffffffffu, rmx, o));
      const double rowmax = sqrt(rmx);
      if (absakk >= alpha * colmax * (colmax / rowmax)) {
      } else if (F::mag(A[pk(imax, imax, pw)]) >= alpha * rowmax) {
        kp = imax;
      } else {
        kstep = 2;
        kp = imax;
      }
    }
    if (lane == 0 && !err && prec) prec[k] = kstep == 2 ? -kp - 1 : kp;
    }
    if (!err) {
      const int p = kstep == 1 ? k : k + 1;
      if (kp != p) {
        // swap_sym_lower_bounded(p, kp) restricted to the block + left segments.
        const int q = kp;
        for (int i = q + 1 + lane; i < pw; i += 32) {
          T t = A[pk(i, p, pw)];
          A[pk(i, p, pw)] = A[pk(i, q, pw)];
          A[pk(i, q, pw)] = t;
        }
        for (int i = p + 1 + lane; i < q; i += 32) {
          T t = A[pk(i, p, pw)];
          A[pk(i, p, pw)] = A[pk(q, i, pw)];
          A[pk(q, i, pw)] = t;
        }
        for (int jj = lane; jj < p; jj += 32) {
          T t = A[pk(p, jj, pw)];
          A[pk(p, jj, pw)] = A[pk(q, jj, pw)];
          A[pk(q, jj, pw)] = t;
        }
        if (lane == 0) {
          T t = A[pk(p, p, pw)];
          A[pk(p, p, pw)] = A[pk(q, q, pw)];
          A[pk(q, q, pw)] = t;
          const int lpv = lp_s[p];
          lp_s[p] = lp_s[q];
          lp_s[q] = lpv;
          swaps[k] = kb + q;
          const int ns = ctl[2];
          swp_p[ns] = kb + p;
          swp_q[ns] = kb + q;
          ctl[2] = ns + 1;
        }
        __syncwarp();
      }
      if (kstep == 1) {
        T dk = A[pk(k, k, pw)];
        if (pfloor >= 0.0) {
          const double m = F::mag(dk);
          if (m < pfloor) {
            dk = m == 0.0 ? F::from_real(pfloor) : F::scale(dk, pfloor / m);
            __syncwarp();
            if (lane == 0) {
              A[pk(k, k, pw)] = dk;
              ++nperturbed;
            }
          }
        } else if (F::is_zero(dk)) {
          err = true;
        }
        if (!err) {
          const T dinv = F::recip(dk);
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const int jj = k + 1 + lane + 32 * t;
            if (jj < pw) {
              const T a = A[pk(jj, k, pw)];
              const T w = F::mul(a, dinv);
              U1[jj] = a;
              L1[jj] = w;
              snap[k * nb + jj] = w;
              A[pk(jj, k, pw)] = w;  // column k finished: the multipliers
            }
          }
          if (lane == 0) dG[k] = dk;
        }
      } else {
        T d11 = A[pk(k, k, pw)], d21 = A[pk(k + 1, k, pw)], d22 = A[pk(k + 1, k + 1, pw)];
        T det = F::sub(F::mul(d11, d22), F::mul(d21, d21));
        const double scale = fmax(fmax(F::mag(d11), F::mag(d22)), F::mag(d21));
        const double growth_floor = 1e-14 * scale * scale;
        if (pfloor >= 0.0) {
          const double fl = fmax(pfloor * pfloor, growth_floor);
          if (F::mag(det) < fl) {
            const double lift = fmax(pfloor, scale * sqrt(1e-14));
            d11 = F::add(d11, F::from_real(lift));
            d22 = F::add(d22, F::from_real(lift));
            det = F::sub(F::mul(d11, d22), F::mul(d21, d21));
            if (F::mag(det) < fl) det = F::add(det, F::from_real(fl));
            if (lane == 0) ++nperturbed;
          }
        } else if (F::mag(det) <= growth_floor) {
          err = true;
        }
        if (!err) {
          const T detinv = F::recip(det);
          if (lane == 0) {
            dG[k] = d11;
            dsG[k] = d21;
            dG[k + 1] = d22;
            kindG[k] = 1;
            kindG[k + 1] = 2;
          }
          for (int i = k + 2 + lane; i < pw; i += 32) {
            const T wik = A[pk(i, k, pw)], wik1 = A[pk(i, k + 1, pw)];
            const T a1 = F::mul(F::sub(F::mul(d22, wik), F::mul(d21, wik1)), detinv);
            const T a2 = F::mul(F::sub(F::mul(d11, wik1), F::mul(d21, wik)), detinv);
            U1[i] = wik;
            U2[i] = wik1;
            L1[i] = a1;
            L2[i] = a2;
            snap[k * nb + i] = a1;
            snap[(k + 1) * nb + i] = a2;
            A[pk(i, k, pw)] = a1;  // columns k, k+1 finished
            A[pk(i, k + 1, pw)] = a2;
          }
        }
      }
    }
    if (lane == 0) {
      if (err) ctl[3] = 1;
      int* cs = cslot + 3 * par;
      cs[0] = k;
      cs[1] = kstep;
      cs[2] = 0;
    }
    return true;
  };
  // Column jj of the trailing update of a step (one warp, lanes over rows):
  // rank-1 with U1 / L1[jj] (skipped for a zero multiplier) or rank-2.
  auto upd_col = [&](int jj, int kstep, const T* L1, const T* L2, const T* U1, const T* U2) {
    const int base = pk(jj, jj, pw) - jj;  // packed index of (i, jj) = base + i
    if (kstep == 1) {
      const T w = L1[jj];
      if (F::is_zero(w)) return;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int i = jj + lane + 32 * t;
        if (i < pw) A[base + i] = F::sub(A[base + i], F::mul(U1[i], w));
      }
    } else {
      const T a1 = L1[jj], a2 = L2[jj];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int i = jj + lane + 32 * t;
        if (i < pw) {
          T x = A[base + i];
          x = F::sub(x, F::mul(U1[i], a1));
          x = F::sub(x, F::mul(U2[i], a2));
          A[base + i] = x;
        }
      }
    }
  };
  if (warp == 0) decide(0, 0, true);
  __syncthreads();
  for (int it = 0;; ++it) {
    const int par = it & 1;
    int k = cslot[3 * par], kstep = cslot[3 * par + 1];
    if (k >= pw || ctl[3]) break;
    if (cslot[3 * par + 2]) {
      // the early decision of step k needed the row maximum: redo it in full
      __syncthreads();
      if (warp == 0) decide(k, par, true);
      __syncthreads();
      if (ctl[3]) break;
      kstep = cslot[3 * par + 1];
    }
    T *L1, *L2, *U1, *U2;
    bufs(par, L1, L2, U1, U2);
    const int kn = k + kstep;
    if (warp == 0) {
      if (kn < pw) {
        upd_col(kn, kstep, L1, L2, U1, U2);
        __syncwarp();
        if (!decide(kn, par ^ 1, false) && lane == 0) {
          int* cs = cslot + 3 * (par ^ 1);
          cs[0] = kn;
          cs[2] = 1;
        }
      } else if (lane == 0) {
        cslot[3 * (par ^ 1)] = kn;
      }
    } else {
      for (int jj = kn + 1 + (warp - 1); jj < pw; jj += NW - 1) upd_col(jj, kstep, L1, L2, U1, U2);
    }
    __syncthreads();
  }
  getf2_finish<T, NT>(fa, s, kb, pw, nb, nrow, ke, fuse, panel, A, lp_s, lpermG, ctl, swp_p, swp_q, supp,
                      reinterpret_cast<int*>(l1), kindG, dG, dsG, snap, swaps, nperturbed, smem_raw);
}

// ---------------------------------------------------------------------------
// getf2, left-looking form (the single-precision fields' tensor engine): the
// same panel-bounded Bunch-Kaufman steps, decisions and outputs as k_getf2,
// but no trailing update of the block.  The block keeps its ORIGINAL values
// in the columns not yet pivoted; step k first forms the column it needs,
//   v[i] = A0(i, c) - sum_{p < k} G(i, p) L(c, p),   i in [k, pw),
// G = L D the unscaled columns of the finished steps, as one GEMV over all
// 16 warps (4 to 16 partial sums per row), for c = k and, when the BK test
// needs the row maximum (or a recorded step names another column), for the
// candidate column too.  The rest of a step runs on the row team, warps 0-3
// (one per SM sub-partition, one row per thread): the partial sums, the
// arg-max, the decision (every team thread takes it from the same values),
// and the multipliers; the interchange, when there is one, on warp 0.  The
// BK tests compare squared moduli, so the decision path has no square roots
// or divisions.  A step costs two block barriers (four with the candidate
// column) and a named barrier of the team.  The sums run in another order
// than the oracle's, so this form is used only where parity is by
// tolerance; k_getf2 stays the bit-exact form.
// ---------------------------------------------------------------------------
template <typename T>
__host__ __device__ constexpr size_t smem_getf2_ll_bytes(int nb) {
  const size_t steps = (size_t)nb * (nb + 1) * sizeof(T)  // A and G, packed lower
                       + (size_t)2 * nb * sizeof(T)       // the formed columns
                       + (size_t)(4 + 6) * 128 * sizeof(T)  // GEMV and look-ahead partial sums
                       + 16 + 32 * 8 + 32 * 4 + 16 * 4 + 4 * (size_t)nb * 4;
  // the fused deep-row replay reuses the same memory after the write-back
  const size_t replay =
      (((size_t)(DEEP_R + 1) * nb * sizeof(T) + 15) & ~size_t(15)) + (size_t)nb * (3 * sizeof(T) + 5) + 16;
  return (steps > replay ? steps : replay) + 64;
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1) k_getf2_ll(FactorArgs fa, const int4* __restrict__ tasks, int nb_small,
                                                 int nb_big) {
  static_assert(NT == 512, "four partial sums of 128 rows");
  using F = Field<T>;
  if (fa.status[0] != 0) return;
  const double pfloor = fa.floor_dev ? *fa.floor_dev : fa.perturb_floor;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, kb = tk.y, slot = tk.z, fuse = tk.w;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int nb = ncol >= 512 ? nb_big : nb_small;
  const int ke = min(kb + nb, ncol), pw = ke - kb;
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  T* dG = reinterpret_cast<T*>(fa.d) + first + kb;
  T* dsG = reinterpret_cast<T*>(fa.dsub) + first + kb;
  unsigned char* kindG = fa.kind + first + kb;
  int* lpermG = fa.lperm + first;
  unsigned char* sc = reinterpret_cast<unsigned char*>(fa.scratch) + (long long)slot * fa.scratch_stride;
  T* snap = reinterpret_cast<T*>(sc);                              // nb x nb
  int* swaps = reinterpret_cast<int*>(snap + (long long)nb * nb);  // nb

  const int npk = pw * (pw + 1) / 2;
  T* A = reinterpret_cast<T*>(smem_raw);  // packed lower: L (pivoted columns), A0 (the rest)
  T* Gs = A + npk;                        // packed lower: G of the pivoted columns
  T* v1 = Gs + npk;                       // formed column k
  T* v2 = v1 + pw;                        // formed candidate column
  T* red = v2 + pw;                       // 4 x 128 partial sums
  double* red_v = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(red + 10 * 128) + 15) & ~uintptr_t(15));
  int* red_i = reinterpret_cast<int*>(red_v + 32);
  int* ctl = red_i + 32;  // [1] scratch [2] nswaps [3] error [4..15] the steps' control words
  int* lp_s = ctl + 16;
  int* swp_p = lp_s + nb;
  int* swp_q = swp_p + nb;
  int* supp = swp_q + nb;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  load_packed_block<T, NT>(A, panel, nrow, kb, pw);
  if (kb == 0)
    for (int p = tid; p < ncol; p += NT) lpermG[p] = p;
  for (int e = tid; e < pw; e += NT) {
    dG[e] = F::zero();
    dsG[e] = F::zero();
    kindG[e] = 0;
    swaps[e] = -1;
  }
  for (int e = tid; e < pw * nb; e += NT) snap[e] = F::zero();
  if (tid < 16) ctl[tid] = 0;  // [2] nswaps, [3] error, [4..15] the steps' control words
  __syncthreads();
  for (int i = tid; i < pw; i += NT) lp_s[i] = lpermG[kb + i];
  __syncthreads();
  const double alpha = (1.0 + sqrt(17.0)) / 8.0;
  int nperturbed = 0;
  const bool reuse = fa.pivot_reuse && fa.pivrec && *fa.pivot_reuse != 0;
  int* prec = fa.pivrec ? fa.pivrec + first + kb : nullptr;

  // Partial sums of column c over the pivoted columns p < k.  The rows
  // [k, pw) take R = 32, 64 or 128 threads each group (the smallest that
  // covers them) and the 512 / R groups split the columns: thread (row k +
  // tid % R, group g = tid / R) sums p = g, g + 512 / R, ... in two
  // interleaved accumulators (independent loads in flight).
  auto groups_of = [&](int k) { return pw - k <= 32 ? 16 : pw - k <= 64 ? 8 : 4; };
  auto gemv = [&](int k, int c) {
    const int ng = groups_of(k), lr = ng == 4 ? 7 : ng == 8 ? 6 : 5;  // R = 512 / ng = 1 << lr
    const int rr = tid & ((1 << lr) - 1), g = tid >> lr, i = k + rr, R = 1 << lr;
    if (i < pw) {
      T acc0 = F::zero(), acc1 = F::zero();
      int p = g;
      for (; p + ng < k; p += 2 * ng) {
        const int cp0 = p * pw - (p * (p + 1)) / 2, cp1 = (p + ng) * pw - ((p + ng) * (p + ng + 1)) / 2;
        acc0 = F::fma_(Gs[cp0 + i], A[cp0 + c], acc0);
        acc1 = F::fma_(Gs[cp1 + i], A[cp1 + c], acc1);
      }
      if (p < k) {
        const int cp = p * pw - (p * (p + 1)) / 2;
        acc0 = F::fma_(Gs[cp + i], A[cp + c], acc0);
      }
      red[g * R + rr] = F::add(acc0, acc1);
    }
  };
  // The row team: warps 0-3 (one per SM sub-partition), thread r owns row
  // k + r of the formed columns.  Its phases synchronise on a named barrier
  // of 128 threads; the other 12 warps only take part in the GEMVs.
  auto team_sync = []() { asm volatile("bar.sync 1, 128;" ::: "memory"); };
  // Team thread r: v[k + r] = A0(k + r, c) - the partial sums (all of the
  // row's partial loads issued before its tree sum).
  // (returns the row's value, zero for a thread past the rows, so the
  // caller's arg-max needs no shared-memory round trip)
  auto form_row = [&](int k, int c, T* v, int r) -> T {
    const int ng = groups_of(k), R = ng == 4 ? 128 : ng == 8 ? 64 : 32, i = k + r;
    T out = F::zero();
    if (r < R && i < pw) {
      const T a = i >= c ? A[pk(i, c, pw)] : A[pk(c, i, pw)];
      T part[16];
#pragma unroll
      for (int g = 0; g < 16; ++g) part[g] = g < ng ? red[g * R + r] : F::zero();
#pragma unroll
      for (int h = 8; h > 0; h >>= 1)
#pragma unroll
        for (int g = 0; g < h; ++g) part[g] = F::add(part[g], part[g + h]);
      out = F::sub(a, part[0]);
      v[i] = out;
    }
    return out;
  };
  // 1 / z with one division (the multipliers only need fp32 accuracy here)
  auto inv = [&](T z) -> T {
    if constexpr (F::complex) {
      const float rz = 1.0f / (z.re * z.re + z.im * z.im);
      return T{z.re * rz, -z.im * rz};
    } else {
      return 1.0f / z;
    }
  };
  // Warp 0 of the team: the interchange of p = k (1x1) or k + 1 (2x2) with q
  // in the unpivoted part (A0), in rows p, q of the pivoted columns (L, G)
  // and of the formed columns, in lperm and the swap log.
  auto interchange = [&](int k, int p, int q) {
    for (int i = q + 1 + lane; i < pw; i += 32) {
      T t = A[pk(i, p, pw)];
      A[pk(i, p, pw)] = A[pk(i, q, pw)];
      A[pk(i, q, pw)] = t;
    }
    for (int i = p + 1 + lane; i < q; i += 32) {
      T t = A[pk(i, p, pw)];
      A[pk(i, p, pw)] = A[pk(q, i, pw)];
      A[pk(q, i, pw)] = t;
    }
    for (int jj = lane; jj < p; jj += 32) {
      T t = A[pk(p, jj, pw)];
      A[pk(p, jj, pw)] = A[pk(q, jj, pw)];
      A[pk(q, jj, pw)] = t;
      if (jj < k) {
        t = Gs[pk(p, jj, pw)];
        Gs[pk(p, jj, pw)] = Gs[pk(q, jj, pw)];
        Gs[pk(q, jj, pw)] = t;
      }
    }
    if (lane == 0) {
      T t = A[pk(p, p, pw)];
      A[pk(p, p, pw)] = A[pk(q, q, pw)];
      A[pk(q, q, pw)] = t;
      t = v1[p];
      v1[p] = v1[q];
      v1[q] = t;
      t = v2[p];
      v2[p] = v2[q];
      v2[q] = t;
      const int lpv = lp_s[p];
      lp_s[p] = lp_s[q];
      lp_s[q] = lpv;
      swaps[k] = kb + q;
      const int ns = ctl[2];
      swp_p[ns] = kb + p;
      swp_q[ns] = kb + q;
      ctl[2] = ns + 1;
    }
  };
  // Team thread r after the interchange: the multipliers of row k + r (1x1)
  // or k + 2 + r (2x2), their G and snapshot entries, and (thread 0) D and
  // the pivot block's entries of A.  Every team thread evaluates the pivot
  // block itself (same values, same result); returns the error flag.
  auto finish_rows = [&](int k, int kstep, int kp, int r) -> bool {
    bool err = false;
    if (kstep == 1) {
      const T* v = kp == k ? v1 : v2;  // a 1x1 step with interchange pivots on the candidate column
      T dk = v[k];
      if (pfloor >= 0.0) {
        const double m = F::mag(dk);
        if (m < pfloor) {
          dk = m == 0.0 ? F::from_real(pfloor) : F::scale(dk, pfloor / m);
          if (r == 0) ++nperturbed;
        }
      } else if (F::is_zero(dk)) {
        err = true;
      }
      if (!err) {
        const T dinv = inv(dk);
        const int i = k + 1 + r;
        if (i < pw) {
          const T a = v[i], w = F::mul(a, dinv);
          Gs[pk(i, k, pw)] = a;
          snap[k * nb + i] = w;
          A[pk(i, k, pw)] = w;
        }
        if (r == 0) {
          A[pk(k, k, pw)] = dk;
          dG[k] = dk;
        }
      }
    } else {
      T d11 = v1[k], d21 = v1[k + 1], d22 = v2[k + 1];
      T det = F::sub(F::mul(d11, d22), F::mul(d21, d21));
      // the growth test |det| <= 1e-14 scale^2 on squares (scale = the
      // largest modulus of the block)
      const double scale2 = fmax(fmax(F::mag2(d11), F::mag2(d22)), F::mag2(d21));
      const double growth_floor = 1e-14 * scale2;
      if (pfloor >= 0.0) {
        const double fl = fmax(pfloor * pfloor, growth_floor);
        if (F::mag2(det) < fl * fl) {
          const double lift = fmax(pfloor, sqrt(scale2) * sqrt(1e-14));
          d11 = F::add(d11, F::from_real(lift));
          d22 = F::add(d22, F::from_real(lift));
          det = F::sub(F::mul(d11, d22), F::mul(d21, d21));
          if (F::mag2(det) < fl * fl) det = F::add(det, F::from_real(fl));
          if (r == 0) ++nperturbed;
        }
      } else if (F::mag2(det) <= growth_floor * growth_floor) {
        err = true;
      }
      if (!err) {
        const T detinv = inv(det);
        if (r == 0) {
          dG[k] = d11;
          dsG[k] = d21;
          dG[k + 1] = d22;
          kindG[k] = 1;
          kindG[k + 1] = 2;
          A[pk(k, k, pw)] = d11;
          A[pk(k + 1, k, pw)] = d21;
          A[pk(k + 1, k + 1, pw)] = d22;
        }
        const int i = k + 2 + r;
        if (i < pw) {
          const T wik = v1[i], wik1 = v2[i];
          const T a1 = F::mul(F::sub(F::mul(d22, wik), F::mul(d21, wik1)), detinv);
          const T a2 = F::mul(F::sub(F::mul(d11, wik1), F::mul(d21, wik)), detinv);
          Gs[pk(i, k, pw)] = wik;
          Gs[pk(i, k + 1, pw)] = wik1;
          snap[k * nb + i] = a1;
          snap[(k + 1) * nb + i] = a2;
          A[pk(i, k, pw)] = a1;
          A[pk(i, k + 1, pw)] = a2;
        }
      }
    }
    return err;
  };

  const bool team = tid < 128;
  const double a2 = alpha * alpha;
  // Look-ahead: while the team finishes step k, warps 4-15 form the partial
  // sums of column k + 1 over the pivoted columns p < k (the rows [k + 1,
  // pw) take R = 32, 64 or 128 of the 384 threads and the 384 / R groups
  // split the columns).  When step k is a 1x1 pivot without interchange, step k + 1 uses
  // them (adding its one missing term, p = k) and skips its GEMV and block
  // barrier.  Control words are double-buffered by iteration parity: with
  // the GEMV barrier skipped, a thread may still read iteration i's words
  // while the team writes iteration i + 1's.
  T* const rs0 = red + 4 * 128;  // two look-ahead buffers of 384 partial sums, by iteration parity
  // log2 of the rows per look-ahead group for column c: the smallest of
  // 32, 64, 128 that covers the rows [c, pw)
  auto la_lr = [&](int c) { return pw - c <= 32 ? 5 : pw - c <= 64 ? 6 : 7; };
  auto spec_gemv = [&](int k, T* out) {
    const int c = k + 1, lr = la_lr(c), ng = 384 >> lr;
    const int u = tid - 128, rr = u & ((1 << lr) - 1), g = u >> lr, i = c + rr;
    if (i < pw) {
      T acc0 = F::zero(), acc1 = F::zero();
      int p = g;
      for (; p + ng < k; p += 2 * ng) {
        const int cp0 = p * pw - (p * (p + 1)) / 2, cp1 = (p + ng) * pw - ((p + ng) * (p + ng + 1)) / 2;
        acc0 = F::fma_(Gs[cp0 + i], A[cp0 + c], acc0);
        acc1 = F::fma_(Gs[cp1 + i], A[cp1 + c], acc1);
      }
      if (p < k) {
        const int cp = p * pw - (p * (p + 1)) / 2;
        acc0 = F::fma_(Gs[cp + i], A[cp + c], acc0);
      }
      out[(g << lr) + rr] = F::add(acc0, acc1);
    }
  };
  // team thread r, look-ahead case: v[k + r] = A0(k + r, k) - the group
  // partials (all loaded, then a tree sum) - G(k + r, k - 1) L(k, k - 1);
  // returns the value (zero past the rows)
  auto form_row_la = [&](int k, const T* part, int r) -> T {
    const int i = k + r;
    T out = F::zero();
    if (i < pw) {
      const T a = A[pk(i, k, pw)];
      const int lr = la_lr(k), ng = 384 >> lr;
      const int cl = (k - 1) * pw - ((k - 1) * k) / 2;  // packed start of column k - 1
      const T gl = F::mul(Gs[cl + i], A[cl + k]);
      T pp[16];
#pragma unroll
      for (int g = 0; g < 16; ++g) pp[g] = g < ng ? part[(g << lr) + r] : F::zero();
#pragma unroll
      for (int h = 8; h > 0; h >>= 1)
#pragma unroll
        for (int g = 0; g < h; ++g) pp[g] = F::add(pp[g], pp[g + h]);
      out = F::sub(F::sub(a, pp[0]), gl);
      v1[i] = out;
    }
    return out;
  };
  for (int k = 0, it = 0; k < pw; ++it) {
    int* cc = ctl + 4 + 6 * (it & 1);         // this iteration: next k, kstep, kp, extra, error
    int* cn = ctl + 4 + 6 * ((it + 1) & 1);   // cn[5]: the next iteration may use the look-ahead
    const bool la = cc[5] != 0;
    if (!la) {
      gemv(k, k);
      __syncthreads();
    }
    if (team) {
      // column k, and per team warp the arg-max of the squared moduli below
      // the diagonal (the BK tests run on squares: no square roots or
      // divisions on the decision path)
      const int r = tid;
      const T vk = la ? form_row_la(k, rs0 + 384 * ((it + 1) & 1), r) : form_row(k, k, v1, r);
      double m2 = -1.0;
      int idx = INT_MAX;
      if (r >= 1 && k + r < pw) {
        m2 = F::mag2(vk);
        idx = k + r;
      }
      warp_argmax(m2, idx);
      if (lane == 0) {
        red_v[warp] = m2;
        red_i[warp] = idx;
      }
      if (r == 0) red_v[4] = F::mag2(vk);
      team_sync();
      // every team thread takes the same decision from the same values
      double col2 = -1.0;
      int imax = INT_MAX;
#pragma unroll
      for (int w = 0; w < 4; ++w) argmax_combine(col2, imax, red_v[w], red_i[w]);
      const double akk2 = red_v[4];
      if (col2 < 0.0) {
        col2 = 0.0;
        imax = k;
      }
      int kstep = 1, kp = k, extra = -1;
      bool err = false;
      if (reuse) {
        const int code = prec[k];
        kstep = code < 0 ? 2 : 1;
        kp = code < 0 ? -code - 1 : code;
        if (kstep == 2 || kp != k) extra = kp;
      } else if (fmax(akk2, col2) == 0.0) {
        err = pfloor < 0.0;
      } else if (akk2 < a2 * col2) {
        extra = imax;
      }
      if (extra < 0 && !err) {
        if (r == 0 && prec && !reuse) prec[k] = k;
        err = finish_rows(k, 1, k, r);
      }
      if (r == 0) {
        if (err) ctl[3] = 1;
        cc[0] = k + 1;
        cc[1] = kstep;
        cc[2] = kp;
        cc[3] = err ? -1 : extra;
        cc[4] = err ? 1 : 0;
        cn[5] = (!err && extra < 0 && k + 1 < pw) ? 1 : 0;
        red_v[5] = akk2;
        red_v[6] = col2;
      }
    } else if (k + 1 < pw) {
      spec_gemv(k, rs0 + 384 * (it & 1));
    }
    __syncthreads();
    if (cc[4]) break;
    const int extra = cc[3];
    if (extra >= 0) {
      gemv(k, extra);
      __syncthreads();
      if (team) {
        const int r = tid;
        const T ve = form_row(k, extra, v2, r);
        int kstep = cc[1], kp = cc[2];
        if (!reuse) {
          // the row maximum of the candidate row: its column over every row
          // of the unpivoted part but itself
          double m2 = 0.0;
          if (k + r < pw && k + r != extra) m2 = F::mag2(ve);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
          if (lane == 0) red_v[8 + warp] = m2;
          team_sync();
          const double rmx = fmax(fmax(red_v[8], red_v[9]), fmax(red_v[10], red_v[11]));
          // |a_kk| rowmax >= alpha colmax^2, |a_rr| >= alpha rowmax, squared
          const double akk2 = red_v[5], col2 = red_v[6];
          kstep = 1;
          kp = k;
          if (akk2 * rmx >= a2 * col2 * col2) {
          } else if (F::mag2(v2[extra]) >= a2 * rmx) {
            kp = extra;
          } else {
            kstep = 2;
            kp = extra;
          }
          if (r == 0 && prec) prec[k] = kstep == 2 ? -kp - 1 : kp;
        }
        const int p = kstep == 1 ? k : k + 1;
        if (kp != p) {
          team_sync();  // every team thread has read v2 / red_v for its decision
          if (warp == 0) interchange(k, p, kp);
        }
        team_sync();
        const bool err = finish_rows(k, kstep, kp, r);
        if (r == 0) {
          if (err) ctl[3] = 1;
          cc[0] = k + kstep;
          cc[4] = err ? 1 : 0;
        }
      }
      __syncthreads();
      if (cc[4]) break;
    }
    k = cc[0];
  }
  getf2_finish<T, NT>(fa, s, kb, pw, nb, nrow, ke, fuse, panel, A, lp_s, lpermG, ctl, swp_p, swp_q, supp,
                      reinterpret_cast<int*>(v1), kindG, dG, dsG, snap, swaps, nperturbed, smem_raw);
}

// ---------------------------------------------------------------------------
// Deep-row replay for tall panels: task = (s, kb, slot, row0); DEEP_R rows.
// ---------------------------------------------------------------------------
template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_deep(FactorArgs fa, const int4* __restrict__ tasks, int nb_small,
                                             int nb_big) {
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, kb = tk.y, slot = tk.z, rs0 = tk.w;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int nb = ncol >= 512 ? nb_big : nb_small;
  const int ke = min(kb + nb, ncol), pw = ke - kb;
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  const unsigned char* sc = reinterpret_cast<const unsigned char*>(fa.scratch) + (long long)slot * fa.scratch_stride;
  const T* snap = reinterpret_cast<const T*>(sc);
  const int* swaps = reinterpret_cast<const int*>(snap + (long long)nb * nb);
  T* X = reinterpret_cast<T*>(smem_raw);
  unsigned char* pmem = smem_raw + (((size_t)(DEEP_R + 1) * nb * sizeof(T) + 15) & ~size_t(15));
  const ReplayProg<T> P =
      load_replay_prog<T, NT>(pmem, pw, nb, swaps, reinterpret_cast<const T*>(fa.d) + first + kb,
                              reinterpret_cast<const T*>(fa.dsub) + first + kb, fa.kind + first + kb);
  __syncthreads();
  replay_deep_rows<T, NT>(panel, nrow, kb, pw, nb, rs0, min(rs0 + DEEP_R, nrow), snap, P, X);
}

// ---------------------------------------------------------------------------
// Block transform of a tall panel: rows [i0, i0 + MM_RB) of M = the replay of
// the same rows of the pw x pw identity (one row per warp, so each step's
// dependency chain is short).  Task (s, kb, slot, i0).
// ---------------------------------------------------------------------------
constexpr int MM_RB = 8;  // identity rows per block-transform CTA (one per warp)

__host__ __device__ constexpr size_t smem_make_m_off_prog(size_t es, int nb) {
  return (((size_t)(MM_RB + 1) * nb * es + 15) & ~size_t(15));
}
__host__ __device__ constexpr size_t smem_make_m_off_slice(size_t es, int nb) {
  return ((smem_make_m_off_prog(es, nb) + (size_t)nb * (3 * es + 4 + 1) + 16) + 15) & ~size_t(15);
}
// snapshot steps staged per slice: the whole block for 4- and 8-byte
// fields, 64 steps for 16-byte ones (a 128-step c64 snapshot is 256 KB)
// (launches of many blocks take 32-step slices: a quarter of the shared
// memory, so several CTAs share an SM)
__host__ __device__ constexpr int make_m_sl(size_t es) { return es >= 16 ? 64 : 128; }
constexpr int MAKE_M_SL_WIDE = 32;
__host__ __device__ constexpr size_t smem_make_m_bytes(size_t es, int nb, int sl) {
  return smem_make_m_off_slice(es, nb) + (size_t)(sl >= nb ? nb : sl + 1) * nb * es + 64;
}

template <typename T, int NT, int SL>
__global__ void __launch_bounds__(NT) k_make_m(FactorArgs fa, const int4* __restrict__ tasks, int nb_small,
                                               int nb_big) {
  static_assert(MM_RB == NT / 32, "one identity row per warp");
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, kb = tk.y, slot = tk.z, i0 = tk.w;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int nb = ncol >= 512 ? nb_big : nb_small;
  const int ke = min(kb + nb, ncol), pw = ke - kb;
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  unsigned char* sc = reinterpret_cast<unsigned char*>(fa.scratch) + (long long)slot * fa.scratch_stride;
  const T* snap = reinterpret_cast<const T*>(sc);
  const int* swaps = reinterpret_cast<const int*>(snap + (long long)nb * nb);
  T* M = reinterpret_cast<T*>(sc + replay_mm_off(nb, sizeof(T)));
  T* X = reinterpret_cast<T*>(smem_raw);
  const ReplayProg<T> P =
      load_replay_prog<T, NT>(smem_raw + smem_make_m_off_prog(sizeof(T), nb), pw, nb, swaps,
                              reinterpret_cast<const T*>(fa.d) + first + kb,
                              reinterpret_cast<const T*>(fa.dsub) + first + kb, fa.kind + first + kb);
  T* S = reinterpret_cast<T*>(smem_raw + smem_make_m_off_slice(sizeof(T), nb));
  __syncthreads();
  // the snapshot in slices of SL steps (the whole block, or two for 16-byte
  // fields, in launches of a few blocks): few staging round trips
  replay_deep_rows<T, NT, true, MM_RB, SL>(panel, nrow, kb, pw, nb, i0, min(i0 + MM_RB, pw), snap, P, X, M, S);
}

// ---------------------------------------------------------------------------
// Deep rows of a tall panel as one product: rows [r0, r0 + MM_ROWS) of the
// panel columns [kb, ke) become A21 M, M the block transform (k_make_m: the
// replay of the identity rows; the replay is linear in the row).  The row
// block is staged in shared memory first (the product overwrites it in
// place), M streams through in mm_cw-column chunks; thread (r = tid %
// MM_ROWS, g = tid / MM_ROWS) owns row r and a contiguous group of columns of
// each chunk, summing over k in ascending order.  Task (s, kb, slot, r0).  Used with the tensor
// engine of every field (the FMA engine replays row by row, in the oracle's
// operation order).
// ---------------------------------------------------------------------------
template <typename T>
__host__ __device__ constexpr int mm_cw() {
  return sizeof(T) >= 16 ? 16 : 32;
}
constexpr int MM_ROWS = 32;  // deep rows per product task
template <typename T>
__host__ __device__ constexpr size_t smem_deep_mm_bytes() {
  return ((size_t)128 * (MM_ROWS + 1) + 2 * 128 * mm_cw<T>()) * sizeof(T) + 16;
}

template <typename T>
__global__ void __launch_bounds__(256) k_deep_mm(FactorArgs fa, const int4* __restrict__ tasks, int nb_small,
                                                 int nb_big) {
  using F = Field<T>;
  constexpr int CW = mm_cw<T>(), NG = 256 / MM_ROWS, NO = CW / NG, LDA = MM_ROWS + 1;
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* As = reinterpret_cast<T*>(smem_raw);  // As[k * LDA + r]
  T* Ms = As + 128 * LDA;                  // 2 x (128 x CW), row-major chunks
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, kb = tk.y, slot = tk.z, r0 = tk.w;
  const int ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int nb = ncol >= 512 ? nb_big : nb_small;
  const int ke = min(kb + nb, ncol), pw = ke - kb;
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  const unsigned char* sc = reinterpret_cast<const unsigned char*>(fa.scratch) + (long long)slot * fa.scratch_stride;
  const T* M = reinterpret_cast<const T*>(sc + replay_mm_off(nb, sizeof(T)));
  const int tid = threadIdx.x, r = tid % MM_ROWS, g = tid / MM_ROWS;
  const int rows = min(MM_ROWS, nrow - r0);
  auto load_chunk = [&](int j0, T* dst) {
    for (int e = tid; e < 128 * CW; e += 256) {
      const int k = e / CW, j = e % CW;
      const bool ok = k < pw && j0 + j < pw;
      const T* src = ok ? M + (long long)k * nb + j0 + j : M;
      cp_async_zfill<sizeof(T)>(dst + e, src, ok);
    }
  };
  for (int e = tid; e < MM_ROWS * 128; e += 256) {
    const int rr = e % MM_ROWS, k = e / MM_ROWS;
    const bool ok = rr < rows && k < pw;
    const T* src = ok ? panel + (r0 + rr) + (long long)(kb + k) * nrow : panel;
    cp_async_zfill<sizeof(T)>(As + k * LDA + rr, src, ok);
  }
  load_chunk(0, Ms);
  cp_async_commit();
  const int nch = (pw + CW - 1) / CW;
  for (int ch = 0; ch < nch; ++ch) {
    if (ch + 1 < nch) load_chunk((ch + 1) * CW, Ms + ((ch + 1) & 1) * 128 * CW);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const T* Mc = Ms + (ch & 1) * 128 * CW + g * NO;
    T acc[NO];
#pragma unroll
    for (int j = 0; j < NO; ++j) acc[j] = F::zero();
#pragma unroll 4
    for (int k = 0; k < pw; ++k) {
      const T a = As[k * LDA + r];
      T m[NO];
      lds_row<T, NO>(Mc + k * CW, m);
#pragma unroll
      for (int j = 0; j < NO; ++j) acc[j] = F::fma_(a, m[j], acc[j]);
    }
    if (r < rows)
#pragma unroll
      for (int j = 0; j < NO; ++j) {
        const int col = ch * CW + g * NO + j;
        if (col < pw) panel[(r0 + r) + (long long)(kb + col) * nrow] = acc[j];
      }
    __syncthreads();  // chunk consumed before its buffer is refilled
  }
}

// ---------------------------------------------------------------------------
// Force-accept floor: max(max_ij |A_scaled ij|, 1) * eps over the assembled
// panels (every stored entry of the equilibrated matrix lands in exactly one
// slot; the other slots are zero).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_panel_absmax(long long m, const T* __restrict__ panel, unsigned long long* __restrict__ out) {
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    v = fmax(v, Field<T>::mag(panel[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __double_as_longlong(v));
}

__global__ void k_force_floor(const unsigned long long* __restrict__ amax, double* __restrict__ floor_out) {
  const double a = __longlong_as_double(*amax);
  *floor_out = fmax(a, 1.0) * 2.220446049250313e-16;
}

// ---------------------------------------------------------------------------
// Incomplete factor (drop_tol): per pivot column p of every panel, drop the
// multipliers below tau * max |L_ip| (rows below the pivot, the 2x2 coupling
// slot excluded) — ldlt_emit_and_free, src/numeric/multifrontal_ldlt.rs:2359.
// One CTA per supernode, one warp per column.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_drop_tol(FactorArgs fa, double tau) {
  using F = Field<T>;
  if (fa.status[0] != 0) return;
  const int s = blockIdx.x;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int p = warp; p < ncol; p += nw) {
    const int i0 = p + (fa.kind[first + p] == 1 ? 2 : 1);
    T* col = panel + (long long)p * nrow;
    double cm = 0.0;
    for (int i = i0 + lane; i < nrow; i += 32) cm = fmax(cm, F::mag(col[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cm = fmax(cm, __shfl_xor_sync(0xffffffffu, cm, o));
    const double thresh = tau * cm;
    for (int i = i0 + lane; i < nrow; i += 32)
      if (F::mag(col[i]) < thresh) col[i] = F::zero();
  }
}

}  // namespace rsd
