// Triangular-solve kernels of the supernodal solve that stream the panels
// at memory bandwidth, and the dependency-chain solve of the wide
// supernodes' diagonal blocks.
//
// Streaming (k_stream): the forward push U_s = L21_s z_s and the backward
// off-diagonal dots L21_s^T x_anc.  An item owns 64 outputs and loops over
// 32-wide reduction units; each unit's 2048-element panel tile and its 32
// right-hand-side rows are copied global -> shared with cp.async (zero
// filled outside the panel), `st_stages<T>(NR)` units in flight, one CTA
// barrier per unit.  Tile layouts keep every lane on consecutive or odd
// strided shared memory:
//   forward  : 64 output rows x 32 reduction columns, S[q * 65 + r]
//   backward : 32 reduction rows x 64 output columns, S[p * 33 + r]
// Thread (x = tid & 63, g = tid >> 6) owns output x and the reduction slice
// [8g, 8g + 8) of every unit; the four slice partials are added in order
// g = 0..3 at the end, so results are deterministic.  The right-hand sides
// read here are final before the launch (forward: z of this level, solved
// by an earlier launch; backward: the ancestors' x, each unit's 32 rows
// read through the supernode's row structure).
//
// Chain (k_chain): every supernode is cut into TB = 64 column blocks whose
// solves form a chain (forward: block i needs z of blocks j < i; backward:
// x of blocks j > i).  One CTA per block and group of at most CH_NR
// right-hand-side columns (the columns' chains are independent):
//   forward : z_i = Linv_i (y_i - sum_{j<i} L_ij z_j)
//   backward: x_i = Linv_i^T (w_i - W_i - sum_{j>i, descending} L_ji^T x_j)
// with Linv_i the precomputed inverse of the unit-lower diagonal block and
// W_i the off-diagonal dots.  The 64 x 64 tiles stream through shared
// memory ahead of the chain; z_j / x_j are read (L2 only) after block j's
// flag.  Items are handed out in ticket order (an atomic counter per launch,
// not blockIdx) and every item waits only on items with smaller tickets,
// whose CTAs have therefore started, so the chain progresses whatever the
// number of resident CTAs.  A finished block is published by one thread
// after a CTA barrier: fence, then a gpu-scope release store of the flag; a
// waiting CTA polls with acquire loads a bounded number of times and on
// timeout raises the launch-wide abort word and a sticky status that the
// host reads after the solve.
// Reference: the column-block substitution of solve_ldlt_block
// (src/dense/ldlt_generic.rs:618-714), reorganised as a dependency chain.
#pragma once

#include "async_copy.cuh"
#include "solve_kernels.cuh"

namespace rsd {

constexpr int WV_NT = 256;
constexpr long WV_POLL_LIMIT = 1L << 21;  // flag polls before a wait gives up
constexpr int ST_UNIT = 2112;             // streamed tile elements (max of 32 x 65 and 64 x 33)
constexpr int CH_UNIT = 64 * 65;          // chain tile elements
constexpr int BWD_CH = 512;               // off-diagonal rows per backward-dot item
constexpr int PUSH_KS = 16;               // column units (of 32) per forward-push item of a wide supernode
// The right-hand sides of a pass are solved as CH_GROUPS independent chains
// of at most CH_NR columns (more CTAs, shorter per-block products).
constexpr int CH_NR = 4;
constexpr int CH_GROUPS = RHS_MAX / CH_NR;
// blocks in a level from which its chains take every column of a pass
constexpr int CH_WIDE_ITEMS = 600;

// Stages in flight: 4, or 3 where the wide elements of 16 right-hand sides
// would otherwise keep a second CTA off the SM.
template <typename T>
__host__ __device__ constexpr int st_stages(int nr) {
  return (sizeof(T) >= 16 || (sizeof(T) >= 8 && nr >= 16)) ? 3 : 4;
}

// Right-hand-side buffers are sized by the pass's column count nr (<=
// RHS_MAX), so a one-column solve keeps several CTAs resident per SM; the
// kernels are instantiated for NR = 1, 4 and 16 register columns (the
// smallest NR >= nr runs) so the inner loops carry no dead columns.
// Streaming: stages of (tile + 32 x nr right-hand sides), then the slice
// partials (4 x nr x 65).
template <typename T>
__host__ __device__ constexpr size_t st_stage_elems(int nr) {
  return (size_t)ST_UNIT + 32 * nr;
}
template <typename T>
__host__ __device__ constexpr size_t st_smem_bytes(int nr) {
  return ((size_t)st_stages<T>(nr) * st_stage_elems<T>(nr) + 4 * 65 * nr) * sizeof(T) + 16;
}
// Chain: one tile slot (its copy overlaps the wait for the dependency's
// flag; after the chain it holds the slice partials), the inverse block,
// right-hand sides (64 x nr) and the block vector (64 x nr).
template <typename T>
__host__ __device__ constexpr size_t ch_smem_bytes(int nr) {
  return ((size_t)2 * CH_UNIT + 64 * nr + 64 * nr) * sizeof(T) + 16;
}

// Wave state (ints): [0] sticky status (nonzero after a timed-out wait;
// cleared by the host when read), then the per-pass region cleared before
// every pass: [1] abort word, [2, 2 + nchain) ticket counters, then the
// forward and the backward block flags.
constexpr int WV_STATE_ABORT = 1;
constexpr int WV_STATE_CTR = 2;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// L2-only loads of vectors written by other CTAs of the same launch.
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ld_cg(const float* p) { return __ldcg(p); }
__device__ __forceinline__ c64 ld_cg(const c64* p) {
  const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
  return c64{v.x, v.y};
}
__device__ __forceinline__ c32 ld_cg(const c32* p) {
  const float2 v = __ldcg(reinterpret_cast<const float2*>(p));
  return c32{v.x, v.y};
}

// Slice partials live at red[(g * NR + c) * 65 + x] (lanes over x write
// consecutive words).  The sum over g = 0..3 in order:
template <typename T, int NR>
__device__ __forceinline__ T slice_sum(const T* red, int x, int c) {
  using F = Field<T>;
  T s = red[c * 65 + x];
  s = F::add(s, red[(NR + c) * 65 + x]);
  s = F::add(s, red[(2 * NR + c) * 65 + x]);
  return F::add(s, red[(3 * NR + c) * 65 + x]);
}
template <typename T, int NR>
__device__ __forceinline__ void store_partials(T* red, const T (&acc)[NR], int x, int g) {
#pragma unroll
  for (int c = 0; c < NR; ++c) red[(g * NR + c) * 65 + x] = acc[c];
}

// ---------------------------------------------------------------------------
// Streaming items.  Forward push (s, r0, nrb): U rows [r0, r0 + 64 nrb) of s
// = L[ncol + r, :] z_s, one 64-row block after another (narrow supernodes
// take several blocks per item so an item streams a few units at least).
// Backward dots (s, i, r0, slot): for the columns of block i, sum over
// off-diagonal rows [ncol + r0, ncol + r0 + BWD_CH) of L[r, p] x_anc[r];
// slot < 0 (the only chunk) writes Wb, else partial sums go to slot `slot`
// (64 x ld each), which the backward chain item of block i adds up in chunk
// order.
// ---------------------------------------------------------------------------
template <typename T, bool FWD>
struct StItem {
  const T* L;
  long long ld;       // panel leading dimension (nrow)
  int r0, rlim;       // tile rows
  int c0, clim;       // tile columns
  const T* V;         // right-hand-side row 0 of the item (row stride a.ld); backward: x in g order
  const int* vrows;   // backward: g of each of the item's rows (x is read through it)
  int vlim;           // right-hand-side rows valid < vlim (relative)
  int cu;             // forward: column units per 64-row block (of this item's column chunk)
  int cb0;            // forward: first column unit of the item
  int nunits;
};

template <typename T, bool FWD>
__device__ __forceinline__ StItem<T, FWD> st_item(const SolveArgs& a, int4 tk) {
  const int s = tk.x;
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  StItem<T, FWD> it;
  it.L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  it.ld = nrow;
  if (FWD) {
    it.r0 = ncol + tk.y; it.rlim = nrow;
    it.c0 = 0; it.clim = ncol;
    it.V = reinterpret_cast<const T*>(a.Ze) + a.c0 + (long long)first * a.ld;
    it.vlim = ncol;
    // z = nrb | first column unit << 8; wide supernodes' items take
    // PUSH_KS column units each (partial sums to slot w)
    it.cb0 = tk.z >> 8;
    it.cu = min(PUSH_KS, (ncol + 31) / 32 - it.cb0);
    if (tk.w < 0) it.cu = (ncol + 31) / 32;
    const int nrb = min(tk.z & 255, (nrow - it.r0 + 63) / 64);
    it.nunits = nrb * it.cu;
  } else {
    it.r0 = ncol + tk.z; it.rlim = min(nrow, it.r0 + BWD_CH);
    it.c0 = tk.y * TB; it.clim = ncol;
    // the ancestors' x straight from the solution vector: row r of the item
    // is g = rs[ncol + r0 + r] (no gathered copy)
    it.V = reinterpret_cast<const T*>(a.Xg) + a.c0;
    it.vrows = a.rs + a.sn_rsoff[s] + ncol + tk.z;
    it.vlim = it.rlim - it.r0;
    it.cu = 1;
    it.cb0 = 0;
    it.nunits = (it.vlim + 31) / 32;
  }
  return it;
}

template <typename T, bool FWD, int NR>
__device__ __forceinline__ void st_issue(T* S, T* Vs, const StItem<T, FWD>& it, int u, int ld, int nr) {
  int rr0, cc0, vr0;
  if constexpr (FWD) {
    const int rb = u / it.cu, cb = it.cb0 + u - rb * it.cu;
    rr0 = it.r0 + 64 * rb; cc0 = 32 * cb; vr0 = 32 * cb;
  } else {
    rr0 = it.r0 + 32 * u; cc0 = it.c0; vr0 = 32 * u;
  }
#pragma unroll
  for (int m = 0; m < 2048 / WV_NT; ++m) {
    const int e = threadIdx.x + WV_NT * m;
    int r, c, dst;
    if constexpr (FWD) {
      r = rr0 + (e & 63); c = cc0 + (e >> 6); dst = (e >> 6) * 65 + (e & 63);
    } else {
      r = rr0 + (e & 31); c = cc0 + (e >> 5); dst = (e >> 5) * 33 + (e & 31);
    }
    const bool ok = r < it.rlim && c < it.clim;
    const T* g = ok ? it.L + r + (long long)c * it.ld : it.L;
    cp_async_zfill<sizeof(T)>(S + dst, g, ok);
  }
  for (int e = threadIdx.x; e < 32 * nr; e += WV_NT) {
    const int k = e / nr, c = e - k * nr, row = vr0 + k;
    const bool ok = row < it.vlim;
    const long long vr = FWD ? row : (ok ? it.vrows[row] : 0);
    const T* g = ok ? it.V + vr * ld + c : it.V;
    cp_async_zfill<sizeof(T)>(Vs + k * NR + c, g, ok);
  }
}

template <typename T, bool FWD, int NR>
__global__ void __launch_bounds__(WV_NT) k_stream(SolveArgs a, const int4* __restrict__ tasks) {
  using F = Field<T>;
  constexpr int NST = st_stages<T>(NR);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nr = a.nrhs, ld = a.ld;
  constexpr int SE = (int)st_stage_elems<T>(NR);
  T* stages = reinterpret_cast<T*>(smem_raw);  // NST x (tile, V rows of stride NR)
  T* red = stages + NST * SE;                  // slice partials, 4 x NR x 65
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x;
  const StItem<T, FWD> it = st_item<T, FWD>(a, tk);
  const int tid = threadIdx.x, x = tid & 63, g = tid >> 6;
  T acc[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) acc[c] = F::zero();
  // slice partials of the finished output block -> U (forward) / Wb / slot
  auto flush = [&](int rb) {
    store_partials<T, NR>(red, acc, x, g);
#pragma unroll
    for (int c = 0; c < NR; ++c) acc[c] = F::zero();
    __syncthreads();
    for (int e = tid; e < 64 * nr; e += WV_NT) {
      const int r = e / nr, c = e - r * nr;
      const T v = slice_sum<T, NR>(red, r, c);
      if (FWD) {
        const int row = it.r0 + 64 * rb + r;
        if (row < it.rlim) {
          if (tk.w < 0) {
            T* Us = reinterpret_cast<T*>(a.U) + a.c0 + a.uoff[s] * ld;
            Us[(long long)(row - a.sn_ncol[s]) * ld + c] = v;
          } else {
            T* part = reinterpret_cast<T*>(a.Wp) + (long long)tk.w * 64 * ld;
            part[(long long)r * ld + c] = v;
          }
        }
      } else if (it.c0 + r < it.clim) {
        if (tk.w < 0) {
          T* Wb = reinterpret_cast<T*>(a.Wb) + a.c0 + (long long)a.sn_first[s] * ld;
          Wb[(long long)(it.c0 + r) * ld + c] = v;
        } else {
          T* part = reinterpret_cast<T*>(a.Wp) + (long long)tk.w * 64 * ld;
          part[(long long)r * ld + c] = v;
        }
      }
    }
  };
#pragma unroll 1
  for (int u = 0; u < NST - 1; ++u) {
    T* S = stages + u * SE;
    if (u < it.nunits) st_issue<T, FWD, NR>(S, S + ST_UNIT, it, u, ld, nr);
    cp_async_commit();
  }
#pragma unroll 1
  for (int u = 0; u < it.nunits; ++u) {
    if (FWD && u > 0 && u % it.cu == 0) flush(u / it.cu - 1);
    cp_async_wait<NST - 2>();
    __syncthreads();  // unit u landed everywhere; unit u - 1's stage and the partials are free
    {
      const int un = u + NST - 1;
      T* Sn = stages + (un % NST) * SE;
      if (un < it.nunits) st_issue<T, FWD, NR>(Sn, Sn + ST_UNIT, it, un, ld, nr);
      cp_async_commit();
    }
    const T* S = stages + (u % NST) * SE;
    const T* V = S + ST_UNIT;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int q = 8 * g + k;
      const T l = FWD ? S[q * 65 + x] : S[x * 33 + q];
      T v[NR];
      lds_row<T, NR>(V + q * NR, v);
#pragma unroll
      for (int c = 0; c < NR; ++c) acc[c] = F::fma_(l, v[c], acc[c]);
    }
  }
  cp_async_wait<0>();
  if (it.nunits > 0) flush(FWD ? (it.nunits - 1) / it.cu : 0);
}

// Forward: sum the column-chunk partials of (s, 64-row block r0) in chunk
// order into U.  Task (s, r0, slot0, nchunks).
template <typename T>
__global__ void __launch_bounds__(WV_NT) k_push_reduce(SolveArgs a, const int4* __restrict__ tasks) {
  using F = Field<T>;
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = tk.y, slot0 = tk.z, nch = tk.w;
  const int off = a.sn_nrow[s] - a.sn_ncol[s];
  const int ld = a.ld, nr = a.nrhs;
  const T* part = reinterpret_cast<const T*>(a.Wp) + (long long)slot0 * 64 * ld;
  T* Us = reinterpret_cast<T*>(a.U) + a.c0 + a.uoff[s] * ld;
  for (int e = threadIdx.x; e < 64 * nr; e += WV_NT) {
    const int r = e / nr, c = e - r * nr;
    if (r0 + r >= off) continue;
    T v = part[(long long)r * ld + c];
    for (int k = 1; k < nch; ++k) v = F::add(v, part[((long long)k * 64 + r) * ld + c]);
    Us[(long long)(r0 + r) * ld + c] = v;
  }
}

// ---------------------------------------------------------------------------
// Chain items (s, 0 / 1 = forward / backward, block i, first flag of s).
// ---------------------------------------------------------------------------

// Wait (thread 0) until flag `f` is set; false on timeout or abort.
__device__ __forceinline__ bool wv_wait(const int* flags, int f, int* state) {
  for (long it = 0; it < WV_POLL_LIMIT; ++it) {
    if (ld_acquire_gpu(flags + f) != 0) return true;
    if (ld_volatile(state + WV_STATE_ABORT) != 0) return false;
  }
  atomicExch(state + WV_STATE_ABORT, 1);
  atomicExch(state, 1);
  return false;
}

// Copy the 64 x 64 tile at (r0, c0) of a column-major source (rows < rlim,
// columns < clim, zero elsewhere) into S[c * 65 + r].
template <typename T>
__device__ __forceinline__ void ch_issue(T* S, const T* src, long long ld, int r0, int rlim, int c0, int clim) {
#pragma unroll
  for (int m = 0; m < 4096 / WV_NT; ++m) {
    const int e = threadIdx.x + WV_NT * m;
    const int r = e & 63, c = e >> 6;
    const bool ok = r0 + r < rlim && c0 + c < clim;
    const T* g = ok ? src + (r0 + r) + (long long)(c0 + c) * ld : src;
    cp_async_zfill<sizeof(T)>(S + c * 65 + r, g, ok);
  }
}

// acc[c] += sum over the thread's 16 reduction entries of the 64 x 64 tile
// S (forward: S[q * 65 + x] = A[x, q]; backward: S[x * 65 + q] = A[q, x])
// times V[q * nr + c].
template <typename T, bool FWD, int NR>
__device__ __forceinline__ void ch_tile_mv(T (&acc)[NR], const T* S, const T* V, int x, int g) {
  using F = Field<T>;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int q = 16 * g + k;
    const T l = FWD ? S[q * 65 + x] : S[x * 65 + q];
    T v[NR];
    lds_row<T, NR>(V + q * NR, v);
#pragma unroll
    for (int c = 0; c < NR; ++c) acc[c] = F::fma_(l, v[c], acc[c]);
  }
}

// gw: right-hand-side columns per chain group (CH_NR, or every column of the
// pass for the levels whose items already fill the GPU: one CTA per block
// then reads the block's inverse and dependency tiles once).
template <typename T, bool FWD, int NR>
__global__ void __launch_bounds__(WV_NT) k_chain(SolveArgs a, const int4* __restrict__ tasks, int ctr, int flag_base,
                                                 int gw) {
  using F = Field<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int sh_t, sh_abort;
  const int ld = a.ld;
  T* S = reinterpret_cast<T*>(smem_raw);  // dependency tile; later the slice partials (4 x NR x 65)
  T* red = S;
  T* Lv = S + CH_UNIT;                    // the inverse block
  T* Vs = Lv + CH_UNIT;                   // 64 x NR
  T* wv = Vs + 64 * NR;                   // 64 x NR
  const int tid = threadIdx.x, x = tid & 63, g = tid >> 6;
  if (tid == 0) {
    sh_t = atomicAdd(a.wstate + WV_STATE_CTR + ctr, 1);
    sh_abort = 0;
  }
  __syncthreads();
  if (ld_volatile(a.wstate + WV_STATE_ABORT) != 0) return;
  const int4 tk = tasks[sh_t];
  const int s = tk.x, i = tk.z, fb = tk.w;
  // column group: columns [cg0, cg0 + nr) of the pass; a group with no
  // columns in this pass has nothing to do (its dependents are in the same
  // group)
  const int cg0 = gw * (tk.y >> 1);
  const int nr = min(gw, a.nrhs - cg0);
  if (nr <= 0) return;
  // flags of group g: flag index (fb + block) * CH_GROUPS + g
  int* flags = a.wstate + flag_base + (long long)fb * CH_GROUPS + (tk.y >> 1);
  const int first = a.sn_first[s], ncol = a.sn_ncol[s], nrow = a.sn_nrow[s];
  const int nblk = (ncol + TB - 1) / TB, nb = min(TB, ncol - i * TB);
  const T* L = reinterpret_cast<const T*>(a.panel) + a.sn_poff[s];
  const T* Li = reinterpret_cast<const T*>(a.linv) + a.linv_off[s] + (long long)i * TB * TB;
  T* Ze = reinterpret_cast<T*>(a.Ze) + a.c0 + cg0 + (long long)first * ld;
  // dependency blocks in chain order: step u is block dep(u)
  const int nd = FWD ? i : nblk - 1 - i;
  auto dep = [&](int u) { return FWD ? u : nblk - 1 - u; };
  auto issue = [&](int u) {
    const int j = dep(u);
    if (FWD) ch_issue<T>(S, L, nrow, i * TB, ncol, j * TB, ncol);
    else ch_issue<T>(S, L, nrow, j * TB, ncol, i * TB, ncol);
  };
  ch_issue<T>(Lv, Li, ncol <= TB ? ncol : TB, 0, nb, 0, nb);
  if (nd > 0) issue(0);
  cp_async_commit();
  // block vector.  Forward: y_i, gathered here — the right-hand side at
  // g = first + lperm[p] minus every push that lands on g, in update-list
  // order (the pull list of g, built at analysis; the pushes are final
  // before this launch), so no separate gather pass.  Backward: w_i - W_i
  // (W_i = off-diagonal dots; for a supernode whose dots were split into
  // row chunks, the chunk partials summed here in chunk order).
  const T* Wb = (!FWD && nrow > ncol) ? reinterpret_cast<const T*>(a.Wb) + a.c0 + cg0 + (long long)first * ld : nullptr;
  const int2 dred = FWD ? make_int2(0, 0) : a.dots_red[s];
  const T* Wpart = reinterpret_cast<const T*>(a.Wp) + (long long)(dred.x + i * dred.y) * 64 * ld + cg0;
  for (int e = tid; e < 64 * NR; e += WV_NT) {
    const int r = e / NR, c = e % NR;
    T v = F::zero();
    if (r < nb && c < nr) {
      if constexpr (FWD) {
        const int gg = first + a.lperm[first + i * TB + r];
        const T* Uc = reinterpret_cast<const T*>(a.U) + a.c0 + cg0 + c;
        v = reinterpret_cast<const T*>(a.Yg)[a.c0 + cg0 + (long long)gg * ld + c];
        const int t0 = a.pull_ptr[gg], t1 = a.pull_ptr[gg + 1];
#pragma unroll 4
        for (int t = t0; t < t1; ++t) v = F::sub(v, Uc[(long long)a.pull_src[t] * ld]);
      } else {
        v = ld_cg(Ze + (long long)(i * TB + r) * ld + c);
        if (dred.y > 1) {
          T w = Wpart[(long long)r * ld + c];
          for (int q = 1; q < dred.y; ++q) w = F::add(w, Wpart[((long long)q * 64 + r) * ld + c]);
          v = F::sub(v, w);
        } else if (Wb) {
          v = F::sub(v, Wb[(long long)(i * TB + r) * ld + c]);
        }
      }
    }
    wv[e] = v;
  }
  T acc[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) acc[c] = F::zero();
#pragma unroll 1
  for (int u = 0; u < nd; ++u) {
    const int j = dep(u);
    if (tid == 0 && !wv_wait(flags, j * CH_GROUPS, a.wstate)) sh_abort = 1;
    cp_async_wait<0>();
    __syncthreads();  // tile u landed; flag j observed
    if (sh_abort) return;
    for (int e = tid; e < 64 * NR; e += WV_NT) {
      const int r = e / NR, c = e % NR;
      Vs[e] = (c < nr && j * TB + r < ncol) ? ld_cg(Ze + (long long)(j * TB + r) * ld + c) : F::zero();
    }
    __syncthreads();
    ch_tile_mv<T, FWD, NR>(acc, S, Vs, x, g);
    __syncthreads();  // tile and right-hand sides consumed
    if (u + 1 < nd) issue(u + 1);
    cp_async_commit();
  }
  cp_async_wait<0>();
  // wv -= sum of the slice partials, then the inverse block
  store_partials<T, NR>(red, acc, x, g);
#pragma unroll
  for (int c = 0; c < NR; ++c) acc[c] = F::zero();
  __syncthreads();
  for (int e = tid; e < 64 * NR; e += WV_NT) {
    const int r = e / NR, c = e % NR;
    wv[e] = (r < nb && c < nr) ? F::sub(wv[e], slice_sum<T, NR>(red, r, c)) : F::zero();
  }
  __syncthreads();
  ch_tile_mv<T, FWD, NR>(acc, Lv, wv, x, g);
  store_partials<T, NR>(red, acc, x, g);
  __syncthreads();
  for (int e = tid; e < 64 * nr; e += WV_NT) {
    const int r = e / nr, c = e - r * nr;
    if (r >= nb) continue;
    const T v = slice_sum<T, NR>(red, r, c);
    Ze[(long long)(i * TB + r) * ld + c] = v;
    if (!FWD) {
      T* Xw = reinterpret_cast<T*>(a.Xg) + a.c0 + cg0;
      Xw[(long long)(first + a.lperm[first + i * TB + r]) * ld + c] = v;
    }
  }
  __syncthreads();
  // the release store orders the CTA's stores above (barrier, then a
  // cumulative gpu-scope release)
  if (tid == 0) st_release_gpu(flags + (long long)i * CH_GROUPS, 1);
}

}  // namespace rsd
