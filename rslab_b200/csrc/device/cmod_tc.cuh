// Tensor-core cmod for the single-precision factor fields (f32, c32):
// the descendant updates of one 128 x 64 target tile accumulate in TMEM with
// tcgen05.mma kind::tf32 in the 3xTF32 split (hi*hi + hi*lo + lo*hi, fp32
// accuracy), and the tile is read-modify-written once at the end.
//
// Task (s, rt << 16 | ct, pair_begin, pair_end): tile rows [128 rt, +128) x
// columns [64 ct, +64) of s's panel.  Pair (k, a, q0, nr << 16 | nc): k's
// off-diagonal rows [a, a+nr) land on tile rows, its rows [q0, q0+nc) on
// tile columns; U = L_k[a.., :] D_k L_k[q0.., :]^T.  The scatter is applied
// while staging: operand row t of A holds the k row that maps to tile row t
// (zero when none), operand row u of B holds the row of G = L_k D_k that
// maps to tile column u, so every pair of every updater adds into the same
// accumulator and the K dimension is the concatenation of the updaters'
// columns.  Complex operands use the real embedding
//   A' = [Ar | Ai],  B' = [[Gr, -Gi], [Gi, Gr]]  ->  A' B'^T = [Re | Im],
// i.e. M = 128, N = 128, and 16 complex columns of k per 32-wide K stage.
// Two stages: staging of chunk i+1 overlaps the MMAs of chunk i; one thread
// issues the MMAs and commits them to the stage's mbarrier, which gates the
// reuse of that stage.  Every wait is bounded; on a timeout the kernel flags
// status 2, drains what it issued (bounded) and frees its TMEM.
// Reference: ll_factor_node cmod, src/numeric/multifrontal_ldlt.rs:2452-2728.
#pragma once

#include "factor_kernels.cuh"
#include "tcgen05.cuh"

namespace rsd {

constexpr int TC_M = 128;                 // target tile rows = UMMA M
constexpr int TC_N = 64;                  // target tile columns
constexpr int TC_NT = 256;                // threads per CTA
constexpr int TC_OPER = 16384;            // bytes of one 128 x 32 fp32 operand tile
constexpr int TC_STAGE = 4 * TC_OPER;     // A hi, A lo, B hi, B lo
constexpr uint32_t TC_TMEM_COLS = 128;

template <typename T> struct TcShape;
template <> struct TcShape<float> {
  static constexpr int kc = 32;  // columns of k per stage
  static constexpr int n = 64;   // UMMA N
};
template <> struct TcShape<c32> {
  static constexpr int kc = 16;
  static constexpr int n = 128;
};

__host__ __device__ constexpr size_t smem_cmod_tc_bytes() {
  return 1024 + 2 * (size_t)TC_STAGE + (TC_M + TC_M + TC_N) * 4 + 64;
}

__device__ __forceinline__ void store_split4(unsigned char* hi_tile, unsigned char* lo_tile, int row, int k4,
                                             const float (&v)[4]) {
  float4 h, l;
  split_tf32(v[0], h.x, l.x);
  split_tf32(v[1], h.y, l.y);
  split_tf32(v[2], h.z, l.z);
  split_tf32(v[3], h.w, l.w);
  const uint32_t off = sw128_off((uint32_t)row, (uint32_t)(4 * k4));
  *reinterpret_cast<float4*>(hi_tile + off) = h;
  *reinterpret_cast<float4*>(lo_tile + off) = l;
}

// Stage one K chunk of pair (k, a, q0) into the operand tiles of a stage.
template <typename T>
__device__ __forceinline__ void tc_stage(unsigned char* stg, const T* __restrict__ LA, const T* __restrict__ LB,
                                         int nrk, int nck, int t0, const int* invrow, const int* invcol,
                                         const T* __restrict__ dk, const T* __restrict__ dsk,
                                         const unsigned char* __restrict__ kindk) {
  using F = Field<T>;
  unsigned char* Ah = stg;
  unsigned char* Al = stg + TC_OPER;
  unsigned char* Bh = stg + 2 * TC_OPER;
  unsigned char* Bl = stg + 3 * TC_OPER;
  const int tid = threadIdx.x;
  if constexpr (Field<T>::complex) {
    {  // A': row t <- k row invrow[t]; chunks 0-3 real parts, 4-7 imaginary parts
      const int row = tid & (TC_M - 1), grp = tid >> 7;
      const int i = invrow[row];
#pragma unroll
      for (int gi = 0; gi < 2; ++gi) {
        const int g = grp + 2 * gi;
        float re[4], im[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int t = t0 + 4 * g + jj;
          T v = F::zero();
          if (i >= 0 && t < nck) v = LA[i + (long long)t * nrk];
          re[jj] = v.re;
          im[jj] = v.im;
        }
        store_split4(Ah, Al, row, g, re);
        store_split4(Ah, Al, row, 4 + g, im);
      }
    }
    {  // B': row u (Re out) = [Gr, -Gi], row 64 + u (Im out) = [Gi, Gr]
      const int u = tid & (TC_N - 1), g = tid >> 6;
      const int j = invcol[u];
      float gr[4], gi[4], ngi[4];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int t = t0 + 4 * g + jj;
        T v = F::zero();
        if (j >= 0 && t < nck) v = ld_G(LB, nrk, j, t, dk, dsk, kindk);
        gr[jj] = v.re;
        gi[jj] = v.im;
        ngi[jj] = -v.im;
      }
      store_split4(Bh, Bl, u, g, gr);
      store_split4(Bh, Bl, u, 4 + g, ngi);
      store_split4(Bh, Bl, TC_N + u, g, gi);
      store_split4(Bh, Bl, TC_N + u, 4 + g, gr);
    }
  } else {
    {
      const int row = tid & (TC_M - 1), grp = tid >> 7;
      const int i = invrow[row];
#pragma unroll
      for (int gi = 0; gi < 4; ++gi) {
        const int g = grp + 2 * gi;
        float v[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int t = t0 + 4 * g + jj;
          v[jj] = (i >= 0 && t < nck) ? LA[i + (long long)t * nrk] : 0.0f;
        }
        store_split4(Ah, Al, row, g, v);
      }
    }
    {
      const int u = tid & (TC_N - 1), grp = tid >> 6;
      const int j = invcol[u];
#pragma unroll
      for (int gi = 0; gi < 2; ++gi) {
        const int g = grp + 4 * gi;
        float v[4];
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const int t = t0 + 4 * g + jj;
          v[jj] = (j >= 0 && t < nck) ? ld_G(LB, nrk, j, t, dk, dsk, kindk) : 0.0f;
        }
        store_split4(Bh, Bl, u, g, v);
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(TC_NT, 1) k_cmod_tc(FactorArgs fa, const int4* __restrict__ tasks,
                                                      const int4* __restrict__ pairs) {
  using F = Field<T>;
  using Sh = TcShape<T>;
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];  // re-aligned to 1024 below
  const uint32_t sraw = smem_u32(smem_raw);
  unsigned char* sm = smem_raw + (((sraw + 1023u) & ~1023u) - sraw);
  int* rs_tile = reinterpret_cast<int*>(sm + 2 * TC_STAGE);  // TC_M
  int* invrow = rs_tile + TC_M;                              // TC_M
  int* invcol = invrow + TC_M;                               // TC_N
  uint64_t* bar = reinterpret_cast<uint64_t*>(invcol + TC_N);  // 2
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);

  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = (tk.y >> 16) * TC_M, c0 = (tk.y & 0xffff) * TC_N;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int rows_here = min(TC_M, nrow - r0), cols_here = min(TC_N, ncol - c0);
  const int* rss = fa.rs + fa.sn_rsoff[s];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid < TC_M) rs_tile[tid] = tid < rows_here ? rss[r0 + tid] : INT_MAX;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, TC_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = idesc_tf32(TC_M, Sh::n);

  const T* dall = reinterpret_cast<const T*>(fa.d);
  const T* dsall = reinterpret_cast<const T*>(fa.dsub);
  const T* pall = reinterpret_cast<const T*>(fa.panel);
  int it = 0;        // K chunks issued
  bool ok = true;    // every wait so far completed (uniform across the CTA)
  for (int u = tk.z; u < tk.w && ok; ++u) {
    const int4 pr = pairs[u];
    const int k = pr.x, a = pr.y, q0 = pr.z, nr = pr.w >> 16, nc = pr.w & 0xffff;
    const int nck = fa.sn_ncol[k], nrk = fa.sn_nrow[k], fk = fa.sn_first[k];
    const int* okr = fa.rs + fa.sn_rsoff[k] + nck;
    __syncthreads();  // the previous pair's staging no longer reads the maps
    if (tid < TC_M) invrow[tid] = -1;
    if (tid < TC_N) invcol[tid] = -1;
    __syncthreads();
    if (tid < nr) invrow[lower_bound_i(rs_tile, 0, rows_here, okr[a + tid])] = tid;
    if (tid < nc) invcol[okr[q0 + tid] - first - c0] = tid;
    __syncthreads();
    const T* Lk = pall + fa.sn_poff[k];
    for (int t0 = 0; t0 < nck; t0 += Sh::kc) {
      const int st = it & 1;
      unsigned char* stg = sm + st * TC_STAGE;
      if (it >= 2) {
        const bool done = mbar_wait_bounded(&bar[st], (uint32_t)(((it >> 1) - 1) & 1));
        if (__syncthreads_or(!done)) {
          ok = false;
          break;
        }
      }
      tc_stage<T>(stg, Lk + nck + a, Lk + nck + q0, nrk, nck, t0, invrow, invcol, dall + fk, dsall + fk,
                  fa.kind + fk);
      fence_proxy_async_smem();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t sa = smem_u32(stg);
        uint32_t acc = it > 0 ? 1u : 0u;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const uint32_t at = sa + (p == 2 ? TC_OPER : 0);
          const uint32_t bt = sa + 2 * TC_OPER + (p == 1 ? TC_OPER : 0);
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            mma_tf32(tmem, desc_sw128(at + 32u * ks), desc_sw128(bt + 32u * ks), idesc, acc);
            acc = 1u;
          }
        }
        mma_commit(&bar[st]);
      }
      ++it;
    }
  }
  // Drain: the last commit covers every MMA issued before it.
  if (it > 0) {
    const int last = it - 1;
    const bool done = mbar_wait_bounded(&bar[last & 1], (uint32_t)((last >> 1) & 1));
    if (__syncthreads_or(!done)) ok = false;
  }
  tc_fence_after();
  if (!ok) {
    if (tid == 0 && atomicCAS(&fa.status[0], 0, 2) == 0) fa.status[1] = s;
  } else if (it > 0) {
    // Epilogue: warp w reads TMEM lanes 32 (w & 3) .. +32 (tile rows) and
    // tile columns 32 (w >> 2) .. +32; P -= U on the lower part only.
    T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
    const int q = warp & 3, h = warp >> 2;
    const int row = 32 * q + lane;
    const uint32_t tl = tmem + ((uint32_t)(32 * q) << 16);
    float re[32];
    tmem_ld32(tl + 32u * h, re);
    if constexpr (Field<T>::complex) {
      float im[32];
      tmem_ld32(tl + (uint32_t)TC_N + 32u * h, im);
      if (row < rows_here) {
        const int gr = r0 + row;
#pragma unroll
        for (int jj = 0; jj < 32; ++jj) {
          const int col = 32 * h + jj, gc = c0 + col;
          if (col < cols_here && gr >= gc) {
            T* p = panel + gr + (long long)gc * nrow;
            T v = *p;
            v.re -= re[jj];
            v.im -= im[jj];
            *p = v;
          }
        }
      }
    } else {
      if (row < rows_here) {
        const int gr = r0 + row;
#pragma unroll
        for (int jj = 0; jj < 32; ++jj) {
          const int col = 32 * h + jj, gc = c0 + col;
          if (col < cols_here && gr >= gc) panel[gr + (long long)gc * nrow] -= re[jj];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TC_TMEM_COLS);
}

}  // namespace rsd
