// Tensor-core descendant updates of the single-precision factor fields (f32,
// c32) computed in the UPDATER's row space, then assembled into the targets.
//
// For every (updater k, target s) pair the update is one dense product
//   W_ks = L21_k[p0.., :] G_k[p0..p1, :]^T,   G_k = L21_k D_k,
// over k's contiguous off-diagonal rows (p0 = the first row landing in s's
// columns).  Only the lower trapezoid is formed: the column tile starting at
// row c0 of k takes k's rows from c0 on.  The three kernels:
//   k_split   once per updater, after its level is factored: writes A = L21_k
//             and B = G_k as row-major, K-contiguous tf32 hi / lo pairs (the
//             3xTF32 split), zero-padded to whole 32-wide K chunks; complex
//             fields use the real embedding A' = [Ar | Ai] per 16-column
//             chunk, B'_re = [Gr | -Gi], B'_im = [Gi | Gr] (so A' B'_re^T =
//             Re U, A' B'_im^T = Im U);
//   k_cmod_mm one 128-row x (<= 64)-column tile of W per CTA: a TMA producer
//             thread loads A hi / lo (128 x 32 boxes) and B hi / lo (16-row
//             boxes) into 128-byte-swizzled K-major stages, one thread issues
//             tcgen05.mma kind::tf32 (hi*hi + hi*lo + lo*hi) into a TMEM
//             accumulator, four epilogue warps promote every window of
//             TC_WIN chunks into fp32 registers (the tensor pipe does not
//             round its accumulation to nearest) and write the tile to the
//             level's W workspace;
//   k_cmod_asm one 128 x 64 target tile per CTA: subtracts, in update order,
//             every pair's W entries that land in the tile (rows r >= column
//             c in k's ordering), through the pairs' inverse row / column
//             maps, and writes the tile once.  Deterministic: no atomics.
// The tensor maps (one per updater and operand) cover this GPU's own split
// pools; no load uses multicast.  Every wait is bounded: on a timeout the
// kernel sets status 2, drains what it issued and frees its TMEM.
// Reference: ll_factor_node cmod, src/numeric/multifrontal_ldlt.rs:2452-2728.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "cmod_tc.cuh"

namespace rsd {

constexpr int MM_M = 128;        // W tile rows (UMMA M)
constexpr int MM_NC = 64;        // W tile columns (complex or real)
constexpr int MM_NS = 3;         // operand stages
constexpr int MM_BOX_B = 16;     // rows of one B box
constexpr int MM_NT = 6 * 32;    // producer warp, MMA warp, 4 epilogue warps
constexpr int MM_SPLIT_ROWS = 256;
constexpr uint32_t MM_TMEM_COLS = 256;  // two 128-column accumulators

// Operand maps of updater k: [0] A hi, [1] A lo, [2] B hi, [3] B lo.
constexpr int MM_MAPS = 4;

// one stage: A hi, A lo (128 rows x 128 B), B hi, B lo (up to 128 rows x 128 B)
constexpr int MM_OPER = MM_M * 128;
constexpr int MM_STAGE = 4 * MM_OPER;
__host__ __device__ constexpr size_t smem_cmod_mm_bytes() { return 1024 + MM_NS * (size_t)MM_STAGE + 128; }

// Split-pool geometry of an updater: K' chunks of 32 fp32 per row.
template <typename T> struct MmShape;
template <> struct MmShape<float> {
  static constexpr int cols_per_chunk = 32;  // k columns per 32-wide K' chunk
  static constexpr int brows = 1;            // B rows per G row (re only)
};
template <> struct MmShape<c32> {
  static constexpr int cols_per_chunk = 16;
  static constexpr int brows = 2;            // B'_re rows, then B'_im rows
};

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 2D tiled TMA load (no multicast) of the box at (x = K' element, y = row)
// into shared memory, completing `bytes` on `bar`.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// ---------------------------------------------------------------------------
// k_split: task (k, r0, chunk, 0): rows [r0, r0 + 256) of k's off-diagonal
// block, K' chunk `chunk`.  One thread per row; reads of L21 are coalesced
// across the warp (consecutive rows of one column), each thread writes its
// row's 32 hi and 32 lo values (128-byte runs).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(MM_SPLIT_ROWS) k_split(FactorArgs fa, const int4* __restrict__ tasks,
                                                         const long long* __restrict__ soff_a,
                                                         const long long* __restrict__ soff_b,
                                                         const int* __restrict__ kpad, float* __restrict__ a_hi,
                                                         float* __restrict__ a_lo, float* __restrict__ b_hi,
                                                         float* __restrict__ b_lo) {
  using F = Field<T>;
  using Sh = MmShape<T>;
  if (fa.status[0] != 0) return;
  const int4 tk = tasks[blockIdx.x];
  const int k = tk.x, r = tk.y + (int)threadIdx.x, ch = tk.z;
  const int first = fa.sn_first[k], ncol = fa.sn_ncol[k], nrow = fa.sn_nrow[k];
  const int m = nrow - ncol;
  if (r >= m) return;
  const int kp = kpad[k];
  const T* L = reinterpret_cast<const T*>(fa.panel) + fa.sn_poff[k] + ncol;  // L21, column stride nrow
  const T* d = reinterpret_cast<const T*>(fa.d) + first;
  const T* ds = reinterpret_cast<const T*>(fa.dsub) + first;
  const unsigned char* kd = fa.kind + first;
  const long long ra = soff_a[k] + (long long)r * kp + 32 * ch;
  const int t0 = ch * Sh::cols_per_chunk;
  if constexpr (!Field<T>::complex) {
    const long long rb = soff_b[k] + (long long)r * kp + 32 * ch;
#pragma unroll 4
    for (int q = 0; q < 32; q += 4) {
      float av[4], gv[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int t = t0 + q + e;
        av[e] = t < ncol ? L[r + (long long)t * nrow] : 0.0f;
        gv[e] = t < ncol ? ld_G(L, nrow, r, t, d, ds, kd) : 0.0f;
      }
      float ah[4], al[4], gh[4], gl[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        split_tf32(av[e], ah[e], al[e]);
        split_tf32(gv[e], gh[e], gl[e]);
      }
      *reinterpret_cast<float4*>(a_hi + ra + q) = make_float4(ah[0], ah[1], ah[2], ah[3]);
      *reinterpret_cast<float4*>(a_lo + ra + q) = make_float4(al[0], al[1], al[2], al[3]);
      *reinterpret_cast<float4*>(b_hi + rb + q) = make_float4(gh[0], gh[1], gh[2], gh[3]);
      *reinterpret_cast<float4*>(b_lo + rb + q) = make_float4(gl[0], gl[1], gl[2], gl[3]);
    }
  } else {
    // B'_re row r and B'_im row r (the im block starts m rows later)
    const long long rre = soff_b[k] + (long long)r * kp + 32 * ch;
    const long long rim = rre + (long long)m * kp;
#pragma unroll 2
    for (int q = 0; q < 16; q += 4) {
      float ar[4], ai[4], gr[4], gi[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int t = t0 + q + e;
        T a = F::zero(), g = F::zero();
        if (t < ncol) {
          a = L[r + (long long)t * nrow];
          g = ld_G(L, nrow, r, t, d, ds, kd);
        }
        ar[e] = a.re;
        ai[e] = a.im;
        gr[e] = g.re;
        gi[e] = g.im;
      }
      float h[4], l[4];
      auto put = [&](float* hi, float* lo, long long off, const float (&v)[4], float sgn) {
#pragma unroll
        for (int e = 0; e < 4; ++e) split_tf32(sgn * v[e], h[e], l[e]);
        *reinterpret_cast<float4*>(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
      };
      put(a_hi, a_lo, ra + q, ar, 1.0f);        // A': Re in 0..15
      put(a_hi, a_lo, ra + 16 + q, ai, 1.0f);   //     Im in 16..31
      put(b_hi, b_lo, rre + q, gr, 1.0f);       // B'_re: Gr
      put(b_hi, b_lo, rre + 16 + q, gi, -1.0f); //        -Gi
      put(b_hi, b_lo, rim + q, gi, 1.0f);       // B'_im: Gi
      put(b_hi, b_lo, rim + 16 + q, gr, 1.0f);  //        Gr
    }
  }
}

// ---------------------------------------------------------------------------
// k_cmod_mm: task (k, r0, c0, nrows | nn << 16) with rows [r0, r0 + nrows)
// and columns [c0, c0 + nn) of k's off-diagonal block (indices relative to
// its first off-diagonal row), written to W at wbase (row stride ldw
// elements of the field).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(MM_NT, 1) k_cmod_mm(FactorArgs fa, const int4* __restrict__ tasks,
                                                      const long long* __restrict__ wbase,
                                                      const int* __restrict__ wld,
                                                      const CUtensorMap* __restrict__ maps,
                                                      const int* __restrict__ kpad, float* __restrict__ W) {
  using Sh = MmShape<T>;
  constexpr bool CX = Field<T>::complex;
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t sraw = smem_u32(smem_raw);
  unsigned char* sm = smem_raw + (((sraw + 1023u) & ~1023u) - sraw);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + MM_NS * MM_STAGE);
  uint64_t* empty = full + MM_NS;
  uint64_t* wbar = empty + MM_NS;  // 2
  uint64_t* pbar = wbar + 2;       // 2
  uint32_t* tslot = reinterpret_cast<uint32_t*>(pbar + 2);

  const int4 tk = tasks[blockIdx.x];
  const int k = tk.x, r0 = tk.y, c0 = tk.z, nrows = tk.w & 0xffff, nn = tk.w >> 16;
  const int m = fa.sn_nrow[k] - fa.sn_ncol[k];
  const int nchunks = kpad[k] / 32;
  const int nr16 = (nn + 15) & ~15;              // B rows per half
  const uint32_t nprime = CX ? 2u * nr16 : nr16; // UMMA N
  const CUtensorMap* mk = maps + (long long)k * MM_MAPS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int i = 0; i < MM_NS; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&wbar[0], 1);
    mbar_init(&wbar[1], 1);
    mbar_init(&pbar[0], 128);
    mbar_init(&pbar[1], 128);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, MM_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  bool ok = true;
  int issued = 0;  // MMA warp: chunks committed
  float acc[128];
#pragma unroll
  for (int j = 0; j < 128; ++j) acc[j] = 0.0f;

  int loaded = 0;  // TMA producer: chunks whose loads were issued
  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      const uint32_t bbytes = nprime * 128u;
      for (int c = 0; c < nchunks; ++c) {
        const int st = c % MM_NS;
        if (c >= MM_NS && !mbar_wait_bounded(&empty[st], (uint32_t)(((c / MM_NS) - 1) & 1))) {
          ok = false;
          break;
        }
        unsigned char* stg = sm + st * MM_STAGE;
        mbar_expect_tx(&full[st], 2u * MM_OPER + 2u * bbytes);
        tma_load_2d(stg, mk + 0, 32 * c, r0, &full[st]);
        tma_load_2d(stg + MM_OPER, mk + 1, 32 * c, r0, &full[st]);
        for (int h = 0; h < (CX ? 2 : 1); ++h)
          for (int b = 0; b < nr16; b += MM_BOX_B) {
            const int row = c0 + b + h * m;  // complex: the B'_im block starts m rows later
            const uint32_t off = (uint32_t)(h * nr16 + b) * 128u;
            tma_load_2d(stg + 2 * MM_OPER + off, mk + 2, 32 * c, row, &full[st]);
            tma_load_2d(stg + 3 * MM_OPER + off, mk + 3, 32 * c, row, &full[st]);
          }
        loaded = c + 1;
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(MM_M, nprime);
      const uint32_t sbase = smem_u32(sm);
      for (int c = 0; c < nchunks && ok; ++c) {
        const int st = c % MM_NS, w = c / TC_WIN;
        if (c % TC_WIN == 0 && w >= 2 && !mbar_wait_bounded(&pbar[w & 1], (uint32_t)(((w - 2) >> 1) & 1))) {
          ok = false;
          break;
        }
        if (!mbar_wait_bounded(&full[st], (uint32_t)((c / MM_NS) & 1))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = sbase + (uint32_t)(st * MM_STAGE);
        const uint32_t dacc = tmem + (uint32_t)(w & 1) * 128u;
        uint32_t accf = (c % TC_WIN) != 0 ? 1u : 0u;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const uint32_t at = sa + (p == 2 ? MM_OPER : 0);              // A hi, A hi, A lo
          const uint32_t bt = sa + 2 * MM_OPER + (p == 1 ? MM_OPER : 0);  // B hi, B lo, B hi
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            mma_tf32(dacc, desc_sw128(at + 32u * ks), desc_sw128(bt + 32u * ks), idesc, accf);
            accf = 1u;
          }
        }
        mma_commit(&empty[st]);
        if (c % TC_WIN == TC_WIN - 1 || c + 1 == nchunks) mma_commit(&wbar[w & 1]);
        issued = c + 1;
      }
    }
  } else {
    // ---------------- epilogue warps: TMEM lanes 32 (warp % 4) .. +31 ----------------
    const int q = warp & 3;
    const int nwin = (nchunks + TC_WIN - 1) / TC_WIN;
    for (int w = 0; w < nwin && ok; ++w) {
      if (!mbar_wait_bounded(&wbar[w & 1], (uint32_t)((w >> 1) & 1))) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint32_t base = tmem + (uint32_t)(w & 1) * 128u + ((uint32_t)(32 * q) << 16);
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        if ((uint32_t)(16 * g) < nprime) {
          float v[16];
          tmem_ld16(base + 16u * g, v);
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[16 * g + j] += v[j];
        }
      }
      tc_fence_before();
      mbar_arrive(&pbar[w & 1]);
    }
  }
  const bool all_ok = __syncthreads_or(!ok) == 0;
  if (warp >= 2 && all_ok) {
    const int row = 32 * (warp & 3) + lane;
    if (row < nrows) {
      float* wr = W + (long long)(CX ? 2 : 1) * (wbase[blockIdx.x] + (long long)row * wld[blockIdx.x]);
      if constexpr (CX) {
        // the imaginary parts start at accumulator column nr16 (16, 32, 48
        // or 64): a compile-time offset per case keeps acc in registers
        auto put = [&](auto off) {
          constexpr int o = decltype(off)::value;
#pragma unroll
          for (int j = 0; j < MM_NC; ++j)
            if (j < nn) *reinterpret_cast<float2*>(wr + 2 * j) = make_float2(acc[j], acc[(o + j) & 127]);
        };
        switch (nr16) {
          case 16: put(std::integral_constant<int, 16>{}); break;
          case 32: put(std::integral_constant<int, 32>{}); break;
          case 48: put(std::integral_constant<int, 48>{}); break;
          default: put(std::integral_constant<int, 64>{}); break;
        }
      } else {
#pragma unroll
        for (int j = 0; j < MM_NC; ++j)
          if (j < nn) wr[j] = acc[j];
      }
    }
  } else if (!all_ok && warp == 1 && lane == 0 && issued > 0) {
    // drain (bounded): the last commit covers every MMA issued before it
    (void)mbar_wait_bounded(&empty[(issued - 1) % MM_NS], (uint32_t)(((issued - 1) / MM_NS) & 1));
  } else if (!all_ok && warp == 0 && lane == 0) {
    // drain (bounded): the TMA loads still in flight land before the CTA exits
    for (int c = std::max(0, loaded - MM_NS); c < loaded; ++c)
      (void)mbar_wait_bounded(&full[c % MM_NS], (uint32_t)((c / MM_NS) & 1));
  }
  if (!all_ok && tid == 0 && atomicCAS(&fa.status[0], 0, 2) == 0) fa.status[1] = k;
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, MM_TMEM_COLS);
}

// ---------------------------------------------------------------------------
// k_cmod_asm: task (s, rt << 16 | ct, pair_begin, pair_end) over the 128 x 64
// tiles of the tensor-core plan; pair u (k, a, q0, nr << 16 | nc) with its
// inverse maps (tile row -> offset from a, tile column -> offset from q0) and
// its W element (a, q0) at wb[u], row stride wl[u].  256 threads: thread
// (row t = tid & 127, half h = tid >> 7) owns tile columns 32 h .. 32 h + 31.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_cmod_asm(FactorArgs fa, const int4* __restrict__ tasks,
                                                  const int4* __restrict__ pairs, const int8_t* __restrict__ maps,
                                                  const long long* __restrict__ wb, const int* __restrict__ wl,
                                                  const float* __restrict__ W) {
  using F = Field<T>;
  if (fa.status[0] != 0) return;
  __shared__ int8_t cmap[2][TC_N];
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = (tk.y >> 16) * TC_M, c0 = (tk.y & 0xffff) * TC_N;
  const int ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int rows_here = min(TC_M, nrow - r0), cols_here = min(TC_N, ncol - c0);
  const int t = threadIdx.x & 127, h = threadIdx.x >> 7;
  T acc[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) acc[j] = F::zero();
  int par = 0;
  for (int u = tk.z; u < tk.w; ++u, par ^= 1) {
    const int4 pr = pairs[u];
    const int8_t* mp = maps + (long long)u * TC_MAP;
    if (threadIdx.x < TC_N) cmap[par][threadIdx.x] = mp[TC_M + threadIdx.x];
    __syncthreads();
    const int i = mp[t];
    if (i >= 0) {
      const int a = pr.y, q0 = pr.z;
      const T* wrow = reinterpret_cast<const T*>(W) + wb[u] + (long long)i * wl[u];
#pragma unroll
      for (int jj = 0; jj < 32; ++jj) {
        const int j = cmap[par][32 * h + jj];
        if (j >= 0 && a + i >= q0 + j) acc[jj] = F::add(acc[jj], wrow[j]);
      }
    }
  }
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  if (t < rows_here)
#pragma unroll
    for (int jj = 0; jj < 32; ++jj) {
      const int col = 32 * h + jj;
      if (col < cols_here && r0 + t >= c0 + col) {
        T* p = panel + (r0 + t) + (long long)(c0 + col) * nrow;
        *p = F::sub(*p, acc[jj]);
      }
    }
}

}  // namespace rsd
