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
//             3xTF32 split), zero-padded to whole 32-wide K chunks.  Complex
//             fields take the 3M form of the product: per 16-column chunk
//             A' = [Ar | Ai], B' = [Gr | Gi] (hi and lo arrays) and the sums
//             As = Ar + Ai, Bs = Gr + Gi as one [hi | lo] array each, so
//               P1 = Ar Gr^T, P2 = Ai Gi^T, P3 = As Bs^T,
//               Re U = P1 - P2,  Im U = P3 - P1 - P2
//             takes three real products of K = 16 (the real embedding took
//             four);
//   k_cmod_mm one 128-row x (<= 64)-column tile of W per CTA: a TMA producer
//             thread loads the A boxes (128 x 32) and B boxes (16-row) into
//             128-byte-swizzled K-major stages, one thread issues
//             tcgen05.mma kind::tf32 (hi*hi + hi*lo + lo*hi) into TMEM
//             accumulators (complex: P1, P2, P3), four epilogue warps promote
//             every window of TC_WIN chunks into fp32 registers (the tensor
//             pipe does not round its accumulation to nearest; complex
//             windows are combined into Re / Im there) and write the tile to
//             the level's W workspace;
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
constexpr int MM_BOX_B = 16;     // rows of one B box
constexpr int MM_NT = 6 * 32;    // producer warp, MMA warp, 4 epilogue warps
constexpr int MM_SPLIT_ROWS = 32;   // rows of one split task
constexpr int MM_SPLIT_NT = 256;    // threads of a split task (8 column groups)
constexpr int MM_SPLIT_LD = 36;     // padded shared-memory row (floats): 4-way bank spread, 16-byte rows
constexpr uint32_t MM_TMEM_COLS = 512;  // two windows of up to 3 x 64 accumulator columns (at 0, 64, 128)
constexpr uint32_t MM_WIN_COLS = 256;   // TMEM columns per window buffer

// Operand maps of updater k: [0] A hi, [1] A lo, [2] B hi, [3] B lo, and for
// complex fields [4] As = [hi | lo] of Ar + Ai, [5] Bs = [hi | lo] of Gr + Gi.
constexpr int MM_MAPS = 6;

// one stage: A boxes of 128 rows x 128 B, B boxes of up to 64 rows x 128 B
constexpr int MM_AOP = MM_M * 128;
constexpr int MM_BOP = MM_NC * 128;

// Split-pool geometry of an updater: K' chunks of 32 fp32 per row.
template <typename T> struct MmShape;
template <> struct MmShape<float> {
  static constexpr int cols_per_chunk = 32;  // k columns per 32-wide K' chunk
  static constexpr int nops = 2;             // A / B arrays: hi, lo
  static constexpr int stages = 4;
};
template <> struct MmShape<c32> {
  static constexpr int cols_per_chunk = 16;
  static constexpr int nops = 3;             // A / B arrays: hi, lo, [sum hi | sum lo]
  static constexpr int stages = 3;
};
template <typename T>
__host__ __device__ constexpr int mm_stage_bytes() { return MmShape<T>::nops * (MM_AOP + MM_BOP); }
template <typename T>
__host__ __device__ constexpr size_t smem_cmod_mm_bytes() {
  return 1024 + MmShape<T>::stages * (size_t)mm_stage_bytes<T>() + 128;
}

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
// k_split: task (k, r0, chunk, 0): rows [r0, r0 + 32) of k's off-diagonal
// block, K' chunk `chunk`.  Phase 1: thread (row, column group) reads L21 and
// forms G = L21 D (ld_G's arithmetic) for its columns, coalesced across the
// rows of a column, splitting into hi / lo rows in shared memory.  Phase 2:
// eight consecutive threads store one row's 128 bytes of each operand, so a
// warp writes four whole rows per store.  The rows of the shared tile are
// padded to 36 floats, which spreads phase 1's column-wise writes over banks.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(MM_SPLIT_NT) k_split(FactorArgs fa, const int4* __restrict__ tasks,
                                                       const long long* __restrict__ soff_a,
                                                       const long long* __restrict__ soff_b,
                                                       const int* __restrict__ kpad, float* __restrict__ a_hi,
                                                       float* __restrict__ a_lo, float* __restrict__ b_hi,
                                                       float* __restrict__ b_lo, float* __restrict__ a_s,
                                                       float* __restrict__ b_s) {
  using F = Field<T>;
  using Sh = MmShape<T>;
  constexpr bool CX = Field<T>::complex;
  constexpr int NOP = CX ? 6 : 4;  // A hi/lo, B hi/lo[, As, Bs]
  __shared__ __align__(16) float tile[NOP][MM_SPLIT_ROWS][MM_SPLIT_LD];
  if (fa.status[0] != 0) return;
  const int4 tk = tasks[blockIdx.x];
  const int k = tk.x, r0 = tk.y, ch = tk.z;
  const int first = fa.sn_first[k], ncol = fa.sn_ncol[k], nrow = fa.sn_nrow[k];
  const int m = nrow - ncol;
  const int kp = kpad[k];
  const T* L = reinterpret_cast<const T*>(fa.panel) + fa.sn_poff[k] + ncol;  // L21, column stride nrow
  const T* d = reinterpret_cast<const T*>(fa.d) + first;
  const T* ds = reinterpret_cast<const T*>(fa.dsub) + first;
  const unsigned char* kd = fa.kind + first;
  const int t0 = ch * Sh::cols_per_chunk;
  const int tid = threadIdx.x, rl = tid % MM_SPLIT_ROWS, grp = tid / MM_SPLIT_ROWS;
  constexpr int GROUPS = MM_SPLIT_NT / MM_SPLIT_ROWS;
  constexpr int PER = Sh::cols_per_chunk / GROUPS;  // columns per thread
  const int r = r0 + rl;
#pragma unroll
  for (int e = 0; e < PER; ++e) {
    const int q = grp * PER + e, t = t0 + q;
    T a = F::zero(), g = F::zero();
    if (r < m && t < ncol) {
      a = L[r + (long long)t * nrow];
      g = ld_G(L, nrow, r, t, d, ds, kd);
    }
    float h, l;
    if constexpr (!CX) {
      split_tf32(a, h, l);
      tile[0][rl][q] = h;
      tile[1][rl][q] = l;
      split_tf32(g, h, l);
      tile[2][rl][q] = h;
      tile[3][rl][q] = l;
    } else {
      split_tf32(a.re, h, l);   // A' = [Ar | Ai], B' = [Gr | Gi]
      tile[0][rl][q] = h;
      tile[1][rl][q] = l;
      split_tf32(a.im, h, l);
      tile[0][rl][16 + q] = h;
      tile[1][rl][16 + q] = l;
      split_tf32(g.re, h, l);
      tile[2][rl][q] = h;
      tile[3][rl][q] = l;
      split_tf32(g.im, h, l);
      tile[2][rl][16 + q] = h;
      tile[3][rl][16 + q] = l;
      split_tf32(a.re + a.im, h, l);  // As = [hi | lo] of Ar + Ai, Bs of Gr + Gi
      tile[4][rl][q] = h;
      tile[4][rl][16 + q] = l;
      split_tf32(g.re + g.im, h, l);
      tile[5][rl][q] = h;
      tile[5][rl][16 + q] = l;
    }
  }
  __syncthreads();
  const long long rowa = soff_a[k] + 32LL * ch, rowb = soff_b[k] + 32LL * ch;
  for (int e = tid; e < MM_SPLIT_ROWS * 8; e += MM_SPLIT_NT) {
    const int rr = e >> 3, q4 = (e & 7) * 4, gr = r0 + rr;
    if (gr >= m) continue;
    const long long oa = rowa + (long long)gr * kp + q4, ob = rowb + (long long)gr * kp + q4;
    *reinterpret_cast<float4*>(a_hi + oa) = *reinterpret_cast<const float4*>(&tile[0][rr][q4]);
    *reinterpret_cast<float4*>(a_lo + oa) = *reinterpret_cast<const float4*>(&tile[1][rr][q4]);
    *reinterpret_cast<float4*>(b_hi + ob) = *reinterpret_cast<const float4*>(&tile[2][rr][q4]);
    *reinterpret_cast<float4*>(b_lo + ob) = *reinterpret_cast<const float4*>(&tile[3][rr][q4]);
    if constexpr (CX) {
      *reinterpret_cast<float4*>(a_s + oa) = *reinterpret_cast<const float4*>(&tile[4][rr][q4]);
      *reinterpret_cast<float4*>(b_s + ob) = *reinterpret_cast<const float4*>(&tile[5][rr][q4]);
    }
  }
}

// ---------------------------------------------------------------------------
// k_cmod_mm: task (k, r0, c0, nrows | nn << 16) with rows [r0, r0 + nrows)
// and columns [c0, c0 + nn) of k's off-diagonal block (indices relative to
// its first off-diagonal row), written to W at wbase (column-major, column
// stride wld elements of the field).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(MM_NT, 1) k_cmod_mm(FactorArgs fa, const int4* __restrict__ tasks,
                                                      const long long* __restrict__ wbase,
                                                      const int* __restrict__ wld,
                                                      const CUtensorMap* __restrict__ maps,
                                                      const int* __restrict__ kpad, float* __restrict__ W) {
  using Sh = MmShape<T>;
  constexpr bool CX = Field<T>::complex;
  constexpr int NS = Sh::stages, NOP = Sh::nops, STAGE = mm_stage_bytes<T>();
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t sraw = smem_u32(smem_raw);
  unsigned char* sm = smem_raw + (((sraw + 1023u) & ~1023u) - sraw);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + NS * STAGE);
  uint64_t* empty = full + NS;
  uint64_t* wbar = empty + NS;  // 2
  uint64_t* pbar = wbar + 2;    // 2
  uint32_t* tslot = reinterpret_cast<uint32_t*>(pbar + 2);

  const int4 tk = tasks[blockIdx.x];
  const int k = tk.x, r0 = tk.y, c0 = tk.z, nrows = tk.w & 0xffff, nn = tk.w >> 16;
  const int nchunks = kpad[k] / 32;
  const uint32_t nr16 = (uint32_t)((nn + 15) & ~15);  // UMMA N = B rows of a box set
  const CUtensorMap* mk = maps + (long long)k * MM_MAPS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int i = 0; i < NS; ++i) {
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
  // promoted tile: real -> acc[j]; complex -> Re in acc[j], Im in acc[64 + j]
  float acc[128];
#pragma unroll
  for (int j = 0; j < 128; ++j) acc[j] = 0.0f;

  // stage layout: A arrays (A hi, A lo[, As]) then B arrays (B hi, B lo[, Bs])
  int loaded = 0;  // TMA producer: chunks whose loads were issued
  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      const uint32_t bbytes = nr16 * 128u;
      for (int c = 0; c < nchunks; ++c) {
        const int st = c % NS;
        if (c >= NS && !mbar_wait_bounded(&empty[st], (uint32_t)(((c / NS) - 1) & 1))) {
          ok = false;
          break;
        }
        unsigned char* stg = sm + st * STAGE;
        mbar_expect_tx(&full[st], (uint32_t)NOP * ((uint32_t)MM_AOP + bbytes));
#pragma unroll
        for (int o = 0; o < NOP; ++o) {
          const int amap = o < 2 ? o : 4, bmap = o < 2 ? 2 + o : 5;
          tma_load_2d(stg + o * MM_AOP, mk + amap, 32 * c, r0, &full[st]);
          for (uint32_t b = 0; b < nr16; b += MM_BOX_B)
            tma_load_2d(stg + NOP * MM_AOP + o * MM_BOP + b * 128u, mk + bmap, 32 * c, c0 + (int)b, &full[st]);
        }
        loaded = c + 1;
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(MM_M, nr16);
      const uint32_t sbase = smem_u32(sm);
      for (int c = 0; c < nchunks && ok; ++c) {
        const int st = c % NS, w = c / TC_WIN;
        if (c % TC_WIN == 0 && w >= 2 && !mbar_wait_bounded(&pbar[w & 1], (uint32_t)(((w - 2) >> 1) & 1))) {
          ok = false;
          break;
        }
        if (!mbar_wait_bounded(&full[st], (uint32_t)((c / NS) & 1))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = sbase + (uint32_t)(st * STAGE), sb = sa + NOP * MM_AOP;
        const uint32_t dacc = tmem + (uint32_t)(w & 1) * MM_WIN_COLS;
        const uint32_t first = (c % TC_WIN) != 0 ? 1u : 0u;
        if constexpr (!CX) {
          uint32_t accf = first;
#pragma unroll
          for (int p = 0; p < 3; ++p) {
            const uint32_t at = sa + (p == 2 ? MM_AOP : 0);   // A hi, A hi, A lo
            const uint32_t bt = sb + (p == 1 ? MM_BOP : 0);   // B hi, B lo, B hi
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
              mma_tf32(dacc, desc_sw128(at + 32u * ks), desc_sw128(bt + 32u * ks), idesc, accf);
              accf = 1u;
            }
          }
        } else {
          // P1 (accumulator columns 0 ..), P2 (64 ..): the Re / Im halves of
          // the A hi / lo and B hi / lo boxes (K steps 0-1 and 2-3)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const uint32_t d = dacc + 64u * (uint32_t)h;
            uint32_t accf = first;
#pragma unroll
            for (int p = 0; p < 3; ++p) {
              const uint32_t at = sa + (p == 2 ? MM_AOP : 0);
              const uint32_t bt = sb + (p == 1 ? MM_BOP : 0);
#pragma unroll
              for (int ks = 2 * h; ks < 2 * h + 2; ++ks) {
                mma_tf32(d, desc_sw128(at + 32u * ks), desc_sw128(bt + 32u * ks), idesc, accf);
                accf = 1u;
              }
            }
          }
          // P3 (128 ..): As and Bs hold [hi | lo] in K steps 0-1 / 2-3
          const uint32_t d = dacc + 128u, at = sa + 2 * MM_AOP, bt = sb + 2 * MM_BOP;
          uint32_t accf = first;
#pragma unroll
          for (int p = 0; p < 3; ++p) {
            const uint32_t ak = p == 2 ? 2u : 0u, bk = p == 1 ? 2u : 0u;  // hi*hi, hi*lo, lo*hi
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
              mma_tf32(d, desc_sw128(at + 32u * (ak + ks)), desc_sw128(bt + 32u * (bk + ks)), idesc, accf);
              accf = 1u;
            }
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
      const uint32_t base = tmem + (uint32_t)(w & 1) * MM_WIN_COLS + ((uint32_t)(32 * q) << 16);
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        if ((uint32_t)(16 * g) < nr16) {
          if constexpr (!CX) {
            float v[16];
            tmem_ld16(base + 16u * g, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[16 * g + j] += v[j];
          } else {
            float v1[16], v2[16];
            tmem_ld16(base + 16u * g, v1);
            tmem_ld16(base + 64u + 16u * g, v2);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              acc[16 * g + j] += v1[j] - v2[j];  // Re = P1 - P2
              v1[j] += v2[j];
            }
            tmem_ld16(base + 128u + 16u * g, v2);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[64 + 16 * g + j] += v2[j] - v1[j];  // Im = P3 - P1 - P2
          }
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
      // W is column-major: the lanes of a warp store 32 consecutive rows
      const long long ld = wld[blockIdx.x];
      float* wr = W + (long long)(CX ? 2 : 1) * (wbase[blockIdx.x] + row);
      if constexpr (CX) {
#pragma unroll
        for (int j = 0; j < MM_NC; ++j)
          if (j < nn) *reinterpret_cast<float2*>(wr + 2 * j * ld) = make_float2(acc[j], acc[64 + j]);
      } else {
#pragma unroll
        for (int j = 0; j < MM_NC; ++j)
          if (j < nn) wr[j * ld] = acc[j];
      }
    }
  } else if (!all_ok && warp == 1 && lane == 0 && issued > 0) {
    // drain (bounded): the last commit covers every MMA issued before it
    (void)mbar_wait_bounded(&empty[(issued - 1) % NS], (uint32_t)(((issued - 1) / NS) & 1));
  } else if (!all_ok && warp == 0 && lane == 0) {
    // drain (bounded): the TMA loads still in flight land before the CTA exits
    for (int c = std::max(0, loaded - NS); c < loaded; ++c)
      (void)mbar_wait_bounded(&full[c % NS], (uint32_t)((c / NS) & 1));
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
// its W element (a, q0) at wb[u], column stride wl[u].  512 threads: thread
// (row t = tid & 127, quarter h = tid >> 7) owns tile columns 16 h .. +15.
// The pairs' maps and descriptors are copied to shared memory in batches of
// ASM_PB (one coalesced copy), so per pair a thread issues only its 16
// independent W loads; every tile element sums its pairs in update order.
// ---------------------------------------------------------------------------
constexpr int ASM_NT = 512;
constexpr int ASM_PB = 48;  // pairs per shared-memory batch
// Two CTAs per SM except for c64, whose 16 accumulators take 64 registers.
template <typename T>
__global__ void __launch_bounds__(ASM_NT, sizeof(T) >= 16 ? 1 : 2)
    k_cmod_asm(FactorArgs fa, const int4* __restrict__ tasks, const int4* __restrict__ pairs,
               const int8_t* __restrict__ maps, const long long* __restrict__ wb, const int* __restrict__ wl,
               const float* __restrict__ W) {
  using F = Field<T>;
  __shared__ __align__(16) int8_t smap[ASM_PB][TC_MAP];
  __shared__ int2 spr[ASM_PB];      // (a, q0)
  __shared__ long long swb[ASM_PB];
  __shared__ int swl[ASM_PB];
  if (fa.status[0] != 0) return;
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = (tk.y >> 16) * TC_M, c0 = (tk.y & 0xffff) * TC_N;
  const int ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int rows_here = min(TC_M, nrow - r0), cols_here = min(TC_N, ncol - c0);
  const int tid = threadIdx.x, t = tid & 127, h = tid >> 7;
  T acc[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) acc[j] = F::zero();
  static_assert(TC_MAP % 16 == 0, "maps copied as int4");
  for (int u0 = tk.z; u0 < tk.w; u0 += ASM_PB) {
    const int nb = min(ASM_PB, tk.w - u0);
    __syncthreads();  // the previous batch is consumed
    const int4* src = reinterpret_cast<const int4*>(maps + (long long)u0 * TC_MAP);
    int4* dstm = reinterpret_cast<int4*>(&smap[0][0]);
    for (int e = tid; e < nb * (TC_MAP / 16); e += ASM_NT) dstm[e] = src[e];
    for (int e = tid; e < nb; e += ASM_NT) {
      const int4 pr = pairs[u0 + e];
      spr[e] = make_int2(pr.y, pr.z);
      swb[e] = wb[u0 + e];
      swl[e] = wl[u0 + e];
    }
    __syncthreads();
    for (int v = 0; v < nb; ++v) {
      const int i = smap[v][t];
      if (i < 0) continue;
      const int2 pr = spr[v];
      int8_t cm[16];
      *reinterpret_cast<int4*>(cm) = *reinterpret_cast<const int4*>(&smap[v][TC_M + 16 * h]);
      // W is column-major: consecutive tile rows read (mostly) consecutive W rows
      const T* wrow = reinterpret_cast<const T*>(W) + swb[v] + i;
      const long long ld = swl[v];
      T w[16];
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) {
        const int j = cm[jj];
        w[jj] = (j >= 0 && pr.x + i >= pr.y + j) ? wrow[j * ld] : F::zero();
      }
#pragma unroll
      for (int jj = 0; jj < 16; ++jj)
        if (cm[jj] >= 0 && pr.x + i >= pr.y + cm[jj]) acc[jj] = F::add(acc[jj], w[jj]);
    }
  }
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s] + (r0 + t);
  if (t < rows_here) {
    // groups of 8: every load of a group before its first store (distinct
    // targets; one round trip per element would serialise the tile)
#pragma unroll
    for (int j0 = 0; j0 < 16; j0 += 8) {
      T old[8];
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        const int col = 16 * h + j0 + jj;
        old[jj] = (col < cols_here && r0 + t >= c0 + col) ? panel[(long long)(c0 + col) * nrow] : F::zero();
      }
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        const int col = 16 * h + j0 + jj;
        if (col < cols_here && r0 + t >= c0 + col)
          panel[(long long)(c0 + col) * nrow] = F::sub(old[jj], acc[j0 + jj]);
      }
    }
  }
}

}  // namespace rsd

namespace rsd {

// ---------------------------------------------------------------------------
// FP64 fields: the same updater-space GEMM tiles on the FP64 tensor cores
// (mma.sync m8n8k4 .f64, DMMA).  Task and W layout as k_cmod_mm; the A
// operand is L21_k (the panel, column stride nrow_k), the B operand G_k (the
// G pool, column stride m_k), staged by cp.async in K chunks (two stages).
// 256 threads: warp (wr, wc) of a 4 x 2 grid owns rows 32 wr .. +31 and
// columns 32 wc .. +31 of the tile, i.e. 4 x 4 m8n8 blocks.  Complex
// products use four real DMMA per block: Re += Ar Br - Ai Bi, Im += Ar Bi +
// Ai Br.  Results agree with the FMA engine to rounding (the DMMA sums its
// four products in its own order); the FMA engine (schur_engine = fma)
// remains the bit-exact reference engine.
// ---------------------------------------------------------------------------
constexpr int DM_NT = 256;
// K chunk and padded shared-memory columns (elements) of the A / B chunks:
// with these strides the fragment loads of a warp (rows g, K columns q) hit
// distinct banks (8-byte elements: stride = 4 mod 16 words; 16-byte
// elements: 2 mod 8 elements).
template <typename T> struct DmShape {
  static constexpr int kc = 16, lda = 132, ldb = 68;
};
template <> struct DmShape<c64> {
  static constexpr int kc = 8, lda = 130, ldb = 66;
};
template <typename T>
__host__ __device__ constexpr size_t smem_cmod_dmm_bytes() {
  return 2 * (size_t)DmShape<T>::kc * (DmShape<T>::lda + DmShape<T>::ldb) * sizeof(T);
}

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <typename T>
__global__ void __launch_bounds__(DM_NT) k_cmod_dmm(FactorArgs fa, const int4* __restrict__ tasks,
                                                   const long long* __restrict__ wbase,
                                                   const int* __restrict__ wld, T* __restrict__ W) {
  using F = Field<T>;
  constexpr bool CX = Field<T>::complex;
  constexpr int KC = DmShape<T>::kc, DM_LDA = DmShape<T>::lda, DM_LDB = DmShape<T>::ldb;
  constexpr int STAGE = KC * (DM_LDA + DM_LDB);
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* stg = reinterpret_cast<T*>(smem_raw);
  const int4 tk = tasks[blockIdx.x];
  const int k = tk.x, r0 = tk.y, c0 = tk.z, nrows = tk.w & 0xffff, nn = tk.w >> 16;
  const int nck = fa.sn_ncol[k], nrk = fa.sn_nrow[k], m = nrk - nck;
  const T* A = reinterpret_cast<const T*>(fa.panel) + fa.sn_poff[k] + nck + r0;  // + t * nrk
  const T* B = reinterpret_cast<const T*>(fa.gpool) + fa.goff[k] + c0;           // + t * m
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wr = warp >> 1, wc = warp & 1;
  const int g = lane >> 2, q = lane & 3;  // fragment group / thread in group

  auto issue = [&](int t0, int st) {
    T* As = stg + st * STAGE;
    T* Bs = As + KC * DM_LDA;
    for (int e = tid; e < KC * MM_M; e += DM_NT) {
      const int t = e / MM_M, r = e % MM_M, tt = t0 + t;
      const bool ok = tt < nck && r < nrows;
      cp_async_zfill<(int)sizeof(T)>(As + t * DM_LDA + r, ok ? A + r + (long long)tt * nrk : A, ok);
    }
    for (int e = tid; e < KC * MM_NC; e += DM_NT) {
      const int t = e / MM_NC, c = e % MM_NC, tt = t0 + t;
      const bool ok = tt < nck && c < nn;
      cp_async_zfill<(int)sizeof(T)>(Bs + t * DM_LDB + c, ok ? B + c + (long long)tt * m : B, ok);
    }
    cp_async_commit();
  };

  // accumulators: [row block i][col block j][2] (complex: re, im pairs)
  double acc[4][4][CX ? 4 : 2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < (CX ? 4 : 2); ++v) acc[i][j][v] = 0.0;

  const int nchunk = (nck + KC - 1) / KC;
  if (nchunk > 0) issue(0, 0);
  for (int c = 0; c < nchunk; ++c) {
    const int st = c & 1;
    if (c + 1 < nchunk) {
      issue((c + 1) * KC, st ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const T* As = stg + st * STAGE;
    const T* Bs = As + KC * DM_LDA;
    const bool active = 32 * wr < nrows && 32 * wc < nn;
    if (active) {
#pragma unroll
      for (int k4 = 0; k4 < KC; k4 += 4) {
        const int t = k4 + q;
        if constexpr (!CX) {
          double a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = As[t * DM_LDA + 32 * wr + 8 * i + g];
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = Bs[t * DM_LDB + 32 * wc + 8 * j + g];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        } else {
          T a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = As[t * DM_LDA + 32 * wr + 8 * i + g];
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = Bs[t * DM_LDB + 32 * wc + 8 * j + g];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              dmma884(acc[i][j][0], acc[i][j][1], a[i].re, b[j].re);   // Re += Ar Br
              dmma884(acc[i][j][0], acc[i][j][1], -a[i].im, b[j].im);  //       - Ai Bi
              dmma884(acc[i][j][2], acc[i][j][3], a[i].re, b[j].im);   // Im += Ar Bi
              dmma884(acc[i][j][2], acc[i][j][3], a[i].im, b[j].re);   //       + Ai Br
            }
        }
      }
    }
    __syncthreads();  // the stage is free for the load after next
  }
  // W[row, col] for row < nrows, col < nn (fragment: row g, columns 2q, 2q+1)
  const long long wb = wbase[blockIdx.x];
  const int ld = wld[blockIdx.x];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = 32 * wr + 8 * i + g;
    if (row >= nrows) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int col = 32 * wc + 8 * j + 2 * q + v;
        if (col >= nn) continue;
        T out;
        if constexpr (CX)
          out = T{acc[i][j][v], acc[i][j][2 + v]};
        else
          out = acc[i][j][v];
        W[wb + row + (long long)col * ld] = out;
      }
  }
}

}  // namespace rsd

namespace rsd {

// ---------------------------------------------------------------------------
// FP64 fields, tensor engine: the deferred in-panel Schur update on DMMA.
// Task (s, kb, r0, c0) as k_schur_tc: trailing-part tile rows [ke + r0,
// +128) x columns [ke + c0, +64) of block [kb, ke) of supernode s, minus
// L21 G^T over the block's columns, G = L21 D formed while it is staged
// (the block's D, dsub and kind in shared memory), on the lower part.  The
// A chunks (L21 rows) arrive by cp.async; the B chunk of step c + 1 is read
// into registers before the products of step c and stored after them, so
// its loads overlap the DMMA.  Warp tiles and fragments as k_cmod_dmm.
// ---------------------------------------------------------------------------
template <typename T>
__host__ __device__ constexpr size_t smem_schur_dmm_bytes() {
  return smem_cmod_dmm_bytes<T>() + (size_t)128 * (2 * sizeof(T) + 1) + 16;
}

// One 128 x 64 tile: tile[row + col ldt] -= sum_t A[row + t lda] G(col, t)
// over t in [0, kdim), G(col, t) = ld_G(B, lda, col, t, d, dsub, kind), for
// row < rows_here, col < cols_here and r0 + row >= c0 + col (the lower part
// of the trailing matrix).  256 threads; every thread calls it.
template <typename T>
__device__ __forceinline__ void dmm_lower_update(const T* A, const T* B, long long lda, int kdim, const T* d,
                                                 const T* dsub, const unsigned char* kind, T* tile, long long ldt,
                                                 int rows_here, int cols_here, int r0, int c0, T* stg) {
  using F = Field<T>;
  constexpr bool CX = Field<T>::complex;
  constexpr int KC = DmShape<T>::kc, DM_LDA = DmShape<T>::lda, DM_LDB = DmShape<T>::ldb;
  constexpr int STAGE = KC * (DM_LDA + DM_LDB);
  constexpr int PB = KC * MM_NC / DM_NT;  // B elements staged per thread per chunk
  static_assert(PB * DM_NT == KC * MM_NC, "B chunk divides over the CTA");
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wr = warp >> 1, wc = warp & 1;
  const int g = lane >> 2, q = lane & 3;

  auto issue_a = [&](int t0, int st) {
    T* As = stg + st * STAGE;
    for (int e = tid; e < KC * MM_M; e += DM_NT) {
      const int t = e / MM_M, r = e % MM_M, tt = t0 + t;
      const bool ok = tt < kdim && r < rows_here;
      cp_async_zfill<(int)sizeof(T)>(As + t * DM_LDA + r, ok ? A + r + (long long)tt * lda : A, ok);
    }
    cp_async_commit();
  };
  T bv[PB];
  auto load_b = [&](int t0) {
#pragma unroll
    for (int u = 0; u < PB; ++u) {
      const int e = tid + u * DM_NT, t = e / MM_NC, c = e % MM_NC, tt = t0 + t;
      bv[u] = (tt < kdim && c < cols_here) ? ld_G(B, lda, c, tt, d, dsub, kind) : F::zero();
    }
  };
  auto store_b = [&](int st) {
    T* Bs = stg + st * STAGE + KC * DM_LDA;
#pragma unroll
    for (int u = 0; u < PB; ++u) {
      const int e = tid + u * DM_NT, t = e / MM_NC, c = e % MM_NC;
      Bs[t * DM_LDB + c] = bv[u];
    }
  };

  double acc[4][4][CX ? 4 : 2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < (CX ? 4 : 2); ++v) acc[i][j][v] = 0.0;

  // warps whose 32 x 32 block lies wholly above the diagonal skip the products
  const bool active = 32 * wr < rows_here && 32 * wc < cols_here && r0 + 32 * wr + 31 >= c0 + 32 * wc;
  const int nchunk = (kdim + KC - 1) / KC;
  if (nchunk > 0) {
    issue_a(0, 0);
    load_b(0);
    store_b(0);
  }
  for (int c = 0; c < nchunk; ++c) {
    const int st = c & 1;
    if (c + 1 < nchunk) {
      issue_a((c + 1) * KC, st ^ 1);
      load_b((c + 1) * KC);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const T* As = stg + st * STAGE;
    const T* Bs = As + KC * DM_LDA;
    if (active) {
#pragma unroll
      for (int k4 = 0; k4 < KC; k4 += 4) {
        const int t = k4 + q;
        if constexpr (!CX) {
          double a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = As[t * DM_LDA + 32 * wr + 8 * i + g];
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = Bs[t * DM_LDB + 32 * wc + 8 * j + g];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        } else {
          T a[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = As[t * DM_LDA + 32 * wr + 8 * i + g];
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = Bs[t * DM_LDB + 32 * wc + 8 * j + g];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              dmma884(acc[i][j][0], acc[i][j][1], a[i].re, b[j].re);   // Re += Ar Br
              dmma884(acc[i][j][0], acc[i][j][1], -a[i].im, b[j].im);  //       - Ai Bi
              dmma884(acc[i][j][2], acc[i][j][3], a[i].re, b[j].im);   // Im += Ar Bi
              dmma884(acc[i][j][2], acc[i][j][3], a[i].im, b[j].re);   //       + Ai Br
            }
        }
      }
    }
    if (c + 1 < nchunk) store_b(st ^ 1);  // that stage was released by the last iteration's barrier
    __syncthreads();
  }
  // tile -= acc on the lower part; per row block every load before its stores
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = 32 * wr + 8 * i + g;
    T old[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int col = 32 * wc + 8 * j + 2 * q + v;
        const bool in = row < rows_here && col < cols_here && r0 + row >= c0 + col;
        old[j][v] = in ? tile[row + (long long)col * ldt] : F::zero();
      }
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int col = 32 * wc + 8 * j + 2 * q + v;
        if (row < rows_here && col < cols_here && r0 + row >= c0 + col) {
          T u;
          if constexpr (CX)
            u = T{acc[i][j][v], acc[i][j][2 + v]};
          else
            u = acc[i][j][v];
          tile[row + (long long)col * ldt] = F::sub(old[j][v], u);
        }
      }
  }
}

template <typename T>
__global__ void __launch_bounds__(DM_NT) k_schur_dmm(FactorArgs fa, const int4* __restrict__ tasks, int nb_small,
                                                    int nb_big) {
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* stg = reinterpret_cast<T*>(smem_raw);
  T* d_s = stg + 2 * DmShape<T>::kc * (DmShape<T>::lda + DmShape<T>::ldb);
  T* ds_s = d_s + 128;
  unsigned char* kd_s = reinterpret_cast<unsigned char*>(ds_s + 128);
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, kb = tk.y, r0 = tk.z, c0 = tk.w;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int nb = ncol >= 512 ? nb_big : nb_small;
  const int ke = min(kb + nb, ncol), pw = ke - kb;
  T* panel = reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s];
  const T* Lb = panel + ke + (long long)kb * nrow;  // the block's L21: row i, column t at Lb[i + t nrow]
  for (int t = threadIdx.x; t < pw; t += DM_NT) {
    d_s[t] = reinterpret_cast<const T*>(fa.d)[first + kb + t];
    ds_s[t] = reinterpret_cast<const T*>(fa.dsub)[first + kb + t];
    kd_s[t] = fa.kind[first + kb + t];
  }
  __syncthreads();
  dmm_lower_update<T>(Lb + r0, Lb + c0, (long long)nrow, pw, d_s, ds_s, kd_s,
                      panel + (ke + r0) + (long long)(ke + c0) * nrow, (long long)nrow,
                      min(MM_M, nrow - ke - r0), min(MM_NC, ncol - ke - c0), r0, c0, stg);
}

// Multifrontal method, FP64 fields on the tensor engine: the contribution
// block of front s, CB -= L21 D L21^T over all ncol columns, in 128 x 64
// tiles (task (s, r0, c0, 0), r0 a multiple of 128 at or below c0) of its
// lower part; D, dsub and kind read through ld_G from the factor's arrays.
template <typename T>
__global__ void __launch_bounds__(DM_NT) k_front_cb_dmm(FactorArgs fa, const int4* __restrict__ tasks) {
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* stg = reinterpret_cast<T*>(smem_raw);
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = tk.y, c0 = tk.z;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s], m = nrow - ncol;
  const T* L21 = reinterpret_cast<const T*>(fa.panel) + fa.sn_poff[s] + ncol;
  T* cb = reinterpret_cast<T*>(fa.cbpool) + fa.cb_off[s];
  dmm_lower_update<T>(L21 + r0, L21 + c0, (long long)nrow, ncol, reinterpret_cast<const T*>(fa.d) + first,
                      reinterpret_cast<const T*>(fa.dsub) + first, fa.kind + first,
                      cb + r0 + (long long)c0 * m, (long long)m, min(MM_M, m - r0), min(MM_NC, m - c0), r0, c0,
                      stg);
}

}  // namespace rsd
