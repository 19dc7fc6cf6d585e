// Tensor-core cmod for the single-precision factor fields (f32, c32):
// the descendant updates of one 128 x 64 target tile accumulate in TMEM with
// tcgen05.mma kind::tf32 in the 3xTF32 split (hi*hi + hi*lo + lo*hi), and the
// tile is read-modify-written once at the end.
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
//
// Pipeline (512 threads, one CTA per SM): the global loads of K chunk c+2
// are issued into a second register set right after chunk c's MMAs, so two
// chunks of loads are in flight behind the tensor work; two shared-memory
// stages gated by mbarriers that tcgen05.commit arrives on; one block
// barrier per chunk.  The inverse scatter maps of every pair (tile row ->
// k row, tile column -> k row, int8) are precomputed at analysis.
// Accuracy: the tensor pipe does not round its accumulation to nearest, so
// the sum runs in windows of TC_WIN chunks over two TMEM accumulators; each
// finished window is added into per-thread fp32 registers (round to nearest)
// while the next window runs on the other accumulator.
// Every wait is bounded; on a timeout the kernel flags status 2, drains what
// it issued (bounded) and frees its TMEM.
// Reference: ll_factor_node cmod, src/numeric/multifrontal_ldlt.rs:2452-2728.
#pragma once

#include "factor_kernels.cuh"
#include "tcgen05.cuh"

namespace rsd {

constexpr int TC_M = 128;                 // target tile rows = UMMA M
constexpr int TC_N = 64;                  // target tile columns
constexpr int TC_NT = 512;                // threads per CTA
constexpr int TC_OPER = 16384;            // bytes of one 128 x 32 fp32 operand tile
constexpr int TC_STAGE = 4 * TC_OPER;     // A hi, A lo, B hi, B lo
constexpr int TC_WIN = 4;                 // K chunks per TMEM accumulation window
constexpr uint32_t TC_ACC_COLS = 128;     // TMEM columns of one accumulator
constexpr uint32_t TC_TMEM_COLS = 2 * TC_ACC_COLS;

template <typename T> struct TcShape;
template <> struct TcShape<float> {
  static constexpr int kc = 32;  // columns of k per stage
  static constexpr int n = 64;   // UMMA N
};
template <> struct TcShape<c32> {
  static constexpr int kc = 16;
  static constexpr int n = 128;
};

constexpr int TC_MAP = TC_M + TC_N;      // bytes of the inverse maps of one pair

__host__ __device__ constexpr size_t smem_cmod_tc_bytes() { return 1024 + 2 * (size_t)TC_STAGE + 64; }

// Per-thread staging values of one K chunk: A' 8 floats, B' 4 floats.
struct TcRegs {
  float a[8];
  float b[4];
};

// hi/lo split of 4 (or 2) consecutive K elements starting at element k of an
// operand row, stored into the hi and lo tiles.
__device__ __forceinline__ void store_split4(unsigned char* hi_tile, unsigned char* lo_tile, int row, int k,
                                             float x0, float x1, float x2, float x3) {
  float4 h, l;
  split_tf32(x0, h.x, l.x);
  split_tf32(x1, h.y, l.y);
  split_tf32(x2, h.z, l.z);
  split_tf32(x3, h.w, l.w);
  const uint32_t off = sw128_off((uint32_t)row, (uint32_t)k);
  *reinterpret_cast<float4*>(hi_tile + off) = h;
  *reinterpret_cast<float4*>(lo_tile + off) = l;
}

__device__ __forceinline__ void store_split2(unsigned char* hi_tile, unsigned char* lo_tile, int row, int k, float x0,
                                             float x1) {
  float2 h, l;
  split_tf32(x0, h.x, l.x);
  split_tf32(x1, h.y, l.y);
  const uint32_t off = sw128_off((uint32_t)row, (uint32_t)k);
  *reinterpret_cast<float2*>(hi_tile + off) = h;
  *reinterpret_cast<float2*>(lo_tile + off) = l;
}

// Global loads of K chunk [t0, t0 + kc) of a pair into registers.
//   c32: A' row tid & 127, complex columns 4 (tid >> 7) .. +4;
//        B' column tid & 63, complex columns 2 (tid >> 6) .. +2.
//   f32: A' row tid & 127, columns 8 (tid >> 7) .. +8;
//        B' column tid & 63, columns 4 (tid >> 6) .. +4.
template <typename T>
__device__ __forceinline__ void tc_load(TcRegs& R, const T* __restrict__ LA, const T* __restrict__ LB, int nrk,
                                        int nck, int t0, const int8_t* __restrict__ map,
                                        const T* __restrict__ dk, const T* __restrict__ dsk,
                                        const unsigned char* __restrict__ kindk) {
  using F = Field<T>;
  const int tid = threadIdx.x;
  const int row = tid & (TC_M - 1), ga = tid >> 7;
  const int u = tid & (TC_N - 1), gb = tid >> 6;
  const int i = map[row], j = map[TC_M + u];
  if constexpr (Field<T>::complex) {
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int t = t0 + 4 * ga + jj;
      T v = F::zero();
      if (i >= 0 && t < nck) v = LA[i + (long long)t * nrk];
      R.a[jj] = v.re;
      R.a[4 + jj] = v.im;
    }
#pragma unroll
    for (int jj = 0; jj < 2; ++jj) {
      const int t = t0 + 2 * gb + jj;
      T v = F::zero();
      if (j >= 0 && t < nck) v = ld_G(LB, nrk, j, t, dk, dsk, kindk);
      R.b[2 * jj] = v.re;
      R.b[2 * jj + 1] = v.im;
    }
  } else {
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
      const int t = t0 + 8 * ga + jj;
      R.a[jj] = (i >= 0 && t < nck) ? LA[i + (long long)t * nrk] : 0.0f;
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int t = t0 + 4 * gb + jj;
      R.b[jj] = (j >= 0 && t < nck) ? ld_G(LB, nrk, j, t, dk, dsk, kindk) : 0.0f;
    }
  }
}

// Registers -> hi/lo operand tiles of a stage (K-major, 128-byte swizzle).
template <typename T>
__device__ __forceinline__ void tc_store(const TcRegs& R, unsigned char* stg) {
  unsigned char* Ah = stg;
  unsigned char* Al = stg + TC_OPER;
  unsigned char* Bh = stg + 2 * TC_OPER;
  unsigned char* Bl = stg + 3 * TC_OPER;
  const int tid = threadIdx.x;
  const int row = tid & (TC_M - 1), ga = tid >> 7;
  const int u = tid & (TC_N - 1), gb = tid >> 6;
  if constexpr (Field<T>::complex) {
    store_split4(Ah, Al, row, 4 * ga, R.a[0], R.a[1], R.a[2], R.a[3]);       // Re(A): K' 0..15
    store_split4(Ah, Al, row, 16 + 4 * ga, R.a[4], R.a[5], R.a[6], R.a[7]);  // Im(A): K' 16..31
    const int k = 2 * gb;
    store_split2(Bh, Bl, u, k, R.b[0], R.b[2]);              // Re out:  Gr
    store_split2(Bh, Bl, u, 16 + k, -R.b[1], -R.b[3]);       //         -Gi
    store_split2(Bh, Bl, TC_N + u, k, R.b[1], R.b[3]);       // Im out:  Gi
    store_split2(Bh, Bl, TC_N + u, 16 + k, R.b[0], R.b[2]);  //          Gr
  } else {
    store_split4(Ah, Al, row, 8 * ga, R.a[0], R.a[1], R.a[2], R.a[3]);
    store_split4(Ah, Al, row, 8 * ga + 4, R.a[4], R.a[5], R.a[6], R.a[7]);
    store_split4(Bh, Bl, u, 4 * gb, R.b[0], R.b[1], R.b[2], R.b[3]);
  }
}

template <int NC>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, float (&v)[NC]);
template <>
__device__ __forceinline__ void tmem_ld_cols<32>(uint32_t taddr, float (&v)[32]) {
  tmem_ld32(taddr, v);
}
template <>
__device__ __forceinline__ void tmem_ld_cols<16>(uint32_t taddr, float (&v)[16]) {
  tmem_ld16(taddr, v);
}

template <typename T>
__global__ void __launch_bounds__(TC_NT, 1) k_cmod_tc(FactorArgs fa, const int4* __restrict__ tasks,
                                                      const int4* __restrict__ pairs,
                                                      const int8_t* __restrict__ maps) {
  using Sh = TcShape<T>;
  constexpr int NC = Sh::n / 4;  // accumulator columns per thread
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];  // re-aligned to 1024 below
  const uint32_t sraw = smem_u32(smem_raw);
  unsigned char* sm = smem_raw + (((sraw + 1023u) & ~1023u) - sraw);
  uint64_t* sbar = reinterpret_cast<uint64_t*>(sm + 2 * TC_STAGE);  // 2 stage barriers
  uint64_t* wbar = sbar + 2;                                        // 2 window barriers
  uint32_t* tslot = reinterpret_cast<uint32_t*>(wbar + 2);

  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = (tk.y >> 16) * TC_M, c0 = (tk.y & 0xffff) * TC_N;
  const int pb = tk.z, pe = tk.w;
  const int ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int rows_here = min(TC_M, nrow - r0), cols_here = min(TC_N, ncol - c0);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    mbar_init(&sbar[0], 1);
    mbar_init(&sbar[1], 1);
    mbar_init(&wbar[0], 1);
    mbar_init(&wbar[1], 1);
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
  auto load_chunk = [&](TcRegs& R, int u, int t0) {
    const int4 pr = pairs[u];
    const int k = pr.x, a = pr.y, q0 = pr.z;
    const int nck = fa.sn_ncol[k], nrk = fa.sn_nrow[k], fk = fa.sn_first[k];
    const T* Lk = pall + fa.sn_poff[k] + nck;
    tc_load<T>(R, Lk + a, Lk + q0, nrk, nck, t0, maps + (long long)u * TC_MAP, dall + fk, dsall + fk, fa.kind + fk);
  };
  // (u, t0) -> the next chunk in (pair, updater column) order
  auto advance = [&](int& u, int& t0) {
    t0 += Sh::kc;
    if (t0 >= fa.sn_ncol[pairs[u].x]) {
      ++u;
      t0 = 0;
    }
  };

  float acc[NC];
#pragma unroll
  for (int j = 0; j < NC; ++j) acc[j] = 0.0f;
  const int q = warp & 3, cg = warp >> 2;  // TMEM lane quarter, column group
  bool ok = true;
  // Add finished window w into the registers (waits for its MMAs).
  auto promote = [&](int w) {
    const bool done = mbar_wait_bounded(&wbar[w & 1], (uint32_t)((w >> 1) & 1));
    if (__syncthreads_or(!done)) {
      ok = false;
      return;
    }
    tc_fence_after();
    float v[NC];
    tmem_ld_cols<NC>(tmem + (uint32_t)(w & 1) * TC_ACC_COLS + ((uint32_t)(32 * q) << 16) + (uint32_t)(cg * NC), v);
#pragma unroll
    for (int j = 0; j < NC; ++j) acc[j] += v[j];
    tc_fence_before();
  };

  int c = 0;   // K chunks issued
  int pw = 0;  // next window to promote
  if (pb < pe) {
    TcRegs R0, R1;  // register sets of the even / odd chunks
    int ul = pb, tl = 0;  // load cursor: two chunks ahead of the issue cursor
    load_chunk(R0, ul, tl);
    advance(ul, tl);
    if (ul < pe) load_chunk(R1, ul, tl);
    int u = pb, t0 = 0;  // issue cursor
    while (u < pe) {
      const int st = c & 1;
      if (c >= 2) {
        const bool done = mbar_wait_bounded(&sbar[st], (uint32_t)(((c >> 1) - 1) & 1));
        if (__syncthreads_or(!done)) {
          ok = false;
          break;
        }
      }
      unsigned char* stg = sm + st * TC_STAGE;
      if (st == 0)
        tc_store<T>(R0, stg);
      else
        tc_store<T>(R1, stg);
      advance(u, t0);
      const bool last = u >= pe;
      fence_proxy_async_smem();
      __syncthreads();
      const int w = c / TC_WIN;
      if (tid == 0) {
        tc_fence_after();
        const uint32_t sa = smem_u32(stg);
        const uint32_t dacc = tmem + (uint32_t)(w & 1) * TC_ACC_COLS;
        uint32_t accf = (c % TC_WIN) != 0 ? 1u : 0u;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const uint32_t at = sa + (p == 2 ? TC_OPER : 0);
          const uint32_t bt = sa + 2 * TC_OPER + (p == 1 ? TC_OPER : 0);
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            mma_tf32(dacc, desc_sw128(at + 32u * ks), desc_sw128(bt + 32u * ks), idesc, accf);
            accf = 1u;
          }
        }
        mma_commit(&sbar[st]);
        if (c % TC_WIN == TC_WIN - 1 || last) mma_commit(&wbar[w & 1]);
      }
      // chunk c + 2 into the register set just stored
      if (ul < pe) {
        advance(ul, tl);
        if (ul < pe) {
          if (st == 0)
            load_chunk(R0, ul, tl);
          else
            load_chunk(R1, ul, tl);
        }
      }
      // window w - 1 is two chunks behind: its MMAs are (nearly) done, and its
      // accumulator is next overwritten by window w + 1, TC_WIN - 2 chunks on
      if (c % TC_WIN == 2 && w >= 1) promote(pw++);
      ++c;
      if (!ok) break;
    }
  }
  if (ok)
    while (pw <= (c - 1) / TC_WIN && c > 0) {
      promote(pw++);
      if (!ok) break;
    }
  if (!ok) {
    // drain what was issued (bounded), then report
    if (c > 0) (void)mbar_wait_bounded(&sbar[(c - 1) & 1], (uint32_t)(((c - 1) >> 1) & 1));
    if (tid == 0 && atomicCAS(&fa.status[0], 0, 2) == 0) fa.status[1] = s;
  } else if (c > 0) {
    // Epilogue: P -= U on the lower part.  Thread (q, cg, lane) holds tile
    // row 32 q + lane and accumulator columns [cg NC, cg NC + NC): for c32
    // columns 0-63 are the real parts and 64-127 the imaginary parts of tile
    // columns 0-63; each thread updates its own component.
    const int row = 32 * q + lane;
    if (row < rows_here) {
      const int gr = r0 + row;
      float* pf = reinterpret_cast<float*>(reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s]);
#pragma unroll
      for (int jj = 0; jj < NC; ++jj) {
        const int colj = cg * NC + jj;
        const int col = Field<T>::complex ? (colj & (TC_N - 1)) : colj;
        const int comp = Field<T>::complex ? (colj >> 6) : 0;
        const int gc = c0 + col;
        if (col < cols_here && gr >= gc) {
          const long long e = gr + (long long)gc * nrow;
          float* p = Field<T>::complex ? pf + 2 * e + comp : pf + e;
          *p -= acc[jj];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TC_TMEM_COLS);
}

}  // namespace rsd
