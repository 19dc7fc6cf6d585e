// The 3xTF32 tensor-core tile pipeline of the single-precision fields, used by
// the deferred in-panel Schur update (k_schur_tc): the update of one 128 x 64
// target tile accumulates in TMEM with tcgen05.mma kind::tf32 in the 3xTF32
// split (hi*hi + hi*lo + lo*hi), and the tile is read-modify-written once at
// the end.  Also here: k_make_g (G_k = L21_k D_k of every updater, read by the
// CUDA-core cmod) and the shared tcgen05 staging helpers.
//
// The pipeline is generic over its operand source (Src): operand row t of A
// holds the source row that maps to tile row t (zero when none), operand row
// u of B the row of G = L D that maps to tile column u, and the K dimension is
// the concatenation of the source's K-ranges.  Complex operands use the real
// embedding
//   A' = [Ar | Ai],  B' = [[Gr, -Gi], [Gi, Gr]]  ->  A' B'^T = [Re | Im],
// i.e. M = 128, N = 128, and 16 complex columns per 32-wide K stage.
// Warp-specialised (one CTA per SM): 16 producer warps load, split and store
// K chunks (A into TMEM, B into three shared-memory stages) and arrive on the
// stage's `full` mbarrier; one MMA warp waits on `full`, issues the 12
// tcgen05.mma of the chunk and commits to the stage's `empty` mbarrier.  No
// block-wide barrier in the main loop.
// Accuracy: the tensor pipe does not round its accumulation to nearest, so
// the sum runs in windows of TC_WIN chunks over two TMEM accumulators; the
// producers add each finished window into per-thread fp32 registers (round
// to nearest) while the next window runs on the other accumulator, and
// signal the MMA warp (`promoted` mbarrier) before the accumulator is reused.
// Every wait is bounded; on a timeout the kernel flags status 2, drains what
// it issued (bounded) and frees its TMEM.
// Reference: ll_cdiv_emit deferred Schur, src/numeric/multifrontal_ldlt.rs:3085-3167.
#pragma once

#include "factor_kernels.cuh"
#include "tcgen05.cuh"

namespace rsd {

constexpr int TC_M = 128;                 // target tile rows = UMMA M
constexpr int TC_N = 64;                  // target tile columns
constexpr int TC_PW = 16;                 // producer warps
constexpr int TC_NP = TC_PW * 32;         // producer threads
constexpr int TC_NT = TC_NP + 32;         // + one MMA-issue warp
constexpr int TC_NS = 4;                  // operand stages
constexpr int TC_OPER = 16384;            // bytes of one 128 x 32 fp32 operand tile
constexpr int TC_STAGE = 2 * TC_OPER;     // B hi, B lo in shared memory (A hi / lo live in TMEM)
constexpr int TC_WIN = 4;                 // K chunks per TMEM accumulation window
constexpr uint32_t TC_ACC_COLS = 128;     // TMEM columns of one accumulator
constexpr uint32_t TC_A_BASE = 2 * TC_ACC_COLS;   // A stages after the two accumulators
constexpr uint32_t TC_A_COLS = 64;                // A hi (32 columns) + A lo (32 columns) per stage
constexpr uint32_t TC_TMEM_COLS = 512;            // 2 x 128 accumulator + 4 x 64 A stage columns
static_assert(TC_A_BASE + TC_NS * TC_A_COLS <= TC_TMEM_COLS, "TMEM budget");

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

// After the stages: the barriers (128 bytes), then the block's D, dsub and
// kind (at most 128 columns of an f32 / c32 block) staged by k_schur_tc.
constexpr int TC_DSTAGE = 128 * (8 + 8 + 1) + 16;
__host__ __device__ constexpr size_t smem_cmod_tc_bytes() {
  return 1024 + TC_NS * (size_t)TC_STAGE + 128 + TC_DSTAGE;
}

// hi/lo split of 4 (or 2) consecutive K elements of an operand row, stored
// at byte offset `off` of the hi and lo tiles.
__device__ __forceinline__ void store_split4(unsigned char* hi_tile, unsigned char* lo_tile, uint32_t off, float x0,
                                             float x1, float x2, float x3) {
  float4 h, l;
  split_tf32(x0, h.x, l.x);
  split_tf32(x1, h.y, l.y);
  split_tf32(x2, h.z, l.z);
  split_tf32(x3, h.w, l.w);
  *reinterpret_cast<float4*>(hi_tile + off) = h;
  *reinterpret_cast<float4*>(lo_tile + off) = l;
}

__device__ __forceinline__ void store_split2(unsigned char* hi_tile, unsigned char* lo_tile, uint32_t off, float x0,
                                             float x1) {
  float2 h, l;
  split_tf32(x0, h.x, l.x);
  split_tf32(x1, h.y, l.y);
  *reinterpret_cast<float2*>(hi_tile + off) = h;
  *reinterpret_cast<float2*>(lo_tile + off) = l;
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

// G_k[r, t] = (L21_k D_k)[r, t] for off-diagonal rows [r0, r0 + MG_ROWS)
// of k and columns [t0, t0 + 32): task (k, t0, r0).  Same arithmetic as
// ld_G; consecutive threads take consecutive rows of one column (coalesced
// loads of L and stores of G).
constexpr int MG_ROWS = 1024;

template <typename T>
__global__ void __launch_bounds__(256) k_make_g(FactorArgs fa, const int4* __restrict__ tasks) {
  if (fa.status[0] != 0) return;
  const int4 tk = tasks[blockIdx.x];
  const int k = tk.x, t0 = tk.y, r0 = tk.z;
  const int first = fa.sn_first[k], ncol = fa.sn_ncol[k], nrow = fa.sn_nrow[k];
  const int off = nrow - ncol, tw = min(32, ncol - t0), r1 = min(off, r0 + MG_ROWS);
  const T* L = reinterpret_cast<const T*>(fa.panel) + fa.sn_poff[k] + ncol;
  T* G = reinterpret_cast<T*>(fa.gpool) + fa.goff[k];
  const T* d = reinterpret_cast<const T*>(fa.d) + first;
  const T* ds = reinterpret_cast<const T*>(fa.dsub) + first;
  const unsigned char* kd = fa.kind + first;
  for (int t = t0; t < t0 + tw; ++t)
#pragma unroll 4
    for (int r = r0 + (int)threadIdx.x; r < r1; r += 256) G[r + (long long)t * off] = ld_G(L, nrow, r, t, d, ds, kd);
}

// The producer / MMA pipeline of one 128 x 64 target tile, generic over the
// operand source: `Src` enumerates the (A, B) K-ranges that accumulate into
// the tile (npairs(), ncols(u)) and opens them (open(Cur&, u, row, col)):
// pointers to the A' source row of tile row `row` and to the B' source row of
// tile column `col` (or -1 when no source row lands there), with their column
// strides.  B' is read from G (plain loads) or formed as L D on the fly
// (Src::kBonfly).  The tile is panel rows [rbase + r0, +128) x columns
// [cbase + c0, +64) of supernode s, rows_here x cols_here of them real;
// P -= U is applied on rows >= columns.
template <typename T>
struct TcCur {
  int u, t0, nck, i, j;
  long long lda, ldb;
  const T* Ar;  // A' source row (column stride lda)
  const T* Br;  // B' source row (column stride ldb)
  const T* dk;  // D of the B' source (on-the-fly G only)
  const T* dsk;
  const unsigned char* kk;
};

template <typename T, typename Src>
__device__ __forceinline__ void tc_tile_pipeline(const FactorArgs& fa, const Src& src, int s, int rbase, int cbase,
                                                 int r0, int c0, int rows_here, int cols_here,
                                                 unsigned char* smem_raw) {
  using F = Field<T>;
  using Sh = TcShape<T>;
  using Cur = TcCur<T>;
  constexpr int NC = Sh::n / 4;  // accumulator columns per producer thread
  const uint32_t sraw = smem_u32(smem_raw);
  unsigned char* sm = smem_raw + (((sraw + 1023u) & ~1023u) - sraw);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + TC_NS * TC_STAGE);  // TC_NS
  uint64_t* empty = full + TC_NS;                                       // TC_NS
  uint64_t* wbar = empty + TC_NS;                                       // 2: window MMAs done
  uint64_t* pbar = wbar + 2;                                            // 2: window promoted
  uint32_t* tslot = reinterpret_cast<uint32_t*>(pbar + 2);

  const int pb = 0, pe = src.npairs();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int i = 0; i < TC_NS; ++i) {
      mbar_init(&full[i], TC_NP);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&wbar[0], 1);
    mbar_init(&wbar[1], 1);
    mbar_init(&pbar[0], TC_NP);
    mbar_init(&pbar[1], TC_NP);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, TC_TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  bool ok = true;
  int nchunks = 0;                         // chunks this thread took part in
  const int q = warp & 3, cg = warp >> 2;  // producers: TMEM lane quarter, column group
  float acc[NC];                           // producers: finished windows, fp32
#pragma unroll
  for (int j = 0; j < NC; ++j) acc[j] = 0.0f;

  if (warp == TC_PW) {
    // ---------------- MMA-issue warp ----------------
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_tf32(TC_M, Sh::n);
      const uint32_t sbase = smem_u32(sm);
      int c = 0;
      for (int u = pb; u < pe && ok; ++u) {
        const int nck = src.ncols(u);
        for (int t0 = 0; t0 < nck; t0 += Sh::kc, ++c) {
          const int st = c % TC_NS, w = c / TC_WIN;
          if (c % TC_WIN == 0 && w >= 2 && !mbar_wait_bounded(&pbar[w & 1], (uint32_t)(((w - 2) >> 1) & 1))) {
            ok = false;
            break;
          }
          if (!mbar_wait_bounded(&full[st], (uint32_t)((c / TC_NS) & 1))) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = sbase + (uint32_t)(st * TC_STAGE);
          const uint32_t dacc = tmem + (uint32_t)(w & 1) * TC_ACC_COLS;
          const uint32_t ahi = tmem + TC_A_BASE + (uint32_t)st * TC_A_COLS;
          uint32_t accf = (c % TC_WIN) != 0 ? 1u : 0u;
#pragma unroll
          for (int p = 0; p < 3; ++p) {
            const uint32_t at = ahi + (p == 2 ? 32u : 0u);  // A hi, A hi, A lo
            const uint32_t bt = sa + (p == 1 ? TC_OPER : 0);  // B hi, B lo, B hi
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
              mma_tf32_at(dacc, at + 8u * ks, desc_sw128(bt + 32u * ks), idesc, accf);
              accf = 1u;
            }
          }
          mma_commit(&empty[st]);
          const bool last = (t0 + Sh::kc >= nck) && (u + 1 == pe);
          if (c % TC_WIN == TC_WIN - 1 || last) mma_commit(&wbar[w & 1]);
        }
      }
      nchunks = c;
    }
  } else {
    // ---------------- producer warps ----------------
    // Fixed per-thread element slots (see the operand layouts above):
    //   c32: A' row tid & 127, complex columns 4 (tid >> 7) .. +4;
    //        B' column tid & 63, complex columns 2 (tid >> 6) .. +2.
    //   f32: A' row tid & 127, columns 8 (tid >> 7) .. +8;
    //        B' column tid & 63, columns 4 (tid >> 6) .. +4.
    const int row = tid & (TC_M - 1), ga = tid >> 7;
    const int ub = tid & (TC_N - 1), gb = tid >> 6;
    uint32_t ob0, ob1 = 0, ob2 = 0, ob3 = 0;
    if constexpr (Field<T>::complex) {
      ob0 = sw128_off(ub, 2 * gb);
      ob1 = sw128_off(ub, 16 + 2 * gb);
      ob2 = sw128_off(TC_N + ub, 2 * gb);
      ob3 = sw128_off(TC_N + ub, 16 + 2 * gb);
    } else {
      ob0 = sw128_off(ub, 4 * gb);
    }
    constexpr int NA = Field<T>::complex ? 4 : 8;  // A columns per thread
    constexpr int NB = Field<T>::complex ? 2 : 4;  // B columns per thread
    const int ta = NA * ga, tb = NB * gb;          // column offsets inside the chunk
    auto promote = [&](int w) {
      if (!mbar_wait_bounded(&wbar[w & 1], (uint32_t)((w >> 1) & 1))) {
        ok = false;
        return;
      }
      tc_fence_after();
      float v[NC];
      tmem_ld_cols<NC>(tmem + (uint32_t)(w & 1) * TC_ACC_COLS + ((uint32_t)(32 * q) << 16) + (uint32_t)(cg * NC), v);
#pragma unroll
      for (int j = 0; j < NC; ++j) acc[j] += v[j];
      tc_fence_before();
      mbar_arrive(&pbar[w & 1]);
    };
    // Chunk cursor: pair u, source columns [t0, t0 + kc); the loads of the
    // next chunk are issued before the current one is stored, so their
    // latency overlaps the stage wait, the split and the stores.
    auto open = [&](Cur& x, int u) {
      src.open(x, u, row, ub);
      x.u = u;
      x.t0 = 0;
      x.nck = src.ncols(u);
    };
    auto load = [&](const Cur& x, T (&va)[NA], T (&vb)[NB]) {
#pragma unroll
      for (int jj = 0; jj < NA; ++jj) {
        const int t = x.t0 + ta + jj;
        va[jj] = (x.i >= 0 && t < x.nck) ? x.Ar[(long long)t * x.lda] : F::zero();
      }
      if constexpr (Src::kBonfly) {
        // G = L D on the fly: the thread's columns and one neighbour on each
        // side (a 2x2 pivot couples a column to one of them) in one batch of
        // independent loads; D, dsub and kind come from shared memory.  The
        // arithmetic is ld_G's.
        T nv[NB + 2];
#pragma unroll
        for (int jj = 0; jj < NB + 2; ++jj) {
          const int t = x.t0 + tb + jj - 1;
          nv[jj] = (x.j >= 0 && t >= 0 && t < x.nck) ? x.Br[(long long)t * x.ldb] : F::zero();
        }
#pragma unroll
        for (int jj = 0; jj < NB; ++jj) {
          const int t = x.t0 + tb + jj;
          T g = F::zero();
          if (x.j >= 0 && t < x.nck) {
            const unsigned char kd = x.kk[t];
            const T a = nv[jj + 1];
            if (kd == 0)
              g = F::mul(a, x.dk[t]);
            else if (kd == 1)
              g = F::add(F::mul(x.dk[t], a), F::mul(x.dsk[t], nv[jj + 2]));
            else
              g = F::add(F::mul(x.dsk[t - 1], nv[jj]), F::mul(x.dk[t], a));
          }
          vb[jj] = g;
        }
      } else {
#pragma unroll
        for (int jj = 0; jj < NB; ++jj) {
          const int t = x.t0 + tb + jj;
          vb[jj] = (x.j >= 0 && t < x.nck) ? x.Br[(long long)t * x.ldb] : F::zero();
        }
      }
    };
    int c = 0, pw = 0;
    if (pb < pe) {
      Cur cur;
      open(cur, pb);
      T va[NA], vb[NB];
      load(cur, va, vb);
      for (;;) {
        Cur nx = cur;
        nx.t0 += Sh::kc;
        bool more = true;
        if (nx.t0 >= nx.nck) {
          if (cur.u + 1 < pe)
            open(nx, cur.u + 1);
          else
            more = false;
        }
        T na[NA], nb2[NB];
        if (more) load(nx, na, nb2);
        const int st = c % TC_NS;
        if (c >= TC_NS && !mbar_wait_bounded(&empty[st], (uint32_t)(((c / TC_NS) - 1) & 1))) {
          ok = false;
          break;
        }
        unsigned char* stg = sm + st * TC_STAGE;
        unsigned char* Bh = stg;
        unsigned char* Bl = stg + TC_OPER;
        // A' hi / lo into this warp's TMEM lanes (row = lane), B' into smem
        tc_fence_after();  // the stage's previous MMAs (empty barrier) precede these stores
        const uint32_t tA = tmem + ((uint32_t)(32 * q) << 16) + TC_A_BASE + (uint32_t)st * TC_A_COLS;
        if constexpr (Field<T>::complex) {
          float h[8], l[8];
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            split_tf32(va[jj].re, h[jj], l[jj]);
            split_tf32(va[jj].im, h[4 + jj], l[4 + jj]);
          }
          tmem_st4(tA + 4u * ga, h[0], h[1], h[2], h[3]);              // Re(A): K' 0..15
          tmem_st4(tA + 16u + 4u * ga, h[4], h[5], h[6], h[7]);        // Im(A): K' 16..31
          tmem_st4(tA + 32u + 4u * ga, l[0], l[1], l[2], l[3]);
          tmem_st4(tA + 48u + 4u * ga, l[4], l[5], l[6], l[7]);
          store_split2(Bh, Bl, ob0, vb[0].re, vb[1].re);                // Re out:  Gr
          store_split2(Bh, Bl, ob1, -vb[0].im, -vb[1].im);              //         -Gi
          store_split2(Bh, Bl, ob2, vb[0].im, vb[1].im);                // Im out:  Gi
          store_split2(Bh, Bl, ob3, vb[0].re, vb[1].re);                //          Gr
        } else {
          float h[8], l[8];
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) split_tf32(va[jj], h[jj], l[jj]);
          tmem_st8(tA + 8u * ga, h);
          tmem_st8(tA + 32u + 8u * ga, l);
          store_split4(Bh, Bl, ob0, vb[0], vb[1], vb[2], vb[3]);
        }
        tmem_wait_st();
        tc_fence_before();
        fence_proxy_async_smem();
        mbar_arrive(&full[st]);
        // window w - 1 is two chunks behind: promote it before the MMA warp
        // needs its accumulator again (window w + 1)
        if (c % TC_WIN == 2 && c >= TC_WIN) promote(pw++);
        ++c;
        if (!more || !ok) break;
        cur = nx;
#pragma unroll
        for (int jj = 0; jj < NA; ++jj) va[jj] = na[jj];
#pragma unroll
        for (int jj = 0; jj < NB; ++jj) vb[jj] = nb2[jj];
      }
    }
    if (ok && c > 0)
      while (pw <= (c - 1) / TC_WIN) {
        promote(pw++);
        if (!ok) break;
      }
    nchunks = c;
  }
  // Every role agrees on the outcome before the epilogue.
  const bool all_ok = __syncthreads_or(!ok) == 0;
  if (warp < TC_PW) {
    if (all_ok && nchunks > 0) {
      // P -= U on the lower part.  Thread (q, cg, lane) holds tile row
      // 32 q + lane and accumulator columns [cg NC, cg NC + NC): for c32
      // columns 0-63 are the real parts and 64-127 the imaginary parts of
      // tile columns 0-63; each thread updates its own component.
      const int nrow = fa.sn_nrow[s];
      const int trow = 32 * q + lane;
      if (trow < rows_here) {
        const int gr = rbase + r0 + trow;
        float* pf = reinterpret_cast<float*>(reinterpret_cast<T*>(fa.panel) + fa.sn_poff[s]);
        // groups of 8: every load of a group before its first store (the
        // targets are distinct; one load-store round trip per element would
        // serialise the tile)
#pragma unroll
        for (int j0 = 0; j0 < NC; j0 += 8) {
          float old[8];
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int colj = cg * NC + j0 + jj;
            const int col = Field<T>::complex ? (colj & (TC_N - 1)) : colj;
            const int comp = Field<T>::complex ? (colj >> 6) : 0;
            const int gc = cbase + c0 + col;
            const long long e = gr + (long long)gc * nrow;
            old[jj] = (col < cols_here && gr >= gc) ? (Field<T>::complex ? pf[2 * e + comp] : pf[e]) : 0.0f;
          }
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int colj = cg * NC + j0 + jj;
            const int col = Field<T>::complex ? (colj & (TC_N - 1)) : colj;
            const int comp = Field<T>::complex ? (colj >> 6) : 0;
            const int gc = cbase + c0 + col;
            if (col < cols_here && gr >= gc) {
              const long long e = gr + (long long)gc * nrow;
              (Field<T>::complex ? pf[2 * e + comp] : pf[e]) = old[jj] - acc[j0 + jj];
            }
          }
        }
      }
    }
  } else if (!all_ok && lane == 0 && nchunks > 0) {
    // drain (bounded): the last commit covers every MMA issued before it
    (void)mbar_wait_bounded(&empty[(nchunks - 1) % TC_NS], (uint32_t)(((nchunks - 1) / TC_NS) & 1));
  }
  if (!all_ok && tid == 0 && atomicCAS(&fa.status[0], 0, 2) == 0) fa.status[1] = s;
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TC_TMEM_COLS);
}


// In-panel (deferred) Schur source of block [kb, ke) of supernode s: one
// K-range of pw columns; A' = L21 rows [ke + r0, ...) of the panel (every
// row real), B' = (L21 D) rows [ke + c0, ...) formed on the fly with the
// block's D.  Reference: ll_cdiv_emit deferred Schur,
// src/numeric/multifrontal_ldlt.rs:3085-3167.
template <typename T>
struct SchurSrc {
  static constexpr bool kBonfly = true;
  const T* L21;  // panel + ke + kb * nrow
  long long nrow;
  int pw, r0, c0, rows_here, cols_here;
  const T* d;
  const T* ds;
  const unsigned char* kd;
  __device__ int npairs() const { return 1; }
  __device__ int ncols(int) const { return pw; }
  __device__ void open(TcCur<T>& x, int, int row, int col) const {
    x.i = row < rows_here ? 0 : -1;
    x.j = col < cols_here ? 0 : -1;
    x.lda = nrow;
    x.ldb = nrow;
    x.Ar = L21 + r0 + row;
    x.Br = L21 + c0 + col;
    x.dk = d;
    x.dsk = ds;
    x.kk = kd;
  }
};

// Task (s, kb, r0, c0): trailing-part tile rows [ke + r0, +128) x columns
// [ke + c0, +64) of block [kb, ke) of supernode s.
template <typename T>
__global__ void __launch_bounds__(TC_NT, 1) k_schur_tc(FactorArgs fa, const int4* __restrict__ tasks, int nb_small,
                                                       int nb_big) {
  if (fa.status[0] != 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];  // re-aligned to 1024 inside
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, kb = tk.y, r0 = tk.z, c0 = tk.w;
  const int first = fa.sn_first[s], ncol = fa.sn_ncol[s], nrow = fa.sn_nrow[s];
  const int nb = ncol >= 512 ? nb_big : nb_small;
  const int ke = min(kb + nb, ncol);
  const int mt = nrow - ke, cw = ncol - ke;
  const T* panel = reinterpret_cast<const T*>(fa.panel) + fa.sn_poff[s];
  // the block's D, dsub and kind into shared memory (after the stages and
  // barriers; the pipeline's first block barrier publishes them)
  const int pw = ke - kb;
  const uint32_t sraw = smem_u32(smem_raw);
  unsigned char* dst = smem_raw + (((sraw + 1023u) & ~1023u) - sraw) + TC_NS * TC_STAGE + 128;
  T* d_s = reinterpret_cast<T*>(dst);
  T* ds_s = d_s + 128;
  unsigned char* kd_s = reinterpret_cast<unsigned char*>(ds_s + 128);
  for (int t = threadIdx.x; t < pw; t += blockDim.x) {
    d_s[t] = reinterpret_cast<const T*>(fa.d)[first + kb + t];
    ds_s[t] = reinterpret_cast<const T*>(fa.dsub)[first + kb + t];
    kd_s[t] = fa.kind[first + kb + t];
  }
  SchurSrc<T> src{panel + ke + (long long)kb * nrow, (long long)nrow, pw, r0, c0,
                  min(TC_M, mt - r0), min(TC_N, cw - c0), d_s, ds_s, kd_s};
  tc_tile_pipeline<T>(fa, src, s, ke, ke, r0, c0, min(TC_M, mt - r0), min(TC_N, cw - c0), smem_raw);
}

}  // namespace rsd
