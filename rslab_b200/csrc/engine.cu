// Host runtime of the B200 LDL^T path: structure upload, the value-independent
// launch plan (one launch group per assembly-tree level), numeric factor and
// multi-RHS solve orchestration on one CUDA stream per handle with CUDA-graph
// capture of the frozen-pattern refactor and of the solve, the device-side
// mixed-precision refinement ladder, and the extern "C" entry points declared
// in include/rslab_b200.h.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rslab_b200.h"
#include "device/factor_kernels.cuh"
#include "device/cmod_tc.cuh"
#include "device/cmod_mm.cuh"
#include "device/solve_kernels.cuh"
#include "device/wave_solve.cuh"
#include "host/host.hpp"

using namespace rsd;
using rslab::RslabError;
using rslab::Status;

namespace {

thread_local std::string g_last_error;

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      throw RslabError(Status::CudaError, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

template <typename T>
T* dalloc(size_t n) {
  void* p = nullptr;
  if (n == 0) n = 1;
  CK(cudaMalloc(&p, n * sizeof(T)));
  return reinterpret_cast<T*>(p);
}
template <typename T>
T* dupload(const std::vector<T>& v, cudaStream_t st) {
  T* p = dalloc<T>(v.size());
  if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return p;
}
struct DFree {
  void operator()(void* p) const {
    if (p) cudaFree(p);
  }
};

// Persistent per-handle device scratch addressed by slot: a slot is
// reallocated only when a request outgrows it, so repeated refinement
// solves run without cudaMalloc / cudaFree.
struct Arena {
  std::vector<std::unique_ptr<void, DFree>> buf;
  std::vector<size_t> cap;
  void* get(int slot, size_t bytes) {
    bytes = std::max<size_t>(bytes, 256);
    if ((int)buf.size() <= slot) {
      buf.resize(slot + 1);
      cap.resize(slot + 1, 0);
    }
    if (cap[slot] < bytes) {
      buf[slot].reset();
      cap[slot] = 0;
      void* p = nullptr;
      CK(cudaMalloc(&p, bytes));
      buf[slot].reset(p);
      cap[slot] = bytes;
    }
    return buf[slot].get();
  }
};
// Arena slots of the mixed-precision driver.
enum ArenaSlot {
  A_R, A_DX, A_AX, A_NB, A_B, A_X, A_BEST, A_MASK, A_BC, A_XC, A_AXC,
  A_GM_PART, A_GM_W, A_GM_R, A_GM_V, A_GM_Z, A_SEGNORM,
  // block GMRES
  A_BG_V0, A_BG_V1, A_BG_Z, A_BG_W, A_BG_AX, A_BG_XC, A_BG_PART, A_BG_DPART, A_BG_PROJ, A_BG_Y, A_BG_NRM,
  A_BG_SCALE, A_BG_COLS, A_BG_B, A_BG_X, A_BG_R, A_BG_CL, A_BG_IB, A_BG_IX
};

size_t elem_size(int dtype) {
  switch (dtype) {
    case RSLAB_F64: return 8;
    case RSLAB_C64: return 16;
    case RSLAB_F32: return 4;
    case RSLAB_C32: return 8;
  }
  throw RslabError(Status::InvalidInput, "unknown dtype");
}

enum LaunchKind {
  L_CMOD, L_GETF2, L_DEEP, L_SCHUR,
  L_FWD_DIAG, L_FWD_PUSH, L_BWD_OFF, L_BWD,
  L_MM_GEMM, L_MM_ASM, L_SPLIT_R, L_SPLIT_C, L_FWD_GATHER, L_EXT_ADD, L_MAKE_G, L_DIAG_INV,
  L_BWD_OFF_RED, L_SCHUR_TC, L_FWD_CHAIN, L_BWD_CHAIN, L_BWD_GATHER, L_DEEP_MM, L_MAKE_M,
  L_FWD_PUSH_RED, L_FRONT_CB,
  L_JOIN_CM  // no kernel: the level's early cmod updates must be complete from here on
};
// Inverse diagonal blocks of a supernode with ncol columns: TB x TB per
// block, or ncol x ncol when it is a single block (leading dimension
// linv_ld).
inline long long linv_elems_of(int ncol) {
  return ncol <= TB ? (long long)ncol * ncol : (long long)((ncol + TB - 1) / TB) * TB * TB;
}

struct Launch {
  int kind;
  long long task_off;  // into the int4 / int2 / int task arrays
  int ntasks;
  int nb_slot;         // getf2/deep: scratch stride nb; chain solves: ticket counter
  int side = 0;        // factor: 1 = may run on the side stream, overlapping the next block's
                       // getf2 / deep-row launches (Schur update beyond the next block);
                       // 2 = on the cmod stream, overlapping the whole level (early
                       // tensor-core cmod of the next level, tagged by nb_slot)
  int narrow = 0;      // getf2: 0, or the block width that sizes the shared memory of a
                       // launch of narrow tasks (the 128-thread kernel); chain solves: 1 =
                       // one chain per block over every column of the pass
};

}  // namespace

// ---------------------------------------------------------------------------
// Analysis handle: host symbolic + device structure + launch plan.
// ---------------------------------------------------------------------------
struct rslab_sym_handle {
  rslab::Symbolic S;
  // independent systems (rslab_analyze_batch): system i owns user columns
  // [seg_begin[i], seg_begin[i+1]) and stored entries [nnz_begin[i], ...);
  // one system otherwise
  std::vector<long long> seg_begin, nnz_begin;
  std::vector<int> seg_of_g;  // system of every analysed (g-order) column
  int panel_nb = 64;
  int n = 0, ns = 0;
  long long nnz = 0;
  long long panel_elems = 0;
  std::vector<long long> poff;
  std::vector<int> nrow;
  // assembly targets (user lower-CSC order)
  std::vector<int> a_row, a_col;
  std::vector<long long> a_dst;
  // full symmetric CSR of A for SpMV
  std::vector<long long> sp_rp, sp_vmap;
  std::vector<int> sp_ci;
  // multifrontal variant: each supernode's contribution block (m x m
  // column-major, m = nrow - ncol) at cb_off[s]; per child its off-diagonal
  // rows' positions in the parent's front (ea_map from ea_moff[c]); extend-add
  // pairs (child, column range [ja, jb)) per (parent, 64-column front tile)
  std::vector<long long> cb_off, ea_moff;
  long long cb_elems = 0;
  std::vector<int> ea_map;
  std::vector<int4> ea_pairs;
  std::vector<int2> ea_rows;  // per pair: the child rows [i0, i1) whose front rows lie in its task's row chunk
  // plan
  std::vector<int4> t4;
  std::vector<int4> cpairs;   // cmod (k, a, q0, nr << 16 | nc) per tile, in update order
  std::vector<int4> t4tc, cpairs_tc;  // the same for the 128 x 64 tensor-core tiles
  std::vector<int8_t> tcmaps;         // per tensor-core pair: 128 + 64 inverse scatter maps
  // tensor-core cmod in the updater's row space (device/cmod_mm.cuh): the
  // W offset of every update-list entry in its target level's buffer, the
  // GEMM tiles (k, r0, c0, nrows | nn << 16) with their W element offsets /
  // column strides, the assembly pairs' W offsets / strides (parallel to
  // cpairs_tc), and the split pools of every updater for the real (32-column
  // chunks) and complex (16-column chunks) fields
  std::vector<long long> upd_woff;
  long long w_elems = 0;              // one level buffer (field elements)
  std::vector<int4> mm_t4;
  std::vector<long long> mm_wb, asm_wb;
  std::vector<int> mm_wl, asm_wl;
  std::vector<int> kpad_r, kpad_c;
  std::vector<long long> soff_a_r, soff_b_r, soff_a_c, soff_b_c;
  long long split_a_r = 0, split_b_r = 0, split_a_c = 0, split_b_c = 0;
  std::vector<int4> sp_r, sp_c;       // split tasks (k, r0, chunk, 0)
  std::vector<long long> goff;        // G_k = L21_k D_k pool offsets ((nrow - ncol) x ncol each)
  long long g_elems = 0;
  int bwd_slots = 0;                  // partial-sum slots of the split push / backward dots (max per level)
  std::vector<long long> linv_off;    // wide supernodes: inverses of their TB x TB diagonal blocks
  long long linv_elems = 0;
  // chain solves: per wide supernode the index of its block-0 flag (-1 for
  // narrow ones), flags per direction, and ticket counters (launches)
  std::vector<int> flag_off;
  int nflags = 0, nwave = 0;
  std::vector<int> t1;
  std::vector<int2> t2;
  std::vector<int4> st4;  // blocked diagonal-solve tasks (s, j0, r0 | c0, 0)
  std::vector<long long> uoff;  // forward-push row offsets (nrow - ncol per supernode)
  long long urows = 0;
  // forward pull lists: for column g, the U rows pushed into it (update order)
  std::vector<int> pull_ptr, pull_src;
  std::vector<int2> dots_red;  // per supernode: (first slot, chunks) of its split backward dots
  std::vector<Launch> fplan, fwdplan, bwdplan;
  int max_getf2_tasks = 0;
  int max_nb = 64;
  double flops_model = 0, flops_proxy = 0;
  // algorithmic real-field flops (multiply + add = 2) per launch kind:
  // [0] assembly, [1] cmod, [2] getf2, [3] deep-row replay, [4] panel Schur
  double kind_flops[6] = {0, 0, 0, 0, 0, 0};
  // device mirrors (uploaded lazily on first factor)
  int device = -1;
  std::vector<std::unique_ptr<void, DFree>> bufs;
  int *d_sn_first = nullptr, *d_sn_ncol = nullptr, *d_sn_nrow = nullptr, *d_rs = nullptr;
  long long *d_poff = nullptr, *d_rsoff = nullptr;
  int *d_upd_ptr = nullptr, *d_upd_k = nullptr, *d_upd_p0 = nullptr, *d_upd_p1 = nullptr;
  int *d_a_row = nullptr, *d_a_col = nullptr, *d_perm = nullptr;
  long long* d_a_dst = nullptr;
  long long *d_sp_rp = nullptr, *d_sp_vmap = nullptr;
  int* d_sp_ci = nullptr;
  int4* d_t4 = nullptr;
  int4* d_cpairs = nullptr;
  int4 *d_t4tc = nullptr, *d_cpairs_tc = nullptr;
  int8_t* d_tcmaps = nullptr;
  int4* d_mm_t4 = nullptr;
  long long *d_mm_wb = nullptr, *d_asm_wb = nullptr;
  int *d_mm_wl = nullptr, *d_asm_wl = nullptr;
  int *d_kpad_r = nullptr, *d_kpad_c = nullptr;
  long long *d_soff_a_r = nullptr, *d_soff_b_r = nullptr, *d_soff_a_c = nullptr, *d_soff_b_c = nullptr;
  int4 *d_sp_r = nullptr, *d_sp_c = nullptr;
  long long* d_goff = nullptr;
  long long *d_cb_off = nullptr, *d_ea_moff = nullptr;
  int* d_ea_map = nullptr;
  int4* d_ea_pairs = nullptr;
  int2* d_ea_rows = nullptr;
  long long* d_linv_off = nullptr;
  int* d_t1 = nullptr;
  int2* d_t2 = nullptr;
  int4* d_st4 = nullptr;
  long long* d_uoff = nullptr;
  int *d_pull_ptr = nullptr, *d_pull_src = nullptr;
  int2* d_dots_red = nullptr;
  int* d_seg_of_row = nullptr;  // system of every user row (batch handles)
  long long* d_seg_begin = nullptr;
  std::mutex mu;
  rslab_analyze_settings settings{};

  template <typename T>
  T* up(const std::vector<T>& v, cudaStream_t st) {
    T* p = dupload(v, st);
    bufs.emplace_back(p);
    return p;
  }

  void ensure_device(cudaStream_t st) {
    std::lock_guard<std::mutex> g(mu);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (device == dev) return;
    if (device >= 0) throw RslabError(Status::InvalidInput, "analysis already bound to another device");
    const auto& s = S;
    std::vector<int> f(ns), c(ns), rs(s.rs.size());
    std::vector<long long> rso(ns);
    for (int i = 0; i < ns; ++i) {
      f[i] = (int)s.sn[i].first_col;
      c[i] = (int)s.sn[i].ncol;
      rso[i] = s.rs_ptr[i];
    }
    for (size_t i = 0; i < s.rs.size(); ++i) rs[i] = (int)s.rs[i];
    std::vector<int> up_(s.upd_ptr.begin(), s.upd_ptr.end()), uk(s.upd.begin(), s.upd.end()),
        u0(s.upd_p0.begin(), s.upd_p0.end()), u1(s.upd_p1.begin(), s.upd_p1.end());
    std::vector<int> perm(s.perm.begin(), s.perm.end());
    d_sn_first = up(f, st);
    d_sn_ncol = up(c, st);
    d_sn_nrow = up(nrow, st);
    d_poff = up(poff, st);
    d_rsoff = up(rso, st);
    d_rs = up(rs, st);
    d_upd_ptr = up(up_, st);
    d_upd_k = up(uk, st);
    d_upd_p0 = up(u0, st);
    d_upd_p1 = up(u1, st);
    d_a_row = up(a_row, st);
    d_a_col = up(a_col, st);
    d_a_dst = up(a_dst, st);
    d_perm = up(perm, st);
    d_sp_rp = up(sp_rp, st);
    d_sp_ci = up(sp_ci, st);
    d_sp_vmap = up(sp_vmap, st);
    d_t4 = up(t4, st);
    d_cpairs = up(cpairs, st);
    d_t4tc = up(t4tc, st);
    d_cpairs_tc = up(cpairs_tc, st);
    d_tcmaps = up(tcmaps, st);
    d_mm_t4 = up(mm_t4, st);
    d_mm_wb = up(mm_wb, st);
    d_mm_wl = up(mm_wl, st);
    d_asm_wb = up(asm_wb, st);
    d_asm_wl = up(asm_wl, st);
    d_kpad_r = up(kpad_r, st);
    d_kpad_c = up(kpad_c, st);
    d_soff_a_r = up(soff_a_r, st);
    d_soff_b_r = up(soff_b_r, st);
    d_soff_a_c = up(soff_a_c, st);
    d_soff_b_c = up(soff_b_c, st);
    d_sp_r = up(sp_r, st);
    d_sp_c = up(sp_c, st);
    d_goff = up(goff, st);
    d_cb_off = up(cb_off, st);
    d_ea_moff = up(ea_moff, st);
    d_ea_map = up(ea_map, st);
    d_ea_pairs = up(ea_pairs, st);
    d_ea_rows = up(ea_rows, st);
    d_linv_off = up(linv_off, st);
    d_t1 = up(t1, st);
    d_t2 = up(t2, st);
    d_st4 = up(st4, st);
    d_uoff = up(uoff, st);
    d_pull_ptr = up(pull_ptr, st);
    d_pull_src = up(pull_src, st);
    d_dots_red = up(dots_red, st);
    if (seg_begin.size() > 2) {
      std::vector<int> sr(n);
      for (size_t i = 0; i + 1 < seg_begin.size(); ++i)
        for (long long r = seg_begin[i]; r < seg_begin[i + 1]; ++r) sr[r] = (int)i;
      d_seg_of_row = up(sr, st);
    }
    d_seg_begin = up(seg_begin, st);
    CK(cudaStreamSynchronize(st));
    device = dev;
  }
};

namespace {

// Append the cmod tiles (tr x tc) of every supernode of a level that has
// updaters: task (s, rt << 16 | ct, pair_begin, pair_end) and its pairs
// (k, a, q0, nr << 16 | nc) in update-list order.
// With `maps`, every pair also gets its inverse scatter maps (tr + tcw
// bytes: for each tile row / column the index of k's row landing there
// inside the pair's run, or -1).
// `lv_of` / [lv_lo, lv_hi]: when given, only updaters whose tree level lies
// in that range contribute pairs (the tensor-core cmod splits a level's
// updates into those final one level earlier and the rest).
void add_cmod_tiles(rslab_sym_handle& H, const std::vector<int64_t>& lvl, int tr, int tcw, std::vector<int4>& tasks,
                    std::vector<int4>& pairs, bool count_flops, std::vector<int8_t>* maps = nullptr,
                    const std::vector<int>* lv_of = nullptr, int lv_lo = 0, int lv_hi = 0,
                    std::vector<long long>* wbase = nullptr, std::vector<int>* wld = nullptr) {
  const auto& S = H.S;
  for (int64_t s : lvl) {
    if (S.upd_ptr[s + 1] == S.upd_ptr[s]) continue;
    const int nc = (int)S.sn[s].ncol, nr = H.nrow[s];
    const int64_t first = S.sn[s].first_col;
    const int64_t* rss = S.rs.data() + S.rs_ptr[s];
    const int ntc = (nc + tcw - 1) / tcw, ntr = (nr + tr - 1) / tr;
    std::vector<std::vector<int4>> tp((size_t)ntc * ntr);
    std::vector<std::vector<int8_t>> tm(maps ? (size_t)ntc * ntr : 0);
    std::vector<std::vector<long long>> twb(wbase ? (size_t)ntc * ntr : 0);
    std::vector<std::vector<int>> twl(wbase ? (size_t)ntc * ntr : 0);
    for (int64_t u = S.upd_ptr[s]; u < S.upd_ptr[s + 1]; ++u) {
      const int64_t k = S.upd[u], p0 = S.upd_p0[u], p1 = S.upd_p1[u];
      if (lv_of && ((*lv_of)[k] < lv_lo || (*lv_of)[k] > lv_hi)) continue;
      const int64_t nck = S.sn[k].ncol;
      const int64_t* ok = S.rs.data() + S.rs_ptr[k] + nck;
      const int64_t nok = S.rs_ptr[k + 1] - S.rs_ptr[k] - nck;
      // local row position of each of k's rows >= p0 in s (merge walk)
      std::vector<int> rel(nok - p0);
      int64_t pos = std::lower_bound(rss, rss + nr, ok[p0]) - rss;
      for (int64_t r = p0; r < nok; ++r) {
        while (rss[pos] < ok[r]) ++pos;
        rel[r - p0] = (int)pos;
      }
      int64_t qa = p0;
      while (qa < p1) {
        const int64_t ct = (ok[qa] - first) / tcw;
        int64_t qb = qa;
        while (qb < p1 && (ok[qb] - first) / tcw == ct) ++qb;
        // k's rows from the column run's first row on: the lower part
        int64_t ra = qa;
        while (ra < nok) {
          const int rt = rel[ra - p0] / tr;
          int64_t rb = ra;
          while (rb < nok && rel[rb - p0] / tr == rt) ++rb;
          tp[(size_t)ct * ntr + rt].push_back(
              make_int4((int)k, (int)ra, (int)qa, (int)(((rb - ra) << 16) | (qb - qa))));
          if (wbase) {  // W element (ra, qa) of the pair's column-major (nok - p0) x (p1 - p0) block
            twb[(size_t)ct * ntr + rt].push_back(H.upd_woff[u] + (qa - p0) * (nok - p0) + (ra - p0));
            twl[(size_t)ct * ntr + rt].push_back((int)(nok - p0));
          }
          if (maps) {
            auto& m = tm[(size_t)ct * ntr + rt];
            const size_t base = m.size();
            m.resize(base + tr + tcw, (int8_t)-1);
            for (int64_t r = ra; r < rb; ++r) m[base + rel[r - p0] - rt * tr] = (int8_t)(r - ra);
            for (int64_t qq = qa; qq < qb; ++qq) m[base + tr + (ok[qq] - first - ct * tcw)] = (int8_t)(qq - qa);
          }
          ra = rb;
        }
        qa = qb;
      }
    }
    for (int ct = 0; ct < ntc; ++ct)
      for (int rt = (ct * tcw) / tr; rt < ntr; ++rt) {
        const auto& v = tp[(size_t)ct * ntr + rt];
        if (v.empty()) continue;
        if (count_flops)
          for (const int4& pq : v) {
            const double nrr = pq.w >> 16, ncc = pq.w & 0xffff;
            // (r, c) pairs with r >= c in k's ordering, times nck multiply-adds
            double cnt = 0;
            for (int cj = 0; cj < (int)ncc; ++cj) {
              const int lo = std::max(pq.y, pq.z + cj);
              cnt += std::max(0, pq.y + (int)nrr - lo);
            }
            H.kind_flops[1] += 2.0 * cnt * (double)S.sn[pq.x].ncol;
          }
        const int pb = (int)pairs.size();
        pairs.insert(pairs.end(), v.begin(), v.end());
        if (maps) {
          const auto& m = tm[(size_t)ct * ntr + rt];
          maps->insert(maps->end(), m.begin(), m.end());
        }
        if (wbase) {
          const auto& b = twb[(size_t)ct * ntr + rt];
          const auto& l = twl[(size_t)ct * ntr + rt];
          wbase->insert(wbase->end(), b.begin(), b.end());
          wld->insert(wld->end(), l.begin(), l.end());
        }
        tasks.push_back(make_int4((int)s, (rt << 16) | ct, pb, (int)pairs.size()));
      }
  }
}

// GEMM tiles of the updater-space tensor-core cmod for the targets of a
// level: for every update-list entry (k -> s) whose updater level lies in
// [lv_lo, lv_hi], column tiles of 64 of k's rows [p0, p1) and, for each, row
// tiles of 128 of k's rows from the column tile's first row to the end (the
// lower trapezoid), with the W offset of the tile's first element.
void add_mm_tiles(rslab_sym_handle& H, const std::vector<int64_t>& lvl, const std::vector<int>& lv_of, int lv_lo,
                  int lv_hi) {
  const auto& S = H.S;
  for (int64_t s : lvl)
    for (int64_t u = S.upd_ptr[s]; u < S.upd_ptr[s + 1]; ++u) {
      const int64_t k = S.upd[u], p0 = S.upd_p0[u], p1 = S.upd_p1[u];
      if (lv_of[k] < lv_lo || lv_of[k] > lv_hi) continue;
      const int64_t m = H.nrow[k] - S.sn[k].ncol;
      for (int64_t c0 = p0; c0 < p1; c0 += MM_NC) {
        const int64_t nn = std::min<int64_t>(MM_NC, p1 - c0);
        for (int64_t r0 = c0; r0 < m; r0 += MM_M) {
          const int64_t nr = std::min<int64_t>(MM_M, m - r0);
          H.mm_t4.push_back(make_int4((int)k, (int)r0, (int)c0, (int)(nr | (nn << 16))));
          H.mm_wb.push_back(H.upd_woff[u] + (c0 - p0) * (m - p0) + (r0 - p0));
          H.mm_wl.push_back((int)(m - p0));
        }
      }
    }
}

// Build panel offsets, assembly targets, SpMV structure and the launch plan.
void build_plan(rslab_sym_handle& H, const int64_t* col_ptr, const int64_t* row_idx) {
  const auto& S = H.S;
  H.n = (int)S.n;
  H.ns = (int)S.sn.size();
  H.nnz = S.nnz;
  const int ns = H.ns, n = H.n;
  H.poff.assign(ns, 0);
  H.nrow.assign(ns, 0);
  long long acc = 0;
  for (int s = 0; s < ns; ++s) {
    long long nr = S.rs_ptr[s + 1] - S.rs_ptr[s];
    H.nrow[s] = (int)nr;
    H.poff[s] = acc;
    acc += nr * S.sn[s].ncol;
    H.flops_model += rslab::supernode_flops(nr, S.sn[s].ncol);
    H.flops_proxy += (double)nr * nr * S.sn[s].ncol;
  }
  H.panel_elems = acc;
  H.uoff.assign(ns, 0);
  H.urows = 0;
  for (int s = 0; s < ns; ++s) {
    H.uoff[s] = H.urows;
    H.urows += H.nrow[s] - S.sn[s].ncol;
  }
  if (H.urows >= (1LL << 31)) throw RslabError(Status::InvalidInput, "forward push buffer exceeds 2^31 rows");
  H.goff.assign(ns, 0);
  H.g_elems = 0;
  for (int s = 0; s < ns; ++s) {
    H.goff[s] = H.g_elems;
    H.g_elems += (long long)(H.nrow[s] - S.sn[s].ncol) * S.sn[s].ncol;
  }
  // multifrontal variant (factor_front + extend-add, multifrontal_ldlt.rs:
  // 901, 1426-1530): contribution blocks, and for every child the position
  // of each of its off-diagonal rows in its parent's front (the parent's row
  // structure: own columns, then its off-diagonal rows)
  H.cb_off.assign(ns, 0);
  H.cb_elems = 0;
  for (int s = 0; s < ns; ++s) {
    const long long m = H.nrow[s] - S.sn[s].ncol;
    H.cb_off[s] = H.cb_elems;
    H.cb_elems += m * m;
  }
  H.ea_moff.assign(ns, 0);
  H.ea_map.clear();
  {
    std::vector<int> par(ns, -1);
    for (int s = 0; s < ns; ++s)
      for (int64_t c : S.sn[s].children) par[c] = s;
    for (int c = 0; c < ns; ++c) {
      H.ea_moff[c] = (long long)H.ea_map.size();
      const int p = par[c];
      const int64_t m = H.nrow[c] - S.sn[c].ncol;
      if (p < 0 || m <= 0) continue;
      const int64_t* rc = S.rs.data() + S.rs_ptr[c] + S.sn[c].ncol;
      const int64_t* rp = S.rs.data() + S.rs_ptr[p];
      const int np = H.nrow[p];
      int64_t pos = 0;
      for (int64_t i = 0; i < m; ++i) {
        while (pos < np && rp[pos] < rc[i]) ++pos;
        if (pos >= np || rp[pos] != rc[i])
          throw RslabError(Status::InvalidInput, "contribution row outside the parent front");
        H.ea_map.push_back((int)pos);
      }
    }
  }
  // updater-space tensor-core cmod: the W block of update-list entry u
  // (k -> s) is k's rows [p0, nok) x its rows [p0, p1), column-major, in the
  // buffer of s's level; split pools per updater, K' padded to 32-wide chunks
  {
    std::vector<int> lev(ns, 0);
    for (size_t li = 0; li < S.by_level.size(); ++li)
      for (int64_t s : S.by_level[li]) lev[s] = (int)li;
    std::vector<long long> acc(S.by_level.size(), 0);
    H.upd_woff.assign(S.upd.size(), 0);
    for (int s = 0; s < ns; ++s)
      for (int64_t u = S.upd_ptr[s]; u < S.upd_ptr[s + 1]; ++u) {
        const int64_t k = S.upd[u];
        const long long nok = H.nrow[k] - S.sn[k].ncol;
        H.upd_woff[u] = acc[lev[s]];
        acc[lev[s]] += (nok - S.upd_p0[u]) * (S.upd_p1[u] - S.upd_p0[u]);
      }
    H.w_elems = 1;
    for (long long v : acc) H.w_elems = std::max(H.w_elems, v);
    H.kpad_r.assign(ns, 0);
    H.kpad_c.assign(ns, 0);
    H.soff_a_r.assign(ns, 0);
    H.soff_b_r.assign(ns, 0);
    H.soff_a_c.assign(ns, 0);
    H.soff_b_c.assign(ns, 0);
    for (int s = 0; s < ns; ++s) {
      const long long nc = S.sn[s].ncol, m = H.nrow[s] - nc;
      H.kpad_r[s] = (int)(32 * ((nc + 31) / 32));
      H.kpad_c[s] = (int)(32 * ((nc + 15) / 16));
      H.soff_a_r[s] = H.split_a_r;
      H.soff_b_r[s] = H.split_b_r;
      H.soff_a_c[s] = H.split_a_c;
      H.soff_b_c[s] = H.split_b_c;
      H.split_a_r += m * H.kpad_r[s];
      H.split_b_r += m * H.kpad_r[s];
      H.split_a_c += m * H.kpad_c[s];
      H.split_b_c += m * H.kpad_c[s];
    }
  }
  H.linv_off.assign(ns, 0);
  H.linv_elems = 0;
  for (int s = 0; s < ns; ++s) {
    H.linv_off[s] = H.linv_elems;
    H.linv_elems += linv_elems_of((int)S.sn[s].ncol);
  }
  H.flag_off.assign(ns, -1);
  H.nflags = 0;
  H.nwave = 0;
  for (int s = 0; s < ns; ++s) {
    H.flag_off[s] = H.nflags;
    H.nflags += (int)((S.sn[s].ncol + TB - 1) / TB);
  }
  // Pull lists: every off-diagonal row r of updater k (U row uoff[k] + r)
  // lands on one column g of an ancestor; list the pushes per g in the
  // ancestor's update-list order so the gather subtracts them in that order.
  H.dots_red.assign(ns, make_int2(0, 0));
  H.pull_ptr.assign(n + 1, 0);
  for (int s = 0; s < ns; ++s)
    for (int64_t u = S.upd_ptr[s]; u < S.upd_ptr[s + 1]; ++u) {
      const int64_t k = S.upd[u];
      const int64_t base = S.rs_ptr[k] + S.sn[k].ncol;
      for (int64_t r = S.upd_p0[u]; r < S.upd_p1[u]; ++r) H.pull_ptr[S.rs[base + r] + 1]++;
    }
  for (int g = 0; g < n; ++g) H.pull_ptr[g + 1] += H.pull_ptr[g];
  H.pull_src.assign(std::max(H.pull_ptr[n], 1), 0);
  {
    std::vector<int> cur(H.pull_ptr.begin(), H.pull_ptr.end() - 1);
    for (int s = 0; s < ns; ++s)
      for (int64_t u = S.upd_ptr[s]; u < S.upd_ptr[s + 1]; ++u) {
        const int64_t k = S.upd[u];
        const int64_t base = S.rs_ptr[k] + S.sn[k].ncol;
        for (int64_t r = S.upd_p0[u]; r < S.upd_p1[u]; ++r)
          H.pull_src[cur[S.rs[base + r]]++] = (int)(H.uoff[k] + r);
      }
  }
  // Assembly targets: user (i, j) -> permuted lower (r, c) -> panel slot.
  std::vector<int> col2sn(n);
  for (int s = 0; s < ns; ++s)
    for (int c = 0; c < S.sn[s].ncol; ++c) col2sn[S.sn[s].first_col + c] = s;
  H.a_row.resize(H.nnz);
  H.a_col.resize(H.nnz);
  H.a_dst.resize(H.nnz);
  for (int j = 0; j < n; ++j)
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
      int i = (int)row_idx[k];
      int gi = (int)S.perm_inv[i], gj = (int)S.perm_inv[j];
      int r = std::max(gi, gj), c = std::min(gi, gj);
      int s = col2sn[c];
      const int64_t* rs = S.rs.data() + S.rs_ptr[s];
      int nr = H.nrow[s];
      int li = (int)(std::lower_bound(rs, rs + nr, (int64_t)r) - rs);
      if (li >= nr || rs[li] != r) throw RslabError(Status::InvalidInput, "assembly target outside row structure");
      H.a_row[k] = i;
      H.a_col[k] = j;
      H.a_dst[k] = H.poff[s] + li + (long long)(c - S.sn[s].first_col) * nr;
    }
  // Full symmetric CSR (rows = user order) with value map into the lower CSC.
  std::vector<long long> cnt(n, 0);
  for (int j = 0; j < n; ++j)
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
      cnt[row_idx[k]]++;
      if (row_idx[k] != j) cnt[j]++;
    }
  H.sp_rp.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) H.sp_rp[i + 1] = H.sp_rp[i] + cnt[i];
  H.sp_ci.assign(H.sp_rp[n], 0);
  H.sp_vmap.assign(H.sp_rp[n], 0);
  std::vector<long long> off(H.sp_rp.begin(), H.sp_rp.end() - 1);
  for (int j = 0; j < n; ++j)
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
      int i = (int)row_idx[k];
      H.sp_ci[off[i]] = j;
      H.sp_vmap[off[i]++] = k;
      if (i != j) {
        H.sp_ci[off[j]] = i;
        H.sp_vmap[off[j]++] = k;
      }
    }

  // Launch plan.
  const int nb_small = H.panel_nb, nb_big = std::max(H.panel_nb, 128);
  H.max_nb = nb_big;
  auto nb_of = [&](int s) { return S.sn[s].ncol >= 512 ? nb_big : nb_small; };
  std::vector<std::vector<Launch>> bw_levels;
  std::vector<int> lv_of(ns, 0);
  for (size_t li = 0; li < S.by_level.size(); ++li)
    for (int64_t s : S.by_level[li]) lv_of[s] = (int)li;
  const int nlev = (int)S.by_level.size();
  for (int li = 0; li < nlev; ++li) {
    const auto& lvl = S.by_level[li];
    // cmod tiles of every panel that has updaters, each with its precomputed
    // list of (updater, row run, column run) pairs in update-list order:
    // TILE x TILE tiles for the CUDA-core kernel, TC_M x TC_N tiles for the
    // tensor-core kernel of the single-precision fields.  The tensor-core
    // updates of the NEXT level from updaters two or more levels below it
    // are final now: they go first, marked to overlap this level (side 2,
    // tag = their level); this level's own launch then adds the updates
    // from the level just below.
    {
      // tensor-core engine: the W tiles of the next level from updaters two
      // or more levels below it (side 2, overlapping this level; tag = the
      // target level, whose parity picks the W buffer) ...
      if (li + 1 < nlev) {
        Launch Le{L_MM_GEMM, (long long)H.mm_t4.size(), 0, li + 1, 2};
        add_mm_tiles(H, S.by_level[li + 1], lv_of, 0, li - 1);
        Le.ntasks = (int)(H.mm_t4.size() - Le.task_off);
        if (Le.ntasks) H.fplan.push_back(Le);
      }
      H.fplan.push_back(Launch{L_JOIN_CM, 0, 0, li});
      Launch L{L_CMOD, (long long)H.t4.size(), 0, 0};
      add_cmod_tiles(H, lvl, TILE, TILE, H.t4, H.cpairs, true);
      L.ntasks = (int)(H.t4.size() - L.task_off);
      if (L.ntasks) H.fplan.push_back(L);
      // ... this level's own tiles from the level just below, then the
      // assembly of every pair of the level into its 128 x 64 target tiles
      Launch Lt{L_MM_GEMM, (long long)H.mm_t4.size(), 0, li};
      add_mm_tiles(H, lvl, lv_of, li - 1, li - 1);
      Lt.ntasks = (int)(H.mm_t4.size() - Lt.task_off);
      if (Lt.ntasks) H.fplan.push_back(Lt);
      Launch La{L_MM_ASM, (long long)H.t4tc.size(), 0, li};
      add_cmod_tiles(H, lvl, TC_M, TC_N, H.t4tc, H.cpairs_tc, false, &H.tcmaps, nullptr, 0, 0, &H.asm_wb, &H.asm_wl);
      La.ntasks = (int)(H.t4tc.size() - La.task_off);
      if (La.ntasks) H.fplan.push_back(La);
    }
    // multifrontal variant: the children's contribution blocks into this
    // level's fronts, per (parent, 64-column front tile), children in order
    {
      Launch Le{L_EXT_ADD, (long long)H.t4.size(), 0, 0};
      for (int64_t s : lvl) {
        const auto& ch = S.sn[s].children;
        if (ch.empty()) continue;
        const int nt = (H.nrow[s] + 63) / 64;
        // tasks: (64-column tile, chunk of EA_ROWS front rows at or below it),
        // so a tall front spreads over many CTAs; targets stay disjoint
        for (int ct = 0; ct < nt; ++ct)
          for (int R0 = (64 * ct / EA_ROWS) * EA_ROWS; R0 < H.nrow[s]; R0 += EA_ROWS) {
            const int pb = (int)H.ea_pairs.size();
            for (int64_t c : ch) {
              const int64_t m = H.nrow[c] - S.sn[c].ncol;
              if (m <= 0) continue;
              const int* mp = H.ea_map.data() + H.ea_moff[c];
              // the child columns j whose front column mp[j] lies in this
              // tile, and the child rows whose front row lies in this chunk
              const int ja = (int)(std::lower_bound(mp, mp + m, 64 * ct) - mp);
              const int jb = (int)(std::lower_bound(mp, mp + m, 64 * ct + 64) - mp);
              const int i0 = std::max(ja, (int)(std::lower_bound(mp, mp + m, R0) - mp));
              const int i1 = (int)(std::lower_bound(mp, mp + m, R0 + EA_ROWS) - mp);
              if (jb > ja && i1 > i0) {
                H.ea_pairs.push_back(make_int4((int)c, ja, jb, 0));
                H.ea_rows.push_back(make_int2(i0, i1));
              }
            }
            if ((int)H.ea_pairs.size() > pb) H.t4.push_back(make_int4((int)s, ct, pb, (int)H.ea_pairs.size()));
          }
      }
      Le.ntasks = (int)(H.t4.size() - Le.task_off);
      if (Le.ntasks) H.fplan.push_back(Le);
    }
    int maxblocks = 0;
    for (int64_t s : lvl) maxblocks = std::max(maxblocks, (int)((S.sn[s].ncol + nb_of(s) - 1) / nb_of(s)));
    for (int b = 0; b < maxblocks; ++b) {
      Launch G{L_GETF2, (long long)H.t4.size(), 0, 0};
      std::vector<int4> deep, make_m, deep_mm, schur, schur_tc, schur_r, schur_tc_r, narrow;
      int slot = 0, launch_nb = 0, narrow_nb = 0;
      for (int64_t s : lvl) {
        int nb = nb_of(s), nc = (int)S.sn[s].ncol, nr = H.nrow[s];
        int kb = b * nb;
        if (kb >= nc) continue;
        int ke = std::min(kb + nb, nc);
        bool fuse = (nr - ke) <= FUSE_DEEP_ROWS;
        // narrow blocks with few deep rows (most leaves of a 3D problem are
        // one to a few columns) go to a 128-thread launch: several CTAs per
        // SM instead of one or two 512-thread ones
        const bool nar = ke - kb <= GETF2_NARROW_PW && nr - ke <= GETF2_NARROW_DEEP;
        (nar ? narrow : H.t4).push_back(make_int4((int)s, kb, slot, fuse ? 1 : 0));
        if (nar) narrow_nb = std::max(narrow_nb, nb);
        launch_nb = std::max(launch_nb, nb);
        if (!fuse) {
          for (int r0 = ke; r0 < nr; r0 += DEEP_R) deep.push_back(make_int4((int)s, kb, slot, r0));
          for (int r0 = ke; r0 < nr; r0 += MM_ROWS) deep_mm.push_back(make_int4((int)s, kb, slot, r0));
          for (int i0 = 0; i0 < ke - kb; i0 += MM_RB) make_m.push_back(make_int4((int)s, kb, slot, i0));
        }
        int mt = nr - ke, cw = nc - ke;
        const double pw = ke - kb;
        H.kind_flops[2] += 2.0 * pw * pw * pw / 3.0;
        H.kind_flops[3] += 2.0 * (double)(nr - ke) * pw * pw / 2.0;
        H.kind_flops[4] += 2.0 * ((double)mt * cw - (double)cw * (cw - 1) / 2.0) * pw;
        // Schur tiles of the next block's columns [ke, ke + nb) first; the
        // rest may overlap the next block's panel factorization
        const int nxt = std::min(nb, cw);
        for (int c0 = 0; c0 < cw; c0 += TILE)
          for (int r0 = c0; r0 < mt; r0 += TILE) (c0 < nxt ? schur : schur_r).push_back(make_int4((int)s, kb, r0, c0));
        for (int c0 = 0; c0 < cw; c0 += TC_N)
          for (int r0 = (c0 / TC_M) * TC_M; r0 < mt; r0 += TC_M)
            (c0 < nxt ? schur_tc : schur_tc_r).push_back(make_int4((int)s, kb, r0, c0));
        ++slot;
      }
      G.ntasks = (int)(H.t4.size() - G.task_off);
      G.nb_slot = launch_nb;
      if (!slot) continue;
      if (G.ntasks) H.fplan.push_back(G);
      if (!narrow.empty()) {
        // the same scratch slots and stride as the wide launch of this block
        Launch Gn{L_GETF2, (long long)H.t4.size(), (int)narrow.size(), launch_nb};
        Gn.narrow = narrow_nb;
        H.t4.insert(H.t4.end(), narrow.begin(), narrow.end());
        H.fplan.push_back(Gn);
      }
      H.max_getf2_tasks = std::max(H.max_getf2_tasks, slot);
      if (!deep.empty()) {
        Launch D{L_DEEP, (long long)H.t4.size(), (int)deep.size(), launch_nb};
        H.t4.insert(H.t4.end(), deep.begin(), deep.end());
        H.fplan.push_back(D);
        // the same rows as one product with the block transform (tensor-core
        // engine of the single-precision fields): M, then A21 M
        Launch Mm{L_MAKE_M, (long long)H.t4.size(), (int)make_m.size(), launch_nb};
        H.t4.insert(H.t4.end(), make_m.begin(), make_m.end());
        H.fplan.push_back(Mm);
        Launch Dm{L_DEEP_MM, (long long)H.t4.size(), (int)deep_mm.size(), launch_nb};
        H.t4.insert(H.t4.end(), deep_mm.begin(), deep_mm.end());
        H.fplan.push_back(Dm);
      }
      if (!schur.empty()) {
        Launch C{L_SCHUR, (long long)H.t4.size(), (int)schur.size(), 0};
        H.t4.insert(H.t4.end(), schur.begin(), schur.end());
        H.fplan.push_back(C);
        Launch Ct{L_SCHUR_TC, (long long)H.t4.size(), (int)schur_tc.size(), 0};
        H.t4.insert(H.t4.end(), schur_tc.begin(), schur_tc.end());
        H.fplan.push_back(Ct);
      }
      if (!schur_r.empty()) {
        Launch C{L_SCHUR, (long long)H.t4.size(), (int)schur_r.size(), 0, 1};
        H.t4.insert(H.t4.end(), schur_r.begin(), schur_r.end());
        H.fplan.push_back(C);
        Launch Ct{L_SCHUR_TC, (long long)H.t4.size(), (int)schur_tc_r.size(), 0, 1};
        H.t4.insert(H.t4.end(), schur_tc_r.begin(), schur_tc_r.end());
        H.fplan.push_back(Ct);
      }
    }
    // multifrontal variant: each front's contribution block, CB -= L21 D L21^T
    // over all its columns, in 64 x 64 tiles of its lower triangle
    {
      Launch Lf{L_FRONT_CB, (long long)H.t4.size(), 0, 0};
      for (int64_t s : lvl) {
        const int m = H.nrow[s] - (int)S.sn[s].ncol;
        for (int c0 = 0; c0 < m; c0 += TILE)
          for (int r0 = c0; r0 < m; r0 += TILE) H.t4.push_back(make_int4((int)s, r0, c0, 0));
      }
      Lf.ntasks = (int)(H.t4.size() - Lf.task_off);
      if (Lf.ntasks) H.fplan.push_back(Lf);
      // the same blocks as 128 x 64 DMMA tiles (FP64 fields, tensor engine)
      Launch Ld{L_FRONT_CB, (long long)H.t4.size(), 0, 0};
      Ld.narrow = 1;
      for (int64_t s : lvl) {
        const int m = H.nrow[s] - (int)S.sn[s].ncol;
        for (int c0 = 0; c0 < m; c0 += TC_N)
          for (int r0 = (c0 / TC_M) * TC_M; r0 < m; r0 += TC_M) H.t4.push_back(make_int4((int)s, r0, c0, 0));
      }
      Ld.ntasks = (int)(H.t4.size() - Ld.task_off);
      if (Ld.ntasks) H.fplan.push_back(Ld);
    }
    // G_k = L21_k D_k of this level's updaters, for the CUDA-core cmod of
    // their ancestors (32-column tasks), and the tensor-core engine's split
    // operands (rows of 256 x one 32-wide K' chunk per task).
    {
      Launch Mg{L_MAKE_G, (long long)H.t4.size(), 0, 0};
      for (int64_t s : lvl) {
        const int off = H.nrow[s] - (int)S.sn[s].ncol;
        for (int t0 = 0; off > 0 && t0 < S.sn[s].ncol; t0 += 32)
          for (int r0 = 0; r0 < off; r0 += MG_ROWS) H.t4.push_back(make_int4((int)s, t0, r0, 0));
      }
      Mg.ntasks = (int)(H.t4.size() - Mg.task_off);
      if (Mg.ntasks) H.fplan.push_back(Mg);
      Launch Sr{L_SPLIT_R, (long long)H.sp_r.size(), 0, 0}, Sc{L_SPLIT_C, (long long)H.sp_c.size(), 0, 0};
      for (int64_t s : lvl) {
        const int off = H.nrow[s] - (int)S.sn[s].ncol;
        for (int r0 = 0; r0 < off; r0 += MM_SPLIT_ROWS) {
          for (int c = 0; c < H.kpad_r[s] / 32; ++c) H.sp_r.push_back(make_int4((int)s, r0, c, 0));
          for (int c = 0; c < H.kpad_c[s] / 32; ++c) H.sp_c.push_back(make_int4((int)s, r0, c, 0));
        }
      }
      Sr.ntasks = (int)(H.sp_r.size() - Sr.task_off);
      Sc.ntasks = (int)(H.sp_c.size() - Sc.task_off);
      if (Sr.ntasks) H.fplan.push_back(Sr);
      if (Sc.ntasks) H.fplan.push_back(Sc);
      // inverses of the diagonal TB-blocks of this level's supernodes (used
      // by the block-chain triangular solves)
      Launch Dv{L_DIAG_INV, (long long)H.t2.size(), 0, 0};
      for (int64_t s : lvl)
        for (int j0 = 0; j0 < S.sn[s].ncol; j0 += TB) H.t2.push_back(make_int2((int)s, j0));
      Dv.ntasks = (int)(H.t2.size() - Dv.task_off);
      if (Dv.ntasks) H.fplan.push_back(Dv);
    }
    // Solve launches for this level.
    // Forward: gather the descendants' pushes into y, solve every
    // supernode's diagonal blocks (block chain, one launch), then stream the
    // push U_s = L21_s z_s.
    // Backward (levels root first): gather the ancestors' x into row order,
    // stream the off-diagonal dots W_s = L21_s^T x_anc (row-chunk partials
    // reduced in chunk order), then the diagonal blocks (block chain).
    {
      int maxb = 0;
      for (int64_t s : lvl) maxb = std::max(maxb, (int)((S.sn[s].ncol + TB - 1) / TB));
      // diagonal blocks: chain items in block order across the level's
      // supernodes (ticket order = dependency order)
      // a level with at least CH_WIDE_ITEMS blocks solves every column of a
      // pass in one chain per block (enough CTAs already); narrower levels
      // split the columns into CH_GROUPS chains of CH_NR
      int items = 0;
      for (int64_t s : lvl) items += (int)((S.sn[s].ncol + TB - 1) / TB);
      const bool wide = items >= CH_WIDE_ITEMS;
      const int ngroups = wide ? 1 : CH_GROUPS;
      if (maxb > 0) {
        Launch W{L_FWD_CHAIN, (long long)H.st4.size(), 0, H.nwave++};
        W.narrow = wide ? 1 : 0;
        for (int b = 0; b < maxb; ++b)
          for (int64_t s : lvl)
            if (b * TB < S.sn[s].ncol)
              for (int g = 0; g < ngroups; ++g) H.st4.push_back(make_int4((int)s, 2 * g, b, H.flag_off[s]));
        W.ntasks = (int)(H.st4.size() - W.task_off);
        H.fwdplan.push_back(W);
      }
      // push items: 64-row blocks, several per item for narrow supernodes
      // (about 8 column units per item)
      // (wide supernodes: PUSH_KS column units per item, partial sums
      // reduced in chunk order by the next launch)
      Launch Pu{L_FWD_PUSH, (long long)H.st4.size(), 0, 0};
      std::vector<int4> pred;
      int pslot = 0;
      for (int64_t s : lvl) {
        const int cu = (int)((S.sn[s].ncol + 31) / 32), off = H.nrow[s] - (int)S.sn[s].ncol;
        if (cu <= PUSH_KS) {
          const int nrb = std::max(1, 8 / cu);
          for (int r0 = 0; r0 < off; r0 += 64 * nrb) H.st4.push_back(make_int4((int)s, r0, nrb, -1));
        } else {
          const int nch = (cu + PUSH_KS - 1) / PUSH_KS;
          for (int r0 = 0; r0 < off; r0 += 64) {
            pred.push_back(make_int4((int)s, r0, pslot, nch));
            for (int q = 0; q < nch; ++q) H.st4.push_back(make_int4((int)s, r0, 1 | ((q * PUSH_KS) << 8), pslot + q));
            pslot += nch;
          }
        }
      }
      Pu.ntasks = (int)(H.st4.size() - Pu.task_off);
      if (Pu.ntasks) H.fwdplan.push_back(Pu);
      H.bwd_slots = std::max(H.bwd_slots, pslot);
      Launch Pr{L_FWD_PUSH_RED, (long long)H.st4.size(), (int)pred.size(), 0};
      H.st4.insert(H.st4.end(), pred.begin(), pred.end());
      if (Pr.ntasks) H.fwdplan.push_back(Pr);

      std::vector<Launch> bw;
      // dots items (s, block, row chunk, slot); a block with several row
      // chunks writes partial sums to slots, reduced in chunk order next
      // (the backward chain item of block i sums a split block's chunk
      // partials itself, in chunk order: slots dots_red[s].x + i * chunks)
      Launch Bo{L_BWD_OFF, (long long)H.st4.size(), 0, 0};
      int slot = 0;
      for (int64_t s : lvl) {
        const int off = H.nrow[s] - (int)S.sn[s].ncol;
        if (off <= 0) continue;
        const int nch = (off + BWD_CH - 1) / BWD_CH;
        if (nch > 1) H.dots_red[s] = make_int2(slot, nch);
        for (int i = 0; i * TB < S.sn[s].ncol; ++i) {
          if (nch == 1) {
            H.st4.push_back(make_int4((int)s, i, 0, -1));
          } else {
            for (int q = 0; q < nch; ++q) H.st4.push_back(make_int4((int)s, i, q * BWD_CH, slot + q));
            slot += nch;
          }
        }
      }
      Bo.ntasks = (int)(H.st4.size() - Bo.task_off);
      if (Bo.ntasks) bw.push_back(Bo);
      H.bwd_slots = std::max(H.bwd_slots, slot);
      if (maxb > 0) {
        Launch W{L_BWD_CHAIN, (long long)H.st4.size(), 0, H.nwave++};
        W.narrow = wide ? 1 : 0;
        for (int dd = 0; dd < maxb; ++dd)
          for (int64_t s : lvl) {
            const int nblk = (int)((S.sn[s].ncol + TB - 1) / TB);
            if (dd < nblk)
              for (int g = 0; g < ngroups; ++g)
                H.st4.push_back(make_int4((int)s, 1 + 2 * g, nblk - 1 - dd, H.flag_off[s]));
          }
        W.ntasks = (int)(H.st4.size() - W.task_off);
        bw.push_back(W);
      }
      bw_levels.push_back(bw);
    }
  }
  // Backward: levels root first.
  for (auto it = bw_levels.rbegin(); it != bw_levels.rend(); ++it)
    for (const Launch& L : *it) H.bwdplan.push_back(L);
}

// Chunk depth of the tile engine for an element size (KChunk<T>::v).
size_t kchunk(size_t es) { return es == 16 ? 16 : 32; }
size_t smem_schur(size_t es) { return 2 * kchunk(es) * TILE * es; }
// Deep-row staging (DEEP_R + 1) x nb plus the replay program, 16-byte aligned.
size_t smem_replay(size_t es, int nb) {
  return (((size_t)(DEEP_R + 1) * nb * es + 15) & ~size_t(15)) + (size_t)nb * (3 * es + 4 + 1) + 16;
}
size_t smem_getf2(size_t es, int nb) {
  size_t a = (size_t)nb * (nb + 1) / 2 * es + 8 * nb * es + 16 + 32 * 8 + 32 * 4 + 16 * 4 + 4 * nb * 4;
  return std::max(a, smem_replay(es, nb)) + 64;
}
size_t smem_deep(size_t es, int nb) { return smem_replay(es, nb) + 64; }
size_t smem_diag_inv(size_t es) { return (size_t)TB * (TB + 1) * 2 * es; }

// Threads of the BK panel kernel: its per-step trailing update is
// latency-bound, so 16 warps hide more of it than 8.
constexpr int GETF2_NT = 512;

// Fields whose descendant updates can run on the tf32 tensor cores.
template <typename T> struct TensorCmod { static constexpr bool ok = false; };
template <> struct TensorCmod<float> { static constexpr bool ok = true; };
template <> struct TensorCmod<c32> { static constexpr bool ok = true; };

// Shared-memory limits of the streamed / chain solve kernels for NR
// right-hand-side columns (NR = 1, 4, RHS_MAX instantiated).
template <typename T, int NR>
void solve_nr_attrs() {
  CK(cudaFuncSetAttribute(k_stream<T, true, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st_smem_bytes<T>(NR)));
  CK(cudaFuncSetAttribute(k_stream<T, false, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st_smem_bytes<T>(NR)));
  CK(cudaFuncSetAttribute(k_chain<T, true, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ch_smem_bytes<T>(NR)));
  CK(cudaFuncSetAttribute(k_chain<T, false, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ch_smem_bytes<T>(NR)));
}

// Launch a streamed (kind 0) or chain (kind 1) solve kernel instantiated for
// the smallest NR in {1, 4, RHS_MAX} that holds nr columns.
template <typename T, bool FWD, int NR>
void launch_solve_nr(int kind, int grid, int nr, const SolveArgs& sa, const int4* tasks, int ctr, int flags,
                     cudaStream_t st, int gw = CH_NR) {
  if (kind == 0)
    k_stream<T, FWD, NR><<<grid, WV_NT, st_smem_bytes<T>(NR), st>>>(sa, tasks);
  else
    k_chain<T, FWD, NR><<<grid, WV_NT, ch_smem_bytes<T>(NR), st>>>(sa, tasks, ctr, flags, gw);
}
template <typename T, bool FWD>
void launch_solve(int kind, int grid, int nr, const SolveArgs& sa, const int4* tasks, int ctr = 0, int flags = 0,
                  cudaStream_t st = nullptr, bool wide = false) {
  if (kind == 1) {  // chain items carry at most CH_NR columns each, or all of them (wide levels)
    if (nr <= 1)
      launch_solve_nr<T, FWD, 1>(kind, grid, nr, sa, tasks, ctr, flags, st);
    else if (nr <= CH_NR || !wide)
      launch_solve_nr<T, FWD, CH_NR>(kind, grid, nr, sa, tasks, ctr, flags, st);
    else
      launch_solve_nr<T, FWD, RHS_MAX>(kind, grid, nr, sa, tasks, ctr, flags, st, RHS_MAX);
    return;
  }
  if (nr <= 1)
    launch_solve_nr<T, FWD, 1>(kind, grid, nr, sa, tasks, ctr, flags, st);
  else if (nr <= 4)
    launch_solve_nr<T, FWD, 4>(kind, grid, nr, sa, tasks, ctr, flags, st);
  else
    launch_solve_nr<T, FWD, RHS_MAX>(kind, grid, nr, sa, tasks, ctr, flags, st);
}

template <typename T>
struct KernelSetup {
  static void configure() {
    static bool done = false;
    if (done) return;
    const size_t es = sizeof(T);
    if constexpr (TensorCmod<T>::ok) {
      CK(cudaFuncSetAttribute(k_cmod_mm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_cmod_mm_bytes<T>()));
      CK(cudaFuncSetAttribute(k_schur_tc<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cmod_tc_bytes()));
    }
    CK(cudaFuncSetAttribute(k_cmod<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cmod_bytes<T>()));
    if constexpr (!TensorCmod<T>::ok) {
      CK(cudaFuncSetAttribute(k_cmod_dmm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_cmod_dmm_bytes<T>()));
      CK(cudaFuncSetAttribute(k_schur_dmm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_schur_dmm_bytes<T>()));
      CK(cudaFuncSetAttribute(k_front_cb_dmm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_cmod_dmm_bytes<T>()));
    }
    CK(cudaFuncSetAttribute(k_schur<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_schur(es)));
    CK(cudaFuncSetAttribute(k_front_cb<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_schur(es)));
    CK(cudaFuncSetAttribute(k_getf2<T, GETF2_NT, getf2_wide_minb(sizeof(T))>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)smem_getf2(es, 128)));
    CK(cudaFuncSetAttribute(k_getf2<T, 256, getf2_mid_minb(sizeof(T))>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)smem_getf2(es, 128)));
    CK(cudaFuncSetAttribute(k_getf2<T, 128, getf2_narrow_minb(sizeof(T))>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_getf2(es, 128)));
    if constexpr (TensorCmod<T>::ok)
      CK(cudaFuncSetAttribute(k_getf2_ll<T, GETF2_NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem_getf2_ll_bytes<T>(128)));
    CK(cudaFuncSetAttribute(k_deep<T, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_deep(es, 128)));
    CK(cudaFuncSetAttribute(k_diag_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_diag_inv(es)));
    CK(cudaFuncSetAttribute(k_deep_mm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_deep_mm_bytes<T>()));
    CK(cudaFuncSetAttribute(k_make_m<T, 32 * MM_RB, make_m_sl(sizeof(T))>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)smem_make_m_bytes(es, 128, make_m_sl(sizeof(T)))));
    CK(cudaFuncSetAttribute(k_make_m<T, 32 * MM_RB, MAKE_M_SL_WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)smem_make_m_bytes(es, 128, MAKE_M_SL_WIDE)));
    solve_nr_attrs<T, 1>();
    solve_nr_attrs<T, 4>();
    solve_nr_attrs<T, RHS_MAX>();
    done = true;
  }
};

inline unsigned grid1(long long m, int tpb = 256) { return (unsigned)((m + tpb - 1) / tpb); }

}  // namespace

// ---------------------------------------------------------------------------
// Factor handle.
// ---------------------------------------------------------------------------
struct rslab_fac_handle {
  rslab_sym_handle* sym = nullptr;
  int dtype = RSLAB_F64;     // field the factor computes in
  int dtype_hi = -1;         // mixed mode: field of the original A (else -1)
  rslab_factor_settings set{};
  cudaStream_t st = nullptr;
  bool own_stream = false;
  std::vector<std::unique_ptr<void, DFree>> bufs;
  void* panel = nullptr;
  void* d = nullptr;
  void* dsub = nullptr;
  unsigned char* kind = nullptr;
  int* lperm = nullptr;
  double* scale = nullptr;
  unsigned long long* rowmax = nullptr;
  void* aval = nullptr;     // A values in the factor field (device)
  void* aval_hi = nullptr;  // mixed mode: original A (device, high precision)
  int* status = nullptr;
  int* h_status = nullptr;  // pinned
  unsigned long long* cnt3 = nullptr;
  double* floor_dev = nullptr;          // force-accept static-pivot floor (device)
  unsigned long long* amax_dev = nullptr;
  void* scratch = nullptr;
  long long scratch_stride = 0;
  void* gpool = nullptr;  // G_k = L21_k D_k of every updater (read by both cmod engines)
  void* cbpool = nullptr; // multifrontal variant: every supernode's contribution block
  void* linv = nullptr;   // inverse diagonal blocks of the wide supernodes
  // updater-space tensor-core cmod (f32 / c32, tensor engine): split operand
  // pools (tf32 hi / lo of L21 and of G; complex fields also the [hi | lo]
  // sums Ar + Ai and Gr + Gi of the 3M product), two level buffers of W, and
  // the TMA tensor maps of every updater's pools (MM_MAPS per supernode)
  float *sp_ahi = nullptr, *sp_alo = nullptr, *sp_bhi = nullptr, *sp_blo = nullptr;
  float *sp_as = nullptr, *sp_bs = nullptr;
  float* wbuf = nullptr;
  CUtensorMap* tmaps = nullptr;
  // static pivot reuse: the pivot record of the last searching factor and the
  // device flag that makes getf2 replay it (read inside the captured graph)
  int* pivrec = nullptr;
  int* pivot_reuse = nullptr;
  bool reuse_on = false;
  // graph of the numeric factor (values read from `aval`)
  cudaGraphExec_t fgraph = nullptr;
  // solve workspace
  int ws_nrhs = 0;
  void *Yg = nullptr, *Ze = nullptr, *Xg = nullptr, *Ub = nullptr, *Wb = nullptr, *bdev = nullptr, *xdev = nullptr;
  void* Wp = nullptr;  // partial sums of the split backward dots
  int* wstate = nullptr;   // wavefront solves: sticky status, abort word, ticket counters, block flags
  int* h_wstat = nullptr;  // pinned copy of the sticky status after each solve
  std::vector<std::unique_ptr<void, DFree>> ws;
  cudaGraphExec_t sgraph = nullptr;
  int sgraph_nrhs = -1;
  // results
  long long ipos = 0, ineg = 0, izero = 0, nperturbed = 0;
  int last_status = 0, failing_sn = -1;
  double factor_ms = 0, solve_ms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // side stream of the factor (lowest priority) and its fork / join events
  cudaStream_t st2 = nullptr, st3 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_cm[2] = {nullptr, nullptr};
  // per-launch rows of the last factor/solve profile
  std::vector<int> tr_kind, tr_grid;
  std::vector<float> tr_ms;
  Arena arena;  // mixed-precision refinement scratch
  // per (system, column) backward errors of the last mixed solve
  std::vector<double> last_be;
  int last_be_nrhs = 0;

  ~rslab_fac_handle() {
    if (fgraph) cudaGraphExecDestroy(fgraph);
    if (sgraph) cudaGraphExecDestroy(sgraph);
    if (h_status) cudaFreeHost(h_status);
    if (h_wstat) cudaFreeHost(h_wstat);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    for (cudaEvent_t e : ev_cm)
      if (e) cudaEventDestroy(e);
    if (st2) cudaStreamDestroy(st2);
    if (st3) cudaStreamDestroy(st3);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own_stream && st) cudaStreamDestroy(st);
  }
  template <typename T>
  T* al(size_t n) {
    T* p = dalloc<T>(n);
    bufs.emplace_back(p);
    return p;
  }
};

namespace {

template <typename T>
FactorArgs make_fargs(rslab_fac_handle& F) {
  auto& H = *F.sym;
  FactorArgs a{};
  a.sn_first = H.d_sn_first;
  a.sn_ncol = H.d_sn_ncol;
  a.sn_nrow = H.d_sn_nrow;
  a.sn_poff = H.d_poff;
  a.sn_rsoff = H.d_rsoff;
  a.rs = H.d_rs;
  a.upd_ptr = H.d_upd_ptr;
  a.upd_k = H.d_upd_k;
  a.upd_p0 = H.d_upd_p0;
  a.upd_p1 = H.d_upd_p1;
  a.panel = F.panel;
  a.d = F.d;
  a.dsub = F.dsub;
  a.kind = F.kind;
  a.lperm = F.lperm;
  a.scratch = F.scratch;
  a.scratch_stride = F.scratch_stride;
  a.status = F.status;
  a.perturb_floor = F.set.on_zero_pivot == RSLAB_PIVOT_PERTURB ? F.set.abs_floor : -1.0;
  a.gpool = F.gpool;
  a.goff = H.d_goff;
  a.floor_dev = F.floor_dev;
  a.pivrec = F.pivrec;
  a.pivot_reuse = F.pivot_reuse;
  a.cbpool = F.cbpool;
  a.cb_off = H.d_cb_off;
  if (F.set.on_zero_pivot == RSLAB_PIVOT_FORCE_ACCEPT) a.perturb_floor = 0.0;
  return a;
}

// Enqueue the whole numeric factor of the values in F.aval on F.st.
struct Prof {
  std::vector<cudaEvent_t> ev;
  std::vector<int> kind;
  std::vector<int> grid;
  std::vector<int> fine;
  void mark(cudaStream_t st, int k, int ntasks = 0, int launch_kind = -1) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    CK(cudaEventRecord(e, st));
    ev.push_back(e);
    kind.push_back(k);
    grid.push_back(ntasks);
    fine.push_back(launch_kind);
  }
  // Per-launch rows (launch kind, grid size, device ms) into the handle.
  void store(std::vector<int>& tk, std::vector<int>& tg, std::vector<float>& tms) const {
    tk.clear();
    tg.clear();
    tms.clear();
    for (size_t i = 1; i < ev.size(); ++i) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, ev[i - 1], ev[i]));
      tk.push_back(fine[i]);
      tg.push_back(grid[i]);
      tms.push_back(ms);
    }
  }
  ~Prof() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

template <typename T>
void enqueue_factor(rslab_fac_handle& F, Prof* prof = nullptr) {
  auto& H = *F.sym;
  const int n = H.n;
  const size_t es = sizeof(T);
  cudaStream_t st = F.st;
  CK(cudaMemsetAsync(F.status, 0, 4 * sizeof(int), st));
  CK(cudaMemsetAsync(F.panel, 0, H.panel_elems * es, st));
  CK(cudaMemsetAsync(F.kind, 0, n, st));
  CK(cudaMemsetAsync(F.d, 0, n * es, st));
  CK(cudaMemsetAsync(F.dsub, 0, n * es, st));
  if (F.set.scaling == RSLAB_SCALING_ONEPASS) {
    CK(cudaMemsetAsync(F.rowmax, 0, n * sizeof(unsigned long long), st));
    if (H.nnz) k_rowmax<T><<<grid1(H.nnz), 256, 0, st>>>(H.nnz, H.d_a_row, H.d_a_col, (const T*)F.aval, F.rowmax);
    k_scale_from_rowmax<<<grid1(n), 256, 0, st>>>(n, F.rowmax, F.scale);
  }
  if (H.nnz)
    k_assemble<T><<<grid1(H.nnz), 256, 0, st>>>(H.nnz, H.d_a_row, H.d_a_col, (const T*)F.aval, F.scale, H.d_a_dst,
                                                (T*)F.panel);
  FactorArgs fa = make_fargs<T>(F);
  const int nb_small = H.panel_nb, nb_big = std::max(H.panel_nb, 128);
  // tensor engine: descendant updates as updater-space GEMM tiles + assembly
  // (tcgen05 3xTF32 for f32 / c32, DMMA for f64 / c64); the single-precision
  // fields also run their panel Schur / deep rows on the tensor-core kernels
  const bool mm = F.set.schur_engine == RSLAB_SCHUR_TENSOR;
  const bool use_tc = TensorCmod<T>::ok && mm;
  // deep rows of tall panels as a product with the block transform on the
  // tensor engine of every field; the FMA engine replays them row by row
  fa.deep_mm = mm ? 1 : 0;
  // multifrontal variant: contribution blocks and extend-add instead of cmod
  const bool mf = F.set.method == RSLAB_METHOD_MULTIFRONTAL;
  if (mf) CK(cudaMemsetAsync(F.cbpool, 0, (size_t)std::max(H.cb_elems, 1LL) * es, st));
  if (F.floor_dev) {
    CK(cudaMemsetAsync(F.amax_dev, 0, sizeof(unsigned long long), st));
    k_panel_absmax<T><<<(unsigned)std::min<long long>(grid1(H.panel_elems), 148LL * 8), 256, 0, st>>>(
        H.panel_elems, (const T*)F.panel, F.amax_dev);
    k_force_floor<<<1, 1, 0, st>>>(F.amax_dev, F.floor_dev);
  }
  if (prof) prof->mark(st, 0);
  // Launches marked `side` (the Schur update beyond the next block) run on
  // the side stream when not profiling; every later launch except the next
  // block's getf2 / deep-row launches waits for them first.
  const bool overlap = prof == nullptr && F.st2 != nullptr && F.set.overlap != 0;
  bool side_pending = false;
  auto runs = [&](const Launch& L) {
    switch (L.kind) {
      case L_CMOD: return !mm && !mf;
      case L_MM_GEMM: case L_MM_ASM: return mm && !mf;
      case L_SPLIT_R: return use_tc && !mf && !Field<T>::complex;
      case L_SPLIT_C: return use_tc && !mf && Field<T>::complex;
      case L_MAKE_G: return !use_tc && !mf;  // G_k of the CUDA-core cmod and of the DMMA tiles
      case L_EXT_ADD: return mf;
      case L_FRONT_CB: return mf && (L.narrow != 0) == (mm && !TensorCmod<T>::ok);  // DMMA tiles or FMA tiles
      case L_DEEP: return !fa.deep_mm;
      case L_MAKE_M: case L_DEEP_MM: return fa.deep_mm != 0;
      case L_SCHUR: return !mm;
      case L_SCHUR_TC: return mm;  // tcgen05 tiles (f32 / c32) or DMMA tiles (f64 / c64)
      default: return true;
    }
  };
  bool cm_pending[2] = {false, false};
  for (const Launch& L : H.fplan) {
    if (!runs(L)) continue;
    cudaStream_t ls = st;
    if (L.kind == L_JOIN_CM) {
      // this level's early updates (forked one level ago) precede all of its work
      if (cm_pending[L.nb_slot & 1]) CK(cudaStreamWaitEvent(st, F.ev_cm[L.nb_slot & 1], 0));
      cm_pending[L.nb_slot & 1] = false;
      continue;
    }
    if (overlap && L.side == 2) {
      CK(cudaEventRecord(F.ev_fork, st));
      CK(cudaStreamWaitEvent(F.st3, F.ev_fork, 0));
      ls = F.st3;
    } else if (overlap && L.side == 1) {
      CK(cudaEventRecord(F.ev_fork, st));
      CK(cudaStreamWaitEvent(F.st2, F.ev_fork, 0));
      ls = F.st2;
    } else if (side_pending && L.kind != L_GETF2 && L.kind != L_DEEP && L.kind != L_MAKE_M &&
               L.kind != L_DEEP_MM) {
      CK(cudaStreamWaitEvent(st, F.ev_join, 0));
      side_pending = false;
    }
    switch (L.kind) {
      case L_CMOD:
        if (mm) continue;
        k_cmod<T><<<L.ntasks, CM_NT, smem_cmod_bytes<T>(), ls>>>(fa, H.d_t4 + L.task_off, H.d_cpairs);
        break;
      case L_MAKE_G:
        k_make_g<T><<<L.ntasks, 256, 0, ls>>>(fa, H.d_t4 + L.task_off);
        break;
      case L_MM_GEMM:
      case L_MM_ASM:
      case L_SPLIT_R:
      case L_SPLIT_C:
        if constexpr (!TensorCmod<T>::ok) {
          // FP64 fields: DMMA tiles from L21 and the G pool, then the same assembly
          T* wb = reinterpret_cast<T*>(F.wbuf) + (size_t)(L.nb_slot & 1) * H.w_elems;
          if (L.kind == L_MM_GEMM)
            k_cmod_dmm<T><<<L.ntasks, DM_NT, smem_cmod_dmm_bytes<T>(), ls>>>(
                fa, H.d_mm_t4 + L.task_off, H.d_mm_wb + L.task_off, H.d_mm_wl + L.task_off, wb);
          else if (L.kind == L_MM_ASM)
            k_cmod_asm<T><<<L.ntasks, ASM_NT, 0, ls>>>(fa, H.d_t4tc + L.task_off, H.d_cpairs_tc, H.d_tcmaps, H.d_asm_wb,
                                                    H.d_asm_wl, F.wbuf + (size_t)(L.nb_slot & 1) * H.w_elems * es / 4);
          else
            continue;
        } else {
          constexpr bool cx = Field<T>::complex;
          const size_t wsz = (size_t)H.w_elems * (cx ? 2 : 1);
          if (L.kind == L_MM_GEMM)
            k_cmod_mm<T><<<L.ntasks, MM_NT, smem_cmod_mm_bytes<T>(), ls>>>(
                fa, H.d_mm_t4 + L.task_off, H.d_mm_wb + L.task_off, H.d_mm_wl + L.task_off, F.tmaps,
                cx ? H.d_kpad_c : H.d_kpad_r, F.wbuf + (L.nb_slot & 1) * wsz);
          else if (L.kind == L_MM_ASM)
            k_cmod_asm<T><<<L.ntasks, ASM_NT, 0, ls>>>(fa, H.d_t4tc + L.task_off, H.d_cpairs_tc, H.d_tcmaps, H.d_asm_wb,
                                                    H.d_asm_wl, F.wbuf + (L.nb_slot & 1) * wsz);
          else
            k_split<T><<<L.ntasks, MM_SPLIT_NT, 0, ls>>>(
                fa, (cx ? H.d_sp_c : H.d_sp_r) + L.task_off, cx ? H.d_soff_a_c : H.d_soff_a_r,
                cx ? H.d_soff_b_c : H.d_soff_b_r, cx ? H.d_kpad_c : H.d_kpad_r, F.sp_ahi, F.sp_alo, F.sp_bhi,
                F.sp_blo, F.sp_as, F.sp_bs);
        }
        break;
      case L_DIAG_INV:
        k_diag_inv<T><<<L.ntasks, DI_NT, smem_diag_inv(es), ls>>>(H.d_t2 + L.task_off, H.d_sn_ncol, H.d_sn_nrow,
                                                                 H.d_poff, (const T*)F.panel, F.status, (T*)F.linv,
                                                                 H.d_linv_off);
        break;
      case L_GETF2: {
        FactorArgs f2 = fa;
        f2.scratch_stride = getf2_scratch_stride(L.nb_slot, (long long)es);
        if (L.narrow) {  // narrow blocks: the bit-exact form on 4 warps, every field
          k_getf2<T, 128, getf2_narrow_minb(sizeof(T))>
              <<<L.ntasks, 128, smem_getf2(es, L.narrow), ls>>>(f2, H.d_t4 + L.task_off, nb_small, nb_big);
          break;
        }
        if constexpr (TensorCmod<T>::ok) {
          // left-looking form (parity by tolerance, like the rest of the
          // engine) for launches of a few blocks, where a block's step
          // latency is the critical path; launches of many blocks take the
          // right-looking form, which fits two CTAs per SM instead of one
          if (use_tc && L.ntasks < GETF2_LL_MAX_TASKS) {
            k_getf2_ll<T, GETF2_NT><<<L.ntasks, GETF2_NT, smem_getf2_ll_bytes<T>(L.nb_slot), ls>>>(
                f2, H.d_t4 + L.task_off, nb_small, nb_big);
            break;
          }
        }
        if (L.ntasks >= GETF2_LL_MAX_TASKS)  // many blocks: 8 warps, more CTAs per SM
          k_getf2<T, 256, getf2_mid_minb(sizeof(T))>
              <<<L.ntasks, 256, smem_getf2(es, L.nb_slot), ls>>>(f2, H.d_t4 + L.task_off, nb_small, nb_big);
        else
          k_getf2<T, GETF2_NT, getf2_wide_minb(sizeof(T))>
              <<<L.ntasks, GETF2_NT, smem_getf2(es, L.nb_slot), ls>>>(f2, H.d_t4 + L.task_off, nb_small, nb_big);
        break;
      }
      case L_DEEP: {
        if (fa.deep_mm) continue;
        FactorArgs f2 = fa;
        f2.scratch_stride = getf2_scratch_stride(L.nb_slot, (long long)es);
        k_deep<T, 256><<<L.ntasks, 256, smem_deep(es, L.nb_slot), ls>>>(f2, H.d_t4 + L.task_off, nb_small, nb_big);
        break;
      }
      case L_MAKE_M: {
        if (!fa.deep_mm) continue;
        FactorArgs f2 = fa;
        f2.scratch_stride = getf2_scratch_stride(L.nb_slot, (long long)es);
        if (L.ntasks >= GETF2_LL_MAX_TASKS)  // many blocks: smaller slices, more CTAs per SM
          k_make_m<T, 32 * MM_RB, MAKE_M_SL_WIDE>
              <<<L.ntasks, 32 * MM_RB, smem_make_m_bytes(es, L.nb_slot, MAKE_M_SL_WIDE), ls>>>(
                  f2, H.d_t4 + L.task_off, nb_small, nb_big);
        else
          k_make_m<T, 32 * MM_RB, make_m_sl(sizeof(T))>
              <<<L.ntasks, 32 * MM_RB, smem_make_m_bytes(es, L.nb_slot, make_m_sl(sizeof(T))), ls>>>(
                  f2, H.d_t4 + L.task_off, nb_small, nb_big);
        break;
      }
      case L_DEEP_MM: {
        if (!fa.deep_mm) continue;
        {
          FactorArgs f2 = fa;
          f2.scratch_stride = getf2_scratch_stride(L.nb_slot, (long long)es);
          k_deep_mm<T><<<L.ntasks, 256, smem_deep_mm_bytes<T>(), ls>>>(f2, H.d_t4 + L.task_off, nb_small, nb_big);
        }
        break;
      }
      case L_SCHUR:
        if (mm) continue;
        k_schur<T><<<L.ntasks, TPB, smem_schur(es), ls>>>(fa, H.d_t4 + L.task_off, nb_small, nb_big);
        break;
      case L_EXT_ADD:
        k_extend_add<T><<<L.ntasks, 256, 0, ls>>>(fa, H.d_t4 + L.task_off, H.d_ea_pairs, H.d_ea_rows, H.d_ea_map,
                                                   H.d_ea_moff);
        break;
      case L_FRONT_CB:
        if constexpr (!TensorCmod<T>::ok) {
          if (L.narrow) {
            k_front_cb_dmm<T><<<L.ntasks, DM_NT, smem_cmod_dmm_bytes<T>(), ls>>>(fa, H.d_t4 + L.task_off);
            break;
          }
        }
        k_front_cb<T><<<L.ntasks, TPB, smem_schur(es), ls>>>(fa, H.d_t4 + L.task_off);
        break;
      case L_SCHUR_TC:
        if (!mm) continue;
        if constexpr (TensorCmod<T>::ok)
          k_schur_tc<T><<<L.ntasks, TC_NT, smem_cmod_tc_bytes(), ls>>>(fa, H.d_t4 + L.task_off, nb_small, nb_big);
        else
          k_schur_dmm<T><<<L.ntasks, DM_NT, smem_schur_dmm_bytes<T>(), ls>>>(fa, H.d_t4 + L.task_off, nb_small,
                                                                            nb_big);
        break;
    }
    if (prof)
      prof->mark(st,
                 (L.kind == L_CMOD || L.kind == L_MAKE_G || L.kind == L_MM_GEMM || L.kind == L_MM_ASM ||
                  L.kind == L_SPLIT_R || L.kind == L_SPLIT_C || L.kind == L_EXT_ADD || L.kind == L_FRONT_CB) ? 1
                 : (L.kind == L_DIAG_INV || L.kind == L_SCHUR_TC)             ? 4
                 : L.kind == L_GETF2                                           ? 2
                 : (L.kind == L_DEEP || L.kind == L_DEEP_MM || L.kind == L_MAKE_M) ? 3
                                                                               : 4,
                 L.ntasks, L.kind);
    if (ls == F.st3) {
      CK(cudaEventRecord(F.ev_cm[L.nb_slot & 1], ls));
      cm_pending[L.nb_slot & 1] = true;
    } else if (ls != st) {
      CK(cudaEventRecord(F.ev_join, ls));
      side_pending = true;
    }
  }
  if (side_pending) CK(cudaStreamWaitEvent(st, F.ev_join, 0));
  for (int q = 0; q < 2; ++q)
    if (cm_pending[q]) CK(cudaStreamWaitEvent(st, F.ev_cm[q], 0));
  if (F.set.drop_tol > 0.0 && H.ns > 0) k_drop_tol<T><<<H.ns, 256, 0, st>>>(fa, F.set.drop_tol);
  CK(cudaMemsetAsync(F.cnt3, 0, 3 * sizeof(unsigned long long), st));
  k_inertia<T><<<grid1(n), 256, 0, st>>>(n, (const T*)F.d, (const T*)F.dsub, F.kind, F.cnt3);
  CK(cudaGetLastError());
}

template <typename T>
void run_factor(rslab_fac_handle& F) {
  auto& H = *F.sym;
  KernelSetup<T>::configure();
  CK(cudaEventRecord(F.ev0, F.st));
  if (F.set.use_graph) {
    if (!F.fgraph) {
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(F.st, cudaStreamCaptureModeThreadLocal));
      try {
        enqueue_factor<T>(F);
      } catch (...) {
        cudaStreamEndCapture(F.st, &g);
        throw;
      }
      CK(cudaStreamEndCapture(F.st, &g));
      // per-node priorities: the panel chain's launches go ahead of the
      // overlapping Schur update when SMs free up
      CK(cudaGraphInstantiate(&F.fgraph, g, cudaGraphInstantiateFlagUseNodePriority));
      cudaGraphDestroy(g);
    }
    CK(cudaGraphLaunch(F.fgraph, F.st));
  } else {
    enqueue_factor<T>(F);
  }
  CK(cudaEventRecord(F.ev1, F.st));
  // status + inertia back to the host
  CK(cudaMemcpyAsync(F.h_status, F.status, 4 * sizeof(int), cudaMemcpyDeviceToHost, F.st));
  unsigned long long c3[3];
  CK(cudaMemcpyAsync(c3, F.cnt3, sizeof(c3), cudaMemcpyDeviceToHost, F.st));
  CK(cudaStreamSynchronize(F.st));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, F.ev0, F.ev1));
  F.factor_ms = ms;
  if (F.h_status[0] == 2) {
    F.last_status = 2;
    throw RslabError(Status::CudaError, "tensor-core pipeline wait timed out in supernode " +
                                            std::to_string(F.h_status[1]));
  }
  F.last_status = F.h_status[0];
  F.failing_sn = F.h_status[0] ? F.h_status[1] : -1;
  F.nperturbed = F.h_status[2];
  F.ipos = (long long)c3[0];
  F.ineg = (long long)c3[1];
  F.izero = (long long)c3[2];
  (void)H;
  if (F.last_status) throw RslabError(Status::NumericallyRankDeficient,
                                      "numerically rank deficient pivot in supernode " + std::to_string(F.failing_sn));
}

// Wave state: sticky status, abort word, one ticket counter per wavefront
// launch, forward and backward block flags.
size_t wave_state_ints(const rslab_sym_handle& H) {
  return (size_t)WV_STATE_CTR + H.nwave + 2 * (size_t)CH_GROUPS * H.nflags;
}

// After a synchronised solve: a timed-out wavefront wait (sticky status set
// by the kernels) is reported and the status cleared.
void wave_check(rslab_fac_handle& F) {
  if (!F.h_wstat || *F.h_wstat == 0) return;
  *F.h_wstat = 0;
  CK(cudaMemsetAsync(F.wstate, 0, sizeof(int), F.st));
  CK(cudaStreamSynchronize(F.st));
  throw RslabError(Status::CudaError, "triangular solve: a wavefront dependency wait timed out");
}

template <typename T>
void ensure_ws(rslab_fac_handle& F, int nrhs) {
  if (F.ws_nrhs >= nrhs) return;
  const size_t es = sizeof(T);
  const long long m = (long long)F.sym->n * nrhs;
  F.ws.clear();
  auto a = [&](size_t bytes) {
    void* p = nullptr;
    CK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
    F.ws.emplace_back(p);
    return p;
  };
  F.Yg = a(m * es);
  F.Ze = a(m * es);
  F.Xg = a(m * es);
  F.Ub = a((size_t)std::max(F.sym->urows, 1LL) * nrhs * es);
  F.Wb = a(m * es);
  F.Wp = a((size_t)std::max(F.sym->bwd_slots, 1) * 64 * nrhs * es);
  F.bdev = a(m * es);
  F.xdev = a(m * es);
  F.wstate = (int*)a(wave_state_ints(*F.sym) * sizeof(int));
  CK(cudaMemsetAsync(F.wstate, 0, wave_state_ints(*F.sym) * sizeof(int), F.st));
  if (!F.h_wstat) {
    CK(cudaMallocHost(&F.h_wstat, sizeof(int)));
    *F.h_wstat = 0;
  }
  F.ws_nrhs = nrhs;
  if (F.sgraph) {
    cudaGraphExecDestroy(F.sgraph);
    F.sgraph = nullptr;
    F.sgraph_nrhs = -1;
  }
}

template <typename T>
SolveArgs make_sargs(rslab_fac_handle& F, int ld, int c0, int nr) {
  auto& H = *F.sym;
  SolveArgs a;
  a.sn_first = H.d_sn_first;
  a.sn_ncol = H.d_sn_ncol;
  a.sn_nrow = H.d_sn_nrow;
  a.sn_poff = H.d_poff;
  a.sn_rsoff = H.d_rsoff;
  a.rs = H.d_rs;
  a.upd_ptr = H.d_upd_ptr;
  a.upd_k = H.d_upd_k;
  a.upd_p0 = H.d_upd_p0;
  a.upd_p1 = H.d_upd_p1;
  a.panel = F.panel;
  a.d = F.d;
  a.dsub = F.dsub;
  a.kind = F.kind;
  a.lperm = F.lperm;
  a.Yg = F.Yg;
  a.Ze = F.Ze;
  a.Xg = F.Xg;
  a.U = F.Ub;
  a.Wb = F.Wb;
  a.uoff = H.d_uoff;
  a.pull_ptr = H.d_pull_ptr;
  a.pull_src = H.d_pull_src;
  a.dots_red = H.d_dots_red;
  a.linv = F.linv;
  a.linv_off = H.d_linv_off;
  a.Wp = F.Wp;
  a.wstate = F.wstate;
  a.ld = ld;
  a.c0 = c0;
  a.nrhs = nr;
  return a;
}

// x = A^-1 b on device buffers (row-major n x nrhs) in the factor's field.
template <typename T>
void enqueue_solve(rslab_fac_handle& F, const T* b, T* x, int nrhs, Prof* prof = nullptr) {
  auto& H = *F.sym;
  const int n = H.n;
  cudaStream_t st = F.st;
  if (prof) prof->mark(st, -1);
  k_perm_in<T><<<grid1((long long)n * nrhs), 256, 0, st>>>(n, nrhs, H.d_perm, F.scale, b, (T*)F.Yg);
  if (prof) prof->mark(st, 0);
  for (int c0 = 0; c0 < nrhs; c0 += RHS_MAX) {
    const int nr = std::min(RHS_MAX, nrhs - c0);
    SolveArgs sa = make_sargs<T>(F, nrhs, c0, nr);
    CK(cudaMemsetAsync(F.wstate + 1, 0, (wave_state_ints(H) - 1) * sizeof(int), st));
    const int fwd_flags = WV_STATE_CTR + H.nwave, bwd_flags = fwd_flags + CH_GROUPS * H.nflags;
    for (const Launch& L : H.fwdplan) {
      switch (L.kind) {
        case L_FWD_CHAIN:
          launch_solve<T, true>(1, L.ntasks, nr, sa, H.d_st4 + L.task_off, L.nb_slot, fwd_flags, st, L.narrow != 0);
          break;
        case L_FWD_PUSH_RED:
          k_push_reduce<T><<<L.ntasks, WV_NT, 0, st>>>(sa, H.d_st4 + L.task_off);
          break;
        default:
          launch_solve<T, true>(0, L.ntasks, nr, sa, H.d_st4 + L.task_off, 0, 0, st);
      }
      if (prof) prof->mark(st, (L.kind == L_FWD_PUSH || L.kind == L_FWD_PUSH_RED) ? 2 : 1, L.ntasks, L.kind);
    }
    k_dsolve<T><<<grid1((long long)n * nr), 256, 0, st>>>(n, sa);
    if (prof) prof->mark(st, 3);
    for (const Launch& L : H.bwdplan) {
      switch (L.kind) {
        case L_BWD_OFF:
          launch_solve<T, false>(0, L.ntasks, nr, sa, H.d_st4 + L.task_off, 0, 0, st);
          break;
        default:  // L_BWD_CHAIN
          launch_solve<T, false>(1, L.ntasks, nr, sa, H.d_st4 + L.task_off, L.nb_slot, bwd_flags, st, L.narrow != 0);
      }
      if (prof)
        prof->mark(st, (L.kind == L_BWD_OFF || L.kind == L_BWD_OFF_RED || L.kind == L_BWD_GATHER) ? 4 : 5, L.ntasks,
                   L.kind);
    }
  }
  k_perm_out<T><<<grid1((long long)n * nrhs), 256, 0, st>>>(n, nrhs, H.d_perm, F.scale, (const T*)F.Xg, x);
  if (prof) prof->mark(st, 0);
  CK(cudaMemcpyAsync(F.h_wstat, F.wstate, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaGetLastError());
}

// Solve with graph capture keyed on nrhs; b, x are the workspace bdev/xdev.
template <typename T>
void solve_ws(rslab_fac_handle& F, int nrhs) {
  KernelSetup<T>::configure();
  if (F.set.use_graph) {
    if (!F.sgraph || F.sgraph_nrhs != nrhs) {
      if (F.sgraph) cudaGraphExecDestroy(F.sgraph);
      F.sgraph = nullptr;
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(F.st, cudaStreamCaptureModeThreadLocal));
      try {
        enqueue_solve<T>(F, (const T*)F.bdev, (T*)F.xdev, nrhs);
      } catch (...) {
        cudaStreamEndCapture(F.st, &g);
        throw;
      }
      CK(cudaStreamEndCapture(F.st, &g));
      CK(cudaGraphInstantiate(&F.sgraph, g, 0));
      cudaGraphDestroy(g);
      F.sgraph_nrhs = nrhs;
    }
    CK(cudaGraphLaunch(F.sgraph, F.st));
  } else {
    enqueue_solve<T>(F, (const T*)F.bdev, (T*)F.xdev, nrhs);
  }
}

template <typename T>
void do_solve(rslab_fac_handle& F, const void* b, void* x, int nrhs, bool on_device) {
  if (F.last_status) throw RslabError(Status::NumericallyRankDeficient, "factor is not valid");
  const size_t es = sizeof(T);
  const long long m = (long long)F.sym->n * nrhs;
  ensure_ws<T>(F, nrhs);
  CK(cudaMemcpyAsync(F.bdev, b, m * es, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, F.st));
  CK(cudaEventRecord(F.ev0, F.st));
  solve_ws<T>(F, nrhs);
  CK(cudaEventRecord(F.ev1, F.st));
  CK(cudaMemcpyAsync(x, F.xdev, m * es, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, F.st));
  CK(cudaStreamSynchronize(F.st));
  wave_check(F);
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, F.ev0, F.ev1));
  F.solve_ms = ms;
}

template <typename T>
void dispatch_field(int dtype, T&& fn) {
  switch (dtype) {
    case RSLAB_F64: fn(double{}); break;
    case RSLAB_C64: fn(c64{}); break;
    case RSLAB_F32: fn(float{}); break;
    case RSLAB_C32: fn(c32{}); break;
    default: throw RslabError(Status::InvalidInput, "unknown dtype");
  }
}

int fail(const RslabError& e) {
  g_last_error = e.what();
  return (int)e.status;
}

}  // namespace

// ---------------------------------------------------------------------------
// Mixed-precision refinement ladder (MixedLdltSolver::solve_to,
// src/numeric/mixed.rs:140-221): x0 = promote(F_lo^-1 demote(b)); plain IR
// with the FP64 residual against the original A while the normwise backward
// error exceeds the target (<= 8 steps, contraction 0.5), then FGMRES(30)
// (max 120) right-preconditioned by the low-precision factor, warm-started at
// the best iterate.  Column-wise for several right-hand sides.
// ---------------------------------------------------------------------------
namespace {

template <typename Hi>
struct MixedCtx {
  using Lo = typename Field<Hi>::Lo;
  rslab_fac_handle& F;
  int n, nrhs;
  cudaStream_t st;
  Hi *r = nullptr, *dx = nullptr, *ax = nullptr;
  unsigned long long* nb = nullptr;
  MixedCtx(rslab_fac_handle& f, int nr) : F(f), n(f.sym->n), nrhs(nr), st(f.st) {
    const size_t bytes = (size_t)n * nrhs * sizeof(Hi);
    r = (Hi*)F.arena.get(A_R, bytes);
    dx = (Hi*)F.arena.get(A_DX, bytes);
    ax = (Hi*)F.arena.get(A_AX, bytes);
    nb = (unsigned long long*)F.arena.get(A_NB, (size_t)std::max(nrhs, 3) * 64 * sizeof(unsigned long long));
  }
  // dx = promote(F_lo^-1 demote(r)) for an n x k block (k <= nrhs, ld = k).
  void precond(const Hi* rr, Hi* out, int k) {
    const long long m = (long long)n * k;
    if (F.dtype_hi < 0 || F.dtype == F.dtype_hi) {  // FP64 tier / plain factor: the matrix's own field
      ensure_ws<Hi>(F, k);
      CK(cudaMemcpyAsync(F.bdev, rr, m * sizeof(Hi), cudaMemcpyDeviceToDevice, st));
      solve_ws<Hi>(F, k);
      CK(cudaMemcpyAsync(out, F.xdev, m * sizeof(Hi), cudaMemcpyDeviceToDevice, st));
      return;
    }
    ensure_ws<Lo>(F, k);
    k_cast_down<Hi, Lo><<<grid1(m), 256, 0, st>>>(m, rr, (Lo*)F.bdev);
    solve_ws<Lo>(F, k);
    k_cast_up<Lo, Hi><<<grid1(m), 256, 0, st>>>(m, (const Lo*)F.xdev, out);
  }
  void residual(const Hi* x, const Hi* b, Hi* rr, int k) {
    auto& H = *F.sym;
    k_residual<Hi><<<grid1((long long)n * k), 256, 0, st>>>(n, k, H.d_sp_rp, H.d_sp_ci, H.d_sp_vmap,
                                                          op_values(), x, b, rr);
  }
  void spmv(const Hi* x, Hi* y, int k) {
    auto& H = *F.sym;
    k_spmv<Hi><<<grid1((long long)n * k), 256, 0, st>>>(n, k, H.d_sp_rp, H.d_sp_ci, H.d_sp_vmap,
                                                      op_values(), x, y);
  }
  // the FP64 operator: the original matrix of a refined handle, the input
  // values of a plain FP64 factor
  const Hi* op_values() const { return (const Hi*)(F.aval_hi ? F.aval_hi : F.aval); }
  // per-column inf norms of up to 3 vectors -> host
  void colmax(const Hi* v, int k, double* out) {
    CK(cudaMemsetAsync(nb, 0, k * sizeof(unsigned long long), st));
    dim3 g(std::min<unsigned>(grid1(n), 1024u), k);
    k_colmax<Hi><<<g, 256, 0, st>>>(n, k, v, nb);
    std::vector<unsigned long long> h(k);
    CK(cudaMemcpyAsync(h.data(), nb, k * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int c = 0; c < k; ++c) {
      double dv;
      std::memcpy(&dv, &h[c], 8);
      out[c] = dv;
    }
  }
};

}  // namespace

// FGMRES for one right-hand side column, all vectors on the device; the
// Hessenberg least-squares and Givens rotations run on the host
// (iterative.rs:822-1037).
template <typename Hi>
static int gmres_column(MixedCtx<Hi>& M, const Hi* b, Hi* x, double tol, int max_iter, int restart);

#include "engine_gmres.inc"

// LdltSolver::solve_refined (src/numeric/sparse_solver.rs:335-375) in the
// factor's field: x = A^-1 b, then for it = 0..max_iter: r = b - A x (stored
// values, full symmetric CSR), keep per column the iterate of smallest
// ||r||_inf, stop at it == max_iter or when every residual is exactly zero,
// else x += A^-1 r.
template <typename T>
static void refined_solve_impl(rslab_fac_handle& F, const void* bsrc, int nrhs, int max_iter, void* xdst,
                               bool on_device) {
  if (F.last_status) throw RslabError(Status::NumericallyRankDeficient, "factor is not valid");
  auto& H = *F.sym;
  const int n = H.n;
  const long long m = (long long)n * nrhs;
  const size_t es = sizeof(T);
  cudaStream_t st = F.st;
  KernelSetup<T>::configure();
  ensure_ws<T>(F, nrhs);
  T* bb = (T*)F.arena.get(A_B, m * es);
  T* xx = (T*)F.arena.get(A_X, m * es);
  T* best = (T*)F.arena.get(A_BEST, m * es);
  T* r = (T*)F.arena.get(A_R, m * es);
  unsigned char* mask = (unsigned char*)F.arena.get(A_MASK, 64 + nrhs);
  unsigned long long* nbits = (unsigned long long*)F.arena.get(A_NB, (size_t)std::max(nrhs, 3) * 64 * 8);
  CK(cudaMemcpyAsync(bb, bsrc, m * es, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  auto solve_into = [&](const T* rhs, T* out) {
    CK(cudaMemcpyAsync(F.bdev, rhs, m * es, cudaMemcpyDeviceToDevice, st));
    solve_ws<T>(F, nrhs);
    CK(cudaMemcpyAsync(out, F.xdev, m * es, cudaMemcpyDeviceToDevice, st));
  };
  solve_into(bb, xx);
  std::vector<double> best_res(nrhs, INFINITY), res(nrhs);
  std::vector<unsigned char> hmask(nrhs);
  std::vector<unsigned long long> hb(nrhs);
  for (int it = 0; it <= max_iter; ++it) {
    k_residual<T><<<grid1(m), 256, 0, st>>>(n, nrhs, H.d_sp_rp, H.d_sp_ci, H.d_sp_vmap, (const T*)F.aval, xx, bb, r);
    CK(cudaMemsetAsync(nbits, 0, nrhs * sizeof(unsigned long long), st));
    dim3 g(std::min<unsigned>(grid1(n), 1024u), nrhs);
    k_colmax<T><<<g, 256, 0, st>>>(n, nrhs, r, nbits);
    CK(cudaMemcpyAsync(hb.data(), nbits, nrhs * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    bool any = false, all_zero = true;
    for (int c = 0; c < nrhs; ++c) {
      std::memcpy(&res[c], &hb[c], 8);
      hmask[c] = res[c] < best_res[c];
      if (hmask[c]) {
        best_res[c] = res[c];
        any = true;
      }
      if (res[c] != 0.0) all_zero = false;
    }
    if (any) {
      CK(cudaMemcpyAsync(mask, hmask.data(), nrhs, cudaMemcpyHostToDevice, st));
      k_copy_cols<T><<<grid1(m), 256, 0, st>>>(m, nrhs, mask, xx, best);
    }
    if (all_zero || it == max_iter) break;
    solve_into(r, r);
    k_axpy1<T><<<grid1(m), 256, 0, st>>>(m, r, xx);
  }
  CK(cudaMemcpyAsync(xdst, best, m * es, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  wave_check(F);
}

namespace {

template <typename Hi>
static void gmres_block_entry(rslab_fac_handle& F, const void* b, int s, double tol, int max_iter, int restart,
                              const void* x0, void* x, bool on_device, int64_t* iters, double* final_res,
                              int* converged) {
  MixedCtx<Hi> M(F, std::min(s, BG_SMAX));
  const long long n = M.n;
  const size_t bytes = (size_t)n * s * sizeof(Hi);
  const cudaMemcpyKind kin = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  Hi* bd = (Hi*)F.arena.get(A_BG_IB, bytes);
  Hi* xd = (Hi*)F.arena.get(A_BG_IX, bytes);
  CK(cudaMemcpyAsync(bd, b, bytes, kin, M.st));
  if (x0)
    CK(cudaMemcpyAsync(xd, x0, bytes, kin, M.st));
  else
    CK(cudaMemsetAsync(xd, 0, bytes, M.st));
  const int gk = std::min(s, BG_SMAX);
  Hi* bk = (Hi*)F.arena.get(A_BG_B, (size_t)n * gk * sizeof(Hi));
  Hi* xk = (Hi*)F.arena.get(A_BG_X, (size_t)n * gk * sizeof(Hi));
  int* dcl = (int*)F.arena.get(A_BG_CL, BG_SMAX * sizeof(int));
  int64_t it = 0;
  bool conv = true;
  for (int g0 = 0; g0 < s; g0 += BG_SMAX) {
    const int k = std::min(BG_SMAX, s - g0);
    std::vector<int> cols(k);
    for (int a = 0; a < k; ++a) cols[a] = g0 + a;
    CK(cudaMemcpyAsync(dcl, cols.data(), k * sizeof(int), cudaMemcpyHostToDevice, M.st));
    k_bg_gather<Hi><<<grid1(n * k), 256, 0, M.st>>>(n, s, k, dcl, bd, bk);
    k_bg_gather<Hi><<<grid1(n * k), 256, 0, M.st>>>(n, s, k, dcl, xd, xk);
    const BlockGmresResult r = gmres_block<Hi>(M, bk, xk, k, tol, max_iter, restart);
    k_bg_scatter<Hi><<<grid1(n * k), 256, 0, M.st>>>(n, s, k, dcl, xk, xd);
    it = std::max<int64_t>(it, r.iters);
    conv = conv && r.converged;
    if (final_res)
      for (int a = 0; a < k; ++a) final_res[g0 + a] = r.final_res[a];
  }
  CK(cudaMemcpyAsync(x, xd, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, M.st));
  CK(cudaStreamSynchronize(M.st));
  wave_check(F);
  if (iters) *iters = it;
  if (converged) *converged = conv ? 1 : 0;
}

}  // namespace

namespace rslab {
// Sets the calling thread's last-error message (for entry points defined in
// other translation units of the library).
void set_last_error(const std::string& msg) { g_last_error = msg; }
// Matrix dimension of a factor handle (-1 for a null handle).
int64_t factor_dimension(const rslab_fac_handle* F) { return F && F->sym ? F->sym->n : -1; }
}  // namespace rslab

extern "C" {

const char* rslab_last_error(void) { return g_last_error.c_str(); }

int rslab_version(void) { return RSLAB_ABI_VERSION; }

void rslab_default_analyze_settings(rslab_analyze_settings* s) {
  s->ordering = RSLAB_ORDER_AMD;
  s->nemin = 16;
  s->relax = 1;
  s->relax_max_width = 256;
  s->relax_max_extra_rows = 64;
  s->hybrid_liu = 1;
  s->panel_nb = 64;
  s->given_perm = nullptr;
}

void rslab_default_factor_settings(rslab_factor_settings* s) {
  s->on_zero_pivot = RSLAB_PIVOT_FAIL;
  s->abs_floor = 0.0;
  s->scaling = RSLAB_SCALING_ONEPASS;
  s->use_graph = 1;
  s->stream = nullptr;
  s->schur_engine = RSLAB_SCHUR_AUTO;
  s->method = RSLAB_METHOD_LEFT_LOOKING;
  s->drop_tol = 0.0;
  s->overlap = 1;
}

int rslab_validate_lower_csc(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, int64_t nnz) {
  try {
    if (n < 0 || !col_ptr || (nnz > 0 && !row_idx)) throw RslabError(Status::InvalidInput, "bad CSC arrays");
    rslab::validate_lower_csc(n, col_ptr, row_idx, nnz);
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  }
}

}  // extern "C"

namespace {

void check_lower_input(int64_t n, const int64_t* col_ptr, const int64_t* row_idx) {
  if (n < 0 || !col_ptr || (n > 0 && !row_idx && col_ptr[n] > 0)) throw RslabError(Status::InvalidInput, "bad CSC");
  if (n >= (int64_t)1 << 31) throw RslabError(Status::InvalidInput, "n too large");
  rslab::validate_lower_csc(n, col_ptr, row_idx, col_ptr[n]);
}

rslab::AnalyzeOptions analyze_options(const rslab_analyze_settings& st) {
  rslab::AnalyzeOptions o;
  o.ordering = (rslab::Ordering)st.ordering;
  o.nemin = st.nemin;
  o.relax = st.relax != 0;
  o.relax_max_width = st.relax_max_width;
  o.relax_max_extra_rows = st.relax_max_extra_rows;
  o.hybrid_liu = st.hybrid_liu != 0;
  o.given_perm = st.given_perm;
  return o;
}

// A handle around a finished host analysis: the device plan is built here.
rslab_sym_handle* make_sym_handle(rslab::Symbolic&& S, const rslab_analyze_settings& st, int64_t n,
                                  const int64_t* col_ptr, const int64_t* row_idx) {
  auto H = std::make_unique<rslab_sym_handle>();
  H->settings = st;
  H->panel_nb = (int)std::min<int64_t>(std::max<int64_t>(st.panel_nb, 8), 128);  // panel kernels hold <= 128 columns
  H->S = std::move(S);
  H->seg_begin = {0, (long long)n};
  H->nnz_begin = {0, (long long)col_ptr[n]};
  build_plan(*H, col_ptr, row_idx);
  return H.release();
}

void fill_estimate(const rslab::MemoryEstimate& e, const rslab::Symbolic& S, rslab_memory_estimate_t* out) {
  out->value_bytes = e.value_bytes;
  out->factor_nnz = e.factor_nnz;
  out->factor_bytes = e.factor_bytes;
  out->panels_all_bytes = e.panels_all_bytes;
  out->panel_live_peak_bytes = e.panel_live_peak_bytes;
  out->transient_peak_bytes = e.transient_peak_bytes;
  out->factor_flops = e.factor_flops;
  out->critical_path_flops = e.critical_path_flops;
  out->max_tree_width = e.max_tree_width;
  out->symbolic_factor_nnz = rslab::symbolic_factor_nnz(S);
  out->mf_transient_peak_bytes = e.mf_transient_peak_bytes;
}

}  // namespace

extern "C" {

int rslab_analyze(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, const rslab_analyze_settings* settings,
                  rslab_sym_handle** out) {
  try {
    if (!out) throw RslabError(Status::InvalidInput, "null output handle");
    *out = nullptr;
    check_lower_input(n, col_ptr, row_idx);
    rslab_analyze_settings st;
    if (settings)
      st = *settings;
    else
      rslab_default_analyze_settings(&st);
    *out = make_sym_handle(rslab::analyze(n, col_ptr, row_idx, analyze_options(st)), st, n, col_ptr, row_idx);
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_symbolic_estimate(const rslab_sym_handle* h, int64_t value_bytes, rslab_memory_estimate_t* est) {
  if (!h || !est || value_bytes <= 0) return fail(RslabError(Status::InvalidInput, "bad estimate arguments"));
  fill_estimate(rslab::estimate_memory(h->S, value_bytes), h->S, est);
  return 0;
}

int rslab_analyze_tuned(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, int64_t value_bytes,
                        rslab_sym_handle** out, int32_t* ordering_used) {
  try {
    if (!out) throw RslabError(Status::InvalidInput, "null output handle");
    *out = nullptr;
    if (value_bytes <= 0) throw RslabError(Status::InvalidInput, "value_bytes must be positive");
    check_lower_input(n, col_ptr, row_idx);
    rslab_analyze_settings st;
    rslab_default_analyze_settings(&st);
    rslab_analyze_settings st_nd = st;
    st_nd.ordering = RSLAB_ORDER_METIS_ND;
    // The ND candidate's analysis runs on a second host thread while the
    // default analysis runs here (the bake-off reads both); it is discarded
    // when the default pattern is below the flop threshold.
    const bool try_nd = n >= RSLAB_ND_BAKEOFF_MIN_N;
    rslab::Symbolic S_nd;
    bool nd_ok = false;  // the ND analysis failed: keep the first pick
    std::thread nd_thread;
    if (try_nd)
      nd_thread = std::thread([&] {
        try {
          S_nd = rslab::analyze(n, col_ptr, row_idx, analyze_options(st_nd));
          nd_ok = true;
        } catch (...) {
          nd_ok = false;
        }
      });
    struct Joiner {
      std::thread& t;
      ~Joiner() {
        if (t.joinable()) t.join();
      }
    } joiner{nd_thread};
    rslab::Symbolic S = rslab::analyze(n, col_ptr, row_idx, analyze_options(st));
    if (nd_thread.joinable()) nd_thread.join();
    if (try_nd) {
      const rslab::MemoryEstimate est = rslab::estimate_memory(S, value_bytes);
      if (est.factor_flops >= (uint64_t)RSLAB_ND_BAKEOFF_MIN_FLOPS) {
        if (nd_ok) {
          const rslab::MemoryEstimate est_nd = rslab::estimate_memory(S_nd, value_bytes);
          const bool flops_win = (double)est_nd.factor_flops < (double)est.factor_flops * RSLAB_ND_BAKEOFF_ADOPT_RATIO;
          const bool fill_ok = rslab::symbolic_factor_nnz(S_nd) <= rslab::symbolic_factor_nnz(S);
          const bool mem_ok = est_nd.panel_live_peak_bytes <= est.panel_live_peak_bytes;
          if (flops_win && fill_ok && mem_ok) {
            S = std::move(S_nd);
            st = st_nd;
          }
        }
      }
    }
    if (ordering_used) *ordering_used = st.ordering;
    *out = make_sym_handle(std::move(S), st, n, col_ptr, row_idx);
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_analyze_batch(int64_t count, const int64_t* n, const int64_t* const* col_ptr,
                        const int64_t* const* row_idx, const rslab_analyze_settings* settings,
                        rslab_sym_handle** out) {
  try {
    if (!out || count <= 0 || !n || !col_ptr || !row_idx) throw RslabError(Status::InvalidInput, "bad batch arguments");
    *out = nullptr;
    rslab_analyze_settings st;
    if (settings)
      st = *settings;
    else
      rslab_default_analyze_settings(&st);
    if (st.ordering == RSLAB_ORDER_GIVEN) throw RslabError(Status::InvalidInput, "batch analysis takes no given permutation");
    rslab::AnalyzeOptions o;
    o.ordering = (rslab::Ordering)st.ordering;
    o.nemin = st.nemin;
    o.relax = st.relax != 0;
    o.relax_max_width = st.relax_max_width;
    o.relax_max_extra_rows = st.relax_max_extra_rows;
    o.hybrid_liu = st.hybrid_liu != 0;
    o.given_perm = nullptr;
    std::vector<rslab::Symbolic> parts((size_t)count);
    std::vector<long long> seg{0}, nz{0};
    for (int64_t i = 0; i < count; ++i) {
      if (n[i] < 0 || !col_ptr[i] || (n[i] > 0 && !row_idx[i] && col_ptr[i][n[i]] > 0))
        throw RslabError(Status::InvalidInput, "bad CSC of system " + std::to_string(i));
      rslab::validate_lower_csc(n[i], col_ptr[i], row_idx[i], col_ptr[i][n[i]]);
      seg.push_back(seg.back() + n[i]);
      nz.push_back(nz.back() + col_ptr[i][n[i]]);
    }
    // the systems' analyses are independent: host threads take systems in
    // turn; each result lands in its own slot, so the merge is unchanged
    {
      std::atomic<int64_t> next{0};
      std::vector<std::string> errs((size_t)count);
      const int nth = (int)std::max<int64_t>(1, std::min<int64_t>(count, std::thread::hardware_concurrency()));
      auto work = [&]() {
        for (int64_t i; (i = next.fetch_add(1)) < count;) {
          try {
            parts[i] = rslab::analyze(n[i], col_ptr[i], row_idx[i], o);
          } catch (const std::exception& e) {
            errs[i] = e.what();
          }
        }
      };
      std::vector<std::thread> pool;
      for (int t = 1; t < nth; ++t) pool.emplace_back(work);
      work();
      for (auto& t : pool) t.join();
      for (int64_t i = 0; i < count; ++i)
        if (!errs[i].empty()) throw RslabError(Status::InvalidInput, "system " + std::to_string(i) + ": " + errs[i]);
    }
    if (seg.back() >= (1LL << 31)) throw RslabError(Status::InvalidInput, "batch too large");
    // block-diagonal lower CSC of the whole batch (user order)
    std::vector<int64_t> cp{0}, ri;
    ri.reserve(nz.back());
    for (int64_t i = 0; i < count; ++i) {
      for (int64_t j = 0; j < n[i]; ++j) {
        for (int64_t k = col_ptr[i][j]; k < col_ptr[i][j + 1]; ++k) ri.push_back(row_idx[i][k] + seg[i]);
        cp.push_back((int64_t)ri.size());
      }
    }
    auto H = std::make_unique<rslab_sym_handle>();
    H->settings = st;
    H->panel_nb = (int)std::min<int64_t>(std::max<int64_t>(st.panel_nb, 8), 128);  // panel kernels hold <= 128 columns
    H->S = rslab::merge_independent(parts);
    H->seg_begin = seg;
    H->nnz_begin = nz;
    build_plan(*H, cp.data(), ri.data());
    *out = H.release();
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_batch_layout(const rslab_sym_handle* h, int64_t* count, int64_t* seg_begin, int64_t* nnz_begin) {
  if (!h || !count) return fail(RslabError(Status::InvalidInput, "null argument"));
  *count = (int64_t)h->seg_begin.size() - 1;
  if (seg_begin) std::copy(h->seg_begin.begin(), h->seg_begin.end(), seg_begin);
  if (nnz_begin) std::copy(h->nnz_begin.begin(), h->nnz_begin.end(), nnz_begin);
  return 0;
}

int rslab_mixed_batch_result(const rslab_fac_handle* F, int64_t cap, double* backward_error, int64_t* count) {
  if (!F || !count) return fail(RslabError(Status::InvalidInput, "null argument"));
  *count = (int64_t)F->last_be.size();
  for (int64_t i = 0; i < std::min<int64_t>(cap, *count); ++i) backward_error[i] = F->last_be[i];
  return 0;
}

void rslab_free_symbolic(rslab_sym_handle* h) { delete h; }

int rslab_symbolic_info(const rslab_sym_handle* h, rslab_symbolic_info_t* info) {
  if (!h || !info) return (int)Status::InvalidInput;
  info->n = h->n;
  info->nnz = h->nnz;
  info->nsuper = h->ns;
  info->nlevels = (int64_t)h->S.by_level.size();
  info->factor_nnz_sym = h->S.factor_nnz_sym;
  info->panel_elems = h->panel_elems;
  info->flops_model = h->flops_model;
  info->flops_proxy = h->flops_proxy;
  info->renumbered = h->S.renumbered;
  info->amd_ncmpa = h->S.amd.ncmpa;
  info->amd_ndense = h->S.amd.n_dense;
  info->amd_ndiv = h->S.amd.ndiv;
  info->amd_nms_ldl = h->S.amd.nms_ldl;
  info->amd_nms_lu = h->S.amd.nms_lu;
  info->n_factor_launches = (int64_t)h->fplan.size();
  info->n_solve_launches = (int64_t)(h->fwdplan.size() + h->bwdplan.size());
  info->tc_tiles = (int64_t)h->t4tc.size();
  info->tc_pairs = (int64_t)h->cpairs_tc.size();
  info->tc_chunks_complex = info->tc_chunks_real = 0;
  for (const int4& pq : h->cpairs_tc) {
    const int64_t nck = h->S.sn[pq.x].ncol;
    info->tc_chunks_complex += (nck + 15) / 16;
    info->tc_chunks_real += (nck + 31) / 32;
  }
  return 0;
}

// perm[n], sn_first/sn_ncol/sn_nrow/sn_level[nsuper], child_ptr[nsuper+1],
// child_idx[nsuper], col_counts[n], parent[n]; any pointer may be null.
int rslab_symbolic_export(const rslab_sym_handle* h, int64_t* perm, int64_t* sn_first, int64_t* sn_ncol,
                          int64_t* sn_nrow, int64_t* sn_level, int64_t* child_ptr, int64_t* child_idx,
                          int64_t* col_counts, int64_t* parent) {
  if (!h) return (int)Status::InvalidInput;
  const auto& S = h->S;
  if (perm) std::copy(S.perm.begin(), S.perm.end(), perm);
  if (col_counts) std::copy(S.col_counts.begin(), S.col_counts.end(), col_counts);
  if (parent) std::copy(S.parent.begin(), S.parent.end(), parent);
  int64_t cp = 0;
  for (int s = 0; s < h->ns; ++s) {
    if (sn_first) sn_first[s] = S.sn[s].first_col;
    if (sn_ncol) sn_ncol[s] = S.sn[s].ncol;
    if (sn_nrow) sn_nrow[s] = h->nrow[s];
    if (sn_level) sn_level[s] = S.level[s];
    if (child_ptr) child_ptr[s] = cp;
    for (int64_t c : S.sn[s].children) {
      if (child_idx) child_idx[cp] = c;
      ++cp;
    }
  }
  if (child_ptr) child_ptr[h->ns] = cp;
  return 0;
}

// Tensor maps of the split pools (cuTensorMapEncodeTiled through the runtime's
// driver entry point): for updater k, A hi / lo over m_k rows and B hi / lo
// over m_k (real) or 2 m_k (complex: B'_re rows, then B'_im rows) rows, each
// row kpad_k fp32 (a multiple of 32: 128-byte aligned rows); boxes of 32
// fp32 x 128 rows (A) and 32 x 16 (B), 128-byte swizzle, out-of-range rows
// read as zero.  The pools are this GPU's own memory.
static void setup_mm_pools(rslab_fac_handle& F) {
  auto& H = *F.sym;
  const bool cx = F.dtype == RSLAB_C32;
  const long long na = std::max(cx ? H.split_a_c : H.split_a_r, 32LL);
  const long long nb = std::max(cx ? H.split_b_c : H.split_b_r, 32LL);
  F.sp_ahi = F.al<float>(na);
  F.sp_alo = F.al<float>(na);
  F.sp_bhi = F.al<float>(nb);
  F.sp_blo = F.al<float>(nb);
  if (cx) {
    F.sp_as = F.al<float>(na);
    F.sp_bs = F.al<float>(nb);
  }
  F.wbuf = F.al<float>((size_t)2 * H.w_elems * (cx ? 2 : 1));
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess)
      throw RslabError(Status::CudaError, "cuTensorMapEncodeTiled is not available");
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  const int ns = H.ns;
  std::vector<CUtensorMap> maps((size_t)std::max(ns, 1) * MM_MAPS);
  std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
  for (int k = 0; k < ns; ++k) {
    const long long m = H.nrow[k] - H.S.sn[k].ncol;
    if (m <= 0) continue;
    const long long kp = cx ? H.kpad_c[k] : H.kpad_r[k];
    const long long oa = cx ? H.soff_a_c[k] : H.soff_a_r[k];
    const long long ob = cx ? H.soff_b_c[k] : H.soff_b_r[k];
    float* bases[MM_MAPS] = {F.sp_ahi + oa, F.sp_alo + oa, F.sp_bhi + ob, F.sp_blo + ob,
                             cx ? F.sp_as + oa : nullptr, cx ? F.sp_bs + ob : nullptr};
    for (int j = 0; j < (cx ? MM_MAPS : 4); ++j) {
      const bool a_side = j < 2 || j == 4;
      const cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)m};
      const cuuint64_t strides[1] = {(cuuint64_t)kp * 4};
      const cuuint32_t box[2] = {32, (cuuint32_t)(a_side ? MM_M : MM_BOX_B)};
      const cuuint32_t estr[2] = {1, 1};
      const CUresult r = encode(&maps[(size_t)k * MM_MAPS + j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, bases[j], dims,
                                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS)
        throw RslabError(Status::CudaError, "cuTensorMapEncodeTiled failed for supernode " + std::to_string(k));
    }
  }
  F.tmaps = reinterpret_cast<CUtensorMap*>(F.al<unsigned char>(maps.size() * sizeof(CUtensorMap)));
  CK(cudaMemcpyAsync(F.tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, F.st));
  CK(cudaStreamSynchronize(F.st));
}

// The matrix values into the handle: straight into the factor's input, or,
// for a refined handle, into the original (FP64) copy and from there demoted
// (or, for the FP64 tier, copied) into the factor's input.
static void load_values(rslab_fac_handle& F, const void* values, cudaMemcpyKind kd) {
  const long long nnz = F.sym->nnz;
  if (F.dtype_hi < 0) {
    CK(cudaMemcpyAsync(F.aval, values, nnz * elem_size(F.dtype), kd, F.st));
    return;
  }
  CK(cudaMemcpyAsync(F.aval_hi, values, nnz * elem_size(F.dtype_hi), kd, F.st));
  if (F.dtype == F.dtype_hi)
    CK(cudaMemcpyAsync(F.aval, F.aval_hi, nnz * elem_size(F.dtype), cudaMemcpyDeviceToDevice, F.st));
  else if (F.dtype_hi == RSLAB_F64)
    k_demote<double, float><<<grid1(nnz), 256, 0, F.st>>>(nnz, (const double*)F.aval_hi, (float*)F.aval);
  else
    k_demote<c64, c32><<<grid1(nnz), 256, 0, F.st>>>(nnz, (const c64*)F.aval_hi, (c32*)F.aval);
}

static int factor_impl(rslab_sym_handle* sym, int dtype, int dtype_hi, const void* values, int on_device,
                       const rslab_factor_settings* settings, rslab_fac_handle** out) {
  try {
    if (!sym || !out) throw RslabError(Status::InvalidInput, "null handle");
    *out = nullptr;
    auto F = std::make_unique<rslab_fac_handle>();
    F->sym = sym;
    F->dtype = dtype;
    F->dtype_hi = dtype_hi;
    if (settings)
      F->set = *settings;
    else
      rslab_default_factor_settings(&F->set);
    if (F->set.method != RSLAB_METHOD_LEFT_LOOKING && F->set.method != RSLAB_METHOD_MULTIFRONTAL)
      throw RslabError(Status::InvalidInput, "method must be RSLAB_METHOD_LEFT_LOOKING or _MULTIFRONTAL");
    if (F->set.schur_engine == RSLAB_SCHUR_AUTO)
      F->set.schur_engine = sym->flops_model >= RSLAB_SCHUR_AUTO_MIN_FLOPS ? RSLAB_SCHUR_TENSOR : RSLAB_SCHUR_FMA;
    if (F->set.schur_engine != RSLAB_SCHUR_TENSOR && F->set.schur_engine != RSLAB_SCHUR_FMA)
      throw RslabError(Status::InvalidInput, "schur_engine must be RSLAB_SCHUR_TENSOR, _FMA or _AUTO");
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    if (F->set.stream) {
      F->st = (cudaStream_t)F->set.stream;
    } else {
      // the panel chain (getf2, deep rows) runs here: highest priority
      CK(cudaStreamCreateWithPriority(&F->st, cudaStreamNonBlocking, prio_hi));
      F->own_stream = true;
    }
    CK(cudaStreamCreateWithPriority(&F->st2, cudaStreamNonBlocking, prio_lo));
    CK(cudaStreamCreateWithPriority(&F->st3, cudaStreamNonBlocking, prio_lo));
    for (cudaEvent_t& e : F->ev_cm) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaEventCreate(&F->ev0));
    CK(cudaEventCreate(&F->ev1));
    CK(cudaEventCreateWithFlags(&F->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&F->ev_join, cudaEventDisableTiming));
    sym->ensure_device(F->st);
    const size_t es = elem_size(dtype);
    const int n = sym->n;
    F->panel = F->al<unsigned char>(sym->panel_elems * es);
    F->d = F->al<unsigned char>(n * es);
    F->dsub = F->al<unsigned char>(n * es);
    F->kind = F->al<unsigned char>(n);
    F->lperm = F->al<int>(n);
    F->pivrec = F->al<int>(std::max(n, 1));
    F->pivot_reuse = F->al<int>(1);
    CK(cudaMemsetAsync(F->pivot_reuse, 0, sizeof(int), F->st));
    F->scale = F->al<double>(n);
    F->rowmax = F->al<unsigned long long>(n);
    F->status = F->al<int>(4);
    F->cnt3 = F->al<unsigned long long>(3);
    F->aval = F->al<unsigned char>(sym->nnz * es);
    CK(cudaMallocHost(&F->h_status, 4 * sizeof(int)));
    const long long nbm = sym->max_nb;
    F->scratch_stride = getf2_scratch_stride(nbm, (long long)es);
    F->scratch = F->al<unsigned char>((size_t)std::max(1, sym->max_getf2_tasks) * F->scratch_stride);
    F->linv = F->al<unsigned char>((size_t)std::max(sym->linv_elems, 1LL) * es);
    if (F->set.on_zero_pivot == RSLAB_PIVOT_FORCE_ACCEPT) {
      F->floor_dev = F->al<double>(1);
      F->amax_dev = F->al<unsigned long long>(1);
    }
    const bool single = dtype == RSLAB_F32 || dtype == RSLAB_C32;
    // descendant-update buffers: the left-looking method only (the
    // multifrontal one updates through its contribution blocks)
    const bool ll = F->set.method == RSLAB_METHOD_LEFT_LOOKING;
    if (ll && F->set.schur_engine == RSLAB_SCHUR_TENSOR) {
      if (single)
        setup_mm_pools(*F);
      else  // FP64 DMMA tiles: the level W buffers (the A / B operands are L21 and G)
        F->wbuf = F->al<float>((size_t)2 * sym->w_elems * es / 4);
    }
    if (ll && !(single && F->set.schur_engine == RSLAB_SCHUR_TENSOR))
      F->gpool = F->al<unsigned char>((size_t)std::max(sym->g_elems, 1LL) * es);
    if (F->set.method == RSLAB_METHOD_MULTIFRONTAL)
      F->cbpool = F->al<unsigned char>((size_t)std::max(sym->cb_elems, 1LL) * es);
    if (F->set.scaling != RSLAB_SCALING_ONEPASS) {
      std::vector<double> ones(n, 1.0);
      CK(cudaMemcpyAsync(F->scale, ones.data(), n * 8, cudaMemcpyHostToDevice, F->st));
      CK(cudaStreamSynchronize(F->st));
    }
    const cudaMemcpyKind kd = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (dtype_hi >= 0) F->aval_hi = F->al<unsigned char>(sym->nnz * elem_size(dtype_hi));
    load_values(*F, values, kd);
    rslab_fac_handle* raw = F.get();
    int rc = 0;
    try {
      dispatch_field(dtype, [&](auto z) { run_factor<decltype(z)>(*raw); });
    } catch (const RslabError& e) {
      if (e.status != Status::NumericallyRankDeficient) throw;
      rc = fail(e);
    }
    *out = F.release();
    return rc;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_factor(rslab_sym_handle* sym, int dtype, const void* values, int values_on_device,
                 const rslab_factor_settings* settings, rslab_fac_handle** out) {
  return factor_impl(sym, dtype, -1, values, values_on_device, settings, out);
}

int rslab_mixed_factor(rslab_sym_handle* sym, int dtype_hi, const void* values_hi, int values_on_device,
                       const rslab_factor_settings* settings, rslab_fac_handle** out) {
  int lo = dtype_hi == RSLAB_F64 ? RSLAB_F32 : dtype_hi == RSLAB_C64 ? RSLAB_C32 : -1;
  if (lo < 0) {
    g_last_error = "mixed factor needs an f64 or c64 matrix";
    return (int)Status::InvalidInput;
  }
  return factor_impl(sym, lo, dtype_hi, values_hi, values_on_device, settings, out);
}

int rslab_tier_factor(rslab_sym_handle* sym, int dtype_hi, int tier, const void* values_hi, int values_on_device,
                      const rslab_factor_settings* settings, rslab_fac_handle** out) {
  if (dtype_hi != RSLAB_F64 && dtype_hi != RSLAB_C64) {
    g_last_error = "tier factor needs an f64 or c64 matrix";
    return (int)Status::InvalidInput;
  }
  if (tier < RSLAB_TIER_FP64 || tier > RSLAB_TIER_TF32X3) {
    g_last_error = "tier must be RSLAB_TIER_FP64, RSLAB_TIER_FP32 or RSLAB_TIER_TF32X3";
    return (int)Status::InvalidInput;
  }
  rslab_factor_settings s;
  if (settings)
    s = *settings;
  else
    rslab_default_factor_settings(&s);
  if (tier == RSLAB_TIER_FP64)
    return factor_impl(sym, dtype_hi, dtype_hi, values_hi, values_on_device, &s, out);
  s.schur_engine = tier == RSLAB_TIER_FP32 ? RSLAB_SCHUR_FMA : RSLAB_SCHUR_TENSOR;
  const int lo = dtype_hi == RSLAB_F64 ? RSLAB_F32 : RSLAB_C32;
  return factor_impl(sym, lo, dtype_hi, values_hi, values_on_device, &s, out);
}

int rslab_refactor(rslab_fac_handle* F, const void* values, int values_on_device) {
  try {
    if (!F) throw RslabError(Status::InvalidInput, "null handle");
    auto& H = *F->sym;
    (void)H;
    load_values(*F, values, values_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice);
    dispatch_field(F->dtype, [&](auto z) { run_factor<decltype(z)>(*F); });
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_set_pivot_reuse(rslab_fac_handle* F, int on) {
  try {
    if (!F) throw RslabError(Status::InvalidInput, "null handle");
    const int v = on ? 1 : 0;
    CK(cudaMemcpyAsync(F->pivot_reuse, &v, sizeof(int), cudaMemcpyHostToDevice, F->st));
    CK(cudaStreamSynchronize(F->st));
    F->reuse_on = v != 0;
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  }
}

int rslab_solve_refined(rslab_fac_handle* F, const void* b, int64_t nrhs, int64_t max_iter, void* x,
                        int on_device) {
  try {
    if (!F || nrhs <= 0) throw RslabError(Status::DimensionMismatch, "nrhs must be positive");
    if (max_iter < 0) throw RslabError(Status::InvalidInput, "max_iter must be non-negative");
    dispatch_field(F->dtype, [&](auto z) {
      refined_solve_impl<decltype(z)>(*F, b, (int)nrhs, (int)max_iter, x, on_device != 0);
    });
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_solve(rslab_fac_handle* F, const void* b, int64_t nrhs, void* x, int on_device) {
  try {
    if (!F || nrhs <= 0) throw RslabError(Status::DimensionMismatch, "nrhs must be positive");
    dispatch_field(F->dtype, [&](auto z) { do_solve<decltype(z)>(*F, b, x, (int)nrhs, on_device != 0); });
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_mixed_solve(rslab_fac_handle* F, const void* b, int64_t nrhs, double target, void* x, int on_device,
                      rslab_mixed_info* info) {
  try {
    if (!F || F->dtype_hi < 0) throw RslabError(Status::InvalidInput, "not a mixed-precision factor");
    if (nrhs <= 0) throw RslabError(Status::DimensionMismatch, "nrhs must be positive");
    if (F->last_status) throw RslabError(Status::NumericallyRankDeficient, "factor is not valid");
    auto t0 = std::chrono::steady_clock::now();
    int rc = 0;
    if (F->dtype_hi == RSLAB_F64)
      rc = mixed_solve_impl<double>(*F, b, (int)nrhs, target, x, on_device != 0, info);
    else
      rc = mixed_solve_impl<c64>(*F, b, (int)nrhs, target, x, on_device != 0, info);
    F->solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_gmres_block(rslab_fac_handle* F, const void* b, int64_t s, double tol, int64_t max_iter, int64_t restart,
                      const void* x0, void* x, int on_device, int64_t* iters, double* final_res, int* converged) {
  try {
    if (!F || !b || !x) throw RslabError(Status::InvalidInput, "null handle or vector");
    if (s <= 0) throw RslabError(Status::DimensionMismatch, "s must be positive");
    if (!(tol > 0.0) || max_iter < 0 || restart < 1)
      throw RslabError(Status::InvalidInput, "tol > 0, max_iter >= 0 and restart >= 1 required");
    if (F->last_status) throw RslabError(Status::NumericallyRankDeficient, "factor is not valid");
    const int op = F->dtype_hi >= 0 ? F->dtype_hi : F->dtype;
    if (op == RSLAB_F64)
      gmres_block_entry<double>(*F, b, (int)s, tol, (int)max_iter, (int)restart, x0, x, on_device != 0, iters,
                                final_res, converged);
    else if (op == RSLAB_C64)
      gmres_block_entry<c64>(*F, b, (int)s, tol, (int)max_iter, (int)restart, x0, x, on_device != 0, iters,
                             final_res, converged);
    else
      throw RslabError(Status::InvalidInput,
                       "block GMRES needs an FP64 operator: a refined handle or an f64 / c64 factor");
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

int rslab_factor_info(const rslab_fac_handle* F, rslab_factor_info_t* info) {
  if (!F || !info) return (int)Status::InvalidInput;
  info->status = F->last_status;
  info->failing_supernode = F->failing_sn;
  info->inertia_pos = F->ipos;
  info->inertia_neg = F->ineg;
  info->inertia_zero = F->izero;
  info->n_perturbed = F->nperturbed;
  info->factor_ms = F->factor_ms;
  info->solve_ms = F->solve_ms;
  info->dtype = F->dtype;
  info->dtype_hi = F->dtype_hi;
  info->multiprocessors = 0;
  info->schur_engine = F->set.schur_engine;
  info->method = F->set.method;
  if (F->sym && F->sym->device >= 0)
    cudaDeviceGetAttribute(&info->multiprocessors, cudaDevAttrMultiProcessorCount, F->sym->device);
  return 0;
}

void* rslab_factor_stream(const rslab_fac_handle* F) { return F ? (void*)F->st : nullptr; }

// One eager solve of the workspace RHS (nrhs columns, filled with ones when
// fill_ones) with a CUDA event after every launch: device ms and launches per
// class ([0] permute in/out, [1] forward diagonal, [2] forward push,
// [3] D solve, [4] backward off-diagonal dots, [5] backward diagonal, [6] total).
int rslab_solve_profile(rslab_fac_handle* F, int64_t nrhs, double* kind_ms, int64_t* kind_launches) {
  try {
    if (!F || nrhs <= 0) throw RslabError(Status::InvalidInput, "bad arguments");
    Prof prof;
    dispatch_field(F->dtype, [&](auto z) {
      using T = decltype(z);
      KernelSetup<T>::configure();
      ensure_ws<T>(*F, (int)nrhs);
      CK(cudaMemsetAsync(F->bdev, 0, (size_t)F->sym->n * nrhs * sizeof(T), F->st));
      enqueue_solve<T>(*F, (const T*)F->bdev, (T*)F->xdev, (int)nrhs, &prof);
    });
    CK(cudaStreamSynchronize(F->st));
    prof.store(F->tr_kind, F->tr_grid, F->tr_ms);
    for (int k = 0; k < 7; ++k) {
      kind_ms[k] = 0;
      kind_launches[k] = 0;
    }
    for (size_t i = 1; i < prof.ev.size(); ++i) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, prof.ev[i - 1], prof.ev[i]));
      kind_ms[prof.kind[i]] += ms;
      kind_ms[6] += ms;
      kind_launches[prof.kind[i]] += 1;
      kind_launches[6] += 1;
    }
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  }
}

// One eager (non-graph) refactor of the current values with a CUDA event
// after every launch: device ms, launch count and algorithmic flops per
// kernel class ([0] equilibration+assembly, [1] cmod, [2] getf2,
// [3] deep-row replay, [4] panel Schur, [5] total).
int rslab_factor_profile(rslab_fac_handle* F, double* kind_ms, int64_t* kind_launches, double* kind_flops) {
  try {
    if (!F) throw RslabError(Status::InvalidInput, "null handle");
    auto& H = *F->sym;
    Prof prof;
    dispatch_field(F->dtype, [&](auto z) {
      using T = decltype(z);
      KernelSetup<T>::configure();
      prof.mark(F->st, -1);
      enqueue_factor<T>(*F, &prof);
    });
    CK(cudaStreamSynchronize(F->st));
    prof.store(F->tr_kind, F->tr_grid, F->tr_ms);
    for (int k = 0; k < 6; ++k) {
      kind_ms[k] = 0;
      kind_launches[k] = 0;
    }
    for (size_t i = 1; i < prof.ev.size(); ++i) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, prof.ev[i - 1], prof.ev[i]));
      int k = prof.kind[i];
      kind_ms[k] += ms;
      kind_ms[5] += ms;
      kind_launches[k] += 1;
      kind_launches[5] += 1;
    }
    const double cplx = (F->dtype == RSLAB_C64 || F->dtype == RSLAB_C32) ? 4.0 : 1.0;
    double tot = 0;
    for (int k = 0; k < 5; ++k) {
      kind_flops[k] = H.kind_flops[k] * cplx;
      tot += kind_flops[k];
    }
    kind_flops[5] = tot;
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  }
}

// Per-launch rows of the last rslab_factor_profile / rslab_solve_profile call:
// launch kind (LaunchKind code, -1 for permutes / D-solve / assembly), grid
// size and device ms; *count = rows available, at most `cap` written.
int rslab_profile_trace(const rslab_fac_handle* F, int64_t cap, int32_t* kind, int32_t* grid, float* ms,
                        int64_t* count) {
  if (!F || !count) return fail(RslabError(Status::InvalidInput, "null argument"));
  const int64_t m = (int64_t)F->tr_ms.size();
  *count = m;
  for (int64_t i = 0; i < std::min(m, cap); ++i) {
    if (kind) kind[i] = F->tr_kind[i];
    if (grid) grid[i] = F->tr_grid[i];
    if (ms) ms[i] = F->tr_ms[i];
  }
  return 0;
}

// Export in the reference LdltFactors layout (src/dense/ldlt_generic.rs:31-66):
// unit diagonal first, rows sorted, exact zeros dropped, the 2x2 coupling row
// skipped.  l_col_ptr[n+1]; call with null value arrays to get nnz first via
// rslab_factor_nnz.
static void export_counts(const rslab_fac_handle* F, std::vector<unsigned char>& panel, std::vector<int>& lperm,
                          std::vector<unsigned char>& kind) {
  auto& H = *F->sym;
  const size_t es = elem_size(F->dtype);
  panel.resize(H.panel_elems * es);
  lperm.resize(H.n);
  kind.resize(H.n);
  CK(cudaMemcpy(panel.data(), F->panel, panel.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(lperm.data(), F->lperm, H.n * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(kind.data(), F->kind, H.n, cudaMemcpyDeviceToHost));
}

static bool is_zero_value(const unsigned char* p, int dtype) {
  // exact zero of the field (both +0 and -0)
  switch (dtype) {
    case RSLAB_F64: {
      double v;
      std::memcpy(&v, p, 8);
      return v == 0.0;
    }
    case RSLAB_C64: {
      double v[2];
      std::memcpy(v, p, 16);
      return v[0] == 0.0 && v[1] == 0.0;
    }
    case RSLAB_F32: {
      float v;
      std::memcpy(&v, p, 4);
      return v == 0.0f;
    }
    default: {
      float v[2];
      std::memcpy(v, p, 8);
      return v[0] == 0.0f && v[1] == 0.0f;
    }
  }
}

static void write_one(unsigned char* dst, int dtype) {
  std::memset(dst, 0, elem_size(dtype));
  if (dtype == RSLAB_F64 || dtype == RSLAB_C64) {
    double one = 1.0;
    std::memcpy(dst, &one, 8);
  } else {
    float one = 1.0f;
    std::memcpy(dst, &one, 4);
  }
}

int rslab_export_factors(const rslab_fac_handle* F, int64_t* l_col_ptr, int64_t* l_row_idx, void* l_values, void* d_diag,
                         void* d_subdiag, uint8_t* two_by_two, int64_t* perm, double* scale, int64_t* nnz_out) {
  try {
    if (!F) throw RslabError(Status::InvalidInput, "null handle");
    auto& H = *F->sym;
    const auto& S = H.S;
    const size_t es = elem_size(F->dtype);
    std::vector<unsigned char> panel, kind;
    std::vector<int> lperm;
    export_counts(F, panel, lperm, kind);
    const int n = H.n;
    std::vector<int64_t> e_of_g(n);
    for (int s = 0; s < H.ns; ++s) {
      const int64_t f0 = S.sn[s].first_col;
      for (int64_t p = 0; p < S.sn[s].ncol; ++p) e_of_g[S.rs[S.rs_ptr[s] + lperm[f0 + p]]] = f0 + p;
    }
    int64_t nnz = 0;
    if (l_col_ptr) l_col_ptr[0] = 0;
    std::vector<std::pair<int64_t, int64_t>> col;  // (row e, panel element index)
    for (int s = 0; s < H.ns; ++s) {
      const int64_t f0 = S.sn[s].first_col, nc = S.sn[s].ncol, nr = H.nrow[s];
      const int64_t* rs = S.rs.data() + S.rs_ptr[s];
      for (int64_t p = 0; p < nc; ++p) {
        col.clear();
        col.push_back({f0 + p, -1});
        int64_t i0 = kind[f0 + p] == 1 ? p + 2 : p + 1;
        for (int64_t i = i0; i < nr; ++i) {
          int64_t idx = H.poff[s] + i + p * nr;
          if (is_zero_value(&panel[idx * es], F->dtype)) continue;
          int64_t g = i < nc ? rs[lperm[f0 + i]] : rs[i];
          col.push_back({e_of_g[g], idx});
        }
        std::sort(col.begin(), col.end());
        for (auto& x : col) {
          if (l_row_idx) l_row_idx[nnz] = x.first;
          if (l_values) {
            unsigned char* dst = (unsigned char*)l_values + nnz * es;
            if (x.second < 0) {
              write_one(dst, F->dtype);
            } else {
              std::memcpy(dst, &panel[x.second * es], es);
            }
          }
          ++nnz;
        }
        if (l_col_ptr) l_col_ptr[f0 + p + 1] = nnz;
      }
    }
    if (nnz_out) *nnz_out = nnz;
    if (d_diag) CK(cudaMemcpy(d_diag, F->d, n * es, cudaMemcpyDeviceToHost));
    if (d_subdiag) CK(cudaMemcpy(d_subdiag, F->dsub, n * es, cudaMemcpyDeviceToHost));
    if (two_by_two)
      for (int e = 0; e < n; ++e) two_by_two[e] = kind[e] == 1;
    if (perm)
      for (int s = 0; s < H.ns; ++s) {
        const int64_t f0 = S.sn[s].first_col;
        for (int64_t p = 0; p < S.sn[s].ncol; ++p) perm[f0 + p] = S.perm[S.rs[S.rs_ptr[s] + lperm[f0 + p]]];
      }
    if (scale) CK(cudaMemcpy(scale, F->scale, n * 8, cudaMemcpyDeviceToHost));
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}

void rslab_free_factor(rslab_fac_handle* F) { delete F; }

int rslab_device_count(int* count) {
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    g_last_error = cudaGetErrorString(e);
    return (int)Status::CudaError;
  }
  return 0;
}

// m successive unit draws of the xorshift64* generator of the synthetic
// workloads from internal state `state` (Rng::unit, src/matgen/mod.rs:62-81);
// returns the advanced state.
uint64_t rslab_rng_units(uint64_t state, int64_t m, double* out) {
  uint64_t x = state;
  for (int64_t i = 0; i < m; ++i) {
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    out[i] = (double)((x * 0x2545F4914F6CDD1Dull) >> 11) / 9007199254740992.0;
  }
  return x;
}

// AMD ordering of a full symmetric pattern, for golden-vector checks.
int rslab_amd_order(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, int64_t* perm, double* stats7) {
  try {
    if (n > 0 && !perm) throw RslabError(Status::InvalidInput, "null perm");
    const rslab::CscPattern p = rslab::checked_full_pattern(n, col_ptr, row_idx);
    rslab::AmdStats st;
    std::vector<int64_t> pr = rslab::amd_order(p, &st);
    std::copy(pr.begin(), pr.end(), perm);
    if (stats7) {
      stats7[0] = st.ncmpa;
      stats7[1] = st.n_dense;
      stats7[2] = st.ndiv;
      stats7[3] = st.nms_ldl;
      stats7[4] = st.nms_lu;
      stats7[5] = st.n_mass_elim;
      stats7[6] = st.n_supervar_merge;
    }
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  }
}

int rslab_metis_order(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, uint64_t seed, int dense_quotient,
                      int64_t dense_threshold, int64_t* perm) {
  try {
    if (n > 0 && !perm) throw RslabError(Status::InvalidInput, "null perm");
    const rslab::CscPattern p = rslab::checked_full_pattern(n, col_ptr, row_idx);
    std::vector<int64_t> pr = rslab::metis_nd_order(p, seed, dense_quotient != 0, dense_threshold);
    std::copy(pr.begin(), pr.end(), perm);
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free dense panel factor.
//
// Some callers cannot allocate device memory while they factor: a solver
// embedded in another library's memory pool, a process whose allocator is
// capped or frozen after start-up, or a real-time loop that must not pay
// cudaMalloc latency or risk an out-of-memory failure mid-run.  For them
// rslab_panel_factor_noalloc runs the blocked Bunch-Kaufman panel kernels
// (getf2, deep-row replay, in-panel Schur) on one caller-owned dense panel
// with every piece of scratch (the per-block multiplier snapshot, swap log,
// the panel's structure and the launch task lists) placed in the file-scope
// array below instead of memory obtained from an allocator.  The structure
// and the task lists are written into that array by a small kernel, so no
// host buffer has to outlive the call.  The array is 1 MiB and, like every
// __device__ variable, is held on each GPU that loads this library until the
// process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t NOALLOC_MAX_NROW = 4096;
constexpr int64_t NOALLOC_MAX_NCOL = 1024;
constexpr size_t NOALLOC_BYTES = size_t(1) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Device address of g_noalloc_scratch on the current device, looked up once
// per device.  In host code the symbol itself is only a host-side stand-in,
// never a device address, so kernels always receive this looked-up pointer.
unsigned char* noalloc_scratch_on_current_device() {
  static std::mutex mu;
  static unsigned char* addr[256] = {};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) throw RslabError(Status::CudaError, "device ordinal out of range");
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    addr[dev] = static_cast<unsigned char*>(p);
  }
  return addr[dev];
}

struct NoallocStruct {  // the one-supernode structure, at offset 0 of the scratch
  int sn_first, sn_ncol, sn_nrow, pad;
  long long sn_poff, sn_rsoff;
};

// The block sequence of one panel, in launch order: for every column block
// its getf2 task, then (unless getf2 replays the deep rows itself) the
// deep-row chunks, then the in-panel Schur tiles.  noalloc_count walks it on
// the host for the launch segments; k_noalloc_plan writes the same tasks on
// the device.
struct NoallocSeg {
  int kind, off, cnt;
};

__host__ __device__ inline int noalloc_schur_tiles(int mt, int cw) {
  int c = 0;
  for (int c0 = 0; c0 < cw && c0 < mt; c0 += TILE) c += (mt - c0 + TILE - 1) / TILE;
  return c;
}

int noalloc_count(int nrow, int ncol, int nb, std::vector<NoallocSeg>& segs) {
  int t = 0;
  for (int kb = 0; kb < ncol; kb += nb) {
    const int ke = std::min(kb + nb, ncol);
    const bool fuse = (nrow - ke) <= FUSE_DEEP_ROWS;
    segs.push_back({L_GETF2, t, 1});
    t += 1;
    if (!fuse) {
      const int cnt = (nrow - ke + DEEP_R - 1) / DEEP_R;
      segs.push_back({L_DEEP, t, cnt});
      t += cnt;
    }
    const int cnt = noalloc_schur_tiles(nrow - ke, ncol - ke);
    if (cnt) segs.push_back({L_SCHUR, t, cnt});
    t += cnt;
  }
  return t;
}

// One CTA: the blocks run in order (every thread keeps the same running
// offset), the tasks of a block are written by all threads.
__global__ void k_noalloc_plan(NoallocStruct* ns, int4* tasks, int nrow, int ncol, int nb) {
  if (threadIdx.x == 0) {
    ns->sn_first = 0;
    ns->sn_ncol = ncol;
    ns->sn_nrow = nrow;
    ns->pad = 0;
    ns->sn_poff = 0;
    ns->sn_rsoff = 0;
  }
  int t = 0;
  for (int kb = 0; kb < ncol; kb += nb) {
    const int ke = min(kb + nb, ncol);
    const bool fuse = (nrow - ke) <= FUSE_DEEP_ROWS;
    if (threadIdx.x == 0) tasks[t] = make_int4(0, kb, 0, fuse ? 1 : 0);
    t += 1;
    if (!fuse) {
      const int cnt = (nrow - ke + DEEP_R - 1) / DEEP_R;
      for (int i = threadIdx.x; i < cnt; i += blockDim.x) tasks[t + i] = make_int4(0, kb, 0, ke + i * DEEP_R);
      t += cnt;
    }
    const int mt = nrow - ke, cw = ncol - ke;
    for (int c0 = 0; c0 < cw && c0 < mt; c0 += TILE) {
      const int cnt = (mt - c0 + TILE - 1) / TILE;
      for (int i = threadIdx.x; i < cnt; i += blockDim.x) tasks[t + i] = make_int4(0, kb, c0 + i * TILE, c0);
      t += cnt;
    }
  }
}

// The kernels' shared-memory limits are raised once per device.
template <typename T>
void noalloc_attrs() {
  static std::mutex mu;
  static bool done[256] = {};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if (done[dev]) return;
  const size_t es = sizeof(T);
  CK(cudaFuncSetAttribute(k_getf2<T, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_getf2(es, 128)));
  CK(cudaFuncSetAttribute(k_deep<T, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_deep(es, 128)));
  CK(cudaFuncSetAttribute(k_schur<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_schur(es)));
  done[dev] = true;
}

template <typename T>
void noalloc_panel(unsigned char* base, T* panel, int nrow, int ncol, int panel_nb, T* d, T* dsub,
                   unsigned char* kind, int* lperm, int* status, cudaStream_t st) {
  const size_t es = sizeof(T);
  const int nb_small = panel_nb, nb_big = std::max(panel_nb, 128);
  const int nb = ncol >= 512 ? nb_big : nb_small;
  std::vector<NoallocSeg> segs;
  const int ntasks = noalloc_count(nrow, ncol, nb, segs);
  const size_t snap_bytes = ((size_t)nb_big * nb_big * es + 3 * nb_big * 4 + 255) / 256 * 256;
  const size_t off_snap = 256, off_tasks = off_snap + snap_bytes;
  const size_t need = off_tasks + (size_t)ntasks * sizeof(int4);
  if (need > NOALLOC_BYTES)
    throw RslabError(Status::InvalidInput, "panel needs " + std::to_string(need) +
                                               " bytes of scratch, more than the allocation-free limit of " +
                                               std::to_string(NOALLOC_BYTES));
  noalloc_attrs<T>();
  k_noalloc_plan<<<1, 256, 0, st>>>(reinterpret_cast<NoallocStruct*>(base),
                                    reinterpret_cast<int4*>(base + off_tasks), nrow, ncol, nb);
  CK(cudaMemsetAsync(status, 0, 4 * sizeof(int), st));
  const NoallocStruct* dn = reinterpret_cast<const NoallocStruct*>(base);
  FactorArgs fa{};
  fa.sn_first = &dn->sn_first;
  fa.sn_ncol = &dn->sn_ncol;
  fa.sn_nrow = &dn->sn_nrow;
  fa.sn_poff = &dn->sn_poff;
  fa.sn_rsoff = &dn->sn_rsoff;
  fa.panel = panel;
  fa.d = d;
  fa.dsub = dsub;
  fa.kind = kind;
  fa.lperm = lperm;
  fa.scratch = base + off_snap;
  fa.scratch_stride = (long long)snap_bytes;
  fa.status = status;
  fa.perturb_floor = -1.0;
  const int4* dt = reinterpret_cast<const int4*>(base + off_tasks);
  for (const NoallocSeg& g : segs) {
    if (g.kind == L_GETF2)
      k_getf2<T, 256><<<g.cnt, 256, smem_getf2(es, nb), st>>>(fa, dt + g.off, nb_small, nb_big);
    else if (g.kind == L_DEEP)
      k_deep<T, 256><<<g.cnt, 256, smem_deep(es, nb), st>>>(fa, dt + g.off, nb_small, nb_big);
    else
      k_schur<T><<<g.cnt, TPB, smem_schur(es), st>>>(fa, dt + g.off, nb_small, nb_big);
  }
  CK(cudaGetLastError());
}

}  // namespace

extern "C" int rslab_panel_factor_noalloc(int dtype, void* panel, int64_t nrow, int64_t ncol, int64_t panel_nb,
                                          void* d, void* dsub, uint8_t* kind, int32_t* lperm, int32_t* status,
                                          void* stream) {
  try {
    if (!panel || !d || !dsub || !kind || !lperm || !status)
      throw RslabError(Status::InvalidInput, "null device pointer");
    if (ncol <= 0 || nrow < ncol) throw RslabError(Status::InvalidInput, "need 0 < ncol <= nrow");
    if (nrow > NOALLOC_MAX_NROW || ncol > NOALLOC_MAX_NCOL)
      throw RslabError(Status::InvalidInput, "panel " + std::to_string(nrow) + " x " + std::to_string(ncol) +
                                                 " exceeds the allocation-free maximum of " +
                                                 std::to_string(NOALLOC_MAX_NROW) + " x " +
                                                 std::to_string(NOALLOC_MAX_NCOL));
    if (panel_nb < 8 || panel_nb > 64) throw RslabError(Status::InvalidInput, "panel_nb must lie in [8, 64]");
    unsigned char* base = noalloc_scratch_on_current_device();
    cudaStream_t st = (cudaStream_t)stream;
    dispatch_field(dtype, [&](auto z) {
      using T = decltype(z);
      noalloc_panel<T>(base, (T*)panel, (int)nrow, (int)ncol, (int)panel_nb, (T*)d, (T*)dsub, kind, lperm,
                       status, st);
    });
    return 0;
  } catch (const RslabError& e) {
    return fail(e);
  } catch (const std::exception& e) {
    return fail(RslabError(Status::InvalidInput, e.what()));
  }
}
