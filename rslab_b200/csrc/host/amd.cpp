// Approximate Minimum Degree ordering on the quotient graph.
//
// Restates the reference AMD (crates/rslab-ordering-core/src/quotient_graph/
// {workspace,algo}.rs driven by crates/rslab-amd/src/lib.rs:amd_order): the
// PE/IW/LEN/NV/ELEN quotient graph with approximate external degrees,
// aggressive element absorption, mass elimination, hash-bucket supervariable
// detection, inline garbage collection and the big-child-last assembly-tree
// postorder.  The reference pins its output byte-for-byte to SuiteSparse AMD,
// so every tie-break (LIFO degree lists, hash modulus, child order) matters and
// is kept exactly; only the code is ours.  All quotient-graph arrays are int32
// as in the reference so the generation-counter overflow guard behaves alike.
#include "host.hpp"

#include <cmath>
#include <cstring>
#include <stdexcept>

namespace rslab {
namespace {

constexpr int32_t NONE = -1;
inline int32_t flip(int32_t x) { return -2 - x; }

// Reset the mark generation when it would overflow (workspace.rs:49-60).
inline int32_t clear_flag(int32_t wflg, int32_t wbig, std::vector<int32_t>& w) {
  if (wflg < 2 || wflg >= wbig) {
    for (auto& x : w)
      if (x != 0) x = 1;
    return 2;
  }
  return wflg;
}

struct QGraph {
  int64_t n = 0;
  size_t iwlen = 0;
  size_t pfree = 0;
  std::vector<int32_t> iw, pe, len, nv, elen, degree, w, head, next, last;
  int32_t wflg = 0, wbig = 0, lemax = 0;
  size_t mindeg = 0;
  uint32_t ncmpa = 0, n_mass_elim = 0, n_supervar_merge = 0;
  size_t nel = 0;
  int32_t ndense = 0;
};

// Workspace construction: ingest the full symmetric pattern (diagonal
// dropped), classify zero-degree / dense / live variables
// (workspace.rs:148-270).
void qg_init(QGraph& g, int64_t n, const int64_t* colptr, const int64_t* rowidx,
             double dense_alpha) {
  if (n >= INT32_MAX) throw RslabError(Status::InvalidInput, "AMD: n too large for int32 indexing");
  g.n = n;
  g.len.assign(n, 0);
  size_t nzaat = 0;
  for (int64_t j = 0; j < n; ++j) {
    size_t cnt = 0;
    for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p)
      if (rowidx[p] != j) ++cnt;
    g.len[j] = (int32_t)cnt;
    nzaat += cnt;
  }
  g.iwlen = nzaat + nzaat / 5 + (size_t)n;
  if (g.iwlen > (size_t)INT32_MAX) throw RslabError(Status::InvalidInput, "AMD: pattern too large");
  g.iw.assign(g.iwlen, 0);
  g.pe.assign(n, 0);
  size_t pfree = 0;
  for (int64_t j = 0; j < n; ++j) {
    g.pe[j] = (int32_t)pfree;
    for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p)
      if (rowidx[p] != j) g.iw[pfree++] = (int32_t)rowidx[p];
  }
  g.pfree = pfree;
  size_t dense;
  if (dense_alpha < 0.0)
    dense = n >= 2 ? (size_t)(n - 2) : 0;
  else
    dense = (size_t)(dense_alpha * std::sqrt((double)n));
  if (dense < 16) dense = 16;
  if (dense > (size_t)n) dense = (size_t)n;

  g.nv.assign(n, 1);
  g.elen.assign(n, 0);
  g.w.assign(n, 1);
  g.degree = g.len;
  g.head.assign(n, NONE);
  g.next.assign(n, NONE);
  g.last.assign(n, NONE);
  g.wbig = INT32_MAX - (int32_t)n;
  g.wflg = 0;
  for (int64_t i = 0; i < n; ++i) {
    size_t deg = (size_t)g.degree[i];
    if (deg == 0) {
      g.elen[i] = flip(1);
      g.nel++;
      g.pe[i] = NONE;
      g.w[i] = 0;
    } else if (deg > dense) {
      g.ndense++;
      g.nv[i] = 0;
      g.elen[i] = NONE;
      g.pe[i] = NONE;
      g.nel++;
    } else {
      int32_t inext = g.head[deg];
      if (inext != NONE) g.last[inext] = (int32_t)i;
      g.next[i] = inext;
      g.head[deg] = (int32_t)i;
    }
  }
}

// Lowest non-empty degree bucket from mindeg upward; LIFO unlink
// (algo.rs:59-84).
int64_t qg_select_pivot(QGraph& g) {
  size_t deg = g.mindeg;
  int32_t me = NONE;
  while (deg < (size_t)g.n) {
    if (g.head[deg] != NONE) {
      me = g.head[deg];
      break;
    }
    ++deg;
  }
  if (me == NONE) return -1;
  g.mindeg = deg;
  int32_t inext = g.next[me];
  if (inext != NONE) g.last[inext] = NONE;
  g.head[deg] = inext;
  return me;
}

inline void unlink_degree(QGraph& g, int32_t i) {
  int32_t ilast = g.last[i], inext = g.next[i];
  if (inext != NONE) g.last[inext] = ilast;
  if (ilast != NONE)
    g.next[ilast] = inext;
  else
    g.head[g.degree[i]] = inext;
}

struct NewElement {
  size_t pme1, pme2_excl;
  int32_t nvpiv;
  size_t degme;
};

// Form the new element `me` (algo.rs:115-314): in place when `me` holds no
// elements, otherwise out of place at pfree with standard absorption of every
// element in me's list, compacting iw when it runs full.
NewElement qg_create_element(QGraph& g, int32_t me) {
  int32_t elenme = g.elen[me];
  int32_t nvpiv = g.nv[me];
  g.nel += (size_t)nvpiv;
  g.nv[me] = -nvpiv;
  size_t degme = 0;
  size_t pme1;
  int64_t pme2;
  if (elenme == 0) {
    pme1 = (size_t)g.pe[me];
    size_t list_end = pme1 + (size_t)g.len[me];
    int64_t pme2s = (int64_t)pme1 - 1;
    for (size_t p = pme1; p < list_end; ++p) {
      int32_t i = g.iw[p];
      int32_t nvi = g.nv[i];
      if (nvi > 0) {
        degme += (size_t)nvi;
        g.nv[i] = -nvi;
        g.iw[++pme2s] = i;
        unlink_degree(g, i);
      }
    }
    pme2 = pme2s;
  } else {
    size_t p = (size_t)g.pe[me];
    size_t pme1_rw = g.pfree;
    size_t slenme = (size_t)(g.len[me] - elenme);
    size_t elenme_u = (size_t)elenme;
    for (size_t knt1 = 1; knt1 <= elenme_u + 1; ++knt1) {
      int32_t e;
      size_t pj, ln;
      if (knt1 > elenme_u) {
        e = me;
        pj = p;
        ln = slenme;
      } else {
        e = g.iw[p++];
        pj = (size_t)g.pe[e];
        ln = (size_t)g.len[e];
      }
      for (size_t knt2 = 1; knt2 <= ln; ++knt2) {
        int32_t i = g.iw[pj++];
        int32_t nvi = g.nv[i];
        if (nvi <= 0) continue;
        if (g.pfree >= g.iwlen) {
          // Compaction: save cursors, tag list heads, slide every live list
          // down, then move the partial new element after them
          // (algo.rs:190-262).
          g.pe[me] = (int32_t)p;
          g.len[me] -= (int32_t)knt1;
          if (g.len[me] == 0) g.pe[me] = NONE;
          g.pe[e] = (int32_t)pj;
          g.len[e] = (int32_t)(ln - knt2);
          if (g.len[e] == 0) g.pe[e] = NONE;
          g.ncmpa++;
          for (int64_t j = 0; j < g.n; ++j) {
            int32_t pn = g.pe[j];
            if (pn >= 0) {
              g.pe[j] = g.iw[pn];
              g.iw[pn] = flip((int32_t)j);
            }
          }
          size_t psrc = 0, pdst = 0, pend = pme1_rw;
          while (psrc < pend) {
            int32_t jm = flip(g.iw[psrc]);
            ++psrc;
            if (jm >= 0) {
              g.iw[pdst] = g.pe[jm];
              g.pe[jm] = (int32_t)pdst;
              ++pdst;
              size_t lenj = (size_t)g.len[jm];
              if (lenj > 0) {
                std::memmove(&g.iw[pdst], &g.iw[psrc], (lenj - 1) * sizeof(int32_t));
                psrc += lenj - 1;
                pdst += lenj - 1;
              }
            }
          }
          size_t p1 = pdst;
          std::memmove(&g.iw[pdst], &g.iw[pme1_rw], (g.pfree - pme1_rw) * sizeof(int32_t));
          pdst += g.pfree - pme1_rw;
          pme1_rw = p1;
          g.pfree = pdst;
          pj = (size_t)g.pe[e];
          p = (size_t)g.pe[me];
        }
        degme += (size_t)nvi;
        g.nv[i] = -nvi;
        g.iw[g.pfree++] = i;
        unlink_degree(g, i);
      }
      if (e != me) {
        g.pe[e] = flip(me);
        g.w[e] = 0;
      }
    }
    pme1 = pme1_rw;
    pme2 = (int64_t)g.pfree - 1;
  }
  g.degree[me] = (int32_t)degme;
  g.pe[me] = (int32_t)pme1;
  g.len[me] = (int32_t)(pme2 - (int64_t)pme1 + 1);
  g.elen[me] = flip(nvpiv + (int32_t)degme);
  g.wflg = clear_flag(g.wflg, g.wbig, g.w);
  size_t pme2_excl = pme2 < (int64_t)pme1 ? pme1 : (size_t)(pme2 + 1);
  return {pme1, pme2_excl, nvpiv, degme};
}

// Degree update, absorption, mass elimination, supervariable detection and
// degree-list re-insertion for one pivot step (algo.rs:332-629).
void qg_finalize_step(QGraph& g, int32_t me, const NewElement& ne, int32_t elenme,
                      bool aggressive, AmdStats& st) {
  size_t degme = ne.degme;
  int32_t nvpiv = ne.nvpiv;
  const size_t pme1 = ne.pme1, pme2e = ne.pme2_excl;

  // Pass 1: w[e] = |Le \ Lme| seeding.
  for (size_t pme = pme1; pme < pme2e; ++pme) {
    int32_t i = g.iw[pme];
    int32_t eln = g.elen[i];
    if (eln > 0) {
      int32_t nvi = -g.nv[i];
      int32_t wnvi = g.wflg - nvi;
      size_t pi = (size_t)g.pe[i];
      for (int32_t k = 0; k < eln; ++k) {
        int32_t e = g.iw[pi + k];
        int32_t we = g.w[e];
        if (we >= g.wflg)
          we -= nvi;
        else if (we != 0)
          we = g.degree[e] + wnvi;
        g.w[e] = we;
      }
    }
  }

  // Pass 2: approximate external degree + hashing.
  for (size_t pme = pme1; pme < pme2e; ++pme) {
    int32_t i = g.iw[pme];
    size_t p1 = (size_t)g.pe[i];
    size_t p2 = p1 + (size_t)g.elen[i];
    size_t pn = p1;
    size_t deg = 0;
    uint64_t hash = 0;
    for (size_t p = p1; p < p2; ++p) {
      int32_t e = g.iw[p];
      int32_t we = g.w[e];
      if (we == 0) continue;
      int32_t dext = we - g.wflg;
      if (aggressive) {
        if (dext > 0) {
          deg += (size_t)dext;
          g.iw[pn++] = e;
          hash += (uint64_t)e;
        } else {
          g.pe[e] = flip(me);
          g.w[e] = 0;
        }
      } else {
        deg += (size_t)dext;
        g.iw[pn++] = e;
        hash += (uint64_t)e;
      }
    }
    g.elen[i] = (int32_t)(pn - p1 + 1);
    size_t p3 = pn;
    size_t p4 = p1 + (size_t)g.len[i];
    for (size_t p = p2; p < p4; ++p) {
      int32_t j = g.iw[p];
      int32_t nvj = g.nv[j];
      if (nvj > 0) {
        deg += (size_t)nvj;
        g.iw[pn++] = j;
        hash += (uint64_t)j;
      }
    }
    if (g.elen[i] == 1 && p3 == pn) {
      // Mass elimination.
      g.pe[i] = flip(me);
      int32_t nvi = -g.nv[i];
      degme -= (size_t)nvi;
      nvpiv += nvi;
      g.nel += (size_t)nvi;
      g.nv[i] = 0;
      g.elen[i] = NONE;
      g.n_mass_elim++;
    } else {
      if ((int32_t)deg < g.degree[i]) g.degree[i] = (int32_t)deg;
      if (p1 != pn) g.iw[pn] = g.iw[p3];
      if (p3 != p1) g.iw[p3] = g.iw[p1];
      g.iw[p1] = me;
      g.len[i] = (int32_t)(pn - p1 + 1);
      size_t h = (size_t)(hash % (uint64_t)g.n);
      int32_t j = g.head[h];
      if (j <= NONE) {
        g.next[i] = flip(j);
        g.head[h] = flip(i);
      } else {
        g.next[i] = g.last[j];
        g.last[j] = i;
      }
      g.last[i] = (int32_t)h;
    }
  }

  int32_t degme_i = (int32_t)degme;
  g.degree[me] = degme_i;
  if (degme_i > g.lemax) g.lemax = degme_i;
  g.wflg += g.lemax;
  g.wflg = clear_flag(g.wflg, g.wbig, g.w);

  // Supervariable detection over each hash chain.
  for (size_t pme = pme1; pme < pme2e; ++pme) {
    int32_t ia = g.iw[pme];
    if (g.nv[ia] >= 0) continue;
    size_t h = (size_t)g.last[ia];
    int32_t jh = g.head[h];
    int32_t i;
    if (jh == NONE) {
      i = NONE;
    } else if (jh < NONE) {
      g.head[h] = NONE;
      i = flip(jh);
    } else {
      i = g.last[jh];
      g.last[jh] = NONE;
    }
    while (i != NONE && g.next[i] != NONE) {
      int32_t ln = g.len[i], eln = g.elen[i], pi = g.pe[i];
      for (int32_t p = pi + 1; p < pi + ln; ++p) g.w[g.iw[p]] = g.wflg;
      int32_t jlast = i;
      int32_t jp = g.next[i];
      while (jp != NONE) {
        bool ok = g.len[jp] == ln && g.elen[jp] == eln;
        if (ok) {
          int32_t pj = g.pe[jp];
          for (int32_t p = pj + 1; p < pj + ln; ++p)
            if (g.w[g.iw[p]] != g.wflg) {
              ok = false;
              break;
            }
        }
        if (ok) {
          g.pe[jp] = flip(i);
          g.nv[i] += g.nv[jp];
          g.nv[jp] = 0;
          g.elen[jp] = NONE;
          jp = g.next[jp];
          g.next[jlast] = jp;
          g.n_supervar_merge++;
        } else {
          jlast = jp;
          jp = g.next[jp];
        }
      }
      g.wflg += 1;
      i = g.next[i];
    }
  }

  // Re-insert survivors with their new degree, compact me's list.
  size_t pw = pme1;
  size_t nleft = (size_t)g.n - g.nel;
  for (size_t pme = pme1; pme < pme2e; ++pme) {
    int32_t i = g.iw[pme];
    int32_t nvi = -g.nv[i];
    if (nvi > 0) {
      g.nv[i] = nvi;
      size_t d = (size_t)g.degree[i] + (size_t)degme_i - (size_t)nvi;
      size_t cap = nleft - (size_t)nvi;
      if (d > cap) d = cap;
      int32_t inext = g.head[d];
      if (inext != NONE) g.last[inext] = i;
      g.next[i] = inext;
      g.last[i] = NONE;
      g.head[d] = i;
      if (d < g.mindeg) g.mindeg = d;
      g.degree[i] = (int32_t)d;
      g.iw[pw++] = i;
    }
  }
  g.nv[me] = nvpiv;
  g.len[me] = (int32_t)(pw - pme1);
  if (g.len[me] == 0) {
    g.pe[me] = NONE;
    g.w[me] = 0;
  }
  if (elenme != 0) g.pfree = pw;

  double f = nvpiv, r = (double)degme_i + (double)g.ndense;
  double lnzme = f * r + (f - 1.0) * f / 2.0;
  double s = f * r * r + r * (f - 1.0) * f + (f - 1.0) * f * (2.0 * f - 1.0) / 6.0;
  st.ndiv += lnzme;
  st.nms_lu += s;
  st.nms_ldl += (s + lnzme) / 2.0;
}

// Iterative DFS over one assembly-tree root (algo.rs:1523-1562).
size_t qg_post_tree(QGraph& g, int32_t root, size_t k) {
  size_t top = 1;
  g.last[0] = root;
  while (top > 0) {
    int32_t i = g.last[top - 1];
    int32_t child0 = g.head[i];
    if (child0 != NONE) {
      size_t count = 0;
      for (int32_t f = child0; f != NONE; f = g.next[f]) ++count;
      size_t new_top = top + count;
      size_t t = new_top;
      int32_t f = child0;
      for (;;) {
        g.last[--t] = f;
        int32_t nf = g.next[f];
        if (nf == NONE) break;
        f = nf;
      }
      top = new_top;
      g.head[i] = NONE;
    } else {
      --top;
      g.w[i] = (int32_t)k++;
    }
  }
  return k;
}

// Un-flip, path-compress absorbed supervariables, postorder the assembly tree
// with the largest front last, expand supervariables and append dense
// variables (algo.rs:1362-1450, 1452-1521).
std::vector<int64_t> qg_finalize_perm(QGraph& g) {
  const int64_t n = g.n;
  std::vector<int64_t> perm(n);
  if (n == 0) return perm;
  for (auto& x : g.pe) x = flip(x);
  for (auto& x : g.elen) x = flip(x);
  for (int64_t i = 0; i < n; ++i) {
    if (g.nv[i] != 0) continue;
    int32_t hi = g.pe[i];
    if (hi == NONE) continue;
    int32_t j = hi;
    while (g.nv[j] == 0) j = g.pe[j];
    int32_t e = j;
    int32_t jj = (int32_t)i;
    while (g.nv[jj] == 0) {
      int32_t jn = g.pe[jj];
      g.pe[jj] = e;
      jj = jn;
    }
  }
  std::fill(g.head.begin(), g.head.end(), NONE);
  std::fill(g.next.begin(), g.next.end(), NONE);
  for (int64_t j = n - 1; j >= 0; --j) {
    if (g.nv[j] > 0) {
      int32_t par = g.pe[j];
      if (par >= 0 && par < n) {
        g.next[j] = g.head[par];
        g.head[par] = (int32_t)j;
      }
    }
  }
  for (int64_t i = 0; i < n; ++i) {
    if (g.nv[i] > 0 && g.head[i] != NONE) {
      int32_t fprev = NONE, bigfprev = NONE, bigf = NONE, maxfr = NONE;
      for (int32_t f = g.head[i]; f != NONE; f = g.next[f]) {
        int32_t fr = g.elen[f];
        if (fr >= maxfr) {
          maxfr = fr;
          bigfprev = fprev;
          bigf = f;
        }
        fprev = f;
      }
      int32_t fnext = g.next[bigf];
      if (fnext != NONE) {
        if (bigfprev != NONE)
          g.next[bigfprev] = fnext;
        else
          g.head[i] = fnext;
        g.next[bigf] = NONE;
        g.next[fprev] = bigf;
      }
    }
  }
  std::fill(g.w.begin(), g.w.end(), NONE);
  size_t k = 0;
  for (int64_t i = 0; i < n; ++i)
    if (g.pe[i] == NONE && g.nv[i] > 0) k = qg_post_tree(g, (int32_t)i, k);
  std::fill(g.head.begin(), g.head.end(), NONE);
  for (int64_t e = 0; e < n; ++e)
    if (g.w[e] != NONE) g.head[g.w[e]] = (int32_t)e;
  std::fill(g.next.begin(), g.next.end(), NONE);
  int32_t nel = 0;
  for (int64_t t = 0; t < n; ++t) {
    int32_t e = g.head[t];
    if (e == NONE) break;
    g.next[e] = nel;
    nel += g.nv[e];
  }
  for (int64_t i = 0; i < n; ++i) {
    if (g.nv[i] == 0) {
      int32_t e = g.pe[i];
      if (e != NONE) {
        g.next[i] = g.next[e];
        g.next[e] += 1;
      } else {
        g.next[i] = nel++;
      }
    }
  }
  for (int64_t i = 0; i < n; ++i) perm[g.next[i]] = i;
  return perm;
}

}  // namespace

std::vector<int64_t> amd_order(const CscPattern& pat, AmdStats* stats_out, double dense_alpha,
                               bool aggressive) {
  QGraph g;
  AmdStats st;
  qg_init(g, pat.n, pat.col_ptr.data(), pat.row_idx.data(), dense_alpha);
  while (g.nel < (size_t)g.n) {
    int64_t me = qg_select_pivot(g);
    if (me < 0) break;
    int32_t elenme = g.elen[me];
    NewElement ne = qg_create_element(g, (int32_t)me);
    qg_finalize_step(g, (int32_t)me, ne, elenme, aggressive, st);
  }
  double f = g.ndense;
  double lnzme = (f - 1.0) * f / 2.0;
  double s = (f - 1.0) * f * (2.0 * f - 1.0) / 6.0;
  st.ndiv += lnzme;
  st.nms_lu += s;
  st.nms_ldl += (s + lnzme) / 2.0;
  st.ncmpa = g.ncmpa;
  st.n_dense = (uint32_t)(g.ndense > 0 ? g.ndense : 0);
  st.n_mass_elim = g.n_mass_elim;
  st.n_supervar_merge = g.n_supervar_merge;
  std::vector<int64_t> perm = qg_finalize_perm(g);
  if (stats_out) *stats_out = st;
  return perm;
}

}  // namespace rslab
