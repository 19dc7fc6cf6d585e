// Multilevel nested-dissection ordering (the MetisND ordering method).
//
// Restates the reference's rslab-metis crate step by step, because the
// permutation (and so the supernode structure) is defined by its tie-breaks:
//   crates/rslab-metis/src/rng.rs             SplitMix64, bounded draws, shuffle
//   crates/rslab-metis/src/graph.rs:1-80      graph of the full pattern (no
//                                             diagonal, no duplicates)
//   crates/rslab-metis/src/coarsen.rs:52-260  sorted heavy-edge matching,
//                                             2-hop fallback, contraction
//   crates/rslab-metis/src/initial_partition.rs:23-200  GGP / BFS bisections
//   crates/rslab-metis/src/fm_refine.rs:32-230          edge FM refinement
//   crates/rslab-metis/src/separator.rs:33-185          Konig vertex cover
//   crates/rslab-metis/src/node_refine.rs:29-463        node-separator FM
//   crates/rslab-metis/src/node_nd.rs:30-408            dissection driver
//   crates/rslab-metis/src/lib.rs:123-140, 204-280      defaults, entry
// Default options only (seed 1, 7 initial trials, coarsen floor 120, AMD on
// subgraphs of <= 200 vertices, 2-hop threshold 0.85, imbalance 0.20, 10 FM
// passes, no dense-column quotient).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <queue>
#include <tuple>
#include <vector>

#include "host.hpp"

namespace rslab {
namespace {

constexpr uint8_t PA = 0, PB = 1, PS = 2;

struct Opts {
  uint64_t seed = 1;
  int niparts = 7;
  int coarsen_floor = 120;
  int nd_to_amd_switch = 200;
  double two_hop = 0.85;
  double max_imbalance = 0.20;
  int fm_passes = 10;
};

struct SplitMix {
  uint64_t s;
  explicit SplitMix(uint64_t seed) : s(seed + 0x9E3779B97F4A7C15ull) {}
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  uint64_t range(uint64_t n) {
    const uint64_t zone = UINT64_MAX - (UINT64_MAX % n);
    for (;;) {
      const uint64_t r = next();
      if (r < zone) return r % n;
    }
  }
  template <typename T>
  void shuffle(std::vector<T>& v) {
    const size_t n = v.size();
    if (n < 2) return;
    for (size_t i = n - 1; i >= 1; --i) std::swap(v[i], v[range(i + 1)]);
  }
};

struct Graph {
  int n = 0;
  std::vector<int> xadj, adj, vw, aw;
  int deg(int v) const { return xadj[v + 1] - xadj[v]; }
};

Graph graph_of(const CscPattern& p) {
  Graph g;
  g.n = (int)p.n;
  g.xadj.assign(1, 0);
  for (int64_t j = 0; j < p.n; ++j) {
    int64_t last = -1;
    for (int64_t k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) {
      const int64_t r = p.row_idx[k];
      if (r == j || r == last) continue;
      g.adj.push_back((int)r);
      last = r;
    }
    g.xadj.push_back((int)g.adj.size());
  }
  g.vw.assign(g.n, 1);
  g.aw.assign(g.adj.size(), 1);
  return g;
}

// ---- coarsening -------------------------------------------------------------

struct Level {
  Graph g;
  std::vector<int> cmap;
};

int two_hop(const Graph& f, std::vector<int>& match, std::vector<int>& cmap) {
  for (int v = 0; v < f.n; ++v) {
    if (match[v] != v) continue;
    int partner = -1;
    for (int k = f.xadj[v]; k < f.xadj[v + 1] && partner < 0; ++k) {
      const int mid = f.adj[k];
      for (int kk = f.xadj[mid]; kk < f.xadj[mid + 1]; ++kk) {
        const int w = f.adj[kk];
        if (w == v) continue;
        if (match[w] == w) {
          partner = w;
          break;
        }
      }
    }
    if (partner >= 0) {
      match[v] = partner;
      match[partner] = v;
    }
  }
  std::fill(cmap.begin(), cmap.end(), -1);
  int cn = 0;
  for (int v = 0; v < f.n; ++v) {
    if (cmap[v] >= 0) continue;
    cmap[v] = cn;
    if (match[v] != v) cmap[match[v]] = cn;
    ++cn;
  }
  return cn;
}

Graph contract(const Graph& f, const std::vector<int>& cmap, int cn) {
  Graph g;
  g.n = cn;
  g.vw.assign(cn, 0);
  for (int v = 0; v < f.n; ++v) g.vw[cmap[v]] += f.vw[v];
  // fine vertices of every coarse vertex, last-inserted first
  std::vector<int> head(cn, -1), next(f.n, -1);
  for (int v = 0; v < f.n; ++v) {
    next[v] = head[cmap[v]];
    head[cmap[v]] = v;
  }
  std::vector<int> marker(cn, -1), wto(cn, 0), touched;
  g.xadj.assign(1, 0);
  for (int c = 0; c < cn; ++c) {
    touched.clear();
    for (int v = head[c]; v >= 0; v = next[v])
      for (int k = f.xadj[v]; k < f.xadj[v + 1]; ++k) {
        const int c2 = cmap[f.adj[k]];
        if (c2 == c) continue;
        if (marker[c2] != c) {
          marker[c2] = c;
          wto[c2] = f.aw[k];
          touched.push_back(c2);
        } else {
          wto[c2] += f.aw[k];
        }
      }
    for (int t : touched) {
      g.adj.push_back(t);
      g.aw.push_back(wto[t]);
    }
    g.xadj.push_back((int)g.adj.size());
  }
  return g;
}

Level coarsen_level(const Graph& f, SplitMix& rng, double two_hop_threshold) {
  std::vector<int> match(f.n, -1), cmap(f.n, -1);
  std::vector<int> order(f.n);
  for (int v = 0; v < f.n; ++v) order[v] = v;
  rng.shuffle(order);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return f.deg(a) < f.deg(b); });
  int cn = 0;
  for (int v : order) {
    if (match[v] != -1) continue;
    int best = -1, best_w = -1;
    for (int k = f.xadj[v]; k < f.xadj[v + 1]; ++k) {
      const int u = f.adj[k];
      if (match[u] != -1) continue;
      const int w = f.aw[k];
      if (w > best_w || (w == best_w && (best < 0 || u < best))) {
        best = u;
        best_w = w;
      }
    }
    if (best >= 0) {
      match[v] = best;
      match[best] = v;
      cmap[v] = cmap[best] = cn;
    } else {
      match[v] = v;
      cmap[v] = cn;
    }
    ++cn;
  }
  const double ratio = (double)cn / (double)std::max(f.n, 1);
  if (ratio > two_hop_threshold && f.n >= 4) cn = two_hop(f, match, cmap);
  return Level{contract(f, cmap, cn), std::move(cmap)};
}

std::vector<Level> coarsen(const Graph& fine, const Opts& o, SplitMix& rng) {
  std::vector<Level> levels;
  int prev = fine.n;
  const Graph* cur = &fine;
  for (;;) {
    if (cur->n <= o.coarsen_floor) break;
    Level lv = coarsen_level(*cur, rng, o.two_hop);
    const int nn = lv.g.n;
    if (nn == 0 || (double)nn > 0.95 * (double)prev) {
      if (nn > 0 && nn < prev) levels.push_back(std::move(lv));
      break;
    }
    prev = nn;
    levels.push_back(std::move(lv));
    cur = &levels.back().g;
  }
  return levels;
}

// ---- initial bisection (coarsest graph) --------------------------------------

int cut_size(const Graph& g, const std::vector<uint8_t>& lab) {
  int64_t cut = 0;
  for (int v = 0; v < g.n; ++v)
    for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) {
      const int u = g.adj[k];
      if (u > v && lab[u] != lab[v]) cut += g.aw[k];
    }
  return (int)std::min<int64_t>(cut, INT32_MAX);
}

int64_t part_weight(const Graph& g, const std::vector<uint8_t>& lab, uint8_t p) {
  int64_t s = 0;
  for (int v = 0; v < g.n; ++v)
    if (lab[v] == p) s += g.vw[v];
  return s;
}

// Greedy graph growing: grow part A from a random seed, always taking the
// boundary vertex of largest cut reduction (first in boundary order on ties).
std::vector<uint8_t> bisect_ggp(const Graph& g, SplitMix& rng, int64_t target_a) {
  const int n = g.n;
  std::vector<uint8_t> lab(n, PB);
  if (n == 0) return lab;
  const int seed = (int)rng.range((uint64_t)n);
  lab[seed] = PA;
  int64_t aw = g.vw[seed];
  std::vector<int> gain(n, 0), wtot(n, 0), boundary;
  std::vector<char> inb(n, 0);
  for (int v = 0; v < n; ++v)
    for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) wtot[v] += g.aw[k];
  auto push_nbrs = [&](int v) {
    for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) {
      const int u = g.adj[k];
      if (lab[u] != PB) continue;
      gain[u] += g.aw[k];
      if (!inb[u]) {
        inb[u] = 1;
        boundary.push_back(u);
      }
    }
  };
  push_nbrs(seed);
  while (aw < target_a && !boundary.empty()) {
    size_t bi = 0;
    int64_t bg = INT64_MIN;
    for (size_t i = 0; i < boundary.size(); ++i) {
      const int v = boundary[i];
      if (lab[v] != PB) continue;
      const int64_t gg = 2 * (int64_t)gain[v] - wtot[v];
      if (gg > bg) {
        bg = gg;
        bi = i;
      }
    }
    const int v = boundary[bi];
    boundary[bi] = boundary.back();  // swap_remove
    boundary.pop_back();
    if (lab[v] != PB) continue;
    lab[v] = PA;
    inb[v] = 0;
    aw += g.vw[v];
    push_nbrs(v);
  }
  return lab;
}

std::vector<uint8_t> bisect_bfs(const Graph& g, SplitMix& rng, int64_t target_a) {
  const int n = g.n;
  std::vector<uint8_t> lab(n, PB);
  if (n == 0) return lab;
  const int seed = (int)rng.range((uint64_t)n);
  std::vector<int> q{seed};
  size_t qh = 0;
  std::vector<char> vis(n, 0);
  vis[seed] = 1;
  int64_t aw = 0;
  while (qh < q.size()) {
    const int v = q[qh++];
    if (aw >= target_a) break;
    lab[v] = PA;
    aw += g.vw[v];
    for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) {
      const int u = g.adj[k];
      if (!vis[u]) {
        vis[u] = 1;
        q.push_back(u);
      }
    }
  }
  return lab;
}

// ---- edge FM refinement --------------------------------------------------------

int refine_bisection(const Graph& g, std::vector<uint8_t>& lab, double max_imb, int passes) {
  const int n = g.n;
  if (n < 2) return cut_size(g, lab);
  int64_t total = 0;
  for (int w : g.vw) total += w;
  const int64_t max_side = (int64_t)std::ceil((1.0 + max_imb) * (double)total / 2.0);
  int pass_cut = cut_size(g, lab);
  // max-heap on (gain, -vertex): largest gain first, lower vertex on ties
  using Item = std::tuple<int, int, int>;  // gain, -v, stamp
  for (int pass = 0; pass < passes; ++pass) {
    const int before = pass_cut;
    std::vector<int> gain(n, 0);
    for (int v = 0; v < n; ++v) {
      int ed = 0, id = 0;
      for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) (lab[g.adj[k]] == lab[v] ? id : ed) += g.aw[k];
      gain[v] = ed - id;
    }
    std::vector<char> locked(n, 0);
    std::priority_queue<Item> heap;
    for (int v = 0; v < n; ++v) heap.emplace(gain[v], -v, gain[v]);
    int cur_cut = pass_cut;
    std::vector<int> moves;
    int64_t a_w = part_weight(g, lab, PA), b_w = total - a_w;
    const bool starts_bal = std::max(a_w, b_w) <= max_side;
    long best_prefix = starts_bal ? 0 : -1;
    int best_cut = pass_cut;
    int no_improve = 0;
    while (!heap.empty()) {
      const auto [gv, nv, stamp] = heap.top();
      heap.pop();
      (void)gv;
      const int v = -nv;
      if (locked[v] || stamp != gain[v]) continue;
      const uint8_t from = lab[v], to = from == PA ? PB : PA;
      if (to == PA) {
        a_w += g.vw[v];
        b_w -= g.vw[v];
      } else {
        a_w -= g.vw[v];
        b_w += g.vw[v];
      }
      const int64_t side_max = std::max(a_w, b_w);
      lab[v] = to;
      cur_cut -= gain[v];
      locked[v] = 1;
      moves.push_back(v);
      for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) {
        const int u = g.adj[k];
        if (locked[u]) continue;
        gain[u] += lab[u] == from ? 2 * g.aw[k] : -2 * g.aw[k];
        heap.emplace(gain[u], -u, gain[u]);
      }
      if (side_max <= max_side) {
        if (best_prefix < 0 || cur_cut < best_cut) {
          best_cut = cur_cut;
          best_prefix = (long)moves.size();
          no_improve = 0;
        } else {
          ++no_improve;
        }
      } else {
        ++no_improve;
      }
      if (no_improve >= 50) break;
    }
    if (best_prefix >= 0) {
      for (size_t i = (size_t)best_prefix; i < moves.size(); ++i) lab[moves[i]] = lab[moves[i]] == PA ? PB : PA;
      pass_cut = best_cut;
    } else {
      pass_cut = cur_cut;
    }
    if (pass_cut == before) break;
  }
  return pass_cut;
}

// ---- edge bisection -> node separator (minimum vertex cover of the cut) ---------

bool augment(int u, const std::vector<std::vector<int>>& adj, std::vector<int>& ma, std::vector<int>& mb,
             std::vector<char>& vis) {
  for (int v : adj[u]) {
    if (vis[v]) continue;
    vis[v] = 1;
    if (mb[v] < 0 || augment(mb[v], adj, ma, mb, vis)) {
      ma[u] = v;
      mb[v] = u;
      return true;
    }
  }
  return false;
}

void construct_separator(const Graph& g, std::vector<uint8_t>& lab) {
  const int n = g.n;
  std::vector<char> ba(n, 0), bb(n, 0);
  for (int v = 0; v < n; ++v) {
    const uint8_t lv = lab[v];
    if (lv != PA && lv != PB) continue;
    for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) {
      const uint8_t lu = lab[g.adj[k]];
      if (lu != lv && (lu == PA || lu == PB)) {
        (lv == PA ? ba : bb)[v] = 1;
        break;
      }
    }
  }
  std::vector<int> al, bl, aidx(n, -1), bidx(n, -1);
  for (int v = 0; v < n; ++v) {
    if (ba[v]) {
      aidx[v] = (int)al.size();
      al.push_back(v);
    }
    if (bb[v]) {
      bidx[v] = (int)bl.size();
      bl.push_back(v);
    }
  }
  if (al.empty() || bl.empty()) return;
  const int na = (int)al.size(), nb = (int)bl.size();
  std::vector<std::vector<int>> adj(na);
  for (int ai = 0; ai < na; ++ai)
    for (int k = g.xadj[al[ai]]; k < g.xadj[al[ai] + 1]; ++k)
      if (bidx[g.adj[k]] >= 0) adj[ai].push_back(bidx[g.adj[k]]);
  std::vector<int> ma(na, -1), mb(nb, -1);
  for (int ai = 0; ai < na; ++ai) {
    std::vector<char> vis(nb, 0);
    augment(ai, adj, ma, mb, vis);
  }
  std::vector<char> za(na, 0), zb(nb, 0);
  std::vector<int> stack;
  for (int ai = 0; ai < na; ++ai)
    if (ma[ai] < 0) {
      za[ai] = 1;
      stack.push_back(ai);
    }
  while (!stack.empty()) {
    const int ai = stack.back();
    stack.pop_back();
    for (int bi : adj[ai])
      if (!zb[bi]) {
        zb[bi] = 1;
        const int m = mb[bi];
        if (m >= 0 && !za[m]) {
          za[m] = 1;
          stack.push_back(m);
        }
      }
  }
  for (int ai = 0; ai < na; ++ai)
    if (!za[ai]) lab[al[ai]] = PS;
  for (int bi = 0; bi < nb; ++bi)
    if (zb[bi]) lab[bl[bi]] = PS;
}

// ---- node-separator refinement ---------------------------------------------------

// Binary max-heap with positions; ties keep their place (strict comparisons),
// which fixes the pop order of equal keys.
struct MaxHeap {
  std::vector<int> heap, pos;
  std::vector<int64_t> key;
  explicit MaxHeap(int n) : pos(n, -1), key(n, 0) {}
  void clear() {
    for (int v : heap) pos[v] = -1;
    heap.clear();
  }
  bool contains(int v) const { return pos[v] >= 0; }
  void swap_at(size_t i, size_t j) {
    std::swap(heap[i], heap[j]);
    pos[heap[i]] = (int)i;
    pos[heap[j]] = (int)j;
  }
  void up(size_t i) {
    while (i > 0) {
      const size_t p = (i - 1) / 2;
      if (key[heap[i]] > key[heap[p]]) {
        swap_at(i, p);
        i = p;
      } else {
        break;
      }
    }
  }
  void down(size_t i) {
    const size_t n = heap.size();
    for (;;) {
      const size_t l = 2 * i + 1, r = 2 * i + 2;
      size_t m = i;
      if (l < n && key[heap[l]] > key[heap[m]]) m = l;
      if (r < n && key[heap[r]] > key[heap[m]]) m = r;
      if (m == i) break;
      swap_at(i, m);
      i = m;
    }
  }
  void insert(int v, int64_t k) {
    key[v] = k;
    pos[v] = (int)heap.size();
    heap.push_back(v);
    up(heap.size() - 1);
  }
  void update(int v, int64_t k) {
    const int64_t old = key[v];
    key[v] = k;
    if (k > old)
      up((size_t)pos[v]);
    else if (k < old)
      down((size_t)pos[v]);
  }
  int pop() {
    if (heap.empty()) return -1;
    const int top = heap[0];
    pos[top] = -1;
    const int last = heap.back();
    heap.pop_back();
    if (!heap.empty()) {
      heap[0] = last;
      pos[last] = 0;
      down(0);
    }
    return top;
  }
};

// Part weights, separator list and, per separator vertex, the weight of its
// neighbours in A and in B.
struct NodeState {
  int64_t pw[3] = {0, 0, 0};
  std::vector<std::array<int64_t, 2>> edeg;
  std::vector<int> bnd, bptr;
  NodeState(const Graph& g, const std::vector<uint8_t>& lab) : edeg(g.n, {0, 0}), bptr(g.n, -1) {
    for (int v = 0; v < g.n; ++v) {
      pw[lab[v]] += g.vw[v];
      if (lab[v] != PS) continue;
      bptr[v] = (int)bnd.size();
      bnd.push_back(v);
      std::array<int64_t, 2> e{0, 0};
      for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) {
        const int u = g.adj[k];
        if (lab[u] != PS) e[lab[u]] += g.vw[u];
      }
      edeg[v] = e;
    }
  }
  void bnd_insert(int v) {
    bptr[v] = (int)bnd.size();
    bnd.push_back(v);
  }
  void bnd_delete(int v) {
    const int p = bptr[v], last = bnd.back();
    bnd[p] = last;
    bptr[last] = p;
    bnd.pop_back();
    bptr[v] = -1;
  }
};

// Pull-in bookkeeping shared by both refinements: separator vertex hv moves
// to side `to`; its neighbours on side `other` join the separator.
template <typename OnPulled>
void move_to_side(const Graph& g, std::vector<uint8_t>& lab, NodeState& st, MaxHeap& q, int hv, int to, int other,
                  OnPulled&& on_pulled, const std::vector<char>* moved) {
  const int64_t hw = g.vw[hv];
  st.bnd_delete(hv);
  st.pw[to] += hw;
  lab[hv] = (uint8_t)to;
  for (int k = g.xadj[hv]; k < g.xadj[hv + 1]; ++k) {
    const int u = g.adj[k];
    if (lab[u] == PS) {
      st.edeg[u][to] += hw;
    } else if (lab[u] == (uint8_t)other) {
      st.bnd_insert(u);
      on_pulled(u);
      lab[u] = PS;
      st.pw[other] -= g.vw[u];
      std::array<int64_t, 2> e{0, 0};
      for (int kk = g.xadj[u]; kk < g.xadj[u + 1]; ++kk) {
        const int w = g.adj[kk];
        if (lab[w] != PS) {
          e[lab[w]] += g.vw[w];
        } else {
          st.edeg[w][other] -= g.vw[u];
          if ((!moved || !(*moved)[w]) && q.contains(w)) q.update(w, g.vw[w] - st.edeg[w][other]);
        }
      }
      st.edeg[u] = e;
      q.insert(u, g.vw[u] - e[other]);
    }
  }
}

int64_t node_refine_1sided(const Graph& g, std::vector<uint8_t>& lab, double max_imb, int niter, SplitMix& rng) {
  const int n = g.n;
  NodeState st(g, lab);
  const int64_t total = st.pw[0] + st.pw[1] + st.pw[2];
  const int64_t badmax = (int64_t)(0.5 * (1.0 + max_imb) * (double)total);
  MaxHeap q(n);
  std::vector<int> swaps, mind, order;
  std::vector<size_t> mptr;
  int to = st.pw[0] < st.pw[1] ? 1 : 0;
  for (int pass = 0; pass < 2 * niter;) {
    const int other = to;
    to = 1 - to;
    q.clear();
    long mincutorder = -1;
    const int64_t initcut = st.pw[2];
    int64_t mincut = st.pw[2];
    order = st.bnd;
    rng.shuffle(order);
    for (int v : order) q.insert(v, g.vw[v] - st.edeg[v][other]);
    const long limit = std::min<long>(3 * (long)st.bnd.size(), 300);
    swaps.clear();
    mind.clear();
    mptr.assign(1, 0);
    int64_t mindiff = std::llabs(st.pw[0] - st.pw[1]);
    for (;;) {
      const int hv = q.pop();
      if (hv < 0) break;
      const int64_t hw = g.vw[hv];
      if (mind.size() + (size_t)g.deg(hv) >= (size_t)(2 * n - 1)) break;
      if (st.pw[to] + hw > badmax) break;
      const int64_t gain = hw - st.edeg[hv][other];
      st.pw[2] -= gain;
      const int64_t newdiff = std::llabs(st.pw[to] + hw - (st.pw[other] - st.edeg[hv][other]));
      const long ns = (long)swaps.size();
      if (st.pw[2] < mincut || (st.pw[2] == mincut && newdiff < mindiff)) {
        mincut = st.pw[2];
        mincutorder = ns;
        mindiff = newdiff;
      } else if (ns - mincutorder > 3 * limit ||
                 (ns - mincutorder > limit && (double)st.pw[2] > 1.10 * (double)mincut)) {
        st.pw[2] += gain;
        break;
      }
      move_to_side(g, lab, st, q, hv, to, other, [&](int u) { mind.push_back(u); }, nullptr);
      swaps.push_back(hv);
      mptr.push_back(mind.size());
    }
    // roll back to the best prefix
    while ((long)swaps.size() > mincutorder + 1) {
      const int hv = swaps.back();
      swaps.pop_back();
      const int64_t hw = g.vw[hv];
      st.pw[2] += hw;
      st.pw[to] -= hw;
      lab[hv] = PS;
      st.bnd_insert(hv);
      std::array<int64_t, 2> e{0, 0};
      for (int k = g.xadj[hv]; k < g.xadj[hv + 1]; ++k) {
        const int u = g.adj[k];
        if (lab[u] == PS)
          st.edeg[u][to] -= hw;
        else
          e[lab[u]] += g.vw[u];
      }
      st.edeg[hv] = e;
      const size_t s = swaps.size();
      for (size_t t = mptr[s]; t < mptr[s + 1]; ++t) {
        const int u = mind[t];
        lab[u] = (uint8_t)other;
        st.pw[other] += g.vw[u];
        st.pw[2] -= g.vw[u];
        st.bnd_delete(u);
        for (int kk = g.xadj[u]; kk < g.xadj[u + 1]; ++kk)
          if (lab[g.adj[kk]] == PS) st.edeg[g.adj[kk]][other] += g.vw[u];
      }
      mptr.pop_back();
    }
    ++pass;
    if (pass % 2 == 0 && (mincutorder == -1 || mincut >= initcut)) break;
  }
  return st.pw[2];
}

void node_balance(const Graph& g, std::vector<uint8_t>& lab, double max_imb, SplitMix& rng) {
  const int n = g.n;
  NodeState st(g, lab);
  const double mult = 0.5 * (1.0 + max_imb);
  if (std::max(st.pw[0], st.pw[1]) < (int64_t)(mult * (double)(st.pw[0] + st.pw[1]))) return;
  const int64_t total = st.pw[0] + st.pw[1] + st.pw[2];
  if (std::llabs(st.pw[0] - st.pw[1]) < 3 * total / std::max(n, 1)) return;
  const int to = st.pw[0] < st.pw[1] ? 0 : 1, other = 1 - to;
  MaxHeap q(n);
  std::vector<char> moved(n, 0);
  std::vector<int> order = st.bnd;
  rng.shuffle(order);
  for (int v : order) q.insert(v, g.vw[v] - st.edeg[v][other]);
  for (;;) {
    const int hv = q.pop();
    if (hv < 0) break;
    const int64_t hw = g.vw[hv];
    moved[hv] = 1;
    const int64_t gain = hw - st.edeg[hv][other];
    const int64_t badmax = (int64_t)(mult * (double)(st.pw[0] + st.pw[1]));
    if (st.pw[to] > st.pw[other]) break;
    if (gain < 0 && st.pw[other] < badmax) break;
    if (st.pw[to] + hw > badmax) continue;
    st.pw[2] -= gain;
    move_to_side(g, lab, st, q, hv, to, other, [](int) {}, &moved);
  }
}

// ---- dissection driver ---------------------------------------------------------

std::vector<uint8_t> multilevel_node_bisection(const Graph& g, const Opts& o, SplitMix& rng) {
  std::vector<Level> levels = coarsen(g, o, rng);
  const Graph& coarsest = levels.empty() ? g : levels.back().g;
  int64_t total = 0;
  for (int w : coarsest.vw) total += w;
  const int64_t target = total / 2;
  std::vector<uint8_t> best(coarsest.n, PA);
  int best_cut = INT32_MAX;
  for (int trial = 0; trial < o.niparts; ++trial) {
    std::vector<uint8_t> lab = trial % 2 == 0 ? bisect_ggp(coarsest, rng, target) : bisect_bfs(coarsest, rng, target);
    const int cut = refine_bisection(coarsest, lab, o.max_imbalance, o.fm_passes);
    if (cut < best_cut) {
      best_cut = cut;
      best = std::move(lab);
    }
  }
  std::vector<uint8_t> lab = std::move(best);
  construct_separator(coarsest, lab);
  node_refine_1sided(coarsest, lab, o.max_imbalance, o.fm_passes, rng);
  for (int li = (int)levels.size() - 1; li >= 0; --li) {
    const Graph& prev = li == 0 ? g : levels[li - 1].g;
    std::vector<uint8_t> proj(prev.n);
    for (int v = 0; v < prev.n; ++v) proj[v] = lab[levels[li].cmap[v]];
    lab = std::move(proj);
    node_balance(prev, lab, o.max_imbalance, rng);
    node_refine_1sided(prev, lab, o.max_imbalance, o.fm_passes, rng);
  }
  return lab;
}

// Subgraph induced by `verts` (local ids in list order), adjacency order kept.
Graph induced(const Graph& g, const std::vector<int>& verts, const std::vector<int>& local) {
  Graph s;
  s.n = (int)verts.size();
  s.xadj.assign(1, 0);
  for (int v : verts) {
    s.vw.push_back(g.vw[v]);
    for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k) {
      const int lu = local[g.adj[k]];
      if (lu >= 0) {
        s.adj.push_back(lu);
        s.aw.push_back(g.aw[k]);
      }
    }
    s.xadj.push_back((int)s.adj.size());
  }
  return s;
}

Graph extract_list(const Graph& g, const std::vector<int>& verts) {
  std::vector<int> local(g.n, -1);
  for (size_t i = 0; i < verts.size(); ++i) local[verts[i]] = (int)i;
  return induced(g, verts, local);
}

// Component labels by depth-first flooding from each unlabelled vertex in order.
int components(const Graph& g, std::vector<int>& cc) {
  cc.assign(g.n, -1);
  int ncc = 0;
  std::vector<int> stack;
  for (int s = 0; s < g.n; ++s) {
    if (cc[s] >= 0) continue;
    cc[s] = ncc;
    stack.assign(1, s);
    while (!stack.empty()) {
      const int v = stack.back();
      stack.pop_back();
      for (int k = g.xadj[v]; k < g.xadj[v + 1]; ++k)
        if (cc[g.adj[k]] < 0) {
          cc[g.adj[k]] = ncc;
          stack.push_back(g.adj[k]);
        }
    }
    ++ncc;
  }
  return ncc;
}

std::vector<std::vector<int>> component_lists(const Graph& g, const std::vector<int>& cc, int ncc) {
  std::vector<std::vector<int>> out(ncc);
  for (int v = 0; v < g.n; ++v) out[cc[v]].push_back(v);
  return out;
}

// AMD on a leaf subgraph: its pattern with the diagonal spliced in (neighbour
// lists are ascending), positions offset.. of the global order.
void amd_leaf(const Graph& s, const std::vector<int>& map, int64_t offset, std::vector<int64_t>& iperm) {
  CscPattern p;
  p.n = s.n;
  p.col_ptr.assign(1, 0);
  for (int v = 0; v < s.n; ++v) {
    bool diag = false;
    for (int k = s.xadj[v]; k < s.xadj[v + 1]; ++k) {
      if (!diag && s.adj[k] > v) {
        p.row_idx.push_back(v);
        diag = true;
      }
      p.row_idx.push_back(s.adj[k]);
    }
    if (!diag) p.row_idx.push_back(v);
    p.col_ptr.push_back((int64_t)p.row_idx.size());
  }
  const std::vector<int64_t> perm = amd_order(p);
  for (size_t pos = 0; pos < perm.size(); ++pos) iperm[map[perm[pos]]] = offset + (int64_t)pos;
}

struct Work {
  Graph g;
  std::vector<int> map;
  int64_t offset;
};

void push_components(std::vector<Work>& work, const Graph& g, const std::vector<int>& map, int64_t offset) {
  std::vector<int> cc;
  const int ncc = components(g, cc);
  const auto lists = component_lists(g, cc, ncc);
  int64_t off = offset;
  for (const auto& verts : lists) {
    std::vector<int> m(verts.size());
    for (size_t i = 0; i < verts.size(); ++i) m[i] = map[verts[i]];
    if (!verts.empty()) work.push_back(Work{extract_list(g, verts), std::move(m), off});
    off += (int64_t)verts.size();
  }
}

std::vector<int64_t> nd_order(const CscPattern& full, const Opts& o) {
  const Graph g = graph_of(full);
  const int n = g.n;
  std::vector<int64_t> iperm(n, -1);
  SplitMix rng(o.seed);
  std::vector<Work> work;
  std::vector<int> ident(n);
  for (int v = 0; v < n; ++v) ident[v] = v;
  push_components(work, g, ident, 0);
  while (!work.empty()) {
    Work w = std::move(work.back());
    work.pop_back();
    const int m = w.g.n;
    if (m == 0) continue;
    if (m == 1) {
      iperm[w.map[0]] = w.offset;
      continue;
    }
    std::vector<int> cc;
    if (components(w.g, cc) > 1) {
      push_components(work, w.g, w.map, w.offset);
      continue;
    }
    if (m <= o.nd_to_amd_switch) {
      amd_leaf(w.g, w.map, w.offset, iperm);
      continue;
    }
    const std::vector<uint8_t> lab = multilevel_node_bisection(w.g, o, rng);
    std::vector<int> av, bv, sv;
    for (int v = 0; v < m; ++v) (lab[v] == PA ? av : lab[v] == PB ? bv : sv).push_back(v);
    const size_t big = std::max(av.size(), bv.size());
    if (av.empty() || bv.empty() || (double)big >= 0.9 * (double)m) {
      amd_leaf(w.g, w.map, w.offset, iperm);
      continue;
    }
    const int64_t na = (int64_t)av.size(), nb = (int64_t)bv.size();
    for (size_t i = 0; i < sv.size(); ++i) iperm[w.map[sv[i]]] = w.offset + na + nb + (int64_t)i;
    std::vector<int> ma(av.size()), mb(bv.size());
    for (size_t i = 0; i < av.size(); ++i) ma[i] = w.map[av[i]];
    for (size_t i = 0; i < bv.size(); ++i) mb[i] = w.map[bv[i]];
    Graph ga = extract_list(w.g, av), gb = extract_list(w.g, bv);
    work.push_back(Work{std::move(ga), std::move(ma), w.offset});
    work.push_back(Work{std::move(gb), std::move(mb), w.offset + na});
  }
  std::vector<int64_t> perm(n, -1);
  for (int v = 0; v < n; ++v) {
    const int64_t p = iperm[v];
    if (p < 0 || p >= n || perm[p] >= 0) throw RslabError(Status::InvalidInput, "nested dissection: invalid order");
    perm[p] = v;
  }
  return perm;
}

}  // namespace

std::vector<int64_t> metis_nd_order(const CscPattern& full, uint64_t seed, bool dense_quotient,
                                    int64_t dense_threshold) {
  Opts o;
  o.seed = seed;
  const int64_t n = full.n;
  if (!dense_quotient || n == 0) return nd_order(full, o);
  // Opt-in quasi-dense column quotient (lib.rs:282-404): columns of
  // off-diagonal degree above max(40, ceil(10 sqrt(n))) (or the given
  // threshold) leave the graph and are appended last, densest first.
  const int64_t thresh =
      dense_threshold >= 0 ? dense_threshold : std::max<int64_t>(40, (int64_t)std::ceil(10.0 * std::sqrt((double)n)));
  std::vector<int64_t> deg(n, 0), dense;
  for (int64_t c = 0; c < n; ++c) {
    for (int64_t k = full.col_ptr[c]; k < full.col_ptr[c + 1]; ++k) deg[c] += full.row_idx[k] != c;
    if (deg[c] > thresh) dense.push_back(c);
  }
  if (dense.empty()) return nd_order(full, o);
  std::sort(dense.begin(), dense.end(), [&](int64_t a, int64_t b) { return deg[a] != deg[b] ? deg[a] > deg[b] : a < b; });
  std::vector<char> is_dense(n, 0);
  for (int64_t c : dense) is_dense[c] = 1;
  std::vector<int64_t> to_orig, local(n, -1);
  for (int64_t c = 0; c < n; ++c)
    if (!is_dense[c]) {
      local[c] = (int64_t)to_orig.size();
      to_orig.push_back(c);
    }
  CscPattern sub;
  sub.n = (int64_t)to_orig.size();
  sub.col_ptr.assign(1, 0);
  for (int64_t c : to_orig) {
    bool diag = false;
    for (int64_t k = full.col_ptr[c]; k < full.col_ptr[c + 1]; ++k) {
      const int64_t r = full.row_idx[k];
      if (r == c || local[r] < 0) continue;
      if (!diag && local[r] > local[c]) {
        sub.row_idx.push_back(local[c]);
        diag = true;
      }
      sub.row_idx.push_back(local[r]);
    }
    if (!diag) sub.row_idx.push_back(local[c]);
    sub.col_ptr.push_back((int64_t)sub.row_idx.size());
  }
  std::vector<int64_t> perm;
  perm.reserve(n);
  for (int64_t l : nd_order(sub, o)) perm.push_back(to_orig[l]);
  perm.insert(perm.end(), dense.begin(), dense.end());
  return perm;
}

}  // namespace rslab
