// ORACLE — test infrastructure only.  Never linked into, or called by, the
// rslab_b200 product; only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load it, as the checker.
//
// The reference's symbolic analysis restated on its own, from the output of a
// fill-reducing ordering (the permutation is an input: the AMD one is pinned
// by the reference's SuiteSparse golden permutations) to the supernode
// partition and the left-looking row structures:
//   symmetric_pattern                       src/sparse/csc.rs:240-291
//   permute_pattern                         src/ordering/amd.rs:21-81
//   EliminationTree::from_pattern / children / roots / subtree_sizes
//                                           src/ordering/elimination_tree.rs:28-103
//   postorder / biased_postorder / merge_bias_partition
//                                           src/ordering/postorder.rs:22-143, 270-290
//   symbolic_prefix_with steps 2-6 + the Renumber pass
//                                           src/symbolic/mod.rs:952-1120
//   column counts (exact)                   src/symbolic/column_counts.rs:97-183
//   pick_amalgamation_strategy              src/symbolic/supernode.rs:222-246
//   find_supernodes (+ relax, root cap)     src/symbolic/supernode.rs:267-482
//   find_fundamental_supernodes             src/symbolic/supernode.rs:605-657
//   predict_merges                          src/symbolic/supernode.rs:678-723
//   analyze_with_inner (knobs, levels)      src/numeric/multifrontal_ldlt.rs:1684-1801
//   compute_supernode_row_structures        src/numeric/multifrontal_ldlt.rs:2121-2152
// Column counts are computed here by a direct row-subtree walk (each row's
// subtree in the elimination tree is traversed once), not by the reference's
// Gilbert-Ng-Peyton scheme: both give the exact counts of L, so the oracle
// reaches the same numbers by an independent route.  Sorts whose keys tie use
// a stable order; the reference's sort_unstable_by_key is an insertion sort
// (stable) for the short child lists that occur here (<= 20 entries).
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

namespace orc_sym {

using Vec = std::vector<int64_t>;

struct Pattern {
  int64_t n = 0;
  Vec cp, ri;
};

// Both triangles of a lower-triangle CSC, rows sorted in every column.
Pattern full_from_lower(int64_t n, const int64_t* cp, const int64_t* ri) {
  Pattern p;
  p.n = n;
  std::vector<Vec> cols(n);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t k = cp[j]; k < cp[j + 1]; ++k) {
      const int64_t i = ri[k];
      cols[j].push_back(i);
      if (i != j) cols[i].push_back(j);
    }
  p.cp.assign(n + 1, 0);
  for (int64_t j = 0; j < n; ++j) {
    std::sort(cols[j].begin(), cols[j].end());
    p.cp[j + 1] = p.cp[j] + (int64_t)cols[j].size();
  }
  p.ri.reserve(p.cp[n]);
  for (auto& c : cols) p.ri.insert(p.ri.end(), c.begin(), c.end());
  return p;
}

// P A P^T for a new-to-old permutation: new column j is old column perm[j]
// with every row relabelled old -> new, rows sorted again.
Pattern permute(const Pattern& a, const Vec& perm) {
  const int64_t n = a.n;
  Vec inv(n);
  for (int64_t k = 0; k < n; ++k) inv[perm[k]] = k;
  Pattern p;
  p.n = n;
  p.cp.assign(n + 1, 0);
  p.ri.reserve(a.ri.size());
  for (int64_t j = 0; j < n; ++j) {
    const int64_t o = perm[j];
    const size_t b = p.ri.size();
    for (int64_t k = a.cp[o]; k < a.cp[o + 1]; ++k) p.ri.push_back(inv[a.ri[k]]);
    std::sort(p.ri.begin() + b, p.ri.end());
    p.cp[j + 1] = (int64_t)p.ri.size();
  }
  return p;
}

// Elimination tree by path-compressed ancestor links; parent -1 = root.
Vec etree(const Pattern& a) {
  const int64_t n = a.n;
  Vec parent(n, -1), anc(n);
  for (int64_t j = 0; j < n; ++j) {
    anc[j] = j;
    for (int64_t k = a.cp[j]; k < a.cp[j + 1]; ++k) {
      int64_t i = a.ri[k];
      if (i >= j) continue;
      int64_t r = i;
      while (anc[r] != r) r = anc[r];
      while (i != r) {  // compress the path to the root just found
        const int64_t nx = anc[i];
        anc[i] = r;
        i = nx;
      }
      if (r != j) {
        parent[r] = j;
        anc[r] = j;
      }
    }
  }
  return parent;
}

Vec subtree_sizes(const Vec& parent) {
  Vec sz(parent.size(), 1);
  for (size_t j = 0; j < parent.size(); ++j)
    if (parent[j] >= 0) sz[parent[j]] += sz[j];
  return sz;
}

// Depth-first postorder: roots by ascending subtree size, at every node its
// children by ascending subtree size; with `bias`, the unbiased children
// first, then the biased ones (each group by size).
void postorder(const Vec& parent, const std::vector<char>* bias, Vec& order, Vec& inv) {
  const int64_t n = (int64_t)parent.size();
  std::vector<Vec> kids(n);
  Vec roots;
  for (int64_t j = 0; j < n; ++j) (parent[j] >= 0 ? kids[parent[j]] : roots).push_back(j);
  const Vec sz = subtree_sizes(parent);
  auto by_size = [&](Vec& v) {
    std::stable_sort(v.begin(), v.end(), [&](int64_t a, int64_t b) { return sz[a] < sz[b]; });
  };
  auto arrange = [&](const Vec& ch) {
    if (!bias) {
      Vec v = ch;
      by_size(v);
      return v;
    }
    Vec early, late;
    for (int64_t c : ch) ((*bias)[c] ? late : early).push_back(c);
    by_size(early);
    by_size(late);
    early.insert(early.end(), late.begin(), late.end());
    return early;
  };
  by_size(roots);
  order.clear();
  order.reserve(n);
  struct Frame {
    int64_t node;
    Vec ch;
    size_t next;
  };
  std::vector<Frame> st;
  for (int64_t r : roots) {
    st.push_back({r, arrange(kids[r]), 0});
    while (!st.empty()) {
      Frame& f = st.back();
      if (f.next < f.ch.size()) {
        const int64_t c = f.ch[f.next++];
        st.push_back({c, arrange(kids[c]), 0});
      } else {
        order.push_back(f.node);
        st.pop_back();
      }
    }
  }
  inv.assign(n, 0);
  for (int64_t k = 0; k < n; ++k) inv[order[k]] = k;
}

// Exact column counts of L (diagonal included): row i of L holds column k iff
// k lies on the etree path from some a_ik (k < i) up to i, so walking those
// paths once per row, stopping at nodes already counted for the row, counts
// every off-diagonal entry of L exactly once.
Vec column_counts(const Pattern& a, const Vec& parent) {
  const int64_t n = a.n;
  Vec cnt(n, 1), mark(n, -1);
  for (int64_t i = 0; i < n; ++i) {
    mark[i] = i;
    for (int64_t q = a.cp[i]; q < a.cp[i + 1]; ++q) {
      int64_t k = a.ri[q];
      if (k >= i) continue;
      while (mark[k] != i) {
        mark[k] = i;
        cnt[k]++;
        k = parent[k];
      }
    }
  }
  return cnt;
}

// Renumber for bushy trees (>= 5% of the internal nodes have two or more
// children), Adjacency for paths.
bool bushy(const Vec& parent) {
  const int64_t n = (int64_t)parent.size();
  if (n == 0) return false;
  Vec nch(n, 0);
  for (int64_t p : parent)
    if (p >= 0) nch[p]++;
  int64_t internal = 0, multi = 0;
  for (int64_t c : nch) {
    internal += c > 0;
    multi += c >= 2;
  }
  if (internal == 0) return false;
  return (double)multi / (double)internal >= 0.05;
}

struct Fund {
  Vec start, ncol, parent;  // parent fundamental supernode or -1
};

// Column j continues the run of j-1 when j is j-1's etree parent, its count
// is one less, and j-1 is its only child.
Fund fundamental(const Vec& parent, const Vec& cc) {
  const int64_t n = (int64_t)parent.size();
  Fund f;
  if (n == 0) return f;
  Vec nch(n, 0), id(n, 0);
  for (int64_t p : parent)
    if (p >= 0) nch[p]++;
  f.start.push_back(0);
  for (int64_t j = 1; j < n; ++j) {
    if (parent[j - 1] == j && cc[j] + 1 == cc[j - 1] && nch[j] == 1) {
      id[j] = id[j - 1];
    } else {
      id[j] = (int64_t)f.start.size();
      f.start.push_back(j);
    }
  }
  const int64_t m = (int64_t)f.start.size();
  f.ncol.assign(m, 0);
  f.parent.assign(m, -1);
  for (int64_t j = 0; j < n; ++j) f.ncol[id[j]]++;
  for (int64_t s = 0; s < m; ++s) {
    const int64_t last = f.start[s] + f.ncol[s] - 1;
    if (parent[last] >= 0) f.parent[s] = id[parent[last]];
  }
  return f;
}

// Columns of every fundamental supernode that the size / trivial-chain rule
// would merge into its parent (adjacency not required).
std::vector<char> merge_bias(const Vec& parent, const Vec& cc, int64_t nemin) {
  std::vector<char> bias(parent.size(), 0);
  const Fund f = fundamental(parent, cc);
  for (size_t s = 0; s < f.start.size(); ++s) {
    const int64_t p = f.parent[s];
    if (p < 0) continue;
    const int64_t cn = f.ncol[s], pn = f.ncol[p];
    const int64_t last = f.start[s] + cn - 1;
    const bool chain = pn == 1 && cc[f.start[p]] + 1 == cc[last];
    const bool small = cn < nemin && pn < nemin;
    if (chain || small)
      for (int64_t c = f.start[s]; c < f.start[s] + cn; ++c) bias[c] = 1;
  }
  return bias;
}

struct Snode {
  int64_t first, ncol, nrow_cc;
  Vec children;
};

int64_t root_of(int64_t s, const Vec& into) {
  while (into[s] >= 0) s = into[s];
  return s;
}

std::vector<Snode> supernodes(const Vec& parent, const Vec& cc, int64_t nemin, int64_t relax_w, int64_t relax_r,
                              bool renumber) {
  const int64_t n = (int64_t)parent.size();
  std::vector<Snode> out;
  if (n == 0) return out;
  const bool relax = relax_w > 0 && n >= 1024;  // RELAX_MIN_N
  const Fund f = fundamental(parent, cc);
  const int64_t m = (int64_t)f.start.size();
  Vec into(m, -1), first = f.start, width = f.ncol;
  const int64_t cap = n >= 1024 ? std::min<int64_t>(n / 20, 2048) : INT64_MAX;
  const bool reverse = relax || renumber;
  for (int64_t it = 0; it < m; ++it) {
    const int64_t s = reverse ? m - 1 - it : it;
    const int64_t p = f.parent[s];
    if (p < 0 || into[s] >= 0) continue;
    const int64_t rs = s, rp = root_of(p, into);
    if (rs == rp) continue;
    const int64_t sf = first[rs], sn = width[rs], pf = first[rp], pn = width[rp];
    if (sf + sn != pf) continue;  // the merged columns must stay contiguous
    const int64_t last = sf + sn - 1;
    const bool chain = pn == 1 && cc[pf] + 1 == cc[last];
    const bool small = sn < nemin && pn < nemin;
    const int64_t merged = sn + pn;
    const bool over_cap = f.parent[rp] < 0 && merged > cap;
    bool relaxed = false;
    if (relax) {
      const int64_t extra = std::max<int64_t>(cc[last] - (1 + cc[pf]), 0);
      relaxed = merged <= relax_w && extra <= relax_r;
    }
    if ((chain || small || relaxed) && !over_cap) {
      into[rs] = rp;
      width[rp] = merged;
      first[rp] = sf;
    }
  }
  Vec newid(m, -1);
  for (int64_t s = 0; s < m; ++s) {
    if (into[s] >= 0) continue;
    newid[s] = (int64_t)out.size();
    out.push_back({first[s], width[s], std::max(cc[first[s]], width[s]), {}});
  }
  for (int64_t s = 0; s < m; ++s) {
    if (into[s] >= 0 || f.parent[s] < 0) continue;
    const int64_t rp = root_of(f.parent[s], into);
    if (rp != s) out[newid[rp]].children.push_back(newid[s]);
  }
  return out;
}

}  // namespace orc_sym

extern "C" {

// The structure of the reference's analyze_with for a given ordering output
// `ord` (new-to-old, before the postorder): final permutation, elimination
// tree, column counts, supernodes (first column, width, row-structure
// height), their children (in supernode order) and assembly-tree levels.
// Arrays sized n (supernode arrays: at most n used; child_ptr n + 1).
// Returns the number of supernodes; *renumbered = 1 when the merge-biased
// postorder was applied.
int64_t oracle_symbolic(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, const int64_t* ord,
                        int64_t nemin, int64_t relax_w, int64_t relax_r, int64_t* perm, int64_t* parent,
                        int64_t* col_counts, int64_t* sn_first, int64_t* sn_ncol, int64_t* sn_nrow,
                        int64_t* sn_level, int64_t* child_ptr, int64_t* child_idx, int32_t* renumbered) {
  using namespace orc_sym;
  *renumbered = 0;
  if (n == 0) {
    child_ptr[0] = 0;
    return 0;
  }
  const Pattern full = full_from_lower(n, col_ptr, row_idx);
  const Vec o(ord, ord + n);
  // postorder of the ordered pattern's etree, composed with the ordering
  const Vec par0 = etree(permute(full, o));
  Vec post, post_inv;
  postorder(par0, nullptr, post, post_inv);
  Vec p(n);
  for (int64_t k = 0; k < n; ++k) p[k] = o[post[k]];
  Pattern pat = permute(full, p);
  Vec par(n);
  for (int64_t k = 0; k < n; ++k) {
    const int64_t q = par0[post[k]];
    par[k] = q >= 0 ? post_inv[q] : -1;
  }
  Vec cc = column_counts(pat, par);
  const bool renumber = bushy(par);
  if (renumber) {
    const std::vector<char> bias = merge_bias(par, cc, nemin);
    if (std::any_of(bias.begin(), bias.end(), [](char b) { return b != 0; })) {
      Vec post2, post2_inv;
      postorder(par, &bias, post2, post2_inv);
      Vec p2(n);
      for (int64_t k = 0; k < n; ++k) p2[k] = p[post2[k]];
      p = p2;
      pat = permute(full, p);
      par = etree(pat);
      cc = column_counts(pat, par);
      *renumbered = 1;
    }
  }
  const std::vector<Snode> sn = supernodes(par, cc, nemin, relax_w, relax_r, renumber);
  const int64_t ns = (int64_t)sn.size();
  // row structures: own columns, then the sorted union of the own columns'
  // rows below the block and the children's off-diagonal rows
  std::vector<Vec> rs(ns);
  Vec level(ns, 0);
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t f = sn[s].first, end = sn[s].first + sn[s].ncol;
    Vec tr;
    for (int64_t j = f; j < end; ++j)
      for (int64_t k = pat.cp[j]; k < pat.cp[j + 1]; ++k)
        if (pat.ri[k] >= end) tr.push_back(pat.ri[k]);
    for (int64_t c : sn[s].children) {
      for (size_t q = (size_t)sn[c].ncol; q < rs[c].size(); ++q)
        if (rs[c][q] >= end) tr.push_back(rs[c][q]);
      level[s] = std::max(level[s], level[c] + 1);
    }
    std::sort(tr.begin(), tr.end());
    tr.erase(std::unique(tr.begin(), tr.end()), tr.end());
    Vec& r = rs[s];
    for (int64_t j = f; j < end; ++j) r.push_back(j);
    r.insert(r.end(), tr.begin(), tr.end());
  }
  std::copy(p.begin(), p.end(), perm);
  std::copy(par.begin(), par.end(), parent);
  std::copy(cc.begin(), cc.end(), col_counts);
  int64_t q = 0;
  for (int64_t s = 0; s < ns; ++s) {
    sn_first[s] = sn[s].first;
    sn_ncol[s] = sn[s].ncol;
    sn_nrow[s] = (int64_t)rs[s].size();
    sn_level[s] = level[s];
    child_ptr[s] = q;
    for (int64_t c : sn[s].children) child_idx[q++] = c;
  }
  child_ptr[ns] = q;
  return ns;
}

}  // extern "C"
