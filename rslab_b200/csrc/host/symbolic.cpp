// Host symbolic analysis for the supernodal LDL^T path.
//
// Restates the reference pipeline that fixes the factor's structure:
//   symmetric pattern -> ordering (AMD) -> etree -> size-sorted postorder ->
//   composed permutation -> relabelled etree -> exact column counts ->
//   amalgamation-strategy pick -> optional merge-biased renumbering ->
//   fundamental supernodes + (relaxed) amalgamation -> Hybrid-Liu child order
//   -> assembly-tree levels -> left-looking row structures and update lists.
// References: src/symbolic/mod.rs:861-1215 (prefix/finish),
// src/symbolic/supernode.rs:222-723, src/ordering/postorder.rs:22-143,
// src/ordering/elimination_tree.rs:28-64, src/symbolic/column_counts.rs:97-183,
// src/numeric/multifrontal_ldlt.rs:1684-1808 (analyze_with_inner),
// :2121-2152 (row structures), :3380-3401 (update lists).
// The structure is value independent, so it is computed once per pattern and
// reused by every numeric factorisation.
#include "host.hpp"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <numeric>

namespace rslab {

void validate_lower_csc(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, int64_t nnz) {
  if (n < 0) throw RslabError(Status::InvalidInput, "n must be non-negative");
  if (col_ptr[0] != 0) throw RslabError(Status::InvalidInput, "col_ptr[0] must be 0");
  if (col_ptr[n] != nnz) throw RslabError(Status::InvalidInput, "col_ptr[n] != nnz");
  for (int64_t j = 0; j < n; ++j)
    if (col_ptr[j + 1] < col_ptr[j])
      throw RslabError(Status::InvalidInput,
                       "col_ptr not monotonically non-decreasing at column " + std::to_string(j));
  for (int64_t j = 0; j < n; ++j) {
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
      int64_t i = row_idx[k];
      if (i < 0 || i >= n)
        throw RslabError(Status::InvalidInput,
                         "row index " + std::to_string(i) + " out of bounds in column " + std::to_string(j));
      if (i < j)
        throw RslabError(Status::InvalidInput, "row index " + std::to_string(i) + " in column " +
                                                   std::to_string(j) + " is upper-triangle");
      if (k > col_ptr[j] && row_idx[k] <= row_idx[k - 1])
        throw RslabError(Status::InvalidInput, "row indices not sorted in column " + std::to_string(j));
    }
  }
}

CscPattern checked_full_pattern(int64_t n, const int64_t* col_ptr, const int64_t* row_idx) {
  if (n < 0) throw RslabError(Status::InvalidInput, "n must be non-negative");
  if (n > INT32_MAX) throw RslabError(Status::InvalidInput, "n exceeds the 32-bit index range");
  if (!col_ptr) throw RslabError(Status::InvalidInput, "null col_ptr");
  if (col_ptr[0] != 0) throw RslabError(Status::InvalidInput, "col_ptr[0] must be 0");
  for (int64_t j = 0; j < n; ++j)
    if (col_ptr[j + 1] < col_ptr[j])
      throw RslabError(Status::InvalidInput,
                       "col_ptr not monotonically non-decreasing at column " + std::to_string(j));
  if (col_ptr[n] > INT32_MAX) throw RslabError(Status::InvalidInput, "nnz exceeds the 32-bit index range");
  if (col_ptr[n] > 0 && !row_idx) throw RslabError(Status::InvalidInput, "null row_idx");
  CscPattern p;
  p.n = n;
  p.col_ptr.assign(n + 1, 0);
  p.row_idx.reserve(col_ptr[n]);
  for (int64_t j = 0; j < n; ++j) {
    int64_t last = -1;
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
      const int64_t i = row_idx[k];
      if (i < 0 || i >= n)
        throw RslabError(Status::InvalidInput,
                         "row index " + std::to_string(i) + " out of bounds in column " + std::to_string(j));
      if (i < last) throw RslabError(Status::InvalidInput, "row indices not sorted in column " + std::to_string(j));
      if (i != last) p.row_idx.push_back(i);  // sorted input: duplicates are adjacent
      last = i;
    }
    p.col_ptr[j + 1] = (int64_t)p.row_idx.size();
  }
  // structural symmetry: entry (i, j) needs (j, i).  The transpose of a
  // column-sorted pattern, filled column by column, is row-sorted too, so the
  // two index arrays must be equal.
  std::vector<int64_t> tp(n + 1, 0), ti(p.row_idx.size());
  for (int64_t i : p.row_idx) tp[i + 1]++;
  for (int64_t j = 0; j < n; ++j) tp[j + 1] += tp[j];
  std::vector<int64_t> fill(tp.begin(), tp.end() - 1);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) ti[fill[p.row_idx[k]]++] = j;
  for (int64_t j = 0; j < n; ++j)
    if (tp[j + 1] != p.col_ptr[j + 1] ||
        !std::equal(ti.begin() + tp[j], ti.begin() + tp[j + 1], p.row_idx.begin() + p.col_ptr[j]))
      throw RslabError(Status::InvalidInput,
                       "pattern is not structurally symmetric (first at column " + std::to_string(j) + ")");
  return p;
}

CscPattern symmetric_pattern(int64_t n, const int64_t* col_ptr, const int64_t* row_idx) {
  CscPattern p;
  p.n = n;
  std::vector<int64_t> cnt(n, 0);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
      int64_t i = row_idx[k];
      cnt[j]++;
      if (i != j) cnt[i]++;
    }
  p.col_ptr.assign(n + 1, 0);
  for (int64_t j = 0; j < n; ++j) p.col_ptr[j + 1] = p.col_ptr[j] + cnt[j];
  p.row_idx.assign(p.col_ptr[n], 0);
  std::vector<int64_t> off(p.col_ptr.begin(), p.col_ptr.end() - 1);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
      int64_t i = row_idx[k];
      p.row_idx[off[j]++] = i;
      if (i != j) p.row_idx[off[i]++] = j;
    }
  for (int64_t j = 0; j < n; ++j) std::sort(p.row_idx.begin() + p.col_ptr[j], p.row_idx.begin() + p.col_ptr[j + 1]);
  return p;
}

CscPattern permute_pattern(const CscPattern& pat, const std::vector<int64_t>& perm) {
  const int64_t n = pat.n;
  std::vector<int64_t> inv(n);
  for (int64_t k = 0; k < n; ++k) inv[perm[k]] = k;
  CscPattern out;
  out.n = n;
  out.col_ptr.assign(n + 1, 0);
  for (int64_t oj = 0; oj < n; ++oj) out.col_ptr[inv[oj] + 1] = pat.col_ptr[oj + 1] - pat.col_ptr[oj];
  for (int64_t j = 0; j < n; ++j) out.col_ptr[j + 1] += out.col_ptr[j];
  out.row_idx.assign(out.col_ptr[n], 0);
  for (int64_t oj = 0; oj < n; ++oj) {
    int64_t nj = inv[oj];
    int64_t dst = out.col_ptr[nj];
    for (int64_t k = pat.col_ptr[oj]; k < pat.col_ptr[oj + 1]; ++k) out.row_idx[dst++] = inv[pat.row_idx[k]];
  }
  for (int64_t j = 0; j < n; ++j)
    std::sort(out.row_idx.begin() + out.col_ptr[j], out.row_idx.begin() + out.col_ptr[j + 1]);
  return out;
}

std::vector<int64_t> etree_from_pattern(const CscPattern& pat) {
  const int64_t n = pat.n;
  std::vector<int64_t> parent(n, -1), anc(n, 0);
  for (int64_t j = 0; j < n; ++j) {
    anc[j] = j;
    for (int64_t k = pat.col_ptr[j]; k < pat.col_ptr[j + 1]; ++k) {
      int64_t i = pat.row_idx[k];
      if (i >= j) continue;
      int64_t r = i;
      while (anc[r] != r) r = anc[r];
      int64_t node = i;
      while (node != r) {
        int64_t nx = anc[node];
        anc[node] = r;
        node = nx;
      }
      if (r != j) {
        parent[r] = j;
        anc[r] = j;
      }
    }
  }
  return parent;
}

namespace {

// Sort by ascending key with ties kept in input order.  The reference uses an
// unstable sort, which is an insertion sort (hence stable) for slices of at
// most 20 elements; longer child lists with tied keys are counted so a caller
// can see where the tie order might differ.
static std::atomic<int64_t> g_long_tie_lists{0};
void sort_by_size(std::vector<int64_t>& v, const std::vector<int64_t>& sizes) {
  std::stable_sort(v.begin(), v.end(), [&](int64_t a, int64_t b) { return sizes[a] < sizes[b]; });
  if (v.size() > 20)
    for (size_t i = 1; i < v.size(); ++i)
      if (sizes[v[i]] == sizes[v[i - 1]]) {
        ++g_long_tie_lists;
        break;
      }
}

}  // namespace

void etree_postorder(const std::vector<int64_t>& parent, const std::vector<uint8_t>* bias,
                     std::vector<int64_t>& post, std::vector<int64_t>& post_inv) {
  const int64_t n = (int64_t)parent.size();
  post.clear();
  post.reserve(n);
  post_inv.assign(n, 0);
  if (n == 0) return;
  std::vector<std::vector<int64_t>> children(n);
  std::vector<int64_t> sizes(n, 1), roots;
  for (int64_t j = 0; j < n; ++j)
    if (parent[j] >= 0) children[parent[j]].push_back(j);
  for (int64_t j = 0; j < n; ++j)
    if (parent[j] >= 0) sizes[parent[j]] += sizes[j];
  for (int64_t j = 0; j < n; ++j)
    if (parent[j] < 0) roots.push_back(j);
  sort_by_size(roots, sizes);
  auto ordered = [&](int64_t node) {
    const auto& ch = children[node];
    if (!bias) {
      std::vector<int64_t> v(ch);
      sort_by_size(v, sizes);
      return v;
    }
    std::vector<int64_t> early, late;
    for (int64_t c : ch) ((*bias)[c] ? late : early).push_back(c);
    sort_by_size(early, sizes);
    sort_by_size(late, sizes);
    early.insert(early.end(), late.begin(), late.end());
    return early;
  };
  struct Frame {
    int64_t node;
    std::vector<int64_t> kids;
    size_t idx;
  };
  std::vector<Frame> stack;
  for (int64_t root : roots) {
    stack.push_back({root, ordered(root), 0});
    while (!stack.empty()) {
      Frame& f = stack.back();
      if (f.idx < f.kids.size()) {
        int64_t c = f.kids[f.idx++];
        stack.push_back({c, ordered(c), 0});
      } else {
        post.push_back(f.node);
        stack.pop_back();
      }
    }
  }
  for (int64_t k = 0; k < n; ++k) post_inv[post[k]] = k;
}

std::vector<int64_t> column_counts(const CscPattern& pat, const std::vector<int64_t>& parent) {
  // Gilbert-Ng-Peyton row-subtree counting on the plain DFS postorder.
  const int64_t n = pat.n;
  std::vector<int64_t> counts(n);
  if (n == 0) return counts;
  std::vector<std::vector<int64_t>> children(n);
  for (int64_t j = 0; j < n; ++j)
    if (parent[j] >= 0) children[parent[j]].push_back(j);
  std::vector<int64_t> post;
  post.reserve(n);
  {
    std::vector<int64_t> nextc(n, 0), stack;
    for (int64_t r = 0; r < n; ++r) {
      if (parent[r] >= 0) continue;
      stack.push_back(r);
      while (!stack.empty()) {
        int64_t node = stack.back();
        if ((size_t)nextc[node] < children[node].size()) {
          stack.push_back(children[node][nextc[node]++]);
        } else {
          post.push_back(node);
          stack.pop_back();
        }
      }
    }
  }
  std::vector<int64_t> post_of(n), first(n);
  for (int64_t k = 0; k < n; ++k) post_of[post[k]] = k;
  first = post_of;
  for (int64_t node : post)
    if (parent[node] >= 0 && first[node] < first[parent[node]]) first[parent[node]] = first[node];
  std::vector<int64_t> delta(n), maxfirst(n, -1), prevleaf(n, -1), anc(n);
  for (int64_t i = 0; i < n; ++i) {
    delta[i] = children[i].empty() ? 1 : 0;
    anc[i] = i;
  }
  for (int64_t i : post) {
    if (parent[i] >= 0) delta[parent[i]] -= 1;
    int64_t fi = first[i];
    for (int64_t k = pat.col_ptr[i]; k < pat.col_ptr[i + 1]; ++k) {
      int64_t q = pat.row_idx[k];
      if (q <= i) continue;
      if (fi > maxfirst[q]) {
        delta[i] += 1;
        int64_t pl = prevleaf[q];
        if (pl != -1) {
          int64_t r = pl;
          while (anc[r] != r) r = anc[r];
          int64_t cur = pl;
          while (cur != r) {
            int64_t nx = anc[cur];
            anc[cur] = r;
            cur = nx;
          }
          delta[r] -= 1;
        }
        prevleaf[q] = i;
        maxfirst[q] = fi;
      }
    }
    if (parent[i] >= 0) anc[i] = parent[i];
  }
  for (int64_t i : post)
    if (parent[i] >= 0) delta[parent[i]] += delta[i];
  for (int64_t i = 0; i < n; ++i) counts[i] = delta[i];
  return counts;
}

namespace {

struct Fundamental {
  std::vector<int64_t> starts, ncols, parent;
};

// Consecutive columns j-1, j share a supernode when parent[j-1]==j, the
// counts drop by one and j has exactly one child (supernode.rs:625-676).
Fundamental find_fundamental(const std::vector<int64_t>& parent, const std::vector<int64_t>& cc) {
  const int64_t n = (int64_t)parent.size();
  Fundamental f;
  if (n == 0) return f;
  std::vector<int64_t> sid(n, 0), nch(n, 0);
  for (int64_t j = 0; j < n; ++j)
    if (parent[j] >= 0) nch[parent[j]]++;
  f.starts.push_back(0);
  for (int64_t j = 1; j < n; ++j) {
    bool same = parent[j - 1] == j && cc[j] + 1 == cc[j - 1] && nch[j] == 1;
    if (same) {
      sid[j] = sid[j - 1];
    } else {
      sid[j] = (int64_t)f.starts.size();
      f.starts.push_back(j);
    }
  }
  const int64_t ns = (int64_t)f.starts.size();
  f.ncols.assign(ns, 0);
  f.parent.assign(ns, -1);
  for (int64_t j = 0; j < n; ++j) f.ncols[sid[j]]++;
  for (int64_t s = 0; s < ns; ++s) {
    int64_t last = f.starts[s] + f.ncols[s] - 1;
    if (parent[last] >= 0) f.parent[s] = sid[parent[last]];
  }
  return f;
}

// Adjacency vs renumber pick from the share of multi-child etree nodes
// (supernode.rs:222-248).
bool pick_renumber(const std::vector<int64_t>& parent) {
  const int64_t n = (int64_t)parent.size();
  if (n == 0) return false;
  std::vector<int64_t> cc(n, 0);
  for (int64_t p : parent)
    if (p >= 0) cc[p]++;
  int64_t leaves = 0, multi = 0;
  for (int64_t c : cc) {
    if (c == 0) ++leaves;
    if (c >= 2) ++multi;
  }
  int64_t internal = n - leaves;
  if (internal == 0) return false;
  return (double)multi / (double)internal >= 0.05;
}

// Desired merges under the chain / size rules, no adjacency requirement
// (supernode.rs:693-723).
std::vector<uint8_t> predict_merges(const std::vector<int64_t>& parent, const std::vector<int64_t>& cc,
                                    int64_t nemin) {
  const int64_t n = (int64_t)parent.size();
  std::vector<uint8_t> bias(n, 0);
  if (n == 0) return bias;
  Fundamental f = find_fundamental(parent, cc);
  for (size_t s = 0; s < f.starts.size(); ++s) {
    int64_t p = f.parent[s];
    if (p < 0) continue;
    int64_t cn = f.ncols[s], pn = f.ncols[p];
    int64_t sf = f.starts[s], pf = f.starts[p];
    int64_t clast = sf + cn - 1;
    bool chain = pn == 1 && cc[pf] + 1 == cc[clast];
    bool size = cn < nemin && pn < nemin;
    if (chain || size)
      for (int64_t c = sf; c < sf + cn; ++c) bias[c] = 1;
  }
  return bias;
}

int64_t find_root(int64_t s, const std::vector<int64_t>& merged) {
  while (merged[s] >= 0) s = merged[s];
  return s;
}

// Fundamental supernodes + chain / size / relaxed amalgamation with the
// root-width cap (supernode.rs:267-465).
std::vector<Supernode> find_supernodes(const std::vector<int64_t>& parent, const std::vector<int64_t>& cc,
                                       const AnalyzeOptions& opt, bool renumber_strategy) {
  const int64_t n = (int64_t)parent.size();
  std::vector<Supernode> out;
  if (n == 0) return out;
  const bool relax = opt.relax && n >= 1024;
  Fundamental f = find_fundamental(parent, cc);
  const int64_t ns = (int64_t)f.starts.size();
  std::vector<int64_t> merged(ns, -1);
  std::vector<int64_t> first = f.starts, ncols = f.ncols;
  const bool reverse = relax || renumber_strategy;
  const int64_t root_cap = n >= 1024 ? std::min<int64_t>(n / 20, 2048) : INT64_MAX;
  for (int64_t it = 0; it < ns; ++it) {
    int64_t s = reverse ? ns - 1 - it : it;
    int64_t p = f.parent[s];
    if (p < 0) continue;
    if (find_root(s, merged) != s) continue;
    int64_t rs = s, rp = find_root(p, merged);
    if (rs == rp) continue;
    int64_t sf = first[rs], sn = ncols[rs], pf = first[rp];
    if (sf + sn != pf) continue;
    int64_t cn = ncols[rs], pn = ncols[rp];
    bool chain = pn == 1 && cc[pf] + 1 == cc[sf + sn - 1];
    bool size = cn < opt.nemin && pn < opt.nemin;
    bool parent_is_root = f.parent[rp] < 0;
    int64_t mn = cn + pn;
    bool cap_exceeded = parent_is_root && mn > root_cap;
    bool relaxed = false;
    if (relax) {
      int64_t clast = sf + sn - 1;
      int64_t extra = cc[clast] - (1 + cc[pf]);
      if (extra < 0) extra = 0;
      relaxed = mn <= opt.relax_max_width && extra <= opt.relax_max_extra_rows;
    }
    if ((chain || size || relaxed) && !cap_exceeded) {
      merged[rs] = rp;
      ncols[rp] = mn;
      first[rp] = sf;
    }
  }
  std::vector<int64_t> newid(ns, 0);
  for (int64_t s = 0; s < ns; ++s) {
    if (merged[s] >= 0) continue;
    Supernode sn;
    sn.first_col = first[s];
    sn.ncol = ncols[s];
    sn.nrow_est = std::max(cc[first[s]], ncols[s]);
    newid[s] = (int64_t)out.size();
    out.push_back(sn);
  }
  for (int64_t s = 0; s < ns; ++s) {
    if (merged[s] >= 0) continue;
    int64_t p = f.parent[s];
    if (p >= 0) {
      int64_t rp = find_root(p, merged);
      if (rp != s) out[newid[rp]].children.push_back(newid[s]);
    }
  }
  return out;
}

}  // namespace

double supernode_flops(int64_t r, int64_t c) {
  double tot = 0;
  for (int64_t m = r - c + 1; m <= r; ++m) tot += (double)m * (double)m - 1.0;
  return tot;
}

Symbolic analyze(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, const AnalyzeOptions& opt) {
  Symbolic S;
  S.n = n;
  S.nnz = col_ptr[n];
  if (n == 0) return S;
  CscPattern full = symmetric_pattern(n, col_ptr, row_idx);

  // Step 1: fill-reducing ordering.
  std::vector<int64_t> ord(n);
  switch (opt.ordering) {
    case Ordering::Amd:
      ord = amd_order(full, &S.amd);
      break;
    case Ordering::MetisND:
      ord = metis_nd_order(full);
      break;
    case Ordering::Natural:
      std::iota(ord.begin(), ord.end(), 0);
      break;
    case Ordering::Given: {
      if (!opt.given_perm) throw RslabError(Status::InvalidInput, "given ordering without a permutation");
      std::vector<uint8_t> seen(n, 0);
      for (int64_t k = 0; k < n; ++k) {
        int64_t v = opt.given_perm[k];
        if (v < 0 || v >= n || seen[v]) throw RslabError(Status::InvalidInput, "given ordering is not a permutation");
        seen[v] = 1;
        ord[k] = v;
      }
      break;
    }
    default:
      throw RslabError(Status::InvalidInput, "ordering method not available in this build");
  }
  S.resolved_ordering = (int)opt.ordering;

  // Steps 2-5: etree of the ordered pattern, size-sorted postorder, composed
  // permutation, relabelled etree.
  CscPattern ord_pat = permute_pattern(full, ord);
  std::vector<int64_t> ord_parent = etree_from_pattern(ord_pat);
  std::vector<int64_t> post, post_inv;
  etree_postorder(ord_parent, nullptr, post, post_inv);
  S.perm.resize(n);
  for (int64_t k = 0; k < n; ++k) S.perm[k] = ord[post[k]];
  S.permuted = permute_pattern(full, S.perm);
  S.parent.assign(n, -1);
  for (int64_t k = 0; k < n; ++k) {
    int64_t op = ord_parent[post[k]];
    S.parent[k] = op >= 0 ? post_inv[op] : -1;
  }
  // Step 6: column counts.
  S.col_counts = column_counts(S.permuted, S.parent);

  // Amalgamation strategy and the merge-biased renumbering.
  bool renumber = pick_renumber(S.parent);
  if (renumber) {
    std::vector<uint8_t> bias = predict_merges(S.parent, S.col_counts, opt.nemin);
    bool any = false;
    for (uint8_t b : bias) any |= b != 0;
    if (any) {
      std::vector<int64_t> post2, post2_inv;
      etree_postorder(S.parent, &bias, post2, post2_inv);
      std::vector<int64_t> np(n);
      for (int64_t k = 0; k < n; ++k) np[k] = S.perm[post2[k]];
      S.perm = np;
      S.permuted = permute_pattern(full, S.perm);
      S.parent = etree_from_pattern(S.permuted);
      S.col_counts = column_counts(S.permuted, S.parent);
      S.renumbered = 1;
    }
  }
  S.perm_inv.assign(n, 0);
  for (int64_t k = 0; k < n; ++k) S.perm_inv[S.perm[k]] = k;
  S.factor_nnz_sym = 0;
  for (int64_t c : S.col_counts) S.factor_nnz_sym += c;

  // Step 7: supernodes.
  S.sn = find_supernodes(S.parent, S.col_counts, opt, renumber);
  const int64_t ns = (int64_t)S.sn.size();

  // Hybrid-Liu child reordering where the contribution stack is large
  // (multifrontal_ldlt.rs:1755-1784).  A scheduling hint only.
  if (opt.hybrid_liu) {
    std::vector<double> cb(ns, 0.0), peak(ns, 0.0);
    for (int64_t s = 0; s < ns; ++s) {
      double cn = (double)(S.sn[s].nrow_est - S.sn[s].ncol);
      cb[s] = cn * cn;
      auto& kids = S.sn[s].children;
      double stack_total = 0;
      for (int64_t c : kids) stack_total += cb[c];
      if (stack_total >= 4000000.0)
        std::stable_sort(kids.begin(), kids.end(),
                         [&](int64_t a, int64_t b) { return (peak[b] - cb[b]) < (peak[a] - cb[a]); });
      double acc = 0, pk = 0;
      for (int64_t c : kids) {
        pk = std::max(pk, acc + peak[c]);
        acc += cb[c];
      }
      peak[s] = std::max(std::max(pk, acc), cb[s]);
    }
  }

  // Assembly-tree levels (multifrontal_ldlt.rs:1786-1801).
  S.level.assign(ns, 0);
  int64_t maxl = 0;
  for (int64_t s = 0; s < ns; ++s) {
    int64_t lv = 0;
    for (int64_t c : S.sn[s].children) lv = std::max(lv, S.level[c] + 1);
    S.level[s] = lv;
    maxl = std::max(maxl, lv);
  }
  S.by_level.assign(maxl + 1, {});
  for (int64_t s = 0; s < ns; ++s) S.by_level[S.level[s]].push_back(s);

  // Row structures: own columns ++ sorted union of the column patterns'
  // trailing rows and the children's off-diagonal rows.
  S.rs_ptr.assign(ns + 1, 0);
  std::vector<std::vector<int64_t>> rs(ns);
  for (int64_t s = 0; s < ns; ++s) {
    const Supernode& sn = S.sn[s];
    int64_t own_last = sn.first_col + sn.ncol;
    std::vector<int64_t> trailing;
    for (int64_t j = sn.first_col; j < own_last; ++j)
      for (int64_t k = S.permuted.col_ptr[j]; k < S.permuted.col_ptr[j + 1]; ++k)
        if (S.permuted.row_idx[k] >= own_last) trailing.push_back(S.permuted.row_idx[k]);
    for (int64_t c : sn.children) {
      int64_t nck = S.sn[c].ncol;
      for (size_t q = (size_t)nck; q < rs[c].size(); ++q)
        if (rs[c][q] >= own_last) trailing.push_back(rs[c][q]);
    }
    std::sort(trailing.begin(), trailing.end());
    trailing.erase(std::unique(trailing.begin(), trailing.end()), trailing.end());
    rs[s].reserve(sn.ncol + trailing.size());
    for (int64_t j = sn.first_col; j < own_last; ++j) rs[s].push_back(j);
    rs[s].insert(rs[s].end(), trailing.begin(), trailing.end());
    S.rs_ptr[s + 1] = S.rs_ptr[s] + (int64_t)rs[s].size();
  }
  S.rs.resize(S.rs_ptr[ns]);
  for (int64_t s = 0; s < ns; ++s) std::copy(rs[s].begin(), rs[s].end(), S.rs.begin() + S.rs_ptr[s]);

  // Update lists: k updates s iff an off-diagonal row of k is a column of s,
  // in increasing k; with the landing range [p0,p1) of k's off-diagonal rows.
  std::vector<int64_t> col2sn(n);
  for (int64_t s = 0; s < ns; ++s)
    for (int64_t c = 0; c < S.sn[s].ncol; ++c) col2sn[S.sn[s].first_col + c] = s;
  std::vector<std::vector<int64_t>> ul(ns);
  for (int64_t k = 0; k < ns; ++k) {
    int64_t nck = S.sn[k].ncol;
    int64_t last = -1;
    for (int64_t q = S.rs_ptr[k] + nck; q < S.rs_ptr[k + 1]; ++q) {
      int64_t s = col2sn[S.rs[q]];
      if (s != last) {
        ul[s].push_back(k);
        last = s;
      }
    }
  }
  S.upd_ptr.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s) S.upd_ptr[s + 1] = S.upd_ptr[s] + (int64_t)ul[s].size();
  S.upd.resize(S.upd_ptr[ns]);
  S.upd_p0.resize(S.upd_ptr[ns]);
  S.upd_p1.resize(S.upd_ptr[ns]);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t f0 = S.sn[s].first_col, f1 = f0 + S.sn[s].ncol;
    for (size_t t = 0; t < ul[s].size(); ++t) {
      int64_t k = ul[s][t];
      const int64_t* ok = S.rs.data() + S.rs_ptr[k] + S.sn[k].ncol;
      int64_t nok = S.rs_ptr[k + 1] - S.rs_ptr[k] - S.sn[k].ncol;
      int64_t p0 = std::lower_bound(ok, ok + nok, f0) - ok;
      int64_t p1 = std::lower_bound(ok, ok + nok, f1) - ok;
      int64_t idx = S.upd_ptr[s] + (int64_t)t;
      S.upd[idx] = k;
      S.upd_p0[idx] = p0;
      S.upd_p1[idx] = p1;
    }
  }
  return S;
}

Symbolic merge_independent(const std::vector<Symbolic>& parts) {
  Symbolic M;
  int64_t coff = 0, soff = 0, nlev = 0;
  for (const auto& P : parts) nlev = std::max<int64_t>(nlev, (int64_t)P.by_level.size());
  M.by_level.assign(nlev, {});
  M.permuted.col_ptr.push_back(0);
  M.rs_ptr.push_back(0);
  M.upd_ptr.push_back(0);
  M.resolved_ordering = parts.empty() ? 0 : parts[0].resolved_ordering;
  for (const auto& P : parts) {
    M.n += P.n;
    M.nnz += P.nnz;
    for (int64_t v : P.perm) M.perm.push_back(v + coff);
    for (int64_t v : P.perm_inv) M.perm_inv.push_back(v + coff);
    for (int64_t v : P.parent) M.parent.push_back(v < 0 ? -1 : v + coff);
    M.col_counts.insert(M.col_counts.end(), P.col_counts.begin(), P.col_counts.end());
    const int64_t pbase = (int64_t)M.permuted.row_idx.size();
    for (size_t j = 1; j < P.permuted.col_ptr.size(); ++j) M.permuted.col_ptr.push_back(P.permuted.col_ptr[j] + pbase);
    for (int64_t r : P.permuted.row_idx) M.permuted.row_idx.push_back(r + coff);
    const int64_t ns = (int64_t)P.sn.size();
    for (int64_t s = 0; s < ns; ++s) {
      Supernode x = P.sn[s];
      x.first_col += coff;
      for (auto& c : x.children) c += soff;
      M.sn.push_back(std::move(x));
      const int64_t rb = (int64_t)M.rs.size();
      for (int64_t q = P.rs_ptr[s]; q < P.rs_ptr[s + 1]; ++q) M.rs.push_back(P.rs[q] + coff);
      (void)rb;
      M.rs_ptr.push_back((int64_t)M.rs.size());
      for (int64_t q = P.upd_ptr[s]; q < P.upd_ptr[s + 1]; ++q) {
        M.upd.push_back(P.upd[q] + soff);
        M.upd_p0.push_back(P.upd_p0[q]);
        M.upd_p1.push_back(P.upd_p1[q]);
      }
      M.upd_ptr.push_back((int64_t)M.upd.size());
      M.level.push_back(P.level[s]);
      M.by_level[P.level[s]].push_back(s + soff);
    }
    M.factor_nnz_sym += P.factor_nnz_sym;
    M.renumbered |= P.renumbered;
    M.amd.ncmpa += P.amd.ncmpa;
    M.amd.n_dense += P.amd.n_dense;
    M.amd.ndiv += P.amd.ndiv;
    M.amd.nms_lu += P.amd.nms_lu;
    M.amd.nms_ldl += P.amd.nms_ldl;
    coff += P.n;
    soff += ns;
  }
  M.permuted.n = M.n;
  return M;
}

MemoryEstimate estimate_memory(const Symbolic& S, int64_t value_bytes) {
  MemoryEstimate e;
  e.value_bytes = value_bytes;
  const int64_t ns = (int64_t)S.sn.size();
  auto nrow = [&](int64_t s) { return S.rs_ptr[s + 1] - S.rs_ptr[s]; };
  // the descendants k whose off-diagonal rows land in s, once each (rows are
  // ascending, so the supernodes they land in come in runs)
  std::vector<int64_t> col_sn(S.n, 0);
  for (int64_t s = 0; s < ns; ++s)
    std::fill(col_sn.begin() + S.sn[s].first_col, col_sn.begin() + S.sn[s].first_col + S.sn[s].ncol, s);
  std::vector<std::vector<int64_t>> upd(ns);
  std::vector<int64_t> refc(ns, 0);
  for (int64_t k = 0; k < ns; ++k) {
    int64_t last = -1;
    for (int64_t q = S.rs_ptr[k] + S.sn[k].ncol; q < S.rs_ptr[k + 1]; ++q) {
      const int64_t s = col_sn[S.rs[q]];
      if (s != last) {
        upd[s].push_back(k);
        refc[k]++;
        last = s;
      }
    }
  }
  auto panel_bytes = [&](int64_t s) { return nrow(s) * S.sn[s].ncol * value_bytes; };
  auto compact_bytes = [&](int64_t s) {
    const int64_t nc = S.sn[s].ncol;
    return (nc * (nc + 1) / 2 + (nrow(s) - nc) * nc) * (value_bytes + 8);
  };
  int64_t panels_all = 0, factor_bytes = 0;
  for (int64_t s = 0; s < ns; ++s) {
    panels_all += panel_bytes(s);
    factor_bytes += compact_bytes(s);
  }
  // the refcount free schedule of the left-looking factor, in postorder
  int64_t live = 0, compact = 0, peak = 0;
  for (int64_t s = 0; s < ns; ++s) {
    live += panel_bytes(s);
    for (int64_t k : upd[s])
      if (--refc[k] == 0) {
        live -= panel_bytes(k);
        compact += compact_bytes(k);
      }
    if (refc[s] == 0) {
      live -= panel_bytes(s);
      compact += compact_bytes(s);
    }
    peak = std::max(peak, live + compact);
  }
  const int64_t input_bytes = S.nnz * (value_bytes + 8);
  const int64_t scratch = (panels_all + factor_bytes) / 4 + 32000000;
  e.panels_all_bytes = panels_all;
  e.factor_bytes = factor_bytes;
  e.factor_nnz = factor_bytes / std::max<int64_t>(value_bytes + 8, 1);
  e.panel_live_peak_bytes = std::max<int64_t>(peak, 0);
  e.transient_peak_bytes = panels_all + factor_bytes + input_bytes + scratch;
  int64_t cb_all = 0;  // sum over supernodes of (nrow - ncol)^2 scalars
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t m = nrow(s) - S.sn[s].ncol;
    cb_all += m * m * value_bytes;
  }
  e.mf_transient_peak_bytes = e.transient_peak_bytes + cb_all;
  std::vector<uint64_t> crit(ns, 0);
  uint64_t cp = 0, flops = 0;
  for (int64_t s = 0; s < ns; ++s) {
    const uint64_t nc = (uint64_t)S.sn[s].ncol, nr = (uint64_t)nrow(s);
    const uint64_t ff = nr * nr * nc;
    flops += ff;
    uint64_t cmax = 0;
    for (int64_t c : S.sn[s].children) cmax = std::max(cmax, crit[c]);
    crit[s] = ff + cmax;
    cp = std::max(cp, crit[s]);
  }
  e.factor_flops = flops;
  e.critical_path_flops = cp;
  int64_t width = ns ? 1 : 0;
  for (const auto& l : S.by_level) width = std::max<int64_t>(width, (int64_t)l.size());
  e.max_tree_width = width;
  return e;
}

}  // namespace rslab
