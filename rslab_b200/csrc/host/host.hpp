// Host-side data structures of the B200 LDL^T path: the lower-triangle CSC
// input, the full symmetric pattern, the symbolic analysis (ordering,
// elimination tree, supernodes, row structures, update lists, level sets) and
// the error type that the C ABI turns into a status code.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace rslab {

// Mirrors the reference error enum (src/error.rs:15-55).
enum class Status : int {
  Ok = 0,
  NumericallyRankDeficient = 1,
  InvalidInput = 2,
  DimensionMismatch = 3,
  CudaError = 4,
  NotCertified = 5,
};

struct RslabError : std::runtime_error {
  Status status;
  RslabError(Status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

// Full symmetric sparsity pattern (both triangles, sorted rows), the input of
// the ordering and the elimination tree (src/sparse/csc.rs:24-29).
struct CscPattern {
  int64_t n = 0;
  std::vector<int64_t> col_ptr;
  std::vector<int64_t> row_idx;
};

// Validation of a lower-triangle CSC (src/sparse/csc.rs:157-237).
void validate_lower_csc(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, int64_t nnz);
// Validation of a full symmetric pattern given to an ordering entry point, as
// Graph::from_csc_pattern (crates/rslab-metis/src/graph.rs:51-86) and
// CscPattern::new check it: col_ptr starts at 0 and never decreases, n and
// nnz fit 32-bit indices, rows lie in [0, n) sorted within each column, and
// the pattern is structurally symmetric.  Returns the pattern with adjacent
// duplicate rows dropped; throws InvalidInput otherwise.
CscPattern checked_full_pattern(int64_t n, const int64_t* col_ptr, const int64_t* row_idx);
// Lower triangle -> full symmetric pattern (src/sparse/csc.rs:240-291).
CscPattern symmetric_pattern(int64_t n, const int64_t* col_ptr, const int64_t* row_idx);
// Relabel a full symmetric pattern by a new-to-old permutation
// (src/ordering/amd.rs:21-81).
CscPattern permute_pattern(const CscPattern& pat, const std::vector<int64_t>& perm);

struct AmdStats {
  uint32_t ncmpa = 0, n_dense = 0, n_mass_elim = 0, n_supervar_merge = 0;
  double ndiv = 0, nms_lu = 0, nms_ldl = 0;
};
std::vector<int64_t> amd_order(const CscPattern& pat, AmdStats* stats = nullptr,
                               double dense_alpha = 10.0, bool aggressive = true);
// Multilevel nested dissection with AMD leaves, default options except the
// seed (crates/rslab-metis/src/lib.rs:184 metis_order, :204 metis_order_full);
// new-to-old permutation.
// dense_quotient: the opt-in quasi-dense column quotient (off in the
// reference's defaults), dense_threshold < 0 = max(40, ceil(10 sqrt(n))).
std::vector<int64_t> metis_nd_order(const CscPattern& pat, uint64_t seed = 1, bool dense_quotient = false,
                                    int64_t dense_threshold = -1);

// Elimination tree: parent[j] > j or -1 (src/ordering/elimination_tree.rs:28-64).
std::vector<int64_t> etree_from_pattern(const CscPattern& pat);
// Children-by-ascending-subtree-size postorder, optionally merge-biased
// (src/ordering/postorder.rs:22-143).
void etree_postorder(const std::vector<int64_t>& parent, const std::vector<uint8_t>* bias,
                     std::vector<int64_t>& post, std::vector<int64_t>& post_inv);
// Exact column counts of L (src/symbolic/column_counts.rs:97-183).
std::vector<int64_t> column_counts(const CscPattern& pat, const std::vector<int64_t>& parent);

enum class Ordering : int { Amd = 0, MetisND = 1, Natural = 2, Given = 3 };

// Analysis knobs (the analyze-time half of SolverSettings,
// src/numeric/multifrontal_ldlt.rs:302-420, defaults :583-614).
struct AnalyzeOptions {
  Ordering ordering = Ordering::Amd;
  int64_t nemin = 16;
  bool relax = true;
  int64_t relax_max_width = 256;
  int64_t relax_max_extra_rows = 64;
  bool hybrid_liu = true;
  const int64_t* given_perm = nullptr;  // used with Ordering::Given
};

struct Supernode {
  int64_t first_col = 0;
  int64_t ncol = 0;
  int64_t nrow_est = 0;  // col_counts-based frontal height
  std::vector<int64_t> children;
};

struct Symbolic {
  int64_t n = 0;
  int64_t nnz = 0;  // stored lower-triangle entries of the analysed pattern
  std::vector<int64_t> perm, perm_inv;  // new-to-old / old-to-new
  CscPattern permuted;                  // full symmetric pattern of P A P^T
  std::vector<int64_t> parent;          // etree of P A P^T
  std::vector<int64_t> col_counts;
  std::vector<Supernode> sn;
  int resolved_ordering = 0;
  int renumbered = 0;  // merge-biased postorder applied
  AmdStats amd;
  // Left-looking structure (src/numeric/multifrontal_ldlt.rs:2121-2152,
  // 3380-3401): per supernode its row structure, and for each supernode the
  // ordered list of descendants whose off-diagonal rows land in its columns.
  std::vector<int64_t> rs_ptr, rs;          // rs[rs_ptr[s]..rs_ptr[s+1])
  std::vector<int64_t> upd_ptr, upd;        // updater k of s
  std::vector<int64_t> upd_p0, upd_p1;      // landing range in k's off-diag rows
  std::vector<int64_t> level;               // assembly-tree level (leaves = 0)
  std::vector<std::vector<int64_t>> by_level;
  int64_t factor_nnz_sym = 0;  // sum of column counts
};

Symbolic analyze(int64_t n, const int64_t* col_ptr, const int64_t* row_idx,
                 const AnalyzeOptions& opt);

// Independent systems as one block-diagonal analysis: system i occupies
// columns [col_off[i], col_off[i+1]); its supernodes, row structures, update
// lists and levels are its own analysis shifted by the offsets, so the
// assembly forest has one tree (or more) per system and level l collects the
// level-l supernodes of every system.
Symbolic merge_independent(const std::vector<Symbolic>& parts);

// A-priori memory and work estimate of an analysis for a scalar of
// value_bytes bytes (LdltSymbolic::estimate_memory,
// src/numeric/sparse_solver.rs:561-660, with estimate_left_looking,
// src/diagnostics.rs:116-175): the refcount free schedule of the left-looking
// factor gives the live panel peak; factor_flops = sum_s nrow^2 ncol.
struct MemoryEstimate {
  int64_t value_bytes = 0, factor_nnz = 0, factor_bytes = 0, panels_all_bytes = 0;
  int64_t panel_live_peak_bytes = 0, transient_peak_bytes = 0;
  uint64_t factor_flops = 0, critical_path_flops = 0;
  int64_t max_tree_width = 0;
  // the multifrontal method's figure: the left-looking one plus every
  // contribution block, all of which it keeps resident on the device
  int64_t mf_transient_peak_bytes = 0;
};
MemoryEstimate estimate_memory(const Symbolic& S, int64_t value_bytes);
// symbolic_factor_nnz (src/numeric/sparse_solver.rs:550-555): the exact
// column-count fill times the 1.2 slack (src/symbolic/mod.rs:1189, 1202).
inline int64_t symbolic_factor_nnz(const Symbolic& S) { return (int64_t)((double)S.factor_nnz_sym * 1.2); }

// Dense partial BK flop model per supernode: F(r,c) = sum_{m=r-c+1}^{r}(m^2-1).
double supernode_flops(int64_t r, int64_t c);

}  // namespace rslab
