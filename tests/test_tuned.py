"""LdltSolver::tuned and its nested-dissection bakeoff
(src/numeric/sparse_solver.rs:108-131, 231-266) over the C ABI
(rslab_analyze_tuned), and the a-priori estimate it compares
(estimate_memory, :561-660).  Host-only: no GPU is touched."""
import numpy as np
import pytest

from rslab_b200 import LdltSymbolic, Ordering, SolverSettings, matgen


def test_c1_pattern_keeps_amd():
    """128^2 2D Laplacian: n >= 10,000 but the AMD analysis predicts < 5e9
    geometric flops, so the bakeoff does not run."""
    a = matgen.c1_matrix()
    sym, s = LdltSymbolic.tuned(a)
    assert s.ordering == Ordering.AMD
    assert sym.estimate_memory().factor_flops < 5e9


def test_small_systems_never_enter_the_bakeoff():
    a = matgen.c2_matrix(20)  # n = 8,000 < 10,000
    _, s = LdltSymbolic.tuned(a)
    assert s.ordering == Ordering.AMD


@pytest.mark.parametrize("which", ["c2", "c4"])
def test_grid_patterns_adopt_metis(which):
    """The C2 (64^3 7-point Helmholtz) and C4 (48^3 27-point) patterns adopt
    MetisND: the ND analysis has < 0.75x the flops, no more fill and no larger
    live-panel peak than the AMD analysis, and the tuned analysis equals a
    plain MetisND analysis."""
    a = matgen.c2_matrix(64) if which == "c2" else matgen.C4System(48).matrix(1.0)
    sym, s = LdltSymbolic.tuned(a)
    assert s.ordering == Ordering.METIS_ND
    amd = LdltSymbolic.analyze_with(a, SolverSettings(ordering=Ordering.AMD))
    nd = LdltSymbolic.analyze_with(a, SolverSettings(ordering=Ordering.METIS_ND))
    e_amd, e_nd = amd.estimate_memory(a.values.dtype), nd.estimate_memory(a.values.dtype)
    assert e_nd.factor_flops < 0.75 * e_amd.factor_flops
    assert nd.symbolic_factor_nnz() <= amd.symbolic_factor_nnz()
    assert e_nd.panel_live_peak_bytes <= e_amd.panel_live_peak_bytes
    ex, en = sym.export(), nd.export()
    for k in ("perm", "sn_first", "sn_ncol", "sn_nrow", "parent"):
        assert np.array_equal(ex[k], en[k]), k


def test_estimate_matches_structure():
    """factor_flops = sum nrow^2 ncol, panels_all = sum nrow ncol x bytes,
    symbolic fill = floor(1.2 x sum of column counts); the live peak lies
    between the largest panel and all panels plus the compact factor."""
    a = matgen.c2_matrix(16)
    sym = LdltSymbolic.analyze(a)
    ex = sym.export()
    r, c = ex["sn_nrow"].astype(np.int64), ex["sn_ncol"].astype(np.int64)
    e = sym.estimate_memory(np.complex128)
    assert e.value_bytes == 16
    assert e.factor_flops == int(np.sum(r * r * c))
    assert e.panels_all_bytes == int(np.sum(r * c)) * 16
    compact = int(np.sum(c * (c + 1) // 2 + (r - c) * c)) * 24
    assert e.factor_bytes == compact and e.factor_nnz == compact // 24
    assert int(np.max(r * c)) * 16 <= e.panel_live_peak_bytes <= e.panels_all_bytes + compact
    assert sym.symbolic_factor_nnz() == int(1.2 * int(np.sum(ex["col_counts"])))
    # the critical path is at least the root chain's own work and at most the total
    assert int(np.max(r * r * c)) <= e.critical_path_flops <= e.factor_flops
    # the multifrontal figure adds every contribution block, (nrow - ncol)^2 scalars each
    assert e.mf_transient_peak_bytes == e.transient_peak_bytes + int(np.sum((r - c) ** 2)) * 16
