"""MetisND ordering (host, no GPU): valid and deterministic permutations,
AMD on graphs at or below the leaf size, contiguous components, and the fill
reduction nested dissection gives on 3D grids.  The reference's own crate
cannot be run here, so the permutation itself is not pinned to it."""
import numpy as np
import pytest

from rslab_b200 import LdltSymbolic, Ordering, SolverSettings, matgen
from rslab_b200.solver import CscMatrix


def _sym(a, o):
    return LdltSymbolic.analyze_with(a, SolverSettings().with_ordering(o))


def _perm(a, o):
    p = np.asarray(_sym(a, o).export()["perm"])
    assert sorted(p.tolist()) == list(range(a.n))
    return p


@pytest.mark.parametrize("make", [lambda: matgen.c1_matrix(40), lambda: matgen.c2_matrix(14),
                                  lambda: matgen.random_sparse_symmetric(900, matgen.Rng(3), 1.0),
                                  lambda: matgen.C4System(9).matrix(1.0)])
def test_valid_and_deterministic(make):
    a = make()
    assert np.array_equal(_perm(a, Ordering.METIS_ND), _perm(a, Ordering.METIS_ND))


def test_small_graph_is_one_amd_leaf():
    a = matgen.c3_matrix(5)  # n = 125 <= 200: the whole graph goes to AMD
    assert np.array_equal(_perm(a, Ordering.METIS_ND), _perm(a, Ordering.AMD))
    ia, ib = _sym(a, Ordering.METIS_ND).info(), _sym(a, Ordering.AMD).info()
    assert ia.factor_nnz_sym == ib.factor_nnz_sym and ia.nsuper == ib.nsuper


def test_nested_dissection_cuts_3d_fill():
    a = matgen.c3_matrix(32)
    nd, amd = _sym(a, Ordering.METIS_ND).info(), _sym(a, Ordering.AMD).info()
    assert nd.flops_model < 0.75 * amd.flops_model
    assert nd.factor_nnz_sym < 0.9 * amd.factor_nnz_sym


def test_disconnected_components():
    """Two disjoint grids: the dissection splits components first, the
    permutation stays valid and the elimination forest has a tree per grid."""
    g1 = matgen.c3_matrix(12)
    g2 = matgen.c1_matrix(30)
    n1 = g1.n
    r1, c1 = np.asarray(g1.row_idx), np.repeat(np.arange(n1), np.diff(np.asarray(g1.col_ptr)))
    r2, c2 = np.asarray(g2.row_idx), np.repeat(np.arange(g2.n), np.diff(np.asarray(g2.col_ptr)))
    a = CscMatrix.from_triplets(n1 + g2.n, np.concatenate([r1, r2 + n1]), np.concatenate([c1, c2 + n1]),
                                np.concatenate([np.asarray(g1.values), np.asarray(g2.values)]))
    _perm(a, Ordering.METIS_ND)
    parent = np.asarray(_sym(a, Ordering.METIS_ND).export()["parent"])
    assert int(np.sum(parent < 0)) >= 2


@pytest.mark.parametrize("side,nnz_m,digits", [(24, 1.53, 2), (40, 14.00, 2), (56, 63.8, 1)])
def test_fill_matches_the_reference_crates_recorded_fill(side, nnz_m, digits):
    """The reference recorded the exact scalar nnz(L) (diagonal included,
    elimination-tree column counts, no supernode padding) of its crate's
    default MetisND on 7-point grids: 24^3 1.53 M, 40^3 14.00 M, 56^3 63.8 M,
    and the 40^3 flop proxy sum(cc^2) 1.53e10
    (dev/research/metis-node-separator-2026-07.md:3-4, 72-74)."""
    a = matgen.c3_matrix(side)
    cc = np.asarray(_sym(a, Ordering.METIS_ND).export()["col_counts"], np.float64)
    assert round(cc.sum() / 1e6, digits) == nnz_m
    if side == 40:
        assert round((cc ** 2).sum() / 1e10, 2) == 1.53


def test_oracle_factor_on_the_dissection_structure():
    """The CPU oracle factors and solves on the MetisND structure: same
    solution as a direct sparse solve, inertia of the shifted Laplacian."""
    import scipy.sparse.linalg as spla

    from oracle.oracle import OracleSolver
    a = matgen.c3_matrix(14)
    sym = _sym(a, Ordering.METIS_ND)
    o = OracleSolver(a, sym.export())
    b = matgen.uniform_rhs(a.n, 2, 5)
    x = o.solve_many(b, 2)
    xr = spla.spsolve(a.to_scipy_full().tocsc(), b)
    assert np.abs(x - xr).max() <= 1e-10 * np.abs(xr).max()
    neg = matgen.negative_eigs_shifted_laplacian((14, 14, 14), 0.1 * matgen.lambda_max((14, 14, 14)))
    assert o.factors().inertia == (a.n - neg, neg, 0)


def test_seeded_fill_on_40_cubed_grid():
    """Other seeds of the same crate, 40^3 grid: the reference recorded 14.3,
    14.5 and 14.9 M for seeds 2-4 (dev/research/metis-node-separator-2026-07.md:72).
    Ours: 14.25, 14.45 and 14.96 M.  Seeds 2 and 3 match the note's one
    decimal; seed 4 reads 0.06 M above it, which is checked here as a bound
    rather than claimed as a match."""
    from rslab_b200.solver import metis_order
    a = matgen.c3_matrix(40)
    full = a.to_scipy_full().tocsc()
    full.sort_indices()
    got = {}
    for seed in (1, 2, 3, 4):
        perm = metis_order(a.n, full.indptr, full.indices, seed)
        assert sorted(perm.tolist()) == list(range(a.n))
        st = SolverSettings().with_ordering(Ordering.GIVEN)
        st.given_perm = perm
        got[seed] = np.asarray(LdltSymbolic.analyze_with(a, st).export()["col_counts"]).sum() / 1e6
    assert round(got[1], 2) == 14.00
    assert round(got[2], 1) == 14.3 and round(got[3], 1) == 14.5
    assert abs(got[4] - 14.9) < 0.1


@pytest.mark.parametrize("shape", ["empty", "one", "diag", "star", "path", "dense", "random", "two_blocks"])
def test_degenerate_graphs_give_permutations(shape):
    import scipy.sparse as sp

    from rslab_b200.solver import metis_order
    n = 3000
    if shape == "empty":
        assert metis_order(0, np.zeros(1, np.int64), np.zeros(0, np.int64)).shape == (0,)
        return
    if shape == "one":
        assert metis_order(1, np.array([0, 1]), np.array([0])).tolist() == [0]
        return
    r = np.arange(1, n)
    a = {"diag": sp.csr_matrix((n, n)),
         "star": sp.csr_matrix((np.ones(n - 1), (r, np.zeros(n - 1))), shape=(n, n)),
         "path": sp.diags([np.ones(n - 1)], [-1]),
         "dense": sp.csr_matrix(np.tril(np.ones((400, 400)), -1)),
         "random": sp.random(n, n, density=5 / n, random_state=1),
         "two_blocks": sp.block_diag([sp.diags([np.ones(1999)], [-1]), np.tril(np.ones((300, 300)), -1)])}[shape]
    a = (a + a.T + sp.eye(a.shape[0])).tocsc()
    a.sort_indices()
    p = metis_order(a.shape[0], a.indptr, a.indices)
    assert sorted(p.tolist()) == list(range(a.shape[0]))


# The reference's dense-quotient tests (crates/rslab-metis/tests/dense_quotient.rs):
# full symmetric pattern of a banded graph plus one near-dense column.

def _pattern(n, edges):
    import scipy.sparse as sp
    r = np.array([e[0] for e in edges] + list(range(n)))
    c = np.array([e[1] for e in edges] + list(range(n)))
    a = sp.csc_matrix((np.ones(len(r)), (r, c)), shape=(n, n))
    a = ((a + a.T) != 0).astype(np.float64).tocsc()
    a.sort_indices()
    return a.indptr, a.indices


def _banded(n, band):
    return [(r, r + 1) for r in range(n - 1)] + [(r, r + band) for r in range(n - band)]


def _with_dense(n, band, col, deg):
    e = _banded(n, band)
    added, step = set(), 1
    while len(added) < deg:
        r = (col + step) % n
        if r != col and r not in added:
            e.append((col, r))
            added.add(r)
        step += 1
    return e


def test_dense_column_lands_at_end_of_perm():
    from rslab_b200.solver import metis_order
    cp, ri = _pattern(1000, _with_dense(1000, 7, 500, 800))
    p = metis_order(1000, cp, ri, dense_quotient=True)
    assert sorted(p.tolist()) == list(range(1000)) and p[-1] == 500


def test_no_dense_column_matches_the_plain_order():
    from rslab_b200.solver import metis_order
    cp, ri = _pattern(600, _banded(600, 11))
    assert np.array_equal(metis_order(600, cp, ri), metis_order(600, cp, ri, dense_quotient=True))


def test_quotient_off_keeps_the_dense_column_inside():
    from rslab_b200.solver import metis_order
    cp, ri = _pattern(1000, _with_dense(1000, 7, 500, 800))
    off = metis_order(1000, cp, ri)
    assert sorted(off.tolist()) == list(range(1000))
    assert metis_order(1000, cp, ri, dense_quotient=True)[-1] == 500


def test_threshold_override_promotes_a_lower_degree_column():
    from rslab_b200.solver import metis_order
    cp, ri = _pattern(200, _with_dense(200, 5, 73, 50))
    assert sorted(metis_order(200, cp, ri).tolist()) == list(range(200))
    p = metis_order(200, cp, ri, dense_quotient=True, dense_threshold=30)
    assert sorted(p.tolist()) == list(range(200)) and p[-1] == 73


@pytest.mark.parametrize("which", ["amd", "metis"])
def test_ordering_entry_points_reject_malformed_patterns(which):
    """The ordering entry points validate their full symmetric pattern as the
    reference's Graph::from_csc_pattern / CscPattern::new do, and return
    InvalidInput instead of reading or writing outside the arrays."""
    from rslab_b200.solver import InvalidInput, amd_order, metis_order

    def run(n, cp, ri):
        cp, ri = np.asarray(cp, np.int64), np.asarray(ri, np.int64)
        return amd_order(n, cp, ri) if which == "amd" else metis_order(n, cp, ri)

    # 3-vertex path 0-1-2 with diagonals: valid
    ok_cp, ok_ri = [0, 2, 5, 7], [0, 1, 0, 1, 2, 1, 2]
    run(3, ok_cp, ok_ri)
    bad = {
        "row out of range": ([0, 2, 5, 7], [0, 1, 0, 1, 9, 1, 2]),
        "negative row": ([0, 2, 5, 7], [0, -1, 0, 1, 2, 1, 2]),
        "col_ptr decreasing": ([0, 5, 2, 7], [0, 1, 0, 1, 2, 1, 2]),
        "col_ptr[0] != 0": ([1, 2, 5, 7], [0, 1, 0, 1, 2, 1, 2]),
        "unsorted column": ([0, 2, 5, 7], [1, 0, 0, 1, 2, 1, 2]),
        "not symmetric": ([0, 2, 4, 6], [0, 1, 1, 2, 1, 2]),
    }
    for what, (cp, ri) in bad.items():
        with pytest.raises(InvalidInput):
            run(3, cp, ri)
        assert what  # message names the case on failure


def test_ordering_entry_points_drop_adjacent_duplicates():
    from rslab_b200.solver import amd_order, metis_order

    cp = np.array([0, 3, 7, 9], np.int64)
    ri = np.array([0, 1, 1, 0, 1, 1, 2, 1, 2], np.int64)
    p, _ = amd_order(3, cp, ri)
    assert sorted(p.tolist()) == [0, 1, 2]
    assert sorted(metis_order(3, cp, ri).tolist()) == [0, 1, 2]
