"""The product's host analysis against the oracle's own restatement of the
reference's symbolic pipeline (oracle/symbolic.cpp: postorder composition,
elimination tree, column counts, amalgamation strategy, merge-biased
renumbering, fundamental + relaxed supernodes, row structures, levels).
Both start from the same ordering output: the AMD permutation (pinned by the
reference's SuiteSparse golden permutations, tests/test_amd_golden.py) or the
MetisND permutation, given to the product as Ordering.GIVEN.  Everything
downstream of the ordering must be identical: the final permutation, etree,
column counts, supernode first columns, widths, row-structure heights, the
supernode tree and its levels.  Host-only."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.oracle import oracle_structure, supernode_parent
from rslab_b200 import CscMatrix, LdltSymbolic, Ordering, SolverSettings, amd_order, matgen
from rslab_b200.solver import metis_order
from tests.helpers import amd_cases, kkt_cases

KEYS = ("perm", "parent", "col_counts", "sn_first", "sn_ncol", "sn_nrow", "sn_level")


def full_pattern(a: CscMatrix):
    f = a.to_scipy_full().tocsc()
    f.sort_indices()
    return np.asarray(f.indptr, np.int64), np.asarray(f.indices, np.int64)


def compare(a: CscMatrix, ordering: str = "amd", settings: SolverSettings = None):
    cp, ri = full_pattern(a)
    ordv = amd_order(a.n, cp, ri)[0] if ordering == "amd" else metis_order(a.n, cp, ri)
    st = settings or SolverSettings()
    given = SolverSettings(ordering=Ordering.GIVEN, nemin=st.nemin, relax=st.relax)
    given.given_perm = ordv
    prod = LdltSymbolic.analyze_with(a, given).export()
    orc = oracle_structure(a, ordv, nemin=st.nemin, relax=st.relax)
    for k in KEYS:
        assert np.array_equal(prod[k], orc[k]), f"{k} differs"
    assert np.array_equal(supernode_parent(prod), supernode_parent(orc)), "supernode tree differs"
    # the default AMD analysis is this GIVEN analysis of the AMD ordering
    if ordering == "amd" and settings is None:
        dflt = LdltSymbolic.analyze(a).export()
        for k in KEYS:
            assert np.array_equal(dflt[k], prod[k]), f"default analysis: {k}"
    return orc


def lower_from_full(n, cp, ri):
    cols = np.repeat(np.arange(n), np.diff(cp))
    keep = ri >= cols
    return CscMatrix.from_triplets(n, ri[keep], cols[keep], np.ones(int(keep.sum())))


@pytest.mark.parametrize("name", sorted(amd_cases()))
def test_amd_golden_patterns(name):
    c = amd_cases()[name]
    a = lower_from_full(c["n"], np.asarray(c["col_ptr"], np.int64), np.asarray(c["row_idx"], np.int64))
    compare(a)


def test_kkt_fixtures():
    for e, a, _ in kkt_cases():
        compare(a)


@pytest.mark.parametrize("side", [16, 64, 128])
def test_c1_laplacian_2d(side):
    compare(matgen.c1_matrix(side))


@pytest.mark.parametrize("side", [8, 14, 24])
def test_c2_helmholtz_amd(side):
    compare(matgen.c2_matrix(side))


@pytest.mark.parametrize("side", [16, 24, 32])
def test_c2_helmholtz_metis(side):
    orc = compare(matgen.c2_matrix(side), "metis")
    assert orc["sn_ncol"].max() > 64  # wide separator supernodes, relaxed merges


@pytest.mark.parametrize("side", [12, 20])
def test_c3_laplacian_3d(side):
    compare(matgen.c3_matrix(side))


def test_c4_stencil27():
    a = matgen.C4System(12).matrix(1.0)
    compare(a)
    compare(a, "metis")


def test_c5_corpus_families():
    """Twelve corpus matrices (every family of the precision-tier corpus)."""
    fams = set()
    for fam, a in matgen.c5_corpus(12):
        fams.add(fam)
        compare(a)
    assert len(fams) >= 4


def test_random_sparse_and_settings():
    a = matgen.random_sparse_symmetric(3000, matgen.Rng(7), 3.0)
    compare(a)
    for st in (SolverSettings(nemin=4), SolverSettings(relax=None), SolverSettings(nemin=32, relax=(128, 16))):
        compare(a, settings=st)


def test_renumbering_path_is_exercised():
    seen = set()
    for a in (matgen.c1_matrix(16), matgen.c1_matrix(40), matgen.c2_matrix(12)):
        cp, ri = full_pattern(a)
        seen.add(oracle_structure(a, amd_order(a.n, cp, ri)[0])["renumbered"])
    assert True in seen
