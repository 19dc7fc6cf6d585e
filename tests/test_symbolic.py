"""Host symbolic analysis against brute-force elimination on small patterns:
etree, exact column counts, supernode partition invariants, and the AMD-based
analysis pipeline options (src/symbolic/mod.rs:861-1215,
src/symbolic/supernode.rs:267-465)."""
import numpy as np
import pytest

from rslab_b200 import CscMatrix, InvalidInput, LdltSymbolic, SolverSettings
from rslab_b200 import matgen


def random_sym(n, density, seed):
    rng = np.random.default_rng(seed)
    m = rng.random((n, n)) < density
    m = np.tril(m | m.T, -1)
    r, c = np.nonzero(m)
    rows = np.concatenate([np.arange(n), r])
    cols = np.concatenate([np.arange(n), c])
    vals = np.concatenate([np.full(n, 4.0), rng.standard_normal(len(r))])
    return CscMatrix.from_triplets(n, rows, cols, vals)


def brute_force_l_pattern(a: CscMatrix, perm):
    n = a.n
    full = (a.to_scipy_full() != 0).toarray()
    p = full[np.ix_(perm, perm)]
    L = np.tril(p).copy()
    for j in range(n):
        rows = np.nonzero(L[j + 1:, j])[0] + j + 1
        for i in rows:
            L[rows[rows >= i], i] = True
    return L


@pytest.mark.parametrize("n,density,seed", [(30, 0.08, 1), (60, 0.05, 2), (120, 0.03, 3)])
def test_etree_and_column_counts_exact(n, density, seed):
    a = random_sym(n, density, seed)
    sym = LdltSymbolic.analyze_with(a, SolverSettings())
    ex = sym.export()
    L = brute_force_l_pattern(a, ex["perm"])
    counts = L.sum(axis=0)
    assert np.array_equal(counts, ex["col_counts"])
    parent = np.array([np.nonzero(L[j + 1:, j])[0][0] + j + 1 if L[j + 1:, j].any() else -1 for j in range(n)])
    assert np.array_equal(parent, ex["parent"])


@pytest.mark.parametrize("relax", [None, (256, 64)])
def test_supernode_partition(relax):
    a = matgen.c1_matrix(48)  # n = 2304 >= 1024, relaxed merges active
    sym = LdltSymbolic.analyze_with(a, SolverSettings(relax=relax))
    ex = sym.export()
    first, ncol, nrow = ex["sn_first"], ex["sn_ncol"], ex["sn_nrow"]
    assert first[0] == 0
    assert np.all(first[1:] == first[:-1] + ncol[:-1])
    assert first[-1] + ncol[-1] == a.n
    assert np.all(nrow >= ncol)
    cc = ex["col_counts"]
    # row structures contain the true L structure of their first column
    assert np.all(nrow >= cc[first] + 0 * ncol)
    # children precede parents (postorder)
    cp, ci = ex["child_ptr"], ex["child_idx"]
    for s in range(len(first)):
        assert np.all(ci[cp[s]:cp[s + 1]] < s)
    if relax is None:
        assert sym.info().nsuper >= 1


def test_fundamental_supernodes_without_amalgamation():
    a = random_sym(80, 0.04, 7)
    sym = LdltSymbolic.analyze_with(a, SolverSettings(nemin=1, relax=None))
    ex = sym.export()
    # with nemin = 1 and no relaxation the row structure is exactly the
    # column count of each supernode's first column
    assert np.array_equal(ex["sn_nrow"], ex["col_counts"][ex["sn_first"]])


def test_perm_is_permutation_and_levels():
    a = matgen.c3_matrix(10)
    sym = LdltSymbolic.analyze(a)
    ex = sym.export()
    assert sorted(ex["perm"]) == list(range(a.n))
    lv = ex["sn_level"]
    cp, ci = ex["child_ptr"], ex["child_idx"]
    for s in range(len(lv)):
        for c in ci[cp[s]:cp[s + 1]]:
            assert lv[c] < lv[s]


def test_invalid_inputs_rejected():
    with pytest.raises(InvalidInput):
        LdltSymbolic.analyze(CscMatrix(2, [0, 1, 2], [1, 0], [1.0, 1.0]))  # upper entry
    with pytest.raises(InvalidInput):
        LdltSymbolic.analyze(CscMatrix(2, [0, 2, 2], [1, 0], [1.0, 1.0]))  # unsorted
    with pytest.raises(InvalidInput):
        CscMatrix.from_triplets(2, [0], [1], [1.0])


def test_given_and_natural_orderings():
    a = random_sym(40, 0.1, 11)
    nat = LdltSymbolic.analyze_with(a, SolverSettings(ordering=2)).export()
    # the natural ordering is only re-postordered
    assert sorted(nat["perm"]) == list(range(40))
    perm = np.random.default_rng(0).permutation(40)
    giv = LdltSymbolic.analyze_with(a, SolverSettings(ordering=3, given_perm=perm)).export()
    assert sorted(giv["perm"]) == list(range(40))


@pytest.mark.parametrize("make", [lambda: random_sym(400, 0.008, 4), lambda: matgen.c3_matrix(8)])
def test_column_counts_exact_under_nested_dissection(make):
    """The same exactness on MetisND structures (graphs above the AMD leaf
    size, so the dissection and its separators are exercised)."""
    a = make()
    ex = LdltSymbolic.analyze_with(a, SolverSettings(ordering=1)).export()
    L = brute_force_l_pattern(a, ex["perm"])
    assert np.array_equal(L.sum(axis=0), ex["col_counts"])
