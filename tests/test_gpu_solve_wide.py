"""The solve's level launches on a pattern whose leaf level has more than 600
blocks (40^3 Helmholtz, MetisND: 1,369 blocks at level 0), so the leaf
chains take every column of a pass in one CTA per block while the upper
levels split the columns into groups of four; the forward chain items pull
their own right-hand sides and the backward chain sums the split dots'
partials.  Per column the operations are those of a one-column solve, so a
many-column solve agrees with single-column solves to rounding; every
column's backward error is at the FP64 level (the oracle's solve of this
size is checked elsewhere, against the same kernels on smaller patterns)."""
import numpy as np
import pytest

from oracle.oracle import backward_error
from rslab_b200 import LdltSymbolic, Ordering, SolverSettings, matgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def factor40():
    a = matgen.c2_matrix(40)
    st = SolverSettings(ordering=Ordering.METIS_ND)
    sym = LdltSymbolic.analyze_with(a, st)
    e = sym.export()
    blocks = np.bincount(np.asarray(e["sn_level"]), weights=(np.asarray(e["sn_ncol"]) + 63) // 64)
    assert blocks.max() >= 600 and blocks.min() < 600  # wide and narrow levels both present
    return a, sym.factor(a, st)


@pytest.mark.parametrize("nrhs", [5, 16, 20])
def test_many_columns_match_single_column_solves(factor40, nrhs):
    a, f = factor40
    b = matgen.uniform_rhs(a.n, nrhs, 11, complex_=True)
    x = f.solve_many(b, nrhs)
    assert backward_error(a, x, b) <= 1e-13
    for c in sorted({0, nrhs // 2, nrhs - 1}):
        xc = f.solve(np.ascontiguousarray(b[:, c]))
        assert np.max(np.abs(x[:, c] - xc)) <= 1e-13 * np.max(np.abs(xc))
