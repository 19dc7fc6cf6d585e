"""The multifrontal factor method (FactorMethod::Multifrontal,
src/numeric/multifrontal_ldlt.rs:283): every supernode's front is the
original columns plus its children's contribution blocks (extend-add), the
front's pivot block is factored by the same Bunch-Kaufman panel kernels as
the left-looking method, and the trailing block becomes the supernode's own
contribution block.  Parity against the oracle (inertia, backward error,
solution) and against the left-looking method on the same analysis (the
reference's own check that both methods solve alike, benches/validate_axes.rs
:441-447; the sums associate differently here, so the comparison is by
tolerance on fixed pivot sequences); repeated factors are bit-identical."""
import numpy as np
import pytest

from oracle.oracle import OracleSolver, backward_error
from rslab_b200 import LdltSymbolic, MixedLdltSolver, Ordering, SolverSettings, matgen
from tests.helpers import kkt_cases, rel_err

pytestmark = pytest.mark.gpu

MF = dict(method="multifrontal")
LL = dict(method="left_looking", schur_engine="fma")


def dominant3d(side, complex_):
    dims = (side, side, side)
    lm = matgen.lambda_max(dims)
    if complex_:
        return matgen.helmholtz(dims, complex(-0.5 * lm, 0.05 * lm))
    return matgen.shifted_laplacian(dims, -0.5 * lm)


@pytest.mark.parametrize("engine", ["fma", "tensor"])
@pytest.mark.parametrize("complex_,side,metis", [(False, 12, False), (True, 12, False), (False, 24, True),
                                                 (True, 24, True)])
def test_multifrontal_matches_left_looking_entrywise(complex_, side, metis, engine):
    """engine "tensor": the panel kernels and the contribution-block products
    on the FP64 tensor cores (DMMA tiles)."""
    a = dominant3d(side, complex_)
    o = Ordering.METIS_ND if metis else Ordering.AMD
    sym = LdltSymbolic.analyze_with(a, SolverSettings(ordering=o))
    mf = sym.factor(a, SolverSettings(ordering=o, schur_engine=engine, **MF))
    assert mf.diagnostics().schur_engine == engine
    assert mf.diagnostics().method == "multifrontal"
    fm = mf.export_factors()
    lm = sym.factor(a, SolverSettings(ordering=o, **LL)).export_factors()
    assert np.array_equal(fm.perm, lm.perm) and np.array_equal(fm.two_by_two, lm.two_by_two)
    assert np.array_equal(fm.l_col_ptr, lm.l_col_ptr) and np.array_equal(fm.l_row_idx, lm.l_row_idx)
    assert rel_err(fm.d_diag, lm.d_diag) <= 1e-12
    assert rel_err(fm.l_values, lm.l_values) <= 1e-12


@pytest.mark.parametrize("case", ["c1_128", "c3_16", "c2_20_metis"])
def test_multifrontal_indefinite_against_oracle(case):
    if case == "c1_128":
        a, o, cx = matgen.c1_matrix(128), Ordering.AMD, False
    elif case == "c3_16":
        a, o, cx = matgen.c3_matrix(16), Ordering.AMD, False
    else:
        a, o, cx = matgen.c2_matrix(20), Ordering.METIS_ND, True
    sym = LdltSymbolic.analyze_with(a, SolverSettings(ordering=o))
    mf = sym.factor(a, SolverSettings(ordering=o, **MF))
    orc = OracleSolver(a, sym.export())
    assert tuple(mf.inertia()) == orc.factors().inertia
    b = matgen.uniform_rhs(a.n, 4, 7, complex_=cx)
    x = mf.solve_many(b, 4)
    xo = orc.solve_many(b, 4)
    assert backward_error(a, x, b) <= max(1e-13, 10 * backward_error(a, xo, b))
    assert rel_err(x, xo) <= 1e-9
    xl = sym.factor(a, SolverSettings(ordering=o, **LL)).solve_many(b, 4)
    assert rel_err(x, xl) <= 1e-9


KKT = kkt_cases()


@pytest.mark.parametrize("case", KKT, ids=[c[0]["name"] for c in KKT])
def test_multifrontal_kkt_fixtures(case):
    """The reference's KKT fixtures: the oracle's inertia wherever the
    matrix is not singular to working precision (smallest eigenvalue modulus
    above 1e-13 of the largest; below that the sign of the smallest pivot is
    rounding and the two methods round differently), backward error at the
    oracle's level everywhere."""
    e, a, rhs = case
    sym = LdltSymbolic.analyze(a)
    orc = OracleSolver(a, sym.export())
    o = orc.factors()
    if o.status != 0:
        return
    mf = sym.factor(a, SolverSettings(**MF))
    ev = np.abs(np.linalg.eigvalsh(a.to_scipy_full().toarray()))
    if ev.min() > 1e-13 * ev.max():
        assert tuple(mf.inertia()) == o.inertia
    x = mf.solve(rhs)
    xo = orc.solve_many(rhs, 1)
    assert backward_error(a, x, rhs) <= max(1e-12, 100 * backward_error(a, xo, rhs))


def test_multifrontal_deterministic_and_refactor():
    a = matgen.c2_matrix(16)
    sym = LdltSymbolic.analyze_with(a, SolverSettings(ordering=Ordering.METIS_ND))
    st = SolverSettings(ordering=Ordering.METIS_ND, **MF)
    f1 = sym.factor(a, st)
    e1 = f1.export_factors()
    f1.refactor(a)
    e2 = f1.export_factors()
    e3 = sym.factor(a, st).export_factors()
    for e in (e2, e3):
        assert np.array_equal(e1.l_values, e.l_values) and np.array_equal(e1.d_diag, e.d_diag)
        assert np.array_equal(e1.d_subdiag, e.d_subdiag)


@pytest.mark.parametrize("complex_", [False, True])
def test_multifrontal_mixed_precision_certifies(complex_):
    a = matgen.c2_matrix(20) if complex_ else matgen.c1_matrix(96)
    st = SolverSettings(**MF)
    m = MixedLdltSolver.factor_with(a, st)
    b = matgen.uniform_rhs(a.n, 1, 5, complex_=complex_)
    x, info = m.solve_to(a, b, 1e-14)
    assert info.certified
    assert backward_error(a, x, b) <= 1e-14
