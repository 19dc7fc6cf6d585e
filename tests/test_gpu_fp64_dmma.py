"""The default descendant-update engine of the FP64 fields: updater-space
GEMM tiles on the FP64 tensor cores (mma.sync m8n8k4 .f64) into a level
workspace, assembled into the targets in update order.  Parity by
tolerance against the bit-exact CUDA-core engine (itself bit-identical to the
oracle): on fixed pivot sequences (diagonally dominant stencils, every pivot
a diagonal 1x1) L and D agree entry by entry within 1e-12 relative; on
indefinite matrices the inertia is exact and backward errors stay at the
FP64 level; the engine is deterministic.  The default engine setting ("auto")
picks these tiles from 2e8 model flops and the bit-exact engine below."""
import numpy as np
import pytest

from oracle.oracle import OracleSolver, backward_error
from rslab_b200 import LdltSymbolic, Ordering, SolverSettings, matgen
from tests.helpers import kkt_cases, rel_err

TENSOR = dict(schur_engine="tensor")

pytestmark = pytest.mark.gpu


def dominant3d(side, complex_):
    dims = (side, side, side)
    lm = matgen.lambda_max(dims)
    if complex_:
        return matgen.helmholtz(dims, complex(-0.5 * lm, 0.05 * lm))
    return matgen.shifted_laplacian(dims, -0.5 * lm)


@pytest.mark.parametrize("complex_,side,metis", [(False, 16, False), (True, 16, False), (False, 28, True),
                                                 (True, 28, True)])
def test_dmma_entrywise_on_fixed_pivot_sequence(complex_, side, metis):
    a = dominant3d(side, complex_)
    st = SolverSettings(ordering=Ordering.METIS_ND if metis else Ordering.AMD, **TENSOR)
    sym = LdltSymbolic.analyze_with(a, st)
    dm = sym.factor(a, st).export_factors()
    fm = sym.factor(a, SolverSettings(ordering=st.ordering, schur_engine="fma")).export_factors()
    assert np.array_equal(dm.perm, fm.perm) and np.array_equal(dm.two_by_two, fm.two_by_two)
    assert np.array_equal(dm.l_col_ptr, fm.l_col_ptr) and np.array_equal(dm.l_row_idx, fm.l_row_idx)
    assert rel_err(dm.d_diag, fm.d_diag) <= 1e-12
    assert rel_err(dm.l_values, fm.l_values) <= 1e-12


@pytest.mark.parametrize("case", ["c1_128", "c3_20", "c2_24_metis"])
def test_dmma_indefinite_inertia_and_backward_error(case):
    if case == "c1_128":
        a, st, cx = matgen.c1_matrix(128), SolverSettings(**TENSOR), False
    elif case == "c3_20":
        a, st, cx = matgen.c3_matrix(20), SolverSettings(**TENSOR), False
    else:
        a, st, cx = matgen.c2_matrix(24), SolverSettings(ordering=Ordering.METIS_ND, **TENSOR), True
    sym = LdltSymbolic.analyze_with(a, st)
    dm = sym.factor(a, st)
    orc = OracleSolver(a, sym.export())
    assert tuple(dm.inertia()) == orc.factors().inertia
    b = matgen.uniform_rhs(a.n, 8, 3, complex_=cx)
    x = dm.solve_many(b, 8)
    xo = orc.solve_many(b, 8)
    assert backward_error(a, x, b) <= max(1e-13, 10 * backward_error(a, xo, b))
    assert rel_err(x, xo) <= 1e-9


def test_dmma_deterministic():
    a = matgen.c2_matrix(20)
    st = SolverSettings(ordering=Ordering.METIS_ND, **TENSOR)
    sym = LdltSymbolic.analyze_with(a, st)
    f1 = sym.factor(a, st).export_factors()
    f2 = sym.factor(a, st).export_factors()
    assert np.array_equal(f1.l_values, f2.l_values) and np.array_equal(f1.d_diag, f2.d_diag)


KKT = kkt_cases()


@pytest.mark.parametrize("case", KKT, ids=[c[0]["name"] for c in KKT])
def test_dmma_kkt_fixtures(case):
    """The reference's KKT fixtures through the DMMA tiles: the oracle's
    inertia wherever the fixture's own second solver agrees with it (where
    it does not, the matrix is singular to working precision and the sign of
    its smallest pivot is rounding), backward error at the oracle's level."""
    e, a, rhs = case
    st = SolverSettings(**TENSOR)
    sym = LdltSymbolic.analyze_with(a, st)
    orc = OracleSolver(a, sym.export())
    o = orc.factors()
    if o.status != 0:
        return
    g = sym.factor(a, st)
    ref, second = e["inertia"], e["mumps_inertia"]
    if (second["positive"], second["negative"], second["zero"]) == (ref["positive"], ref["negative"], ref["zero"]):
        assert tuple(g.inertia()) == o.inertia
    x = g.solve(rhs)
    xo = orc.solve_many(rhs, 1)
    assert backward_error(a, x, rhs) <= max(1e-12, 100 * backward_error(a, xo, rhs))


def test_auto_engine_by_size():
    small = matgen.c1_matrix(48)
    sym = LdltSymbolic.analyze(small)
    assert sym.info().flops_model < 2e8
    assert sym.factor(small).diagnostics().schur_engine == "fma"
    big = dominant3d(28, True)
    st = SolverSettings(ordering=Ordering.METIS_ND)
    sym = LdltSymbolic.analyze_with(big, st)
    assert sym.info().flops_model >= 2e8
    assert sym.factor(big, st).diagnostics().schur_engine == "tensor"
    assert sym.factor(big, SolverSettings(ordering=Ordering.METIS_ND, schur_engine="fma")).diagnostics().schur_engine == "fma"
