"""The GPU numeric path on MetisND structures (the C2 configuration's
ordering, and the one LdltSolver::tuned adopts on 3D grids) against the CPU
oracle on the same seeded inputs.  Tolerances: FP64 factors within 1e-12
relative with identical inertia and pivot sequence, solves within 1e-10 of
the oracle's solution; the tensor-core (c32, 3xTF32) engine: exact inertia on
real indefinite grids, certified normwise backward error <= 1e-14 after FP64
refinement, and forward error against the FP64 oracle's solution <= 1e-10."""
import numpy as np
import pytest

from oracle.oracle import OracleSolver, backward_error
from rslab_b200 import LdltSolver, LdltSymbolic, MixedLdltSolver, Ordering, SolverSettings, matgen
from tests.helpers import rel_err
from tests.test_gpu_parity import check_factors

pytestmark = pytest.mark.gpu

# oracle comparisons run the bit-exact CUDA-core engine (exact pivot
# sequences); the mixed paths run the default tensor-core engine
ND = SolverSettings(ordering=Ordering.METIS_ND, schur_engine="fma")
ND_T = SolverSettings(ordering=Ordering.METIS_ND)


def nd_both(a):
    sym = LdltSymbolic.analyze_with(a, ND)
    gpu = sym.factor(a, ND)
    orc = OracleSolver(a, sym.export(), panel_nb=ND.panel_nb)
    return sym, gpu, orc


@pytest.mark.parametrize("side", [16, 20, 24])
def test_metis_helmholtz_fp64_matches_oracle(side):
    a = matgen.c2_matrix(side)
    sym, gpu, orc = nd_both(a)
    check_factors(gpu, orc, a.n)
    b = matgen.uniform_rhs(a.n, 16, 1, complex_=True)
    x = gpu.solve_many(b, 16)
    xo = orc.solve_many(b, 16)
    assert rel_err(x, xo) <= 1e-10
    assert backward_error(a, x, b) <= max(1e-13, 10 * backward_error(a, xo, b))


@pytest.mark.parametrize("side", [16, 24])
def test_metis_real_laplacian_fp64_matches_oracle_and_analytic_inertia(side):
    a = matgen.c3_matrix(side)
    sym, gpu, orc = nd_both(a)
    g, _ = check_factors(gpu, orc, a.n)
    dims = (side,) * 3
    neg = matgen.negative_eigs_shifted_laplacian(dims, 0.1 * matgen.lambda_max(dims))
    assert tuple(g.inertia) == (a.n - neg, neg, 0)


@pytest.mark.parametrize("side", [24, 32])
def test_metis_tensor_engine_inertia_and_certificate(side):
    """c32 factor with tensor-core descendant updates on a real indefinite
    grid: the inertia is exact (the analytic count), and the FP64 ladder
    certifies 1e-14 against the original matrix."""
    a = matgen.c3_matrix(side)
    dims = (side,) * 3
    neg = matgen.negative_eigs_shifted_laplacian(dims, 0.1 * matgen.lambda_max(dims))
    m = MixedLdltSolver.factor_with(a, ND_T)
    assert tuple(m.inertia()) == (a.n - neg, neg, 0)
    b = matgen.uniform_rhs(a.n, 4, 2)
    x, info = m.solve_to(a, b, 1e-14)
    assert info.certified and info.backward_error <= 1e-14
    assert backward_error(a, x, b) <= 1e-14


def test_metis_helmholtz_40_fp64_and_mixed_against_oracle():
    """The largest C2-family case the oracle factors in seconds: FP64 factor
    within 1e-12 of the oracle's; the mixed (c32 tensor-core) solution's
    forward error measured against the oracle's FP64 solution."""
    a = matgen.c2_matrix(40)
    sym, gpu, orc = nd_both(a)
    check_factors(gpu, orc, a.n)
    b = matgen.uniform_rhs(a.n, 16, 1, complex_=True)
    xo = orc.solve_many(b, 16)
    assert rel_err(gpu.solve_many(b, 16), xo) <= 1e-10
    m = MixedLdltSolver.factor_with(a, ND_T, sym=sym)
    x, info = m.solve_to(a, b, 1e-14)
    assert info.certified and info.backward_error <= 1e-14
    assert backward_error(a, x, b) <= 1e-14
    assert rel_err(x, xo) <= 1e-10


def test_default_entry_point_takes_the_bakeoff_pick():
    """LdltSolver.factor (LdltSolver::tuned, default engines) on a 32^3
    Helmholtz pattern adopts MetisND; its inertia equals the oracle's on that
    structure and its solution agrees within 1e-10."""
    a = matgen.c2_matrix(32)
    sym, s = LdltSymbolic.tuned(a)
    assert s.ordering == Ordering.METIS_ND
    gpu = LdltSolver.factor(a)
    orc = OracleSolver(a, sym.export())
    assert tuple(gpu.inertia()) == orc.factors().inertia
    b = matgen.uniform_rhs(a.n, 4, 1, complex_=True)
    assert rel_err(gpu.solve_many(b, 4), orc.solve_many(b, 4)) <= 1e-10
