"""The CPU oracle pinned to the reference's known answers before it is
trusted as the parity checker:
  * hand-computed solves (src/dense/ldlt_generic.rs:837-915);
  * inertia signatures (src/numeric/sparse_solver.rs:1007-1033);
  * MUMPS inertia of the reference's KKT fixtures (tests/data/parity);
  * the analytic inertia of shifted Dirichlet Laplacians (separable spectrum).
"""
import numpy as np
import pytest

from oracle.oracle import OracleSolver, backward_error, mixed_solve
from rslab_b200 import CscMatrix, LdltSymbolic, SolverSettings
from rslab_b200 import matgen
from tests.helpers import kkt_cases


def oracle_for(a, **kw):
    return OracleSolver(a, LdltSymbolic.analyze(a).export(), **kw)


def test_antidiagonal_2x2_real():
    a = CscMatrix.from_triplets(2, [0, 1, 1], [0, 0, 1], [0.0, 1.0, 0.0])
    o = oracle_for(a)
    assert np.allclose(o.solve_many(np.array([3.0, 5.0]), 1), [5.0, 3.0], atol=1e-12)
    f = o.factors()
    assert f.inertia == (1, 1, 0)
    assert f.two_by_two[0]


def test_antidiagonal_2x2_complex():
    a = CscMatrix.from_triplets(2, [0, 1, 1], [0, 0, 1], np.array([0, 1, 0], dtype=complex))
    x = oracle_for(a).solve_many(np.array([1 + 1j, 2 - 1j]), 1)
    assert np.allclose(x, [2 - 1j, 1 + 1j], atol=1e-12)


def test_indefinite_5x5_residual():
    e = [(0, 0, 1.0), (1, 0, 3.0), (1, 1, 2.0), (2, 0, 0.5), (2, 1, -1.0), (2, 2, -4.0), (3, 1, 2.0), (3, 2, 1.0),
         (3, 3, 0.0), (4, 0, -2.0), (4, 3, 3.0), (4, 4, 1.0)]
    r, c, v = zip(*e)
    a = CscMatrix.from_triplets(5, r, c, v)
    b = np.array([1.0, -2.0, 3.0, 0.5, -1.5])
    x = oracle_for(a).solve_many(b, 1)
    assert np.max(np.abs(a.to_scipy_full() @ x - b)) < 1e-10


def test_diagonal_inertia_signature():
    a = CscMatrix.from_triplets(5, range(5), range(5), [2.0, -3, 4, -1, 5])
    assert oracle_for(a).factors().inertia == (3, 2, 0)


@pytest.mark.parametrize("side", [16, 40, 96])
def test_shifted_laplacian_analytic_inertia(side):
    dims = (side, side)
    a = matgen.c1_matrix(side)
    f = oracle_for(a).factors()
    neg = matgen.negative_eigs_shifted_laplacian(dims, 0.3 * matgen.lambda_max(dims))
    assert f.inertia == (a.n - neg, neg, 0)


def test_3d_shifted_laplacian_analytic_inertia():
    dims = (12, 12, 12)
    a = matgen.c3_matrix(12)
    f = oracle_for(a).factors()
    neg = matgen.negative_eigs_shifted_laplacian(dims, 0.1 * matgen.lambda_max(dims))
    assert f.inertia == (a.n - neg, neg, 0)


KKT = kkt_cases()
# Fixtures on which the oracle's panel-bounded BK (no delayed pivots) matches
# the MUMPS inertia; the reference manifest marks the others as inertia
# failures of the reference solver itself or they need a delayed pivot.
MUMPS_MATCH = [c for c in KKT if c[0]["name"] not in {
    "ACOPP14_0001", "ACOPP14_0003", "ACOPP30_0000", "CERI651CLS_0486", "CERI651CLS_0487", "CERI651DLS_0618",
    "DALLASS_0026", "HATFLDG_0003", "HATFLDG_0004", "HATFLDG_0005", "HATFLDG_0006", "HYDCAR20_0000",
    "SWOPF_0000"}]


@pytest.mark.parametrize("case", MUMPS_MATCH, ids=[c[0]["name"] for c in MUMPS_MATCH])
def test_kkt_inertia_matches_mumps(case):
    e, a, rhs = case
    o = oracle_for(a)
    f = o.factors()
    exp = e["mumps_inertia"]
    assert f.status == 0
    assert f.inertia == (exp["positive"], exp["negative"], exp["zero"])
    x = o.solve_many(rhs, 1)
    assert backward_error(a, x, rhs) < 1e-6


def test_singular_block_rejected_and_perturb_rescues():
    e, a, rhs = next(c for c in KKT if c[0]["name"] == "HYDCAR20_0000")
    assert oracle_for(a).factors().status == 1
    o = oracle_for(a, perturb_floor=1e-10)
    f = o.factors()
    assert f.status == 0 and f.n_perturbed > 0


def test_mixed_oracle_certifies_laplacian():
    a = matgen.c1_matrix(40)
    sym = LdltSymbolic.analyze(a)
    lo = OracleSolver(a, sym.export(), dtype=np.float32)
    b = matgen.uniform_rhs(a.n, 1, 0)
    x, info = mixed_solve(lo, a, b, 64 * 2.220446049250313e-16)
    hi = OracleSolver(a, sym.export()).solve_many(b, 1)
    assert info["certified"]
    assert np.max(np.abs(x - hi)) / np.max(np.abs(hi)) < 1e-10
