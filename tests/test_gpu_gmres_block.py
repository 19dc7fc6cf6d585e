"""Block GMRES on the GPU (rslab_gmres_block) with a factored handle as the
preconditioner, against the numpy oracle of the reference's gmres_block and
against direct solves; and the refinement ladder's block GMRES-IR stage."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.krylov import gmres_block as oracle_gmres_block
from oracle.oracle import backward_error
from rslab_b200 import LdltSymbolic, MixedLdltSolver, SolverSettings, matgen
from rslab_b200 import _native as N
from rslab_b200.krylov import gmres_block
from rslab_b200.tiers import tier_settings

pytestmark = pytest.mark.gpu


def _full(a):
    n = a.n
    cp = np.asarray(a.col_ptr)
    col = np.repeat(np.arange(n), np.diff(cp))
    low = sp.csr_matrix((np.asarray(a.values), (np.asarray(a.row_idx), col)), shape=(n, n))
    return low + low.T - sp.diags(low.diagonal())


def _relres(a, x, b):
    r = b - _full(a) @ x
    bn = np.linalg.norm(b, axis=0)
    return np.linalg.norm(r, axis=0) / np.where(bn > 0, bn, 1.0)


def test_refined_c32_handle_preconditions_block_gmres():
    a = matgen.c2_matrix(12)
    b = matgen.uniform_rhs(a.n, 5, 3, complex_=True)
    h = MixedLdltSolver.factor(a)
    r = gmres_block(h, b, 1e-13)
    assert r.converged and 1 <= r.iters <= 10
    assert np.all(r.final_res <= 1e-13)
    assert np.all(_relres(a, r.x, b) <= 2e-13)
    xd = LdltSymbolic.analyze(a).factor(a).solve_many(b, 5)
    assert np.abs(r.x - xd).max() <= 1e-9 * np.abs(xd).max()


def test_matches_the_oracle_with_the_same_preconditioner():
    """The oracle's block GMRES driven by the same c32 factor (a plain c32
    factor of cast(A) is the refined handle's factor): same step count within
    one, same solution within the tolerance."""
    a = matgen.c2_matrix(12)
    b = matgen.uniform_rhs(a.n, 4, 5, complex_=True)
    h = MixedLdltSolver.factor(a)
    r = gmres_block(h, b, 1e-13, restart=8)
    a32 = type(a)(a.n, a.col_ptr, a.row_idx, np.asarray(a.values).astype(np.complex64))
    lo = LdltSymbolic.analyze(a32).factor(a32)
    full = _full(a)

    def pre(rr):
        z = lo.solve_many(np.ascontiguousarray(rr).astype(np.complex64), rr.shape[1])
        return np.asarray(z).reshape(rr.shape).astype(np.complex128)

    xo, ito, convo, fro = oracle_gmres_block(lambda v: full @ v, pre, b, 1e-13, 120, 8)
    assert convo and r.converged
    assert abs(ito - r.iters) <= 1
    assert np.abs(r.x - xo).max() <= 1e-10 * np.abs(xo).max()


def test_fp64_factor_needs_one_step_and_real_handles_work():
    a = matgen.c3_matrix(14)
    b = matgen.uniform_rhs(a.n, 3, 2)
    f64 = LdltSymbolic.analyze(a).factor(a)
    r = gmres_block(f64, b, 1e-13)
    assert r.converged and r.iters <= 1
    h32 = MixedLdltSolver.factor(a)
    r2 = gmres_block(h32, b, 1e-13)
    assert r2.converged and np.all(_relres(a, r2.x, b) <= 2e-13)


def test_many_columns_zero_column_and_warm_start():
    a = matgen.c3_matrix(12)
    b = matgen.uniform_rhs(a.n, 20, 4)  # two groups of columns
    b[:, 7] = 0.0
    h = MixedLdltSolver.factor(a)
    r = gmres_block(h, b, 1e-12)
    assert r.converged and np.all(r.x[:, 7] == 0) and r.final_res[7] == 0
    assert np.all(_relres(a, r.x, b)[np.arange(20) != 7] <= 2e-12)
    r2 = gmres_block(h, b, 1e-10, x0=r.x)
    assert r2.converged and r2.iters == 0


def test_f32_factor_is_rejected_as_operator():
    a = matgen.c3_matrix(8)
    a32 = type(a)(a.n, a.col_ptr, a.row_idx, np.asarray(a.values).astype(np.float32))
    f32 = LdltSymbolic.analyze(a32).factor(a32)
    with pytest.raises(Exception):
        gmres_block(f32, np.ones(a.n, np.float32), 1e-10)


def test_ladder_gmres_ir_certifies_a_hard_matrix():
    """A random sparse symmetric matrix from the tier corpus on which plain
    IR stagnates with the c32 factor: the ladder's GMRES-IR stage runs
    (gmres_iters > 0) and certifies every column."""
    fam, a = list(matgen.c5_corpus(202, 5))[201]
    assert fam == "random_sparse"
    b = matgen.uniform_rhs(a.n, 4, 17)
    h = MixedLdltSolver.factor_tier(a, N.TIER_TF32X3, tier_settings())
    x, info = h.solve_to(a, b, 1e-14)
    assert info.certified and info.gmres_iters > 0
    assert backward_error(a, x, b) <= 1e-14
