"""`rslab_b200.ldlt(A)` — the drop-in for RSLAB's Python `rslab.ldlt`
(python/rslab/__init__.py:155, python/src/lib.rs:861-948): scipy input,
dtype-selected field, solve / solve_many / refine, preconditioner (static
pivoting), force_accept and drop_tol, checked by residuals and, for
drop_tol, entry by entry against the oracle's factor with the reference's
per-column drop rule (multifrontal_ldlt.rs:2359-2367) applied on the host.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.oracle import OracleSolver
from rslab_b200 import LdltSymbolic, NumericallyRankDeficient, SolverSettings, ldlt, matgen

pytestmark = pytest.mark.gpu


def sym_dominant(n, seed, complex_=False, nnz_per_row=5):
    rng = np.random.default_rng(seed)
    m = sp.random(n, n, density=nnz_per_row / n, format="csc", random_state=rng)
    if complex_:
        m = m + 1j * sp.random(n, n, density=nnz_per_row / n, format="csc", random_state=rng)
    a = m + m.T + sp.eye(n) * (2.0 * nnz_per_row + 1.0)
    return a.tocsc()


def rel_res(A, x, b):
    return float(np.linalg.norm(A @ x - b) / max(np.linalg.norm(b), 1.0))


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-5)])
def test_ldlt_real(dtype, tol):
    A = sym_dominant(300, 1).astype(dtype)
    b = np.linspace(-1, 1, 300).astype(dtype)
    f = ldlt(A)
    assert f.dtype == np.dtype(dtype).name
    assert f.n == 300 and f.factor_nnz >= 300
    assert f.inertia == (300, 0, 0)
    assert rel_res(A.astype(np.float64), f.solve(b).astype(np.float64), b) < tol


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-12), (np.complex64, 1e-5)])
def test_ldlt_complex_symmetric(dtype, tol):
    A = sym_dominant(250, 2, complex_=True).astype(dtype)
    assert abs(A - A.T).max() == 0  # complex-symmetric, not Hermitian
    b = (np.arange(250) % 7 - 3 + 1j).astype(dtype)
    f = ldlt(A)
    assert f.dtype == np.dtype(dtype).name
    assert rel_res(A.astype(np.complex128), f.solve(b).astype(np.complex128), b) < tol


def test_full_or_triangular_input_same_factor():
    A = sym_dominant(120, 3)
    b = np.ones(120)
    x1 = ldlt(A).solve(b)
    x2 = ldlt(sp.tril(A)).solve(b)
    assert np.array_equal(x1, x2)


def test_solve_many_matches_columns():
    A = sym_dominant(160, 4)
    B = np.random.default_rng(5).standard_normal((160, 6))
    f = ldlt(A)
    X = f.solve_many(np.ascontiguousarray(B))
    assert X.shape == (160, 6)
    for c in range(6):
        assert rel_res(A, X[:, c], B[:, c]) < 1e-12


def test_indefinite_inertia_matches_analytic():
    # shifted 2D Laplacian: the negative-eigenvalue count is analytic
    a = matgen.c1_matrix(32)
    A = sp.csc_matrix((a.values, a.row_idx, a.col_ptr), shape=(a.n, a.n))
    f = ldlt(A)
    dims = (32, 32)
    neg = matgen.negative_eigs_shifted_laplacian(dims, 0.3 * matgen.lambda_max(dims))
    assert f.inertia == (a.n - neg, neg, 0)


def test_preconditioner_refine_recovers_accuracy():
    # a zero diagonal entry coupled to one neighbour: the static-pivot factor
    # plus refinement against A reaches full accuracy
    A = sym_dominant(200, 6).tolil()
    A[17, 17] = 0.0
    A[17, :] = 0.0
    A[:, 17] = 0.0
    A[17, 17] = 0.0
    A[17, 18] = A[18, 17] = 1.0
    A = A.tocsc()
    b = np.ones(200)
    f = ldlt(A, preconditioner=1e-4)
    x = f.solve(b, refine=20)
    assert rel_res(A, x, b) < 1e-10


def test_force_accept_on_zero_pivot():
    A = sp.diags([2.0, 0.0, 3.0]).tocsc()
    with pytest.raises(NumericallyRankDeficient):
        ldlt(A)
    f = ldlt(A, force_accept=True)
    assert f.n_perturbed == 1


def test_dtype_mismatch_rejected():
    f = ldlt(sym_dominant(50, 7))
    with pytest.raises(ValueError):
        f.solve(np.ones(50, dtype=np.float32))


def drop_rule(lf, tau):
    """The reference's per-column drop on an exported CSC factor."""
    cp, ri, lv = lf.l_col_ptr, lf.l_row_idx, lf.l_values
    keep = np.ones(len(lv), bool)
    for j in range(len(cp) - 1):
        sl = slice(cp[j], cp[j + 1])
        rows, vals = ri[sl], lv[sl]
        off = rows != j
        cm = np.max(np.abs(vals[off])) if off.any() else 0.0
        keep[sl] = (~off) | (np.abs(vals) >= tau * cm)
    # every column keeps at least its unit diagonal, so no column is empty
    kept = np.add.reduceat(keep.astype(np.int64), cp[:-1])
    return ri[keep], lv[keep], np.concatenate([[0], np.cumsum(kept)])


def test_drop_tol_matches_oracle_rule():
    a = matgen.c3_matrix(12)
    tau = 0.05
    sym = LdltSymbolic.analyze(a)
    # the bit-exact engine: the kept entries are compared with the oracle's exactly
    full = sym.factor(a, SolverSettings(drop_tol=None, schur_engine="fma")).export_factors()
    inc = sym.factor(a, SolverSettings(drop_tol=tau, schur_engine="fma")).export_factors()
    ref = OracleSolver(a, sym.export()).factors()
    r_idx, r_val, r_ptr = drop_rule(ref, tau)
    assert len(inc.l_values) < len(full.l_values)
    assert np.array_equal(inc.l_row_idx, r_idx)
    assert np.array_equal(inc.l_values, r_val)
    assert np.array_equal(inc.l_col_ptr, r_ptr)
    # as a preconditioner for refinement on a diagonally dominant system
    A = sym_dominant(400, 8, nnz_per_row=12)
    f = ldlt(A, drop_tol=tau)
    assert f.factor_nnz < ldlt(A).factor_nnz
    b = np.ones(400)
    assert rel_res(A, f.solve(b, refine=40), b) < 1e-10


@pytest.mark.parametrize("complex_", [False, True])
def test_method_multifrontal_solves_alike(complex_):
    """`method="multifrontal"` factors with contribution blocks and
    extend-add; it solves like the left-looking default (the reference's LL
    vs MF check is a 1e-9 solution tolerance, multifrontal_ldlt.rs:3865-3883)
    with the same inertia."""
    A = sym_dominant(400, 6, complex_=complex_)
    b = np.linspace(-1, 1, 400) + (0.5j if complex_ else 0.0)
    ll, mf = ldlt(A), ldlt(A, method="multifrontal")
    assert mf.inertia == ll.inertia
    xl, xm = ll.solve(b), mf.solve(b)
    assert np.max(np.abs(xm - xl)) <= 1e-9 * np.max(np.abs(xl))
    assert rel_res(A, xm, b) < 1e-12
