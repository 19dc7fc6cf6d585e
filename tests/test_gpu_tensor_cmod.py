"""Tensor-core (tcgen05, 3xTF32) descendant updates of the f32 / c32 factor.

The single-precision fields run their cmod updates on the tensor cores by
default: 3xTF32 split products with fp32 accumulation, fp32-level accuracy but
not the oracle's operation order, so parity is by tolerance here (the
bit-exact CUDA-core engine, schur_engine="fma", is pinned against the oracle
in test_gpu_parity.py).  The checks: exact inertia (analytic for shifted
Laplacians), the same pivot sequence as the fp32 FMA factor on matrices
without near-tie pivots, D within fp32 rounding of it, and solve backward
errors at fp32 level.
"""
import numpy as np
import pytest

from oracle.oracle import backward_error
from rslab_b200 import LdltSymbolic, MixedLdltSolver, SolverSettings, matgen

pytestmark = pytest.mark.gpu

CASES = {
    # (matrix, field): 2D real (many small updaters), 3D real with supernodes
    # wider than 128 and tall panels (several 128-row tiles, many K chunks),
    # 3D complex-symmetric Helmholtz
    "f32_2d": (lambda: matgen.c1_matrix(64), np.float32),
    "f32_3d": (lambda: matgen.c3_matrix(20), np.float32),
    "c32_3d": (lambda: matgen.c2_matrix(16), np.complex64),
}


def factor_pair(name):
    mk, dt = CASES[name]
    a = mk()
    sym = LdltSymbolic.analyze(a)
    aa = a.astype(dt)
    tc = sym.factor(aa, SolverSettings(schur_engine="tensor"))
    fma = sym.factor(aa, SolverSettings(schur_engine="fma"))
    return a, aa, sym, tc, fma


@pytest.mark.parametrize("name", list(CASES))
def test_tensor_cmod_matches_fma_factor(name):
    a, aa, sym, tc, fma = factor_pair(name)
    ft, ff = tc.export_factors(), fma.export_factors()
    assert tuple(ft.inertia) == tuple(ff.inertia)
    assert np.array_equal(ft.two_by_two, ff.two_by_two)
    assert np.array_equal(ft.perm, ff.perm)
    scale = float(np.max(np.abs(ff.d_diag)))
    assert float(np.max(np.abs(ft.d_diag - ff.d_diag))) <= 1e-4 * scale
    b = matgen.uniform_rhs(a.n, 4, 7, complex_=np.iscomplexobj(aa.values))
    xt = tc.solve_many(b.astype(aa.values.dtype), 4)
    xf = fma.solve_many(b.astype(aa.values.dtype), 4)
    bt = backward_error(a, xt.astype(np.complex128 if np.iscomplexobj(xt) else np.float64), b)
    bf = backward_error(a, xf.astype(np.complex128 if np.iscomplexobj(xf) else np.float64), b)
    assert bt <= max(1e-5, 10 * bf), (bt, bf)


def test_tensor_cmod_analytic_inertia_3d():
    a, aa, sym, tc, fma = factor_pair("f32_3d")
    side = 20
    dims = (side, side, side)
    neg = matgen.negative_eigs_shifted_laplacian(dims, 0.1 * matgen.lambda_max(dims))
    assert tuple(tc.inertia()) == (a.n - neg, neg, 0)


def test_tensor_cmod_deterministic():
    mk, dt = CASES["c32_3d"]
    a = mk().astype(dt)
    sym = LdltSymbolic.analyze(a)
    f1 = sym.factor(a).export_factors()
    f2 = sym.factor(a).export_factors()
    assert np.array_equal(f1.l_values, f2.l_values) and np.array_equal(f1.d_diag, f2.d_diag)


@pytest.mark.parametrize("kind", ["real", "complex"])
def test_mixed_with_tensor_cmod_certifies(kind):
    a = matgen.c3_matrix(16) if kind == "real" else matgen.c2_matrix(16)
    sym = LdltSymbolic.analyze(a)
    m = MixedLdltSolver.factor_with(a, SolverSettings(schur_engine="tensor"), sym=sym)
    b = matgen.uniform_rhs(a.n, 8, 3, complex_=(kind == "complex"))
    x, info = m.solve_to(a, b, 1e-14)
    assert info.certified
    assert backward_error(a, x, b) <= 1e-14
