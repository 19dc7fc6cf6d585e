"""Tensor-core (tcgen05, 3xTF32) descendant updates of the f32 / c32 factor.

The single-precision fields run their cmod updates on the tensor cores by
default: 3xTF32 split products with fp32 accumulation, fp32-level accuracy but
not the oracle's operation order, so parity is by tolerance here (the
bit-exact CUDA-core engine, schur_engine="fma", is pinned against the oracle
in test_gpu_parity.py).  The checks: on a fixed pivot sequence (diagonally
dominant stencils) L and D agree with the FP64 factor to fp32 level entry by
entry; on indefinite matrices exact inertia (analytic for shifted
Laplacians) and fp32-level solve backward errors (there, grid Laplacians hold
exact magnitude ties that rounding at the fp32 level may break either way,
so the pivot sequences of the two engines need not agree).
"""
import numpy as np
import pytest

from oracle.oracle import backward_error
from rslab_b200 import LdltSymbolic, MixedLdltSolver, SolverSettings, matgen

pytestmark = pytest.mark.gpu

def spd3d(side, complex_):
    """Diagonally dominant 3D stencils: Bunch-Kaufman takes every diagonal
    1x1 pivot in order, so both engines follow the same pivot sequence and
    their factors compare entry by entry."""
    dims = (side, side, side)
    lm = matgen.lambda_max(dims)
    if complex_:
        return matgen.helmholtz(dims, complex(-0.5 * lm, 0.05 * lm))
    return matgen.shifted_laplacian(dims, -0.5 * lm)


CASES = {
    # (matrix, field): 2D real indefinite (many small updaters), 3D real
    # indefinite with supernodes wider than 128 and tall panels (several
    # 128-row tiles, many K chunks), 3D complex-symmetric Helmholtz
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


def as_hi(x):
    return x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)


@pytest.mark.parametrize("complex_,side,metis", [(False, 20, False), (True, 20, False), (False, 28, True),
                                                 (True, 28, True)])
def test_tensor_cmod_entrywise_on_fixed_pivot_sequence(complex_, side, metis):
    """MetisND structures add wide separator updaters: updates of more than
    64 columns (several W column tiles), taller than 128 rows, many K chunks."""
    a = spd3d(side, complex_)
    dt = np.complex64 if complex_ else np.float32
    from rslab_b200 import Ordering
    sym = LdltSymbolic.analyze_with(a, SolverSettings(ordering=Ordering.METIS_ND if metis else Ordering.AMD))
    f64 = sym.factor(a).export_factors()
    tc = sym.factor(a.astype(dt), SolverSettings(schur_engine="tensor")).export_factors()
    fma = sym.factor(a.astype(dt), SolverSettings(schur_engine="fma")).export_factors()
    for f in (tc, fma):
        assert np.array_equal(f.two_by_two, f64.two_by_two) and np.array_equal(f.perm, f64.perm)
        assert np.array_equal(f.l_col_ptr, f64.l_col_ptr) and np.array_equal(f.l_row_idx, f64.l_row_idx)
    ld = float(np.max(np.abs(as_hi(tc.d_diag) - f64.d_diag) / np.abs(f64.d_diag)))
    ll = float(np.max(np.abs(as_hi(tc.l_values) - f64.l_values)) / np.max(np.abs(f64.l_values)))
    ld_f = float(np.max(np.abs(as_hi(fma.d_diag) - f64.d_diag) / np.abs(f64.d_diag)))
    # fp32-level agreement with the FP64 factor, like the fp32 FMA engine
    assert ld <= 2e-6 and ll <= 2e-6, (ld, ll, ld_f)


@pytest.mark.parametrize("name", list(CASES))
def test_tensor_cmod_indefinite_inertia_and_backward_error(name):
    a, aa, sym, tc, fma = factor_pair(name)
    assert tuple(tc.inertia()) == tuple(fma.inertia())
    b = matgen.uniform_rhs(a.n, 4, 7, complex_=np.iscomplexobj(aa.values))
    xt = tc.solve_many(b.astype(aa.values.dtype), 4)
    xf = fma.solve_many(b.astype(aa.values.dtype), 4)
    bt = backward_error(a, as_hi(xt), b)
    bf = backward_error(a, as_hi(xf), b)
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
    st = SolverSettings(schur_engine="tensor")
    f1 = sym.factor(a, st).export_factors()
    f2 = sym.factor(a, st).export_factors()
    assert np.array_equal(f1.l_values, f2.l_values) and np.array_equal(f1.d_diag, f2.d_diag)


@pytest.mark.parametrize("nb", [32, 64])
def test_tensor_engine_with_panel_widths(nb):
    """The tensor engine's panel kernels (left-looking getf2, block transform
    of the deep rows, tensor-core in-panel Schur) with 32- and 64-wide blocks
    (128 for the wide separators): on a fixed pivot sequence the factor
    agrees with the FP64 one at fp32 level."""
    from rslab_b200 import Ordering
    a = spd3d(24, True)
    st = SolverSettings(ordering=Ordering.METIS_ND, panel_nb=nb)
    sym = LdltSymbolic.analyze_with(a, st)
    f64 = sym.factor(a, SolverSettings(ordering=Ordering.METIS_ND, panel_nb=nb, schur_engine="fma")).export_factors()
    tc = sym.factor(a.astype(np.complex64),
                    SolverSettings(ordering=Ordering.METIS_ND, panel_nb=nb, schur_engine="tensor")).export_factors()
    assert np.array_equal(tc.perm, f64.perm)
    ld = float(np.max(np.abs(as_hi(tc.d_diag) - f64.d_diag) / np.abs(f64.d_diag)))
    ll = float(np.max(np.abs(as_hi(tc.l_values) - f64.l_values)) / np.max(np.abs(f64.l_values)))
    assert ld <= 2e-6 and ll <= 2e-6, (ld, ll)


@pytest.mark.parametrize("kind", ["real", "complex"])
def test_mixed_with_tensor_cmod_certifies(kind):
    a = matgen.c3_matrix(16) if kind == "real" else matgen.c2_matrix(16)
    sym = LdltSymbolic.analyze(a)
    m = MixedLdltSolver.factor_with(a, SolverSettings(schur_engine="tensor"), sym=sym)
    b = matgen.uniform_rhs(a.n, 8, 3, complex_=(kind == "complex"))
    x, info = m.solve_to(a, b, 1e-14)
    assert info.certified
    assert backward_error(a, x, b) <= 1e-14
