"""GPU numeric path (librslab_b200.so through its C ABI) against the CPU
oracle on the same seeded inputs.  Tolerances (FP64 paths): factor L and D
within 1e-12 relative (max-abs over the union pattern, relative to the
oracle's max), identical inertia and pivot sequence (two_by_two + pivot
permutation) on matrices without near-tie pivots, solve backward error
<= 1e-13 or within 10x the oracle's, mixed-precision solves certified at
64 eps against the original matrix."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle.oracle import OracleSolver, backward_error, mixed_solve
from rslab_b200 import (CscMatrix, LdltSolver, LdltSymbolic, MixedLdltSolver, NumericallyRankDeficient,
                        SolverSettings, ZeroPivotAction)
from rslab_b200 import matgen
from tests.helpers import kkt_cases, rel_err

pytestmark = pytest.mark.gpu

EPS = 2.220446049250313e-16


def both(a, settings=None, dtype=None):
    # the bit-exact CUDA-core engine: the oracle's operation order, so pivot
    # sequences and factors compare exactly (the default FP64 engine, DMMA
    # tiles, is checked by tolerance in test_gpu_fp64_dmma.py)
    settings = settings or SolverSettings(schur_engine="fma")
    sym = LdltSymbolic.analyze_with(a, settings)
    aa = a if dtype is None else a.astype(dtype)
    gpu = sym.factor(aa, settings)
    orc = OracleSolver(aa, sym.export(), panel_nb=settings.panel_nb)
    return sym, gpu, orc


def l_matrix(f, n):
    return sp.csc_matrix((f.l_values, f.l_row_idx, f.l_col_ptr), shape=(n, n))


def _first_diff(a, b):
    idx = np.nonzero(a != b)[0]
    return int(idx[0]) if len(idx) else -1


def check_factors(gpu, orc, n, tol=1e-12, pivots=True):
    """GPU vs oracle factors.  The GPU kernels use the oracle's operation order
    (non-contracted elementwise ops, FMA-accumulated Schur products in
    ascending order), so the factors are expected bit-identical; the assertion
    is the 1e-12 relative tolerance."""
    g = gpu.export_factors()
    o = orc.factors()
    assert o.status == 0
    assert tuple(g.inertia) == o.inertia
    if pivots:
        assert np.array_equal(g.two_by_two, o.two_by_two), \
            f"2x2 pivot pattern differs first at e={_first_diff(g.two_by_two, o.two_by_two)}"
        assert np.array_equal(g.perm, o.perm), f"pivot permutation differs first at e={_first_diff(g.perm, o.perm)}"
    assert rel_err(g.scale, o.scale) == 0.0
    assert rel_err(g.d_diag, o.d_diag) <= tol, f"D differs first at e={_first_diff(g.d_diag, o.d_diag)}"
    assert rel_err(g.d_subdiag, o.d_subdiag) <= tol
    dl = abs(l_matrix(g, n) - l_matrix(o, n)).max()
    assert dl / max(abs(o.l_values).max(), 1e-300) <= tol
    return g, o


def bit_identical(g, o) -> bool:
    return (np.array_equal(g.d_diag, o.d_diag) and np.array_equal(g.l_col_ptr, o.l_col_ptr)
            and np.array_equal(g.l_row_idx, o.l_row_idx) and np.array_equal(g.l_values, o.l_values))


def test_antidiagonal_2x2():
    a = CscMatrix.from_triplets(2, [0, 1, 1], [0, 0, 1], [0.0, 1.0, 0.0])
    s = LdltSolver.factor(a)
    assert np.allclose(s.solve(np.array([3.0, 5.0])), [5.0, 3.0], atol=1e-12)
    assert tuple(s.inertia()) == (1, 1, 0)
    ac = a.astype(np.complex128)
    sc = LdltSolver.factor(ac)
    assert np.allclose(sc.solve(np.array([1 + 1j, 2 - 1j])), [2 - 1j, 1 + 1j], atol=1e-12)


def test_diagonal_inertia():
    a = CscMatrix.from_triplets(5, range(5), range(5), [2.0, -3, 4, -1, 5])
    assert tuple(LdltSolver.factor(a).inertia()) == (3, 2, 0)


@pytest.mark.parametrize("side", [16, 40, 128])
def test_shifted_laplacian_2d(side):
    a = matgen.c1_matrix(side)
    sym, gpu, orc = both(a)
    g, o = check_factors(gpu, orc, a.n)
    dims = (side, side)
    neg = matgen.negative_eigs_shifted_laplacian(dims, 0.3 * matgen.lambda_max(dims))
    assert tuple(g.inertia) == (a.n - neg, neg, 0)
    b = matgen.uniform_rhs(a.n, 1, 0)
    x = gpu.solve(b)
    xo = orc.solve_many(b, 1)
    assert rel_err(x, xo) <= 1e-10
    assert backward_error(a, x, b) <= max(1e-13, 10 * backward_error(a, xo, b))


@pytest.mark.parametrize("side", [8, 14])
def test_helmholtz_3d_complex(side):
    a = matgen.c2_matrix(side)
    sym, gpu, orc = both(a)
    check_factors(gpu, orc, a.n)
    b = matgen.uniform_rhs(a.n, 16, 1, complex_=True)
    x = gpu.solve_many(b, 16)
    xo = orc.solve_many(b, 16)
    assert rel_err(x, xo) <= 1e-10
    assert backward_error(a, x, b) <= max(1e-13, 10 * backward_error(a, xo, b))


def test_wide_supernodes_multi_block():
    # dense-ish 3D problem: supernodes wider than one 64-column panel block,
    # tall deep-row replays and the deferred in-panel Schur update
    a = matgen.c3_matrix(20)
    sym, gpu, orc = both(a)
    assert sym.export()["sn_ncol"].max() > 128
    g, o = check_factors(gpu, orc, a.n)
    assert bit_identical(g, o)


@pytest.mark.parametrize("kind", ["f64", "c64", "f32", "c32"])
def test_factor_bit_identical_to_oracle(kind):
    dt = {"f64": np.float64, "c64": np.complex128, "f32": np.float32, "c32": np.complex64}[kind]
    a = matgen.c2_matrix(12) if kind.startswith("c") else matgen.c1_matrix(48)
    # single-precision descendant updates on the CUDA cores: the oracle's operation order
    sym, gpu, orc = both(a, settings=SolverSettings(schur_engine="fma"), dtype=dt)
    g = gpu.export_factors()
    o = orc.factors()
    assert tuple(g.inertia) == o.inertia
    assert bit_identical(g, o)


@pytest.mark.parametrize("nrhs", [1, 5, 16, 21])
def test_multi_rhs_matches_columnwise(nrhs):
    a = matgen.c3_matrix(10)
    s = LdltSolver.factor(a)
    b = matgen.uniform_rhs(a.n, nrhs, 3)
    x = s.solve_many(b, nrhs).reshape(a.n, nrhs)
    b2 = b.reshape(a.n, nrhs)
    for c in range(nrhs):
        xc = s.solve(b2[:, c].copy())
        assert rel_err(x[:, c], xc) <= 1e-13


KKT = kkt_cases()


@pytest.mark.parametrize("case", KKT, ids=[c[0]["name"] for c in KKT])
def test_kkt_fixtures_match_oracle(case):
    e, a, rhs = case
    sym = LdltSymbolic.analyze(a)
    orc = OracleSolver(a, sym.export())
    o = orc.factors()
    if o.status != 0:
        with pytest.raises(NumericallyRankDeficient):
            sym.factor(a)
        return
    gpu = sym.factor(a)
    g = gpu.export_factors()
    assert tuple(g.inertia) == o.inertia
    x = gpu.solve(rhs)
    xo = orc.solve_many(rhs, 1)
    assert backward_error(a, x, rhs) <= max(1e-12, 100 * backward_error(a, xo, rhs))


def test_static_pivoting_matches_oracle():
    e, a, rhs = next(c for c in KKT if c[0]["name"] == "HYDCAR20_0000")
    st = SolverSettings.preconditioner(1e-10)
    st.schur_engine = "fma"
    sym = LdltSymbolic.analyze(a)
    gpu = sym.factor(a, st)
    o = OracleSolver(a, sym.export(), perturb_floor=1e-10).factors()
    assert gpu.n_perturbed() == o.n_perturbed > 0
    assert tuple(gpu.inertia()) == o.inertia


def test_refactor_same_pattern():
    a = matgen.c1_matrix(40)
    sym = LdltSymbolic.analyze(a)
    s = sym.factor(a)
    a2 = CscMatrix(a.n, a.col_ptr, a.row_idx, a.values * 1.5 + 0.01)
    s.refactor(a2)
    ref = sym.factor(a2)
    b = matgen.uniform_rhs(a.n, 1, 5)
    assert np.array_equal(s.solve(b), ref.solve(b))


def test_graph_and_eager_bit_identical_and_deterministic():
    a = matgen.c2_matrix(10)
    sym = LdltSymbolic.analyze(a)
    b = matgen.uniform_rhs(a.n, 4, 9, complex_=True)
    xs = []
    for use_graph in (True, False, True):
        st = SolverSettings(use_graph=use_graph)
        s = sym.factor(a, st)
        xs.append(s.solve_many(b, 4))
    assert np.array_equal(xs[0], xs[1]) and np.array_equal(xs[0], xs[2])


@pytest.mark.parametrize("kind", ["real", "complex"])
def test_mixed_precision_certifies(kind):
    a = matgen.c1_matrix(64) if kind == "real" else matgen.c2_matrix(12)
    sym = LdltSymbolic.analyze(a)
    m = MixedLdltSolver.factor_with(a, SolverSettings(), sym=sym)
    b = matgen.uniform_rhs(a.n, 1, 0, complex_=(kind == "complex"))
    x, info = m.solve(a, b)
    assert info.certified and info.backward_error <= 64 * EPS
    assert backward_error(a, x, b) <= 64 * EPS * 1.01
    lo = OracleSolver(a, sym.export(), dtype=np.float32 if kind == "real" else np.complex64)
    xo, io = mixed_solve(lo, a, b, 64 * EPS)
    assert io["certified"]
    assert rel_err(x, xo) <= 1e-9


def test_mixed_multi_rhs_target():
    a = matgen.c2_matrix(12)
    sym = LdltSymbolic.analyze(a)
    m = MixedLdltSolver.factor_with(a, SolverSettings(), sym=sym)
    b = matgen.uniform_rhs(a.n, 16, 1, complex_=True)
    x, info = m.solve_to(a, b, 1e-14)
    assert info.certified
    assert backward_error(a, x, b) <= 1e-14


def test_rank_deficient_reports_supernode():
    a = CscMatrix.from_triplets(3, [0, 1, 2], [0, 1, 2], [1.0, 0.0, 2.0])
    with pytest.raises(NumericallyRankDeficient):
        LdltSolver.factor(a)
