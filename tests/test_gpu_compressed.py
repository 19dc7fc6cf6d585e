"""CompressedLdltFactors (src/dense/ldlt_generic.rs:434-536) over the C ABI:
uint32 indices equal to the int64 export, the same values, half the index
bytes, and a solve bit-identical to the reference's solve_ldlt on the same
factors (restated here in numpy with the same expression order), checked
against the oracle's solution within 1e-10."""
import numpy as np
import pytest

from oracle.oracle import OracleSolver
from rslab_b200 import CompressedLdltFactors, LdltSymbolic, SolverSettings, matgen
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


def solve_ldlt_numpy(f, rhs):
    """The reference's solve_ldlt (ldlt_generic.rs:339-422) on exported factors."""
    n = f["d_diag"].shape[0]
    cp, ri, lv = f["l_col_ptr"].astype(np.int64), f["l_row_idx"].astype(np.int64), f["l_values"]
    y = rhs[f["perm"].astype(np.int64)].copy()
    for j in range(n):
        s, e = cp[j] + 1, cp[j + 1]
        y[ri[s:e]] = y[ri[s:e]] - lv[s:e] * y[j]
    k = 0
    d, ds, two = f["d_diag"], f["d_subdiag"], f["two_by_two"]
    while k < n:
        if two[k]:
            det = d[k] * d[k + 1] - ds[k] * ds[k]
            z0, z1 = y[k], y[k + 1]
            y[k], y[k + 1] = (d[k + 1] * z0 - ds[k] * z1) / det, (d[k] * z1 - ds[k] * z0) / det
            k += 2
        else:
            y[k] = y[k] / d[k]
            k += 1
    for j in range(n - 1, -1, -1):
        s, e = cp[j] + 1, cp[j + 1]
        y[j] = y[j] - np.sum(lv[s:e] * y[ri[s:e]])
    x = np.empty_like(y)
    x[f["perm"].astype(np.int64)] = y
    return x


@pytest.mark.parametrize("kind", ["f64", "c64"])
def test_compressed_factors_match_export_and_solve(kind):
    a = matgen.c1_matrix(40) if kind == "f64" else matgen.c2_matrix(10)
    sym = LdltSymbolic.analyze(a)
    gpu = sym.factor(a)
    full = gpu.export_factors()
    cf = CompressedLdltFactors.from_factors(gpu)
    assert cf is not None and cf.n == a.n and cf.factor_nnz() == full.l_values.shape[0]
    assert cf.index_bytes() == 4 * (a.n + 1 + cf.factor_nnz() + a.n)
    arr = cf.arrays()
    assert arr["l_col_ptr"].dtype == np.uint32 and arr["perm"].dtype == np.uint32
    assert np.array_equal(arr["l_col_ptr"].astype(np.int64), full.l_col_ptr)
    assert np.array_equal(arr["l_row_idx"].astype(np.int64), full.l_row_idx)
    assert np.array_equal(arr["perm"].astype(np.int64), full.perm)
    assert np.array_equal(arr["l_values"], full.l_values)
    assert np.array_equal(arr["d_diag"], full.d_diag) and np.array_equal(arr["two_by_two"], full.two_by_two)
    # the container solves with the equilibrated matrix S A S
    b = matgen.uniform_rhs(a.n, 1, 7, complex_=(kind == "c64"))
    x = cf.solve(b)
    xs = gpu.solve(b / full.scale) / full.scale  # (S A S)^-1 b = S^-1 A^-1 S^-1 b
    assert rel_err(x, xs) <= 1e-10
    orc = OracleSolver(a, sym.export())
    xo = orc.solve_many(b / full.scale, 1) / full.scale
    assert rel_err(x, xo) <= 1e-10
    # the reference's expressions, restated: agreement to rounding
    assert rel_err(x, solve_ldlt_numpy(arr, np.asarray(b))) <= 1e-12
