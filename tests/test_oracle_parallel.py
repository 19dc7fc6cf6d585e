"""The oracle's timing mode (OpenBLAS products, level-parallel schedule; the
timed CPU baseline) against its exact mode (plain loops in the reference's
operation order; the checker), on the oracle's own symbolic structure.
Host-only.  The two differ only in GEMM summation order: same pivots and
inertia on these matrices, factors within 1e-12 relative, solutions within
1e-10.  The chunked multi-column solve (solve_ldlt_many) is bit-identical to
the single block solve."""
import numpy as np
import pytest

from oracle.oracle import OracleSolver, backward_error, oracle_structure, set_parallel
from rslab_b200 import amd_order, matgen
from rslab_b200.solver import metis_order
from tests.helpers import rel_err


def structure(a, ordering):
    f = a.to_scipy_full().tocsc()
    f.sort_indices()
    cp, ri = np.asarray(f.indptr, np.int64), np.asarray(f.indices, np.int64)
    o = amd_order(a.n, cp, ri)[0] if ordering == "amd" else metis_order(a.n, cp, ri)
    return oracle_structure(a, o)


@pytest.mark.parametrize("case", ["c2_24_metis", "c3_16_amd", "c1_64_amd", "c2_20_c32"])
def test_timing_mode_matches_exact_mode(case):
    if case == "c2_24_metis":
        a, ordering, dt, tol = matgen.c2_matrix(24), "metis", None, 1e-12
    elif case == "c3_16_amd":
        a, ordering, dt, tol = matgen.c3_matrix(16), "amd", None, 1e-12
    elif case == "c1_64_amd":
        a, ordering, dt, tol = matgen.c1_matrix(64), "amd", None, 1e-12
    else:
        a, ordering, dt, tol = matgen.c2_matrix(20), "metis", np.complex64, 1e-4
    ex = structure(a, ordering)
    nrhs = 16
    b = matgen.uniform_rhs(a.n, nrhs, 3, complex_=np.iscomplexobj(a.values))
    try:
        set_parallel(False)
        ref = OracleSolver(a, ex, dtype=dt)
        fr = ref.factors()
        xr = ref.solve_many(b, nrhs)
        set_parallel(True, threads=4)
        fast = OracleSolver(a, ex, dtype=dt)
        ff = fast.factors()
        xf = fast.solve_many(b, nrhs)
    finally:
        set_parallel(False)
    assert fr.status == 0 and ff.status == 0
    assert ff.inertia == fr.inertia
    assert np.array_equal(ff.perm, fr.perm) and np.array_equal(ff.two_by_two, fr.two_by_two)
    assert rel_err(ff.d_diag, fr.d_diag) <= tol
    assert np.array_equal(ff.l_col_ptr, fr.l_col_ptr)
    assert rel_err(ff.l_values, fr.l_values) <= tol
    assert rel_err(xf, xr) <= (1e-10 if dt is None else 1e-3)
    if dt is None:
        assert backward_error(a, xf, b) <= max(1e-13, 10 * backward_error(a, xr, b))


def test_chunked_solve_is_bit_identical():
    a = matgen.c2_matrix(24)
    ex = structure(a, "amd")
    b = matgen.uniform_rhs(a.n, 24, 5, complex_=True)
    try:
        set_parallel(False)
        o = OracleSolver(a, ex)
        set_parallel(False, threads=1)
        x1 = o.solve_many(b, 24)          # one block solve
        set_parallel(False, threads=6)
        x6 = o.solve_many(b, 24)          # six column chunks
        cols = [o.solve_many(np.ascontiguousarray(b[:, c]), 1) for c in (0, 7, 23)]
    finally:
        set_parallel(False, threads=0)
    assert np.array_equal(x1, x6)
    for c, xc in zip((0, 7, 23), cols):
        assert np.array_equal(x6[:, c], xc)
