"""Batched independent systems on the GPU: one analysis handle, one launch
per assembly-tree level across all systems.  The batch factor of every
system is bit-identical to factoring it alone (same update lists and tile
order, same kernels), and the mixed-precision solve certifies every
(system, column) separately."""
import numpy as np
import pytest

from oracle.oracle import backward_error
from rslab_b200 import LdltSymbolic, SolverSettings, matgen
from rslab_b200.batch import BatchSystems, analyze_batch, factor_batch, mixed_solve_batch

pytestmark = pytest.mark.gpu


def systems():
    # C3-shaped: shifted 3D Laplacians of uneven sides, plus 2D ones
    return [matgen.c3_matrix(s) for s in (6, 11, 9, 14)] + [matgen.c1_matrix(20), matgen.c1_matrix(13)]


# The engine is pinned: "auto" picks by the analysis' size, and the merged
# batch is larger than any of its systems.
@pytest.mark.parametrize("engine", ["fma", "tensor"])
def test_batch_factor_bit_identical_to_single_factors(engine):
    st = SolverSettings(schur_engine=engine)
    sy = systems()
    b = BatchSystems(sy)
    sym = analyze_batch(b)
    fb = factor_batch(b, sym, st).export_factors()
    off = 0
    for a in sy:
        f = LdltSymbolic.analyze(a).factor(a, st).export_factors()
        sl = slice(off, off + a.n)
        assert np.array_equal(fb.d_diag[sl], f.d_diag)
        assert np.array_equal(fb.d_subdiag[sl], f.d_subdiag)
        assert np.array_equal(fb.two_by_two[sl], f.two_by_two)
        assert np.array_equal(fb.perm[sl], f.perm + off)
        off += a.n
    total = [0, 0, 0]
    for a in sy:
        i = LdltSymbolic.analyze(a).factor(a, st).inertia()
        total = [total[0] + i.positive, total[1] + i.negative, total[2] + i.zero]
    assert tuple(fb.inertia) == tuple(total)


def test_batch_solve_matches_single_solves():
    st = SolverSettings(schur_engine="fma")
    sy = systems()
    b = BatchSystems(sy)
    sym = analyze_batch(b)
    s = factor_batch(b, sym, st)
    rhs = [matgen.uniform_rhs(a.n, 4, 10 + i) for i, a in enumerate(sy)]
    xs = b.split(s.solve_many(b.stack_rhs(rhs), 4))
    for a, r, x in zip(sy, rhs, xs):
        x1 = LdltSymbolic.analyze(a).factor(a, st).solve_many(r, 4)
        assert np.array_equal(x, x1)


def test_batch_mixed_certifies_every_system():
    sy = systems()
    b = BatchSystems(sy)
    sym = analyze_batch(b)
    rhs = [matgen.uniform_rhs(a.n, 4, 20 + i) for i, a in enumerate(sy)]
    xs, res = mixed_solve_batch(b, sym, rhs, 1e-14, SolverSettings())
    assert res.info.certified
    assert res.backward_error.shape == (len(sy), 4)
    assert np.all(res.certified)
    for a, r, x, be in zip(sy, rhs, xs, res.backward_error):
        for c in range(4):
            got = backward_error(a, x[:, c], r[:, c])
            assert got <= 1e-14 and be[c] <= 1e-14
            # at ~1e-16 the residual itself is rounding noise of b - A x: the
            # device and host evaluations agree to within that noise
            assert abs(got - be[c]) <= 1e-15
