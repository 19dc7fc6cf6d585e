"""Static pivot reuse (rslab_set_pivot_reuse): getf2 replays the pivot steps
recorded by the last searching factor.  Where the search would choose the
same steps the replayed factor is bit-identical to a searching one; across a
frequency sweep the replayed factors, refined in FP64, certify every
frequency, with a searching refactor as the fallback."""
import numpy as np
import pytest

from oracle.oracle import backward_error
from rslab_b200 import CscMatrix, LdltSymbolic, SolverSettings, matgen
from rslab_b200.sweep import frequency_sweep, sweep_settings

pytestmark = pytest.mark.gpu


def same(f, g):
    return (np.array_equal(f.perm, g.perm) and np.array_equal(f.two_by_two, g.two_by_two)
            and np.array_equal(f.d_diag, g.d_diag) and np.array_equal(f.l_values, g.l_values))


@pytest.mark.parametrize("dt", [np.float64, np.complex64])
def test_replayed_pivots_reproduce_the_searching_factor(dt):
    a = matgen.c1_matrix(48) if dt == np.float64 else matgen.c2_matrix(12)
    a = a.astype(dt)
    st = SolverSettings(scaling="identity")
    sym = LdltSymbolic.analyze_with(a, st)
    f = sym.factor(a, st)
    ref = f.export_factors()
    f.reuse_pivots(True)
    f.refactor(a)
    assert same(f.export_factors(), ref)
    # doubling every value (exact in floating point, no equilibration)
    # doubles every magnitude the search compares: the same steps, and the
    # replayed factor equals a fresh searching factor of the new values
    a2 = CscMatrix(a.n, a.col_ptr, a.row_idx, a.values * dt(2.0))
    f.refactor(a2)
    fresh = sym.factor(a2, st).export_factors()
    assert same(f.export_factors(), fresh)
    f.reuse_pivots(False)
    f.refactor(a2)
    assert same(f.export_factors(), fresh)


def test_sweep_with_pivot_reuse_certifies():
    c4 = matgen.C4System(side=10, seed=3)
    omegas = c4.omegas(64)[::9]
    b = matgen.uniform_rhs(c4.n, 8, 4, complex_=True)
    mats = [c4.matrix(w) for w in omegas]
    stats = {}
    out = list(frequency_sweep(mats, b, 1e-14, sweep_settings(), reuse_pivots=True, stats=stats))
    assert stats["reused"] == len(omegas) - 1
    for i, x, info in out:
        assert info.certified and info.backward_error <= 1e-14
        assert backward_error(mats[i], x, b) <= 1e-14
