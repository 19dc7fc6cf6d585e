"""The oracle on the sweep and tier-corpus matrix families (no GPU): its
FP64 factor + solve agrees with a direct sparse solve, its inertia with the
dense spectrum (real families), and its static pivoting (perturb-to-floor)
still gives a solve that refinement can certify."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from oracle.oracle import OracleSolver, backward_error, mixed_solve
from rslab_b200 import LdltSymbolic, matgen
from rslab_b200.sweep import sweep_settings


def _check_solve(a, nrhs=3, seed=1):
    b = matgen.uniform_rhs(a.n, nrhs, seed, complex_=np.iscomplexobj(a.values))
    sym = LdltSymbolic.analyze_with(a, sweep_settings())
    o = OracleSolver(a, sym.export())
    assert o.status == 0
    x = o.solve_many(b, nrhs)
    xr = spla.spsolve(a.to_scipy_full().tocsc(), b)
    assert np.abs(x - xr).max() <= 1e-9 * np.abs(xr).max()
    assert backward_error(a, x, b) <= 1e-13
    return o


@pytest.mark.parametrize("k", [0, 31, 63])
def test_sweep_matrices(k):
    c4 = matgen.C4System(side=6, seed=3)
    _check_solve(c4.matrix(c4.omegas(64)[k]))


def test_heldout_helmholtz27_family():
    _check_solve(matgen.c5_heldout(7, 6))


@pytest.mark.parametrize("idx", range(6))
def test_corpus_families(idx):
    fams = {}
    for fam, a in matgen.c5_corpus(60, 5):
        if a.n <= 3000 and fam not in fams:
            fams[fam] = a
    fam = matgen.C5_FAMILIES[idx]
    if fam not in fams:
        pytest.skip(f"no small {fam} matrix in the first 60")
    a = fams[fam]
    o = _check_solve(a)
    if not np.iscomplexobj(a.values):
        ev = np.linalg.eigvalsh(a.to_scipy_full().toarray())
        tol = 1e-9 * np.abs(ev).max()
        assert tuple(o.factors().inertia) == (int((ev > tol).sum()), int((ev < -tol).sum()), 0)


def test_oracle_mixed_refinement_on_a_sweep_matrix():
    c4 = matgen.C4System(side=6, seed=3)
    a = c4.matrix(c4.omegas(64)[40])
    b = matgen.uniform_rhs(a.n, 1, 2, complex_=True)
    sym = LdltSymbolic.analyze_with(a, sweep_settings())
    lo = OracleSolver(a, sym.export(), dtype=np.complex64)
    x, info = mixed_solve(lo, a, b, 1e-14)
    assert info["certified"] and backward_error(a, x, b) <= 1e-14
