"""Frequency sweep on the GPU: one analysis, refactor per frequency, FP64
refinement to 1e-14 (the same-pattern sweep workload, small grid)."""
import numpy as np
import pytest

from oracle.oracle import backward_error
from rslab_b200 import matgen
from rslab_b200.solver import MixedLdltSolver
from rslab_b200.sweep import frequency_sweep, sweep_settings

pytestmark = pytest.mark.gpu


def test_sweep_certifies_every_frequency_and_matches_fresh_factors():
    c4 = matgen.C4System(side=10, seed=3)
    omegas = c4.omegas(64)[[0, 21, 42, 63]]
    b = matgen.uniform_rhs(c4.n, 8, 4, complex_=True)
    mats = [c4.matrix(w) for w in omegas]
    out = list(frequency_sweep(mats, b, target=1e-14))
    assert len(out) == len(omegas)
    for i, x, info in out:
        assert info.certified and info.backward_error <= 1e-14
        # recomputed on the host from the stored lower triangle
        assert backward_error(mats[i], x, b) <= 1e-14
        # a fresh factor of the same matrix reaches the same solution
        xf, inf2 = MixedLdltSolver.factor_with(mats[i], sweep_settings()).solve_to(mats[i], b, 1e-14)
        assert inf2.certified
        assert np.abs(x - xf).max() <= 1e-10 * max(np.abs(xf).max(), 1.0)
