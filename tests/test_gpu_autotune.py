"""The autotuner (rslab_b200.autotune): every candidate schedule / engine
certifies the same solve, the choice is the fastest certified candidate (or
the default within the tie margin), and a second call on the same pattern is
served from the cache."""
import numpy as np
import pytest

from rslab_b200 import LdltSymbolic, matgen
from rslab_b200.autotune import DEFAULT, candidates, tune_mixed

pytestmark = pytest.mark.gpu


def test_autotune_mixed_chooses_a_certified_fastest_candidate():
    a = matgen.c2_matrix(16)
    b = matgen.uniform_rhs(a.n, 4, 1, complex_=True)
    sym = LdltSymbolic.analyze(a)
    cands = candidates(panel_widths=(64, 32))
    res = tune_mixed(a, b, sym=sym, cands=cands, reps=2, warmup=1)
    assert set(res.seconds) == set(cands)
    assert all(res.certified.values())
    best = min(res.seconds.values())
    assert res.chosen == DEFAULT or res.seconds[res.chosen] == best
    assert res.seconds[res.chosen] <= best * 1.02 + 1e-12
    again = tune_mixed(a, b, sym=sym, cands=cands)
    assert again is res
    s = res.settings()
    assert (s.schur_engine, s.overlap, s.panel_nb) == res.chosen
