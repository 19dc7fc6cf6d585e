"""AMD ordering pinned to the reference's SuiteSparse golden permutations
(crates/rslab-amd/tests/oracle_match.rs:146-160): exact permutation and the
ncmpa / n_dense / ndiv / nms_ldl / nms_lu counters."""
import numpy as np
import pytest

from rslab_b200 import amd_order
from tests.helpers import amd_cases

CASES = amd_cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_amd_matches_suitesparse(name):
    c = CASES[name]
    perm, st = amd_order(c["n"], c["col_ptr"], c["row_idx"])
    assert list(perm) == c["perm"], f"{name}: permutation mismatch"
    for k in ("ncmpa", "n_dense", "ndiv", "nms_ldl", "nms_lu"):
        assert st[k] == c[k], f"{name}: {k} {st[k]} != {c[k]}"


def test_mass_elimination_and_supervariables_fire():
    c = CASES["grid_7x7"]
    _, st = amd_order(c["n"], c["col_ptr"], c["row_idx"])
    assert st["n_mass_elim"] > 0
    assert st["n_supervar_merge"] > 0
