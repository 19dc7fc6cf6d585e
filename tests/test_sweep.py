"""The frequency-sweep workload generator (no GPU): A(w) = K - w^2 M + i w C
on the 27-point pattern, and the sweep's default static-pivoting settings."""
import numpy as np
import scipy.sparse as sp

from rslab_b200 import matgen
from rslab_b200.solver import ZeroPivotAction
from rslab_b200.sweep import sweep_settings


def test_c4_system_structure_and_formula():
    c4 = matgen.C4System(side=8, seed=3)
    assert c4.n == 512
    K = c4.K.to_scipy_full()
    # 27-point stencil: interior rows hold 27 entries, off-diagonals are -1
    nnz_rows = (K != 0).sum(axis=1).A1
    assert nnz_rows.max() == 27 and nnz_rows.min() == 8
    off = (K - sp.diags(K.diagonal())).tocsr()
    off.eliminate_zeros()
    assert set(np.unique(off.data)) == {-1.0}
    d = K.diagonal()
    assert d.min() >= 26.0 and d.max() <= 26.1
    assert 0.5 <= c4.mdiag.min() and c4.mdiag.max() <= 1.5
    w = c4.omegas(64)
    assert len(w) == 64 and np.isclose(w[0], 0.1 * np.sqrt(c4.lambda_mid)) and np.isclose(w[-1], 2 * np.sqrt(c4.lambda_mid))
    om = w[17]
    A = c4.matrix(om).to_scipy_full()
    ref = K.astype(np.complex128) * (1 + 0.01j * om) - om * om * sp.diags(c4.mdiag)
    assert abs(A - ref).max() < 1e-12
    assert abs(A - A.T).max() == 0.0


def test_c4_matrix_is_deterministic_and_pattern_fixed():
    a = matgen.C4System(side=6, seed=3)
    b = matgen.C4System(side=6, seed=3)
    x, y = a.matrix(1.3), b.matrix(2.1)
    assert np.array_equal(x.col_ptr, y.col_ptr) and np.array_equal(x.row_idx, y.row_idx)
    assert np.array_equal(a.K.values, b.K.values) and np.array_equal(a.mdiag, b.mdiag)


def test_sweep_settings_use_static_pivoting():
    st = sweep_settings()
    assert st.on_zero_pivot == ZeroPivotAction.perturb_to_eps(1e-10)
