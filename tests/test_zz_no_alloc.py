"""rslab_panel_factor_noalloc — the allocation-free dense panel factor — checked
through the C ABI against the regular rslab_factor entry point.

Callers that cannot allocate device memory at factor time (graph-captured
code, foreign or frozen allocators, real-time loops) use this entry point;
its scratch lives in a static device array.  A dense symmetric matrix
analysed with the natural ordering is a single supernode, so rslab_factor
runs the same panel kernels on the same panel: the outputs must agree within
the 1e-12 relative tolerance of the other parity tests (they are expected to
be bit-identical).  Two calls in a row check that state left in the shared
scratch by one call does not leak into the next.
"""
import ctypes as C

import numpy as np
import pytest

from rslab_b200 import CscMatrix, LdltSymbolic, Ordering, SolverSettings
from rslab_b200 import _native as N

pytestmark = pytest.mark.gpu

TOL = 1e-12


def dense_indefinite(n, seed, complex_):
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((n, n))
    if complex_:
        m = m + 1j * rng.standard_normal((n, n))
    a = (m + m.T) / 2  # complex-symmetric, not Hermitian
    a[np.arange(n), np.arange(n)] += np.where(np.arange(n) % 3 == 0, 0.0, 2.0)
    return a


def lower_csc(a):
    n = a.shape[0]
    r, c = np.tril_indices(n)
    order = np.lexsort((r, c))
    r, c = r[order], c[order]
    return CscMatrix.from_triplets(n, r, c, a[r, c])


def rel(x, y):
    return float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))


@pytest.mark.parametrize("n,complex_", [(300, False), (300, True), (700, False)])
def test_noalloc_matches_regular_entry_point(n, complex_):
    import torch

    a = dense_indefinite(n, 11 + n, complex_)
    dt = np.complex128 if complex_ else np.float64
    code = N.C64 if complex_ else N.F64
    A = lower_csc(a.astype(dt))
    st = SolverSettings(ordering=Ordering.NATURAL, relax=None, scaling="identity")
    sym = LdltSymbolic.analyze_with(A, st)
    assert sym.info().nsuper == 1
    ref = sym.factor(A, st).export_factors()

    dev = torch.device("cuda", 0)
    tdt = torch.complex128 if complex_ else torch.float64
    host_panel = np.asfortranarray(np.tril(a).astype(dt))
    for call in range(2):
        panel = torch.from_numpy(host_panel.ravel(order="F").copy()).to(dev)
        d = torch.zeros(n, dtype=tdt, device=dev)
        dsub = torch.zeros(n, dtype=tdt, device=dev)
        kind = torch.zeros(n, dtype=torch.uint8, device=dev)
        lperm = torch.zeros(n, dtype=torch.int32, device=dev)
        status = torch.full((4,), -1, dtype=torch.int32, device=dev)
        rc = N.lib.rslab_panel_factor_noalloc(code, C.c_void_p(panel.data_ptr()), n, n, 64,
                                              C.c_void_p(d.data_ptr()), C.c_void_p(dsub.data_ptr()),
                                              C.c_void_p(kind.data_ptr()), C.c_void_p(lperm.data_ptr()),
                                              C.c_void_p(status.data_ptr()), None)
        assert rc == 0, N.last_error()
        torch.cuda.synchronize()
        assert int(status[0].item()) == 0, f"call {call}: status {status.tolist()}"
        d_h, ds_h = d.cpu().numpy(), dsub.cpu().numpy()
        kind_h, lperm_h = kind.cpu().numpy(), lperm.cpu().numpy()
        assert np.array_equal(kind_h == 1, ref.two_by_two), f"call {call}: 2x2 pattern"
        assert np.array_equal(lperm_h, ref.perm), f"call {call}: pivot order"
        assert rel(d_h, ref.d_diag) <= TOL
        assert rel(ds_h, ref.d_subdiag) <= TOL
        Lp = np.tril(panel.cpu().numpy().reshape((n, n), order="F"), -1)
        Lr = np.zeros((n, n), dtype=dt)
        cols = np.repeat(np.arange(n), np.diff(ref.l_col_ptr))
        Lr[ref.l_row_idx, cols] = ref.l_values
        Lr = np.tril(Lr, -1)
        assert rel(Lp, Lr) <= TOL, f"call {call}: L"


def test_noalloc_rejects_oversized_panel():
    rc = N.lib.rslab_panel_factor_noalloc(N.F64, C.c_void_p(1), 5000, 10, 64, C.c_void_p(1), C.c_void_p(1),
                                          C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None)
    assert rc == 2
    assert "allocation-free maximum" in N.last_error()
