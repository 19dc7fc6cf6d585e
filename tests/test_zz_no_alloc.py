"""rslab_panel_factor_noalloc — the allocation-free dense panel factor — checked
through the C ABI against the regular rslab_factor entry point.

Callers that cannot allocate device memory at factor time (foreign or frozen
allocators, real-time loops) use this entry point; its scratch lives in a
static device array.  A dense symmetric matrix analysed with the natural
ordering is a single supernode, so rslab_factor runs the same panel kernels
on the same panel: the outputs must agree within the 1e-12 relative
tolerance of the other parity tests (1e-5 in f32; they are expected to be
bit-identical).  A panel with off-diagonal rows below its fully-summed block
(nrow > ncol) is checked by reconstruction: the pivoted block equals
L11 D L11^T and the off-diagonal rows equal L21 D L11^T.  Two calls in a row
check that state left in the shared scratch by one call does not leak into
the next.
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


_FIELD = {np.float64: (N.F64, "float64"), np.complex128: (N.C64, "complex128"),
          np.float32: (N.F32, "float32")}


def noalloc_factor(host_panel, nrow, ncol, dt):
    """One call of the allocation-free entry point on a copy of host_panel
    (nrow x ncol, column-major); returns the panel and the pivot arrays."""
    import torch

    dev = torch.device("cuda", 0)
    code, tname = _FIELD[dt]
    tdt = getattr(torch, tname)
    panel = torch.from_numpy(np.asfortranarray(host_panel).ravel(order="F").copy()).to(dev)
    d = torch.zeros(ncol, dtype=tdt, device=dev)
    dsub = torch.zeros(ncol, dtype=tdt, device=dev)
    kind = torch.zeros(ncol, dtype=torch.uint8, device=dev)
    lperm = torch.zeros(ncol, dtype=torch.int32, device=dev)
    status = torch.full((4,), -1, dtype=torch.int32, device=dev)
    rc = N.lib.rslab_panel_factor_noalloc(code, C.c_void_p(panel.data_ptr()), nrow, ncol, 64,
                                          C.c_void_p(d.data_ptr()), C.c_void_p(dsub.data_ptr()),
                                          C.c_void_p(kind.data_ptr()), C.c_void_p(lperm.data_ptr()),
                                          C.c_void_p(status.data_ptr()), None)
    assert rc == 0, N.last_error()
    torch.cuda.synchronize()
    return (panel.cpu().numpy().reshape((nrow, ncol), order="F"), d.cpu().numpy(), dsub.cpu().numpy(),
            kind.cpu().numpy(), lperm.cpu().numpy(), status.cpu().numpy())


@pytest.mark.parametrize("n,dt", [(300, np.float64), (300, np.complex128), (700, np.float64), (300, np.float32)])
def test_noalloc_matches_regular_entry_point(n, dt):
    complex_ = dt == np.complex128
    tol = 1e-5 if dt == np.float32 else TOL
    a = dense_indefinite(n, 11 + n, complex_)
    A = lower_csc(a.astype(dt))
    # f32: the regular entry point's CUDA-core engine runs the same in-panel kernels
    st = SolverSettings(ordering=Ordering.NATURAL, relax=None, scaling="identity", schur_engine="fma")
    sym = LdltSymbolic.analyze_with(A, st)
    assert sym.info().nsuper == 1
    ref = sym.factor(A, st).export_factors()

    host_panel = np.tril(a).astype(dt)
    for call in range(2):
        Lp, d_h, ds_h, kind_h, lperm_h, status = noalloc_factor(host_panel, n, n, dt)
        assert int(status[0]) == 0, f"call {call}: status {status.tolist()}"
        assert np.array_equal(kind_h == 1, ref.two_by_two), f"call {call}: 2x2 pattern"
        assert np.array_equal(lperm_h, ref.perm), f"call {call}: pivot order"
        assert rel(d_h, ref.d_diag) <= tol
        assert rel(ds_h, ref.d_subdiag) <= tol
        Lp = np.tril(Lp, -1)
        Lr = np.zeros((n, n), dtype=dt)
        cols = np.repeat(np.arange(n), np.diff(ref.l_col_ptr))
        Lr[ref.l_row_idx, cols] = ref.l_values
        Lr = np.tril(Lr, -1)
        assert rel(Lp, Lr) <= tol, f"call {call}: L"


def block_d(d, dsub, kind):
    """D of the factor: 1x1 pivots and symmetric 2x2 blocks (kind 1 marks a
    block's first column, dsub its off-diagonal)."""
    n = d.shape[0]
    D = np.diag(d).astype(d.dtype)
    for k in np.nonzero(kind == 1)[0]:
        D[k + 1, k] = D[k, k + 1] = dsub[k]
    return D


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
def test_noalloc_panel_with_offdiagonal_rows(dt):
    """A 600 x 300 panel: the 300 fully-summed columns on top of 300 rows that
    the panel's pivots do not touch."""
    nrow, ncol = 600, 300
    complex_ = dt == np.complex128
    a = dense_indefinite(nrow, 5, complex_).astype(dt)
    host_panel = np.tril(a)[:, :ncol].copy()
    A11, A21 = a[:ncol, :ncol], a[ncol:, :ncol]
    first = None
    for call in range(2):
        P, d_h, ds_h, kind_h, lperm_h, status = noalloc_factor(host_panel, nrow, ncol, dt)
        assert int(status[0]) == 0, f"call {call}: status {status.tolist()}"
        assert sorted(lperm_h.tolist()) == list(range(ncol))
        L11 = np.tril(P[:ncol], -1) + np.eye(ncol, dtype=dt)
        L21 = P[ncol:]
        D = block_d(d_h, ds_h, kind_h)
        p = lperm_h.astype(np.int64)
        scale = np.max(np.abs(a))
        assert rel(L11 @ D @ L11.T, A11[np.ix_(p, p)]) <= 1e-10, call
        assert float(np.max(np.abs(L21 @ D @ L11.T - A21[:, p]))) <= 1e-10 * scale, call
        if first is None:
            first = (P, d_h, lperm_h)
        else:  # the second call sees the first call's scratch: same result
            assert np.array_equal(first[2], lperm_h) and np.array_equal(first[0], P) and np.array_equal(first[1], d_h)


def test_noalloc_rejects_oversized_panel():
    rc = N.lib.rslab_panel_factor_noalloc(N.F64, C.c_void_p(1), 5000, 10, 64, C.c_void_p(1), C.c_void_p(1),
                                          C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None)
    assert rc == 2
    assert "allocation-free maximum" in N.last_error()
