"""The block GMRES oracle on the host: exact and approximate
preconditioners, deflation of columns that converge at different speeds,
zero columns, warm starts, complex-symmetric operators."""
import numpy as np

from oracle.krylov import gmres_block, givens, well_conditioned_dim


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    return q @ np.diag(np.linspace(1.0, 50.0, n)) @ q.T


def test_exact_preconditioner_converges_in_one_step():
    a = _spd(40, 1)
    b = np.random.default_rng(2).normal(size=(40, 3))
    ainv = np.linalg.inv(a)
    x, it, conv, fr = gmres_block(lambda v: a @ v, lambda r: ainv @ r, b, 1e-12, 50, 10)
    assert conv and it == 1 and np.all(fr <= 1e-12)
    assert np.allclose(x, np.linalg.solve(a, b), rtol=0, atol=1e-10)


def test_single_precision_preconditioner_refines_to_double():
    a = _spd(60, 3) - 20.0 * np.eye(60)  # indefinite
    b = np.random.default_rng(4).normal(size=(60, 4))
    ainv32 = np.linalg.inv(a.astype(np.float32)).astype(np.float64)
    x, it, conv, fr = gmres_block(lambda v: a @ v, lambda r: ainv32 @ r, b, 1e-13, 60, 20)
    assert conv and 1 < it < 20
    assert np.allclose(x, np.linalg.solve(a, b), rtol=0, atol=1e-9 * np.abs(np.linalg.solve(a, b)).max())


def test_columns_deflate_at_their_own_speed():
    n = 50
    a = np.diag(np.linspace(1.0, 10.0, n))
    b = np.zeros((n, 3))
    b[0, 0] = 1.0                      # an eigenvector: one step
    b[:, 1] = 1.0                      # every eigenvalue: many steps
    b[:5, 2] = 1.0
    x, it, conv, fr = gmres_block(lambda v: a @ v, lambda r: r, b, 1e-12, 200, 60)
    assert conv and np.all(fr <= 1e-12)
    assert np.allclose(a @ x, b, atol=1e-10)


def test_zero_column_and_warm_start():
    a = _spd(30, 5)
    b = np.random.default_rng(6).normal(size=(30, 2))
    b[:, 1] = 0
    x, it, conv, fr = gmres_block(lambda v: a @ v, lambda r: r, b, 1e-12, 100, 30)
    assert conv and np.all(x[:, 1] == 0) and fr[1] == 0
    x2, it2, conv2, _ = gmres_block(lambda v: a @ v, lambda r: r, b, 1e-10, 100, 30, x0=x)
    assert conv2 and it2 == 0


def test_complex_symmetric_operator():
    rng = np.random.default_rng(7)
    m = rng.normal(size=(30, 30)) + 1j * rng.normal(size=(30, 30))
    a = m + m.T + 30 * np.eye(30)
    b = rng.normal(size=(30, 2)) + 1j * rng.normal(size=(30, 2))
    x, it, conv, fr = gmres_block(lambda v: a @ v, lambda r: r, b, 1e-12, 200, 40)
    assert conv and np.allclose(a @ x, b, atol=1e-9)


def test_helpers():
    c, s = givens(3.0, 4.0)
    assert abs(c - 0.6) < 1e-15 and abs(s - 0.8) < 1e-15
    h = np.diag([1.0, 1e-20, 2.0])
    assert well_conditioned_dim(h, 3) == 1 and well_conditioned_dim(h, 0) == 0
