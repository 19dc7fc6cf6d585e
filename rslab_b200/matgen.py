"""Seeded synthetic matrices with the shapes of the LDL^T benchmark workloads.

Mirrors the reference generators (src/matgen/mod.rs:62-95 `Rng`, xorshift64*;
src/matgen/stencil.rs:47-134 `laplacian_weights` / `laplacian` / `helmholtz`)
so the same seed gives the same matrix, and adds the workloads that the
reference does not ship: the shifted 2D/3D Laplacians, the 3D Helmholtz shift
and the 27-point stencil.  All matrices are returned as lower-triangle
CscMatrix objects.
"""
from __future__ import annotations

import math

import numpy as np

from .solver import CscMatrix

MASK = (1 << 64) - 1


class Rng:
    """xorshift64* (src/matgen/mod.rs:62-95)."""

    def __init__(self, seed: int):
        self.s = ((seed ^ 0x9E3779B97F4A7C15) | 1) & MASK

    def next_u64(self) -> int:
        x = self.s
        x ^= x >> 12
        x ^= (x << 25) & MASK
        x ^= x >> 27
        self.s = x
        return (x * 0x2545F4914F6CDD1D) & MASK

    def unit(self) -> float:
        return (self.next_u64() >> 11) / float(1 << 53)

    def range(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * self.unit()

    def units(self, m: int) -> np.ndarray:
        """m successive unit() draws (same sequence), generated natively."""
        import ctypes as C
        from . import _native as N
        out = np.empty(m, dtype=np.float64)
        self.s = int(N.lib.rslab_rng_units(C.c_uint64(self.s), m, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out


def _lower_csc(n, diag, rows, cols, w) -> CscMatrix:
    r = np.concatenate([np.arange(n), rows])
    c = np.concatenate([np.arange(n), cols])
    v = np.concatenate([diag, w])
    return CscMatrix.from_triplets(n, r, c, v)


def laplacian_weights(dims):
    """(diag, rows, cols, w) of the Dirichlet grid Laplacian (unit weights)."""
    dims = list(dims)
    nd = len(dims)
    n = int(np.prod(dims))
    stride = [1] * nd
    for d in range(1, nd):
        stride[d] = stride[d - 1] * dims[d - 1]
    idx = np.arange(n)
    diag = np.zeros(n)
    rows, cols = [], []
    for d in range(min(nd, 3)):
        c = (idx // stride[d]) % dims[d]
        inner = c + 1 < dims[d]
        i = idx[inner]
        j = i + stride[d]
        diag[i] += 1.0
        diag[j] += 1.0
        rows.append(j)
        cols.append(i)
        diag[~inner] += 1.0          # + boundary ghost
        diag[c == 0] += 1.0          # - boundary ghost
    rows = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    cols = np.concatenate(cols) if cols else np.zeros(0, np.int64)
    return diag, rows, cols, -np.ones(len(rows))


def lambda_max(dims) -> float:
    """Largest eigenvalue of -Delta_h with Dirichlet ends: sum_d 2 + 2 cos(pi/(N_d+1))."""
    return float(sum(2.0 + 2.0 * math.cos(math.pi / (m + 1)) for m in dims))


def shifted_laplacian(dims, sigma: float) -> CscMatrix:
    """A = -Delta_h - sigma I (real symmetric, indefinite once sigma > lambda_min)."""
    diag, rows, cols, w = laplacian_weights(dims)
    n = int(np.prod(dims))
    return _lower_csc(n, diag - sigma, rows, cols, w)


def helmholtz(dims, k2: complex) -> CscMatrix:
    """Complex-symmetric A = -Delta_h - k2 I (src/matgen/stencil.rs:114-134)."""
    diag, rows, cols, w = laplacian_weights(dims)
    n = int(np.prod(dims))
    return _lower_csc(n, diag.astype(np.complex128) - k2, rows, cols, w.astype(np.complex128))


def stencil27(side: int, rng: Rng):
    """3D 27-point stencil K (off-diagonal -1, diagonal 26 + U[0, 0.1]) as
    (diag, rows, cols, w) lower-triangle arrays."""
    n = side ** 3
    idx = np.arange(n)
    x, y, z = idx % side, (idx // side) % side, idx // (side * side)
    rows, cols = [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                off = dx + dy * side + dz * side * side
                if off <= 0:
                    continue
                ok = (x + dx >= 0) & (x + dx < side) & (y + dy >= 0) & (y + dy < side) & (z + dz >= 0) & (z + dz < side)
                i = idx[ok]
                rows.append(i + off)
                cols.append(i)
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    diag = 26.0 + 0.1 * rng.units(n)
    return diag, rows, cols, -np.ones(len(rows))


def uniform_rhs(n: int, nrhs: int, seed: int, complex_: bool = False) -> np.ndarray:
    """Row-major n x nrhs right-hand sides, entries U[-1, 1) from Rng(seed)
    (real then imaginary draw per entry for complex)."""
    rng = Rng(seed)
    m = n * nrhs * (2 if complex_ else 1)
    u = 2.0 * rng.units(m) - 1.0
    if complex_:
        u = u[0::2] + 1j * u[1::2]
    b = u.reshape(n, nrhs)
    return b[:, 0].copy() if nrhs == 1 else b


# Workloads -------------------------------------------------------------------

def c1_matrix(side: int = 128) -> CscMatrix:
    """2D 5-point Dirichlet Laplacian minus 0.3 lambda_max (real, indefinite)."""
    dims = (side, side)
    return shifted_laplacian(dims, 0.3 * lambda_max(dims))


def c2_matrix(side: int = 64) -> CscMatrix:
    """3D 7-point Helmholtz -Delta_h - k2 (1 + 0.05 i) I, k2 = 0.2 lambda_max."""
    dims = (side, side, side)
    k2 = 0.2 * lambda_max(dims)
    return helmholtz(dims, k2 * (1.0 + 0.05j))


def c3_matrix(side: int) -> CscMatrix:
    """3D 7-point Laplacian shifted by 0.1 lambda_max."""
    dims = (side, side, side)
    return shifted_laplacian(dims, 0.1 * lambda_max(dims))


def c3_sides(count: int = 512, seed: int = 2, lo: int = 12, hi: int = 40) -> list:
    """Cube sides of the batched workload: uniform integers in [lo, hi] from Rng(seed)."""
    rng = Rng(seed)
    return [lo + min(int(u * (hi - lo + 1)), hi - lo) for u in rng.units(count)]


def c3_batch(count: int = 512, seed: int = 2, lo: int = 12, hi: int = 40) -> list:
    """The batched workload: `count` shifted 3D Laplacians (shift 0.1 lambda_max)."""
    return [c3_matrix(s) for s in c3_sides(count, seed, lo, hi)]


class C4System:
    """The same-pattern frequency-sweep workload A(w) = K - w^2 M + i w C:
    K the 3D 27-point stencil on a side^3 grid (off-diagonal -1, diagonal
    26 + U[0, 0.1]), M diagonal U[0.5, 1.5], C = 0.01 K, complex symmetric.
    The frequencies are `count` points evenly spaced in [0.1, 2] sqrt(l_mid),
    l_mid the centre of K's Gershgorin interval (the stencil's spectrum lies
    inside it).  Draws: K's diagonal, then M's, from Rng(seed)."""

    def __init__(self, side: int = 48, seed: int = 3):
        rng = Rng(seed)
        diag, rows, cols, w = stencil27(side, rng)
        self.side = side
        self.n = side ** 3
        self.mdiag = 0.5 + rng.units(self.n)
        self.K = _lower_csc(self.n, diag, rows, cols, w)
        # Gershgorin: K_ii -/+ (number of stencil neighbours of i)
        deg = np.bincount(rows, minlength=self.n) + np.bincount(cols, minlength=self.n)
        self.lambda_mid = 0.5 * (float(np.min(diag - deg)) + float(np.max(diag + deg)))
        cp = self.K.col_ptr
        self._diag_pos = np.asarray(cp[:-1], np.int64)  # (j, j) is the first entry of column j
        assert np.array_equal(np.asarray(self.K.row_idx)[self._diag_pos], np.arange(self.n))

    def omegas(self, count: int = 64) -> np.ndarray:
        return np.linspace(0.1, 2.0, count) * math.sqrt(self.lambda_mid)

    def matrix(self, omega: float) -> CscMatrix:
        """A(omega) on K's lower-triangle pattern (complex128)."""
        v = np.asarray(self.K.values, np.float64) * (1.0 + 0.01j * omega)
        v[self._diag_pos] -= omega * omega * self.mdiag
        return CscMatrix(self.n, self.K.col_ptr, self.K.row_idx, v)


def stencil27_lambda_max(side: int) -> float:
    """Largest eigenvalue of the 27-point operator 26 I - (neighbour sum) with
    Dirichlet ends: 27 - prod_d (1 + 2 cos t_d), minimised at one t_d =
    side pi/(side+1) and two t_d = pi/(side+1)."""
    c = math.cos(math.pi / (side + 1))
    return 27.0 - (1.0 - 2.0 * c) * (1.0 + 2.0 * c) ** 2


def normals(rng: Rng, m: int) -> np.ndarray:
    """m N(0, 1) draws by the Box-Muller transform of 2m unit draws."""
    u = rng.units(2 * m).reshape(m, 2)
    return np.sqrt(-2.0 * np.log1p(-u[:, 0])) * np.cos(2.0 * math.pi * u[:, 1])


def random_sparse_symmetric(n: int, rng: Rng, shift: float) -> CscMatrix:
    """Symmetric n x n: every row draws 8-30 partner columns (uniform) with
    N(0, 1) values (the symmetric pair shares the value; repeats add), the
    diagonal is N(0, 1) + shift."""
    k = 8 + np.minimum((rng.units(n) * 23).astype(np.int64), 22)
    rows = np.repeat(np.arange(n), k)
    cols = np.minimum((rng.units(int(k.sum())) * n).astype(np.int64), n - 1)
    vals = normals(rng, len(rows))
    keep = rows != cols
    r, c, v = np.maximum(rows, cols)[keep], np.minimum(rows, cols)[keep], vals[keep]
    diag = normals(rng, n) + shift
    return _lower_csc(n, diag, r, c, v)


C5_FAMILIES = ("laplacian2d", "laplacian3d", "stencil27", "random_sparse", "helmholtz27", "helmholtz7")


def c5_corpus(count: int = 2000, seed: int = 5):
    """The precision-tier training corpus: `count` seeded matrices, yielded
    as (family, CscMatrix).  Family uniform over C5_FAMILIES, parameters from
    Rng(seed) in order:
      laplacian2d   side U{16..160}, -Delta_h - s lambda_max I, s U[0, 0.6]
      laplacian3d   side U{8..40},   s U[0, 0.4]
      stencil27     side U{8..32},   27-point K - s lambda_max I, s U[0, 0.5]
      random_sparse n U{500..8000},  8-30 N(0,1) entries per row, shift U[-1, 1] sqrt(19)
      helmholtz27   side U{8..32},   K - k2 (1 + i eta) I, k2 = U[0.05, 0.3] lambda_max, eta U[0, 0.05]
      helmholtz7    side U{8..40},   7-point, same k2 / eta draws (complex)
    The stencils' random diagonals and the random patterns draw from
    Rng(seed * 1000003 + index)."""
    rng = Rng(seed)

    def uint(lo, hi):
        return lo + min(int(rng.unit() * (hi - lo + 1)), hi - lo)

    for idx in range(count):
        fam = C5_FAMILIES[uint(0, len(C5_FAMILIES) - 1)]
        sub = Rng(seed * 1000003 + idx)
        if fam == "laplacian2d":
            side = uint(16, 160)
            dims = (side, side)
            a = shifted_laplacian(dims, rng.range(0.0, 0.6) * lambda_max(dims))
        elif fam == "laplacian3d":
            side = uint(8, 40)
            dims = (side, side, side)
            a = shifted_laplacian(dims, rng.range(0.0, 0.4) * lambda_max(dims))
        elif fam == "stencil27":
            side = uint(8, 32)
            s = rng.range(0.0, 0.5)
            diag, rows, cols, w = stencil27(side, sub)
            a = _lower_csc(side ** 3, diag - s * stencil27_lambda_max(side), rows, cols, w)
        elif fam == "random_sparse":
            n = uint(500, 8000)
            a = random_sparse_symmetric(n, sub, rng.range(-1.0, 1.0) * math.sqrt(19.0))
        else:
            side = uint(8, 32) if fam == "helmholtz27" else uint(8, 40)
            k2 = rng.range(0.05, 0.3)
            eta = rng.range(0.0, 0.05)
            if fam == "helmholtz27":
                diag, rows, cols, w = stencil27(side, sub)
                lam = stencil27_lambda_max(side)
            else:
                diag, rows, cols, w = laplacian_weights((side, side, side))
                lam = lambda_max((side, side, side))
            shift = k2 * lam * (1.0 + 1j * eta)
            a = _lower_csc(side ** 3, diag.astype(np.complex128) - shift, rows, cols, w.astype(np.complex128))
        yield fam, a


def c5_heldout(side: int = 80, seed: int = 6) -> CscMatrix:
    """The held-out evaluation matrix of the precision-tier network: 27-point
    complex Helmholtz K - k2 (1 + 0.02 i) I on a side^3 grid, k2 = 0.15
    lambda_max (K's diagonal 26 + U[0, 0.1] from Rng(seed))."""
    diag, rows, cols, w = stencil27(side, Rng(seed))
    shift = 0.15 * stencil27_lambda_max(side) * (1.0 + 0.02j)
    return _lower_csc(side ** 3, diag.astype(np.complex128) - shift, rows, cols, w.astype(np.complex128))


def negative_eigs_shifted_laplacian(dims, sigma: float) -> int:
    """Exact count of eigenvalues of -Delta_h - sigma I below zero (separable spectrum)."""
    ev = None
    for m in dims:
        e = 2.0 - 2.0 * np.cos(np.arange(1, m + 1) * np.pi / (m + 1))
        ev = e if ev is None else (ev[:, None] + e[None, :]).ravel()
    return int(np.sum(ev < sigma))
