"""Block GMRES with a factored handle as the preconditioner.

`gmres_block(solver, b, tol, max_iter, restart, x0)` mirrors the reference's
`gmres_block(op, b, s, precond, tol, max_iter, restart, x0)`
(src/numeric/iterative.rs:1881) for a factored solver used as preconditioner: the operator
is the handle's FP64 matrix and the preconditioner its factor
(`impl Preconditioner for LdltSolver`, iterative.rs:178-190).  The iteration
runs on the GPU (rslab_gmres_block); `b` is an n x s array (a 1-D b is one
column) and the result carries the reference's BlockKrylovResult fields.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native as N
from .solver import DimensionMismatch, InvalidInput, _check


@dataclass
class BlockKrylovResult:
    x: np.ndarray
    iters: int
    converged: bool
    final_res: np.ndarray


def gmres_block(solver, b, tol: float, max_iter: int = 120, restart: int = 30,
                x0: Optional[np.ndarray] = None) -> BlockKrylovResult:
    """`solver`: an LdltSolver of an f64 / c64 matrix or a MixedLdltSolver
    (any tier).  Relative residual ||b_c - A x_c|| / ||b_c|| <= tol per column."""
    h = getattr(solver, "_h", None)
    if not h:
        raise InvalidInput("gmres_block needs a factored LdltSolver or MixedLdltSolver")
    n = solver._sym.n
    dt = np.dtype(solver.dtype)
    if dt not in (np.dtype(np.float64), np.dtype(np.complex128)):
        raise InvalidInput("gmres_block needs an FP64 operator (an f64 / c64 handle)")
    b = np.asarray(b)
    one = b.ndim == 1
    bb = np.ascontiguousarray(b.reshape(n, -1) if one else b, dtype=dt)
    if bb.shape[0] != n:
        raise DimensionMismatch(n, bb.shape[0])
    s = bb.shape[1]
    xx = np.empty_like(bb)
    x0c = None
    if x0 is not None:
        x0c = np.ascontiguousarray(np.asarray(x0).reshape(n, s), dtype=dt)
    it = C.c_int64()
    conv = C.c_int()
    fr = np.zeros(s, np.float64)
    _check(N.lib.rslab_gmres_block(h, bb.ctypes.data_as(C.c_void_p), s, float(tol), int(max_iter), int(restart),
                                   None if x0c is None else x0c.ctypes.data_as(C.c_void_p),
                                   xx.ctypes.data_as(C.c_void_p), 0, C.byref(it),
                                   fr.ctypes.data_as(C.POINTER(C.c_double)), C.byref(conv)))
    return BlockKrylovResult(xx[:, 0] if one else xx, int(it.value), bool(conv.value), fr)
