"""`ldlt(A)` — the GPU-backed counterpart of RSLAB's Python entry point
`rslab.ldlt` (python/rslab/__init__.py:155-262, native `ldlt_factor`
python/src/lib.rs:861-948) and its `Ldlt` handle (lib.rs:201, :500-660).

Same call shape and keyword meaning: the lower triangle of `A` is extracted
(duplicates summed), the dtype of `A` picks the field (float64, float32,
complex128, complex64 — complex matrices are complex-symmetric, not
Hermitian), the analysis uses the default settings, and the keywords layer on
top.  `threads` sizes the reference's CPU pool and has no effect here;
`method` ('left_looking' / 'multifrontal') picks the numeric schedule (the
same pivoting; the factors agree to rounding); `memory` ('low' / 'eager')
only changes the reference's CPU memory profile, never the factor, so it is
validated and otherwise ignored (every panel here is resident on the device).
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .solver import (CscMatrix, InvalidInput, LdltSolver, LdltSymbolic, SolverSettings,
                     ZeroPivotAction)

_DTYPES = (np.float64, np.float32, np.complex128, np.complex64)


def _lower_csc(A) -> CscMatrix:
    import scipy.sparse as sp
    if sp.issparse(A):
        M = A.tocsc()
    else:
        M = sp.csc_matrix(np.asarray(A))
    if M.shape[0] != M.shape[1]:
        raise InvalidInput(f"matrix must be square, got {M.shape}")
    if M.dtype.type not in _DTYPES:
        raise InvalidInput(f"unsupported dtype {M.dtype}: expected float64, float32, complex128, or complex64")
    L = sp.tril(M, format="csc")
    L.sum_duplicates()
    L.sort_indices()
    return CscMatrix(M.shape[0], L.indptr.astype(np.int64), L.indices.astype(np.int64), L.data)


class Ldlt:
    """A factored symmetric matrix with its original lower triangle kept for
    refinement (the reference's `Ldlt` pyclass)."""

    def __init__(self, solver: LdltSolver, a: CscMatrix, sym: LdltSymbolic):
        self._s = solver
        self._a = a
        self._sym = sym

    @property
    def n(self) -> int:
        return self._s.n

    @property
    def factor_nnz(self) -> int:
        return self._s.factor_nnz()

    @property
    def n_perturbed(self) -> int:
        return self._s.n_perturbed()

    @property
    def inertia(self) -> tuple:
        i = self._s.inertia()
        return (i.positive, i.negative, i.zero)

    @property
    def dtype(self) -> str:
        return np.dtype(self._s.dtype).name

    def _rhs(self, b) -> np.ndarray:
        b = np.asarray(b)
        if b.dtype != np.dtype(self._s.dtype):
            raise ValueError("rhs dtype does not match the factor dtype")
        return np.ascontiguousarray(b)

    def solve(self, b, refine: int = 0) -> np.ndarray:
        """x = A^-1 b; `refine` > 0 adds that many refinement steps against A."""
        b = self._rhs(b)
        if b.ndim != 1 or b.shape[0] != self.n:
            raise ValueError(f"rhs must have shape ({self.n},)")
        if refine > 0:
            return self._s.solve_refined(self._a, b, int(refine))
        return self._s.solve(b)

    def solve_many(self, b) -> np.ndarray:
        """X = A^-1 B for a C-contiguous n x nrhs block (one pass for all columns)."""
        b = self._rhs(b)
        if b.ndim != 2 or b.shape[0] != self.n:
            raise ValueError(f"rhs must have shape ({self.n}, nrhs)")
        nrhs = b.shape[1]
        x = self._s.solve_many(b, nrhs)
        return x.reshape(self.n, nrhs)


def ldlt(A, *, threads: Optional[int] = None, preconditioner: Optional[float] = None,
         drop_tol: Optional[float] = None, method: str = "left_looking", memory: str = "low",
         force_accept: bool = False) -> Ldlt:
    """Factor a symmetric (or complex-symmetric) matrix P^T A P = L D L^T on the GPU."""
    if method not in ("left_looking", "leftlooking", "ll", "multifrontal", "mf"):
        raise ValueError(f"method must be 'left_looking' or 'multifrontal', got '{method}'")
    if memory not in ("low", "low_memory", "eager"):
        raise ValueError(f"memory must be 'low' or 'eager', got '{memory}'")
    if threads is not None and threads < 0:
        raise ValueError("threads must be non-negative")
    a = _lower_csc(A)
    st = SolverSettings(method="multifrontal" if method in ("multifrontal", "mf") else "left_looking")
    if preconditioner is not None:
        st.on_zero_pivot = ZeroPivotAction.perturb_to_eps(float(preconditioner))
    elif force_accept:
        st.on_zero_pivot = ZeroPivotAction.force_accept()
    if drop_tol is not None:
        st.drop_tol = float(drop_tol)
    sym = LdltSymbolic.analyze_with(a, st)
    return Ldlt(sym.factor(a, st), a, sym)
