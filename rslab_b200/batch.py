"""Many independent symmetric systems factored and solved together.

The reference factors independent systems one `LdltSymbolic::factor` call at
a time (src/numeric/sparse_solver.rs:677); here they share one analysis
handle whose assembly forest holds every system's tree, so each level of
every system goes out in the same launch (`rslab_analyze_batch`).  Each
system keeps exactly the structure its own `LdltSymbolic::analyze` gives.

`BatchSystems` concatenates the systems' values and right-hand sides in input
order and splits results back; `MixedLdltSolver` on a batch certifies every
(system, column) separately (`MixedBatchResult.backward_error`).

`shard_by_weight` assigns systems to ranks for one-process-per-GPU runs: the
systems are independent, so ranks exchange no data, only optional per-system
statistics at the end (`gather_stats`).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N
from .solver import (CscMatrix, InvalidInput, LdltSolver, LdltSymbolic, MixedInfo, MixedLdltSolver,
                     SolverSettings, _check, _p64)


class BatchSystems:
    """Independent lower-CSC systems (same field) laid out block-diagonally."""

    def __init__(self, systems: Sequence[CscMatrix]):
        if not systems:
            raise InvalidInput("empty batch")
        dt = {np.asarray(a.values).dtype for a in systems}
        if len(dt) != 1:
            raise InvalidInput("all systems of a batch must share one dtype")
        self.systems = list(systems)
        self.n = np.array([a.n for a in systems], np.int64)
        self.seg = np.concatenate([[0], np.cumsum(self.n)]).astype(np.int64)
        self.nnz = np.array([a.nnz for a in systems], np.int64)
        self.nz = np.concatenate([[0], np.cumsum(self.nnz)]).astype(np.int64)

    @property
    def count(self) -> int:
        return len(self.systems)

    @property
    def total_n(self) -> int:
        return int(self.seg[-1])

    def values(self) -> np.ndarray:
        return np.concatenate([np.asarray(a.values) for a in self.systems])

    def as_matrix(self) -> CscMatrix:
        """The block-diagonal lower CSC of the whole batch (values concatenated)."""
        cps, ris = [np.zeros(1, np.int64)], []
        for a, off, nzo in zip(self.systems, self.seg[:-1], self.nz[:-1]):
            cps.append(np.asarray(a.col_ptr[1:], np.int64) + nzo)
            ris.append(np.asarray(a.row_idx, np.int64) + off)
        return CscMatrix(self.total_n, np.concatenate(cps), np.concatenate(ris) if ris else np.zeros(0, np.int64),
                         self.values())

    def stack_rhs(self, bs: Sequence[np.ndarray]) -> np.ndarray:
        """Row-major (sum n) x nrhs block from per-system n_i x nrhs blocks."""
        return np.ascontiguousarray(np.concatenate([np.asarray(b) for b in bs], axis=0))

    def split(self, x: np.ndarray) -> List[np.ndarray]:
        return [x[self.seg[i]:self.seg[i + 1]] for i in range(self.count)]


def analyze_batch(batch: BatchSystems, opts: Optional[SolverSettings] = None) -> LdltSymbolic:
    """One analysis handle over every system of the batch."""
    opts = opts or SolverSettings()
    for a in batch.systems:
        a.validate()
    s, keep = opts._analyze_c()
    cps = [np.ascontiguousarray(a.col_ptr, np.int64) for a in batch.systems]
    ris = [np.ascontiguousarray(a.row_idx, np.int64) for a in batch.systems]
    cp_arr = (N.i64p * batch.count)(*[_p64(c) for c in cps])
    ri_arr = (N.i64p * batch.count)(*[_p64(r) for r in ris])
    n_arr = np.ascontiguousarray(batch.n)
    h = C.c_void_p()
    _check(N.lib.rslab_analyze_batch(batch.count, _p64(n_arr), cp_arr, ri_arr, C.byref(s), C.byref(h)))
    del keep, cps, ris
    return LdltSymbolic(h, batch.total_n, int(batch.nz[-1]), opts)


def batch_layout(sym: LdltSymbolic):
    cnt = C.c_int64(0)
    _check(N.lib.rslab_batch_layout(sym._h, C.byref(cnt), None, None))
    seg = np.zeros(cnt.value + 1, np.int64)
    nz = np.zeros(cnt.value + 1, np.int64)
    _check(N.lib.rslab_batch_layout(sym._h, C.byref(cnt), _p64(seg), _p64(nz)))
    return seg, nz


@dataclass
class MixedBatchResult:
    info: MixedInfo
    backward_error: np.ndarray  # systems x nrhs
    certified: np.ndarray       # systems x nrhs booleans


def mixed_batch_result(solver: MixedLdltSolver, count: int, nrhs: int, target: float,
                       info: MixedInfo) -> MixedBatchResult:
    cnt = C.c_int64(0)
    be = np.zeros(count * nrhs, np.float64)
    _check(N.lib.rslab_mixed_batch_result(solver._h, be.size, be.ctypes.data_as(C.POINTER(C.c_double)),
                                          C.byref(cnt)))
    be = be[: cnt.value].reshape(count, nrhs)
    return MixedBatchResult(info, be, be <= target)


def factor_batch(batch: BatchSystems, sym: LdltSymbolic, opts: Optional[SolverSettings] = None) -> LdltSolver:
    return sym.factor(batch.as_matrix(), opts)


def mixed_solve_batch(batch: BatchSystems, sym: LdltSymbolic, rhs: Sequence[np.ndarray], target: float,
                      opts: Optional[SolverSettings] = None):
    """Low-precision factor of every system + FP64 refinement certified per
    (system, column); returns the per-system solutions and the result."""
    a = batch.as_matrix()
    m = MixedLdltSolver.factor_with(a, opts or SolverSettings(), sym=sym)
    b = batch.stack_rhs(rhs)
    nrhs = 1 if b.ndim == 1 else b.shape[1]
    x, info = m.solve_to(a, b, target)
    return batch.split(x), mixed_batch_result(m, batch.count, nrhs, target, info)


# ---------------------------------------------------------------------------
# Sharding across ranks (one process per GPU).
# ---------------------------------------------------------------------------


def shard_by_weight(weights: Sequence[float], world_size: int) -> List[List[int]]:
    """Longest-processing-time assignment of units to ranks: heaviest first,
    each to the currently lightest rank (ties to the lower rank).  Returns the
    unit indices of every rank in ascending order.  Deterministic."""
    if world_size <= 0:
        raise InvalidInput("world_size must be positive")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    load = [0.0] * world_size
    out: List[List[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(weights[i])
    return [sorted(v) for v in out]


def gather_stats(local: dict, world_size: int) -> List[dict]:
    """All ranks' per-unit statistics (a host-side all-gather of small dicts;
    the only communication of a sharded batch).  Single-process: [local]."""
    if world_size == 1:
        return [local]
    import torch.distributed as dist
    out: List[Optional[dict]] = [None] * world_size
    dist.all_gather_object(out, local)
    return out  # type: ignore[return-value]
