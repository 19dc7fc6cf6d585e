"""Same-pattern frequency sweeps: one analysis, one low-precision factor
handle, then per frequency a refactor (the captured factor graph replayed on
the new values) and a solve refined in FP64 to the target backward error.

The reference factors every frequency from scratch through
`MixedLdltSolver::factor` (src/numeric/mixed.rs:234) and `solve_to` (:267);
here the symbolic analysis and the launch plan are reused and each refactor
replays the factor graph, which is what keeps a 64-point sweep cheap.  Zero
pivots follow the settings' `on_zero_pivot` (static pivoting by default, as
the workload asks).
"""
from __future__ import annotations

from typing import Iterator, Optional, Sequence, Tuple

import numpy as np

from .solver import CscMatrix, LdltSymbolic, MixedInfo, MixedLdltSolver, SolverSettings


def sweep_settings() -> SolverSettings:
    """Static pivoting: a pivot below 1e-10 (scaled matrix) is perturbed to
    that floor instead of failing the factor; IR certifies the result."""
    return SolverSettings.preconditioner(1e-10)


def frequency_sweep(matrices, b: np.ndarray, target: float = 1e-14, settings: Optional[SolverSettings] = None,
                    reuse_pivots: bool = False,
                    stats: Optional[dict] = None) -> Iterator[Tuple[int, np.ndarray, MixedInfo]]:
    """Yield (index, x, info) for every matrix of `matrices` (an iterable of
    CscMatrix on one pattern), solving A_i x = b to `target`.

    reuse_pivots: static pivot reuse (the counterpart of the reference's
    static-pivot sweep, src/numeric/multifrontal_lu.rs:3551): the first
    matrix is factored with the Bunch-Kaufman search, which records its
    pivot steps, and the following refactors replay them without searching;
    a frequency whose refined solve does not certify is refactored with the
    search (which records its steps afresh) and solved again.  `stats`
    (optional) receives the counts of reused and re-searched factors."""
    st = settings or sweep_settings()
    solver = None
    if stats is not None:
        stats.update(reused=0, searched=0, refactored_after_failure=0)
    for i, a in enumerate(matrices):
        if solver is None:
            sym = LdltSymbolic.analyze_with(a, st)
            solver = MixedLdltSolver.factor_with(a, st, sym=sym)
            if stats is not None:
                stats["searched"] += 1
            if reuse_pivots:
                solver.reuse_pivots(True)
            x, info = solver.solve_to(a, b, target)
            yield i, x, info
            continue
        solver.refactor(a)
        if stats is not None:
            stats["reused" if reuse_pivots else "searched"] += 1
        x, info = solver.solve_to(a, b, target)
        if reuse_pivots and not info.certified:
            solver.reuse_pivots(False)
            solver.refactor(a)
            solver.reuse_pivots(True)
            x, info = solver.solve_to(a, b, target)
            if stats is not None:
                stats["refactored_after_failure"] += 1
        yield i, x, info


def shard_frequencies(count: int, rank: int, world_size: int) -> list:
    """The frequency indices one rank sweeps: index i goes to rank
    i mod world_size.  Every frequency costs the same (one pattern, one
    factor graph), so round-robin balances to within one frequency; the
    ranks need no exchange until the per-frequency certificates are gathered
    (`gather_certificates`)."""
    if world_size <= 0 or not 0 <= rank < world_size:
        raise ValueError("need 0 <= rank < world_size")
    return list(range(rank, count, world_size))


def gather_certificates(local: dict, world_size: int) -> list:
    """Every rank's per-frequency records (a host-side all-gather of small
    dicts, the only communication of a sharded sweep)."""
    from .batch import gather_stats
    return gather_stats(local, world_size)
