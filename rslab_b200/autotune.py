"""Autotuner for the factor's tile shapes and launch schedule.

The reference picks its settings by a fixed heuristic (LdltSolver::tuned,
src/numeric/sparse_solver.rs:108-131) or a learned model of CPU timings
(factor_auto); on the GPU the choices that matter are different, so this
module measures them on the actual pattern and keeps the fastest.  The knobs
are value independent, so a pattern is tuned once and the choice reused for
every refactor of it (frequency sweeps, batches, time steps):

  schur_engine  the refined factor's precision tier and update engine: an
                f32 / c32 factor with tcgen05 tensor-core GEMM tiles
                ("tensor") or CUDA-core tiles ("fma"), or the FP64 factor
                under the same refinement ladder ("fp64": the cheapest when
                the single-precision factor needs many corrections)
  overlap       launch schedule: side streams overlapping independent work
                (the Schur update beyond the next block, the next level's
                early updates) or one in-order stream
  panel_nb      Bunch-Kaufman block width of the panel kernels (getf2, deep
                rows and in-panel Schur tiles): 64 or 32 (supernodes of 512
                or more columns use 128 either way); an analysis-time knob,
                tuned only when `panel_widths` lists more than one width

Every candidate runs `warmup` untimed and `reps` timed steps (refactor +
solve to the target backward error, host buffers in and out, the same for
every candidate); the fastest median wins, ties within `tie_rel` go to the
default.  The numeric result does not depend on the choice beyond rounding:
every candidate is a complete, certified solve.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .solver import LdltSymbolic, MixedLdltSolver, SolverSettings

Candidate = Tuple[str, bool, int]  # (schur_engine, overlap, panel_nb)
DEFAULT: Candidate = ("tensor", True, 64)


@dataclass
class TuneResult:
    chosen: Candidate
    seconds: Dict[Candidate, float]      # median step time per candidate
    certified: Dict[Candidate, bool]
    tuning_seconds: float
    fingerprint: tuple
    history: List[Tuple[Candidate, float]] = field(default_factory=list)

    def settings(self, base: Optional[SolverSettings] = None) -> SolverSettings:
        """The chosen knobs as settings; for the "fp64" tier the engine field
        keeps its default (use `fp64` to pick the factor call)."""
        s = base or SolverSettings()
        eng, s.overlap, s.panel_nb = self.chosen
        s.schur_engine = "tensor" if eng == "fp64" else eng
        return s

    @property
    def fp64(self) -> bool:
        return self.chosen[0] == "fp64"

    def table(self) -> dict:
        return {f"{e}/{'overlap' if o else 'in-order'}/nb{nb}": round(t * 1e3, 3)
                for (e, o, nb), t in sorted(self.seconds.items(), key=lambda kv: kv[1])}


_CACHE: Dict[tuple, TuneResult] = {}


def fingerprint(sym: LdltSymbolic, dtype) -> tuple:
    inf = sym.info()
    return (int(inf.n), int(inf.nnz), int(inf.nsuper), int(inf.nlevels), round(float(inf.flops_model), -6),
            np.dtype(dtype).str)


def candidates(engines: Sequence[str] = ("tensor", "fma"), overlaps: Sequence[bool] = (True, False),
               panel_widths: Sequence[int] = (64,)) -> List[Candidate]:
    out = [(e, o, nb) for nb in panel_widths for e in engines for o in overlaps]
    out.sort(key=lambda c: c != DEFAULT)  # the default first
    return out


def tune_mixed(a, b, target: float = 1e-14, sym: Optional[LdltSymbolic] = None,
               cands: Optional[Sequence[Candidate]] = None, reps: int = 2, warmup: int = 1,
               tie_rel: float = 0.02, use_cache: bool = True) -> TuneResult:
    """Tune the mixed-precision path (MixedLdltSolver: f32 / c32 factor +
    FP64 refinement) of matrix `a` with right-hand sides `b`.  `sym` is the
    analysis to reuse for the default panel width (others are analysed
    here)."""
    cands = list(cands or candidates())
    sym = sym or LdltSymbolic.analyze(a)
    key = fingerprint(sym, np.asarray(a.values).dtype) + (tuple(cands), float(target))
    if use_cache and key in _CACHE:
        return _CACHE[key]
    t_all = time.perf_counter()
    syms = {sym.settings.panel_nb: sym}
    secs: Dict[Candidate, float] = {}
    cert: Dict[Candidate, bool] = {}
    hist: List[Tuple[Candidate, float]] = []
    for c in cands:
        eng, ovl, nb = c
        if nb not in syms:
            s_an = SolverSettings(ordering=sym.settings.ordering, panel_nb=nb)
            syms[nb] = LdltSymbolic.analyze_with(a, s_an)
        st = SolverSettings(ordering=syms[nb].settings.ordering, schur_engine="tensor" if eng == "fp64" else eng,
                            overlap=ovl, panel_nb=nb)
        if eng == "fp64":
            from . import _native as N
            m = MixedLdltSolver.factor_tier(a, N.TIER_FP64, st, sym=syms[nb])
        else:
            m = MixedLdltSolver.factor_with(a, st, sym=syms[nb])
        ok = True
        times = []
        for it in range(warmup + reps):
            t0 = time.perf_counter()
            m.refactor(a)
            _, info = m.solve_to(a, b, target)
            dt = time.perf_counter() - t0
            ok = ok and bool(info.certified)
            if it >= warmup:
                times.append(dt)
                hist.append((c, dt))
        del m
        secs[c] = float(np.median(times))
        cert[c] = ok
    # fastest certified candidate; within tie_rel of the default, keep the default
    ok_c = [c for c in cands if cert[c]] or list(cands)
    best = min(ok_c, key=lambda c: secs[c])
    if DEFAULT in secs and cert.get(DEFAULT, False) and secs[DEFAULT] <= secs[best] * (1.0 + tie_rel):
        best = DEFAULT
    res = TuneResult(best, secs, cert, time.perf_counter() - t_all, key, hist)
    if use_cache:
        _CACHE[key] = res
    return res
