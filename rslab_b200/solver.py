"""Host-side mirror of RSLAB's symmetric direct-solver API over the C ABI.

Same names, argument meaning and error behaviour as the reference:
  CscMatrix            src/sparse/csc.rs:15 (lower triangle, sorted, duplicates summed)
  SolverSettings       src/numeric/multifrontal_ldlt.rs:302 (defaults :583-614)
  LdltSymbolic         src/numeric/sparse_solver.rs:457-711 (analyze once, factor many)
  LdltSolver           src/numeric/sparse_solver.rs:40-375
  MixedLdltSolver      src/numeric/mixed.rs:225-291, MixedInfo :81
  Inertia              src/inertia.rs:11
  RslabError family    src/error.rs:15-55
All numeric work runs in librslab_b200.so on the GPU; this module only moves
arrays across the boundary.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import NamedTuple, Optional

import numpy as np

from . import _native as N

# ---------------------------------------------------------------------------
# Errors (src/error.rs).
# ---------------------------------------------------------------------------


class RslabError(Exception):
    """Base of the reference error enum."""


class NumericallyRankDeficient(RslabError):
    pass


class InvalidInput(RslabError):
    pass


class DimensionMismatch(RslabError):
    def __init__(self, expected: int, got: int):
        super().__init__(f"dimension mismatch: expected {expected}, got {got}")
        self.expected = expected
        self.got = got


class CudaError(RslabError):
    pass


def _check(rc: int) -> None:
    if rc == 0:
        return
    msg = N.last_error()
    if rc == 1:
        raise NumericallyRankDeficient(msg)
    if rc == 2:
        raise InvalidInput(msg)
    if rc == 3:
        raise DimensionMismatch(-1, -1) from RslabError(msg)
    if rc == 4:
        raise CudaError(msg)
    raise RslabError(f"status {rc}: {msg}")


_DT = {np.dtype(np.float64): N.F64, np.dtype(np.complex128): N.C64,
       np.dtype(np.float32): N.F32, np.dtype(np.complex64): N.C32}
_NP = {v: k for k, v in _DT.items()}


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def _p64(a: np.ndarray):
    return a.ctypes.data_as(N.i64p)


# ---------------------------------------------------------------------------
# CSC container.
# ---------------------------------------------------------------------------


class CscMatrix:
    """Lower-triangle CSC, rows sorted within each column (csc.rs:15)."""

    def __init__(self, n: int, col_ptr, row_idx, values):
        self.n = int(n)
        self.col_ptr = _i64(col_ptr)
        self.row_idx = _i64(row_idx)
        self.values = np.ascontiguousarray(values)
        if self.values.dtype not in _DT:
            self.values = self.values.astype(np.float64)

    @classmethod
    def from_triplets(cls, n: int, rows, cols, vals) -> "CscMatrix":
        """Entries must be lower (row >= col); duplicates are summed (csc.rs:41-105)."""
        rows = _i64(rows)
        cols = _i64(cols)
        vals = np.asarray(vals)
        if not (len(rows) == len(cols) == len(vals)):
            raise InvalidInput("triplet arrays must have equal length")
        if len(cols) and (cols.min() < 0 or cols.max() >= n):
            raise InvalidInput(f"column index out of bounds for n={n}")
        if len(rows) and (rows.min() < 0 or rows.max() >= n):
            raise InvalidInput(f"row index out of bounds for n={n}")
        if np.any(rows < cols):
            k = int(np.nonzero(rows < cols)[0][0])
            raise InvalidInput(f"triplet {k} ({rows[k]}, {cols[k]}) is upper-triangle; "
                               "CscMatrix stores only the lower triangle (row >= col)")
        key = cols * max(n, 1) + rows
        order = np.argsort(key, kind="stable")
        key_s = key[order]
        uniq, start = np.unique(key_s, return_index=True)
        summed = np.add.reduceat(vals[order], start) if len(vals) else vals
        ucols = uniq // max(n, 1)
        urows = uniq % max(n, 1)
        col_ptr = np.zeros(n + 1, dtype=np.int64)
        np.add.at(col_ptr, ucols + 1, 1)
        col_ptr = np.cumsum(col_ptr)
        return cls(n, col_ptr, urows, summed)

    @property
    def nnz(self) -> int:
        return int(self.row_idx.shape[0])

    def validate(self) -> None:
        n = self.n
        if self.col_ptr.shape[0] != n + 1:
            raise InvalidInput(f"col_ptr length {self.col_ptr.shape[0]} != n+1={n + 1}")
        if self.row_idx.shape[0] != self.values.shape[0]:
            raise InvalidInput("row_idx and values length mismatch")
        if self.col_ptr[0] != 0:
            raise InvalidInput(f"col_ptr[0] must be 0, got {self.col_ptr[0]}")
        if self.col_ptr[n] != self.row_idx.shape[0]:
            raise InvalidInput("col_ptr[n] != nnz")
        # monotone col_ptr, row bounds, lower triangle, sorted columns: one
        # native pass (rslab_validate_lower_csc)
        cp = np.ascontiguousarray(self.col_ptr, np.int64)
        ri = np.ascontiguousarray(self.row_idx, np.int64)
        _check(N.lib.rslab_validate_lower_csc(n, _p64(cp), _p64(ri), int(ri.shape[0])))

    def astype(self, dtype) -> "CscMatrix":
        return CscMatrix(self.n, self.col_ptr, self.row_idx, self.values.astype(dtype))

    def to_scipy_full(self):
        import scipy.sparse as sp
        L = sp.csc_matrix((self.values, self.row_idx, self.col_ptr), shape=(self.n, self.n))
        D = sp.diags(L.diagonal())
        return (L + L.T - D).tocsr()

    def symv(self, x: np.ndarray) -> np.ndarray:
        """y = A x from the stored lower triangle (csc.rs:294-308), on the host."""
        return self.to_scipy_full() @ x


# ---------------------------------------------------------------------------
# Settings / results.
# ---------------------------------------------------------------------------


class Ordering:
    AMD = N.ORDER_AMD
    METIS_ND = N.ORDER_METIS_ND
    NATURAL = N.ORDER_NATURAL
    GIVEN = N.ORDER_GIVEN


@dataclass
class ZeroPivotAction:
    """`Fail` (exact) or `PerturbToEps(abs_floor)` (static pivoting)."""
    kind: str = "fail"
    abs_floor: float = 0.0

    @staticmethod
    def fail() -> "ZeroPivotAction":
        return ZeroPivotAction("fail")

    @staticmethod
    def perturb_to_eps(abs_floor: float) -> "ZeroPivotAction":
        return ZeroPivotAction("perturb", float(abs_floor))

    @staticmethod
    def force_accept() -> "ZeroPivotAction":
        """Accept tiny pivots: static pivoting at max(max|A_scaled|, 1) * eps
        (the left-looking path, multifrontal_ldlt.rs:3355-3358)."""
        return ZeroPivotAction("force_accept")


@dataclass
class SolverSettings:
    on_zero_pivot: ZeroPivotAction = field(default_factory=ZeroPivotAction.fail)
    ordering: int = Ordering.AMD
    nemin: int = 16
    relax: Optional[tuple] = (256, 64)
    reorder_hybrid_liu: bool = True
    panel_nb: int = 64
    scaling: str = "onepass"  # or "identity"
    use_graph: bool = True
    given_perm: Optional[np.ndarray] = None
    # descendant updates: "tensor" (GEMM tiles: 3xTF32 tcgen05 for f32 / c32,
    # FP64 DMMA for f64 / c64), "fma" (CUDA cores in the oracle's operation
    # order, bit-exact) or "auto" (tensor from 2e8 model flops, else fma)
    schur_engine: str = "auto"
    # incomplete factor: drop |L_ip| < drop_tol * max_i |L_ip| per column
    drop_tol: Optional[float] = None
    # schedule of the factor's launches: side streams overlap independent
    # work (True) or everything runs in order on one stream (False)
    overlap: bool = True
    # FactorMethod (multifrontal_ldlt.rs:283): "left_looking" (default) or
    # "multifrontal" (fronts with contribution blocks and extend-add)
    method: str = "left_looking"

    @staticmethod
    def exact() -> "SolverSettings":
        return SolverSettings()

    @staticmethod
    def preconditioner(abs_floor: float) -> "SolverSettings":
        return SolverSettings(on_zero_pivot=ZeroPivotAction.perturb_to_eps(abs_floor))

    def with_pivot(self, p: ZeroPivotAction) -> "SolverSettings":
        self.on_zero_pivot = p
        return self

    def with_ordering(self, o: int) -> "SolverSettings":
        self.ordering = o
        return self

    def with_nemin(self, nemin: int) -> "SolverSettings":
        self.nemin = nemin
        return self

    def with_relax(self, relax) -> "SolverSettings":
        self.relax = relax
        return self

    def with_panel_nb(self, nb: int) -> "SolverSettings":
        self.panel_nb = nb
        return self

    def with_scaling(self, s: str) -> "SolverSettings":
        self.scaling = s
        return self

    def _analyze_c(self):
        s = N.AnalyzeSettings()
        N.lib.rslab_default_analyze_settings(C.byref(s))
        s.ordering = self.ordering
        s.nemin = self.nemin
        if self.relax is None:
            s.relax = 0
        else:
            s.relax = 1
            s.relax_max_width, s.relax_max_extra_rows = self.relax
        s.hybrid_liu = int(self.reorder_hybrid_liu)
        s.panel_nb = self.panel_nb
        keep = None
        if self.ordering == Ordering.GIVEN:
            keep = _i64(self.given_perm)
            s.given_perm = _p64(keep)
        return s, keep

    def _factor_c(self, stream=None):
        s = N.FactorSettings()
        N.lib.rslab_default_factor_settings(C.byref(s))
        if self.on_zero_pivot.kind == "perturb":
            s.on_zero_pivot = N.PIVOT_PERTURB
            s.abs_floor = self.on_zero_pivot.abs_floor
        elif self.on_zero_pivot.kind == "force_accept":
            s.on_zero_pivot = N.PIVOT_FORCE_ACCEPT
        s.drop_tol = float(self.drop_tol) if self.drop_tol else 0.0
        s.scaling = N.SCALING_ONEPASS if self.scaling == "onepass" else N.SCALING_IDENTITY
        s.use_graph = int(self.use_graph)
        s.stream = stream
        engines = {"tensor": N.SCHUR_TENSOR, "fma": N.SCHUR_FMA, "auto": N.SCHUR_AUTO}
        if self.schur_engine not in engines:
            raise ValueError(f"schur_engine must be one of {sorted(engines)}")
        s.schur_engine = engines[self.schur_engine]
        s.overlap = int(bool(self.overlap))
        methods = {"left_looking": N.METHOD_LEFT_LOOKING, "multifrontal": N.METHOD_MULTIFRONTAL}
        if self.method not in methods:
            raise ValueError(f"method must be one of {sorted(methods)}")
        s.method = methods[self.method]
        return s


class Inertia(NamedTuple):
    positive: int
    negative: int
    zero: int


@dataclass
class MixedInfo:
    ir_iters: int
    gmres_iters: int
    backward_error: float
    certified: bool


@dataclass
class MemoryEstimate:
    """A-priori memory / work estimate of an analysis (MemoryEstimate,
    src/diagnostics.rs:14-53; computed as LdltSymbolic::estimate_memory,
    src/numeric/sparse_solver.rs:561-660)."""
    value_bytes: int
    factor_nnz: int
    factor_bytes: int
    panels_all_bytes: int
    panel_live_peak_bytes: int
    transient_peak_bytes: int
    factor_flops: int
    critical_path_flops: int
    max_tree_width: int
    mf_transient_peak_bytes: int = 0  # the multifrontal method's figure (every contribution block resident)


@dataclass
class StageReport:
    """One timed stage of a factorization (StageReport, src/diagnostics.rs:220-228)."""
    name: str
    wall_ms: float
    flops: int
    bytes: int


@dataclass
class Diagnostics:
    """Per-call factor diagnostics (Diagnostics, src/diagnostics.rs:235-240):
    the reference's stages / threads / factor_nnz / estimate, plus the
    device-side figures of this build.  `threads` is the number of
    multiprocessors of the GPU the factor ran on (the reference reports its
    CPU worker count)."""
    factor_ms: float
    solve_ms: float
    factor_nnz: int
    flops: float
    flops_proxy: float
    n_supernodes: int
    n_levels: int
    threads: int = 0
    estimate: Optional[MemoryEstimate] = None
    stages: list = field(default_factory=list)
    schur_engine: str = ""   # the descendant-update engine the factor ran with
    method: str = ""         # left_looking or multifrontal

    def total_ms(self) -> float:
        return sum(s.wall_ms for s in self.stages)


@dataclass
class LdltFactors:
    """The reference factor container (src/dense/ldlt_generic.rs:31-66)."""
    n: int
    l_col_ptr: np.ndarray
    l_row_idx: np.ndarray
    l_values: np.ndarray
    d_diag: np.ndarray
    d_subdiag: np.ndarray
    two_by_two: np.ndarray
    perm: np.ndarray
    n_perturbed: int
    inertia: Inertia
    scale: np.ndarray


# ---------------------------------------------------------------------------
# Analysis / factor handles.
# ---------------------------------------------------------------------------


class LdltSymbolic:
    """Phase-1 analysis of a pattern, reusable across value sets."""

    def __init__(self, handle, n: int, nnz: int, settings: SolverSettings):
        self._h = handle
        self.n = n
        self.nnz = nnz
        self.settings = settings

    @classmethod
    def analyze(cls, a: CscMatrix) -> "LdltSymbolic":
        return cls.analyze_with(a, SolverSettings())

    @classmethod
    def analyze_with(cls, a: CscMatrix, opts: SolverSettings) -> "LdltSymbolic":
        a.validate()
        s, keep = opts._analyze_c()
        h = C.c_void_p()
        _check(N.lib.rslab_analyze(a.n, _p64(a.col_ptr), _p64(a.row_idx), C.byref(s), C.byref(h)))
        del keep
        return cls(h, a.n, a.nnz, opts)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(N, "lib", None)  # None during interpreter shutdown
        if h and lib is not None:
            lib.rslab_free_symbolic(h)
            self._h = None

    def info(self) -> N.SymbolicInfo:
        inf = N.SymbolicInfo()
        _check(N.lib.rslab_symbolic_info(self._h, C.byref(inf)))
        return inf

    def n_levels(self) -> int:
        return int(self.info().nlevels)

    def estimate_memory(self, dtype=np.float64) -> MemoryEstimate:
        """A-priori estimate for a scalar of `dtype` (estimate_memory::<T>)."""
        e = N.MemoryEstimateC()
        _check(N.lib.rslab_symbolic_estimate(self._h, np.dtype(dtype).itemsize, C.byref(e)))
        return MemoryEstimate(int(e.value_bytes), int(e.factor_nnz), int(e.factor_bytes), int(e.panels_all_bytes),
                              int(e.panel_live_peak_bytes), int(e.transient_peak_bytes), int(e.factor_flops),
                              int(e.critical_path_flops), int(e.max_tree_width), int(e.mf_transient_peak_bytes))

    def symbolic_factor_nnz(self) -> int:
        """Exact symbolic fill x 1.2 slack (sparse_solver.rs:550-555)."""
        e = N.MemoryEstimateC()
        _check(N.lib.rslab_symbolic_estimate(self._h, 8, C.byref(e)))
        return int(e.symbolic_factor_nnz)

    @classmethod
    def tuned(cls, a: CscMatrix) -> tuple:
        """LdltSolver::tuned (sparse_solver.rs:108-131): the default analysis,
        then on large systems the nested-dissection bakeoff (:231-266) that
        adopts MetisND only on a clear predicted-flops win with no regression
        in exact fill or live-panel peak.  Returns (analysis, settings)."""
        a.validate()
        vals = np.asarray(a.values)
        vb = vals.dtype.itemsize if vals.dtype in _DT else 8
        h = C.c_void_p()
        used = C.c_int32(0)
        _check(N.lib.rslab_analyze_tuned(a.n, _p64(a.col_ptr), _p64(a.row_idx), vb, C.byref(h), C.byref(used)))
        s = SolverSettings(ordering=int(used.value))
        return cls(h, a.n, a.nnz, s), s

    def export(self) -> dict:
        inf = self.info()
        n, ns = int(inf.n), int(inf.nsuper)
        out = {k: np.zeros(n, np.int64) for k in ("perm", "col_counts", "parent")}
        for k in ("sn_first", "sn_ncol", "sn_nrow", "sn_level", "child_idx"):
            out[k] = np.zeros(max(ns, 1), np.int64)
        out["child_ptr"] = np.zeros(ns + 1, np.int64)
        _check(N.lib.rslab_symbolic_export(
            self._h, _p64(out["perm"]), _p64(out["sn_first"]), _p64(out["sn_ncol"]), _p64(out["sn_nrow"]),
            _p64(out["sn_level"]), _p64(out["child_ptr"]), _p64(out["child_idx"]), _p64(out["col_counts"]),
            _p64(out["parent"])))
        for k in ("sn_first", "sn_ncol", "sn_nrow", "sn_level"):
            out[k] = out[k][:ns]
        out["child_idx"] = out["child_idx"][: int(out["child_ptr"][-1])]
        return out

    def _check_pattern(self, a: CscMatrix) -> None:
        a.validate()
        if a.n != self.n or a.nnz != self.nnz:
            raise InvalidInput("factor_numeric: matrix does not match the analyzed pattern")

    def factor(self, a: CscMatrix, opts: Optional[SolverSettings] = None, stream=None) -> "LdltSolver":
        self._check_pattern(a)
        opts = opts or self.settings
        vals = np.ascontiguousarray(a.values)
        if vals.dtype not in _DT:
            raise InvalidInput(f"unsupported dtype {vals.dtype}")
        fs = opts._factor_c(stream)
        h = C.c_void_p()
        rc = N.lib.rslab_factor(self._h, _DT[vals.dtype], vals.ctypes.data_as(C.c_void_p), 0, C.byref(fs),
                                C.byref(h))
        solver = LdltSolver(h, self, vals.dtype) if h else None
        _check(rc)
        return solver

    def factor_device(self, dtype, values_ptr: int, opts: Optional[SolverSettings] = None, stream=None):
        """Factor values already resident in device memory (a raw pointer)."""
        opts = opts or self.settings
        fs = opts._factor_c(stream)
        h = C.c_void_p()
        rc = N.lib.rslab_factor(self._h, _DT[np.dtype(dtype)], C.c_void_p(values_ptr), 1, C.byref(fs), C.byref(h))
        solver = LdltSolver(h, self, np.dtype(dtype)) if h else None
        _check(rc)
        return solver


class LdltSolver:
    """A factored matrix; solves against many right-hand sides."""

    def __init__(self, handle, sym: LdltSymbolic, dtype):
        self._h = handle
        self._sym = sym
        self.dtype = np.dtype(dtype)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(N, "lib", None)  # None during interpreter shutdown
        if h and lib is not None:
            lib.rslab_free_factor(h)
            self._h = None

    @classmethod
    def factor(cls, a: CscMatrix) -> "LdltSolver":
        """Settings from the heuristic pick LdltSolver::tuned (sparse_solver.rs:94-97)."""
        sym, s = LdltSymbolic.tuned(a)
        return sym.factor(a, s)

    @classmethod
    def factor_with(cls, a: CscMatrix, opts: SolverSettings) -> "LdltSolver":
        return LdltSymbolic.analyze_with(a, opts).factor(a, opts)

    @property
    def n(self) -> int:
        return self._sym.n

    def refactor(self, a: CscMatrix) -> None:
        self._sym._check_pattern(a)
        vals = np.ascontiguousarray(a.values, dtype=self.dtype)
        _check(N.lib.rslab_refactor(self._h, vals.ctypes.data_as(C.c_void_p), 0))

    def reuse_pivots(self, on: bool = True) -> None:
        """Static pivot reuse: the following refactors replay the pivot steps
        of the last factor that searched (rslab_set_pivot_reuse)."""
        _check(N.lib.rslab_set_pivot_reuse(self._h, int(bool(on))))

    def _info(self) -> N.FactorInfo:
        inf = N.FactorInfo()
        _check(N.lib.rslab_factor_info(self._h, C.byref(inf)))
        return inf

    def inertia(self) -> Inertia:
        i = self._info()
        return Inertia(int(i.inertia_pos), int(i.inertia_neg), int(i.inertia_zero))

    def n_perturbed(self) -> int:
        return int(self._info().n_perturbed)

    def factor_nnz(self) -> int:
        nnz = C.c_int64()
        _check(N.lib.rslab_export_factors(self._h, None, None, None, None, None, None, None, None, C.byref(nnz)))
        return int(nnz.value)

    def diagnostics(self) -> Diagnostics:
        """Diagnostics of this factor (LdltSolver::diagnostics, sparse_solver.rs:57;
        filled as LdltSymbolic::factor does, :692-705)."""
        i = self._info()
        si = self._sym.info()
        nnz = self.factor_nnz()
        entry_bytes = self.dtype.itemsize + 8
        return Diagnostics(i.factor_ms, i.solve_ms, nnz, si.flops_model, si.flops_proxy, int(si.nsuper),
                           int(si.nlevels), threads=int(i.multiprocessors),
                           estimate=self._sym.estimate_memory(self.dtype),
                           stages=[StageReport("factor", float(i.factor_ms), int(si.flops_model), nnz * entry_bytes)],
                           schur_engine="fma" if i.schur_engine == N.SCHUR_FMA else "tensor",
                           method="multifrontal" if i.method == N.METHOD_MULTIFRONTAL else "left_looking")

    def stream(self) -> int:
        return int(N.lib.rslab_factor_stream(self._h) or 0)

    def solve(self, rhs) -> np.ndarray:
        b = np.ascontiguousarray(rhs, dtype=self.dtype)
        if b.shape[0] != self.n:
            raise DimensionMismatch(self.n, b.shape[0])
        return self.solve_many(b, 1).reshape(self.n)

    def solve_many(self, b, nrhs: int) -> np.ndarray:
        b = np.ascontiguousarray(b, dtype=self.dtype).reshape(-1)
        if nrhs <= 0 or b.shape[0] != self.n * nrhs:
            raise DimensionMismatch(self.n * nrhs, b.shape[0])
        x = np.empty_like(b)
        _check(N.lib.rslab_solve(self._h, b.ctypes.data_as(C.c_void_p), nrhs, x.ctypes.data_as(C.c_void_p), 0))
        return x.reshape(self.n, nrhs) if nrhs > 1 else x

    def solve_device(self, b_ptr: int, nrhs: int, x_ptr: int) -> None:
        _check(N.lib.rslab_solve(self._h, C.c_void_p(b_ptr), nrhs, C.c_void_p(x_ptr), 1))

    def solve_refined(self, a: CscMatrix, rhs, max_iter: int) -> np.ndarray:
        """Iterative refinement against the factored matrix (sparse_solver.rs:335-375),
        on the GPU: residuals from the stored values, per-column best iterate."""
        if a.n != self.n:
            raise DimensionMismatch(self.n, a.n)
        self._sym._check_pattern(a)
        b = np.ascontiguousarray(rhs, dtype=self.dtype)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        if b.shape[0] != self.n:
            raise DimensionMismatch(self.n, b.shape[0])
        x = np.empty_like(b)
        _check(N.lib.rslab_solve_refined(self._h, b.ctypes.data_as(C.c_void_p), nrhs, int(max_iter),
                                         x.ctypes.data_as(C.c_void_p), 0))
        return x

    def export_factors(self) -> LdltFactors:
        n = self.n
        nnz = self.factor_nnz()
        lcp = np.zeros(n + 1, np.int64)
        lri = np.zeros(max(nnz, 1), np.int64)
        lv = np.zeros(max(nnz, 1), self.dtype)
        d = np.zeros(n, self.dtype)
        ds = np.zeros(n, self.dtype)
        two = np.zeros(n, np.uint8)
        perm = np.zeros(n, np.int64)
        scale = np.zeros(n, np.float64)
        _check(N.lib.rslab_export_factors(
            self._h, _p64(lcp), _p64(lri), lv.ctypes.data_as(C.c_void_p), d.ctypes.data_as(C.c_void_p),
            ds.ctypes.data_as(C.c_void_p), two.ctypes.data_as(C.POINTER(C.c_uint8)), _p64(perm),
            scale.ctypes.data_as(C.POINTER(C.c_double)), None))
        return LdltFactors(n, lcp, lri[:nnz], lv[:nnz], d, ds, two.astype(bool), perm, self.n_perturbed(),
                           self.inertia(), scale)


class CompressedLdltFactors:
    """CompressedLdltFactors (src/dense/ldlt_generic.rs:434-536): the factor
    in the LdltFactors layout with uint32 index arrays and pivot permutation
    (half the index bytes), held on the host; `solve` is the reference's
    solve_ldlt on these factors, bit for bit.  Like the reference container it
    holds the factors of the equilibrated matrix S A S (S = the factor's
    `scale`), so `solve` solves with S A S."""

    def __init__(self, handle, dtype):
        self._h = handle
        self.dtype = np.dtype(dtype)
        n, nnz, ib, dt = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        _check(N.lib.rslab_cfac_info(handle, C.byref(n), C.byref(nnz), C.byref(ib), C.byref(dt)))
        self.n, self._nnz, self._index_bytes = int(n.value), int(nnz.value), int(ib.value)

    @classmethod
    def from_factors(cls, solver: "LdltSolver") -> Optional["CompressedLdltFactors"]:
        """The compressed copy of `solver`'s factor, or None when n or nnz(L)
        does not fit 32 bits (the reference's from_factors returns None)."""
        h = C.c_void_p()
        rc = N.lib.rslab_compress_factors(solver._h, C.byref(h))
        if rc == 2 and "32 bits" in N.last_error():
            return None
        _check(rc)
        return cls(h, solver.dtype)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(N, "lib", None)
        if h and lib is not None:
            lib.rslab_free_cfac(h)
            self._h = None

    def factor_nnz(self) -> int:
        return self._nnz

    def index_bytes(self) -> int:
        return self._index_bytes

    def arrays(self) -> dict:
        n, nnz = self.n, self._nnz
        u32 = C.POINTER(C.c_uint32)
        out = {"l_col_ptr": np.zeros(n + 1, np.uint32), "l_row_idx": np.zeros(max(nnz, 1), np.uint32),
               "l_values": np.zeros(max(nnz, 1), self.dtype), "d_diag": np.zeros(n, self.dtype),
               "d_subdiag": np.zeros(n, self.dtype), "two_by_two": np.zeros(n, np.uint8),
               "perm": np.zeros(n, np.uint32)}
        _check(N.lib.rslab_cfac_export(
            self._h, out["l_col_ptr"].ctypes.data_as(u32), out["l_row_idx"].ctypes.data_as(u32),
            out["l_values"].ctypes.data_as(C.c_void_p), out["d_diag"].ctypes.data_as(C.c_void_p),
            out["d_subdiag"].ctypes.data_as(C.c_void_p), out["two_by_two"].ctypes.data_as(C.POINTER(C.c_uint8)),
            out["perm"].ctypes.data_as(u32)))
        out["l_row_idx"] = out["l_row_idx"][:nnz]
        out["l_values"] = out["l_values"][:nnz]
        out["two_by_two"] = out["two_by_two"].astype(bool)
        return out

    def solve(self, rhs) -> np.ndarray:
        b = np.ascontiguousarray(rhs, dtype=self.dtype).reshape(-1)
        if b.shape[0] != self.n:
            raise DimensionMismatch(self.n, b.shape[0])
        x = np.empty_like(b)
        _check(N.lib.rslab_cfac_solve(self._h, b.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p)))
        return x


CERT_FACTOR = 64.0
EPS_F64 = 2.220446049250313e-16


class MixedLdltSolver:
    """Low-precision factor of cast(A), refined to double precision (mixed.rs:225)."""

    def __init__(self, handle, sym: LdltSymbolic, dtype_hi):
        self._h = handle
        self._sym = sym
        self.dtype = np.dtype(dtype_hi)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(N, "lib", None)  # None during interpreter shutdown
        if h and lib is not None:
            lib.rslab_free_factor(h)
            self._h = None

    @classmethod
    def factor(cls, a: CscMatrix) -> "MixedLdltSolver":
        """Factor cast(A) with the heuristic pick LdltSolver::tuned on the
        low-precision matrix (mixed.rs:232-243)."""
        vals = np.asarray(a.values)
        lo = np.complex64 if np.iscomplexobj(vals) else np.float32
        sym, s = LdltSymbolic.tuned(a.astype(lo))
        sym.nnz = a.nnz
        return cls.factor_with(a, s, sym=sym)

    @classmethod
    def factor_with(cls, a: CscMatrix, opts: SolverSettings, sym: Optional[LdltSymbolic] = None,
                    stream=None) -> "MixedLdltSolver":
        sym = sym or LdltSymbolic.analyze_with(a, opts)
        sym._check_pattern(a)
        vals = np.ascontiguousarray(a.values)
        if vals.dtype not in (np.dtype(np.float64), np.dtype(np.complex128)):
            raise InvalidInput("mixed factor needs an f64 or c64 matrix")
        fs = opts._factor_c(stream)
        h = C.c_void_p()
        rc = N.lib.rslab_mixed_factor(sym._h, _DT[vals.dtype], vals.ctypes.data_as(C.c_void_p), 0, C.byref(fs),
                                      C.byref(h))
        out = cls(h, sym, vals.dtype) if h else None
        _check(rc)
        return out

    @classmethod
    def factor_tier(cls, a: CscMatrix, tier: int, opts: Optional[SolverSettings] = None,
                    sym: Optional[LdltSymbolic] = None, stream=None) -> "MixedLdltSolver":
        """The refined factor in precision tier `tier` (N.TIER_FP64 / TIER_FP32 /
        TIER_TF32X3; the tier sets the descendant-update engine).  TIER_FP64
        factors in the matrix's own field and refines with the same ladder."""
        opts = opts or SolverSettings()
        sym = sym or LdltSymbolic.analyze_with(a, opts)
        sym._check_pattern(a)
        vals = np.ascontiguousarray(a.values)
        if vals.dtype not in (np.dtype(np.float64), np.dtype(np.complex128)):
            raise InvalidInput("tier factor needs an f64 or c64 matrix")
        fs = opts._factor_c(stream)
        h = C.c_void_p()
        rc = N.lib.rslab_tier_factor(sym._h, _DT[vals.dtype], int(tier), vals.ctypes.data_as(C.c_void_p), 0,
                                     C.byref(fs), C.byref(h))
        out = cls(h, sym, vals.dtype) if h else None
        _check(rc)
        return out

    def refactor(self, a: CscMatrix) -> None:
        self._sym._check_pattern(a)
        vals = np.ascontiguousarray(a.values, dtype=self.dtype)
        _check(N.lib.rslab_refactor(self._h, vals.ctypes.data_as(C.c_void_p), 0))

    def reuse_pivots(self, on: bool = True) -> None:
        """Static pivot reuse: the following refactors replay the pivot steps
        of the last factor that searched (rslab_set_pivot_reuse)."""
        _check(N.lib.rslab_set_pivot_reuse(self._h, int(bool(on))))

    def solve(self, a: CscMatrix, b) -> tuple:
        return self.solve_to(a, b, CERT_FACTOR * EPS_F64)

    def solve_to(self, a: CscMatrix, b, target_backward_error: float, out: Optional[np.ndarray] = None) -> tuple:
        """`out` (optional, not in the reference API): a C-contiguous array of
        b's shape and dtype that receives the solution, e.g. page-locked
        host memory so the device-to-host copy runs at full speed."""
        if a.n != self._sym.n:
            raise DimensionMismatch(self._sym.n, a.n)
        b = np.ascontiguousarray(b, dtype=self.dtype)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        if b.shape[0] != self._sym.n:
            raise DimensionMismatch(self._sym.n, b.shape[0])
        if out is not None:
            if out.shape != b.shape or out.dtype != b.dtype or not out.flags["C_CONTIGUOUS"]:
                raise InvalidInput("out must be C-contiguous with the shape and dtype of b")
            x = out
        else:
            x = np.empty_like(b)
        info = N.MixedInfoC()
        _check(N.lib.rslab_mixed_solve(self._h, b.ctypes.data_as(C.c_void_p), nrhs, float(target_backward_error),
                                       x.ctypes.data_as(C.c_void_p), 0, C.byref(info)))
        return x, MixedInfo(int(info.ir_iters), int(info.gmres_iters), float(info.backward_error),
                            bool(info.certified))

    def inertia(self) -> Inertia:
        inf = N.FactorInfo()
        _check(N.lib.rslab_factor_info(self._h, C.byref(inf)))
        return Inertia(int(inf.inertia_pos), int(inf.inertia_neg), int(inf.inertia_zero))

    def diagnostics(self) -> N.FactorInfo:
        inf = N.FactorInfo()
        _check(N.lib.rslab_factor_info(self._h, C.byref(inf)))
        return inf

    def stream(self) -> int:
        return int(N.lib.rslab_factor_stream(self._h) or 0)


KINDS = ("assembly", "cmod", "getf2", "deep_replay", "panel_schur", "total")


def factor_profile(handle) -> dict:
    """Per-kernel-class device ms, launches and algorithmic flops of one eager
    refactor (the measurement aid behind bench.py's roofline line)."""
    ms = (C.c_double * 6)()
    nl = (C.c_int64 * 6)()
    fl = (C.c_double * 6)()
    _check(N.lib.rslab_factor_profile(handle, ms, nl, fl))
    return {k: {"ms": ms[i], "launches": int(nl[i]), "flops": fl[i]} for i, k in enumerate(KINDS)}


SOLVE_KINDS = ("permute", "fwd_diag", "fwd_push", "dsolve", "bwd_off", "bwd_diag", "total")


def solve_profile(handle, nrhs: int) -> dict:
    """Per-kernel-class device ms and launches of one eager solve."""
    ms = (C.c_double * 7)()
    nl = (C.c_int64 * 7)()
    _check(N.lib.rslab_solve_profile(handle, nrhs, ms, nl))
    return {k: {"ms": ms[i], "launches": int(nl[i])} for i, k in enumerate(SOLVE_KINDS)}


LAUNCH_KINDS = ("cmod", "getf2", "deep_replay", "panel_schur", "fwd_diag", "fwd_push", "bwd_off", "bwd_diag",
                "cmod_mm", "cmod_asm", "split_r", "split_c", "fwd_gather", "extend_add", "make_g", "diag_inv",
                "bwd_off_reduce", "schur_tc", "fwd_chain", "bwd_chain", "bwd_gather", "deep_mm", "make_m", "push_reduce",
                "front_cb", "join")


def profile_trace(handle) -> list:
    """Per-launch (kind, grid, ms) rows of the handle's last factor/solve profile."""
    cnt = C.c_int64(0)
    _check(N.lib.rslab_profile_trace(handle, 0, None, None, None, C.byref(cnt)))
    m = int(cnt.value)
    kind = (C.c_int32 * max(m, 1))()
    grid = (C.c_int32 * max(m, 1))()
    ms = (C.c_float * max(m, 1))()
    _check(N.lib.rslab_profile_trace(handle, m, kind, grid, ms, C.byref(cnt)))
    return [(LAUNCH_KINDS[kind[i]] if kind[i] >= 0 else "other", int(grid[i]), float(ms[i])) for i in range(m)]


def amd_order(n: int, col_ptr, row_idx) -> tuple:
    """AMD on a full symmetric pattern; returns (perm, stats dict)."""
    cp = _i64(col_ptr)
    ri = _i64(row_idx)
    perm = np.zeros(n, np.int64)
    st = (C.c_double * 7)()
    _check(N.lib.rslab_amd_order(n, _p64(cp), _p64(ri), _p64(perm), st))
    keys = ("ncmpa", "n_dense", "ndiv", "nms_ldl", "nms_lu", "n_mass_elim", "n_supervar_merge")
    return perm, {k: st[i] for i, k in enumerate(keys)}


def metis_order(n: int, col_ptr, row_idx, seed: int = 1, dense_quotient: bool = False,
                dense_threshold: Optional[int] = None) -> np.ndarray:
    """MetisND on a full symmetric pattern (new-to-old permutation); the
    keywords are MetisOptions' seed, dense_quotient_enabled and
    dense_quotient_threshold (crates/rslab-metis/src/lib.rs:90-122)."""
    cp = _i64(col_ptr)
    ri = _i64(row_idx)
    perm = np.zeros(n, np.int64)
    _check(N.lib.rslab_metis_order(n, _p64(cp), _p64(ri), C.c_uint64(seed), int(dense_quotient),
                                   -1 if dense_threshold is None else int(dense_threshold), _p64(perm)))
    return perm


def device_count() -> int:
    c = C.c_int(0)
    N.lib.rslab_device_count(C.byref(c))
    return int(c.value)
