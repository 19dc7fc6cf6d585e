"""ORACLE — test infrastructure only (see oracle.cpp).

ctypes wrapper of oracle/_build/liboracle.so, the C++ restatement of the
reference CPU LDL^T path.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg may import this module; the rslab_b200 product never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_DT = {np.dtype(np.float64): 0, np.dtype(np.complex128): 1, np.dtype(np.float32): 2, np.dtype(np.complex64): 3}
i64p = C.POINTER(C.c_int64)
vp = C.c_void_p


def build() -> Path:
    srcs = [HERE / "oracle.cpp", HERE / "symbolic.cpp", HERE / "build_oracle.sh"]
    if not LIB.exists() or any(LIB.stat().st_mtime < s.stat().st_mtime for s in srcs):
        subprocess.run(["bash", str(HERE / "build_oracle.sh")], check=True, stdout=subprocess.DEVNULL)
    return LIB


def _load():
    build()
    lib = C.CDLL(str(LIB))
    lib.oracle_factor.restype = vp
    lib.oracle_factor.argtypes = [C.c_int, C.c_int64, i64p, i64p, vp, i64p, C.c_int64, i64p, i64p, i64p, i64p,
                                  C.c_int, C.c_double, C.c_double, C.c_int64, C.POINTER(C.c_int)]
    lib.oracle_factor_nnz.restype = C.c_int64
    lib.oracle_factor_nnz.argtypes = [vp]
    lib.oracle_export.restype = None
    lib.oracle_export.argtypes = [vp, i64p, i64p, vp, vp, vp, C.POINTER(C.c_uint8), i64p, C.POINTER(C.c_double),
                                  i64p]
    lib.oracle_solve.restype = C.c_int
    lib.oracle_solve.argtypes = [vp, vp, C.c_int64, vp]
    lib.oracle_mixed_solve.restype = C.c_int
    lib.oracle_mixed_solve.argtypes = [vp, C.c_int, C.c_int64, i64p, i64p, vp, vp, C.c_double, vp, i64p,
                                       C.POINTER(C.c_double), C.POINTER(C.c_int)]
    lib.oracle_symv.restype = None
    lib.oracle_symv.argtypes = [C.c_int, C.c_int64, i64p, i64p, vp, vp, vp]
    lib.oracle_free.restype = None
    lib.oracle_free.argtypes = [vp]
    lib.oracle_set_parallel.restype = C.c_int
    lib.oracle_set_parallel.argtypes = [C.c_int, C.c_char_p, C.c_int]
    lib.oracle_symbolic.restype = C.c_int64
    lib.oracle_symbolic.argtypes = [C.c_int64, i64p, i64p, i64p, C.c_int64, C.c_int64, C.c_int64] + [i64p] * 9 + \
        [C.POINTER(C.c_int32)]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _p(a):
    return a.ctypes.data_as(i64p)


def openblas_path() -> str:
    """The ILP64 OpenBLAS that numpy ships (numpy.libs/libscipy_openblas64_*.so)."""
    import glob
    import os

    d = os.path.join(os.path.dirname(os.path.dirname(np.__file__)), "numpy.libs")
    hits = sorted(glob.glob(os.path.join(d, "libscipy_openblas64_*.so")))
    if not hits:
        raise RuntimeError(f"no libscipy_openblas64_*.so under {d}")
    return hits[0]


def set_parallel(fast: bool, threads: int = 0) -> None:
    """Timing mode (BLAS products, level-parallel schedule) on or off; off is
    the exact checker.  threads 0 = all cores."""
    path = openblas_path().encode() if fast else b""
    if lib().oracle_set_parallel(int(fast), path, int(threads)) != 0:
        raise RuntimeError("oracle: OpenBLAS did not load")


def oracle_structure(a, ordering: np.ndarray, nemin: int = 16, relax=(256, 64)) -> dict:
    """The reference's symbolic analysis (oracle/symbolic.cpp) of the lower
    CSC pattern of `a` for the ordering output `ordering` (new-to-old, before
    the postorder): a dict with the keys of LdltSymbolic.export() (perm,
    parent, col_counts, sn_first, sn_ncol, sn_nrow = row-structure heights,
    sn_level, child_ptr, child_idx) plus `renumbered`."""
    n = a.n
    cp = np.ascontiguousarray(a.col_ptr, np.int64)
    ri = np.ascontiguousarray(a.row_idx, np.int64)
    o = np.ascontiguousarray(ordering, np.int64)
    out = {k: np.zeros(max(n, 1), np.int64) for k in ("perm", "parent", "col_counts", "sn_first", "sn_ncol",
                                                      "sn_nrow", "sn_level", "child_idx")}
    out["child_ptr"] = np.zeros(n + 1, np.int64)
    ren = C.c_int32(0)
    rw, rr = (relax if relax is not None else (0, 0))
    ns = lib().oracle_symbolic(n, _p(cp), _p(ri), _p(o), nemin, rw, rr, _p(out["perm"]), _p(out["parent"]),
                               _p(out["col_counts"]), _p(out["sn_first"]), _p(out["sn_ncol"]), _p(out["sn_nrow"]),
                               _p(out["sn_level"]), _p(out["child_ptr"]), _p(out["child_idx"]), C.byref(ren))
    for k in ("perm", "parent", "col_counts"):
        out[k] = out[k][:n]
    for k in ("sn_first", "sn_ncol", "sn_nrow", "sn_level"):
        out[k] = out[k][:ns]
    out["child_ptr"] = out["child_ptr"][: ns + 1]
    out["child_idx"] = out["child_idx"][: int(out["child_ptr"][-1])]
    out["renumbered"] = bool(ren.value)
    return out


def supernode_parent(ex: dict) -> np.ndarray:
    """Parent supernode of every supernode (-1 for roots) from a structure
    dict's child lists (their order is a scheduling choice, the sets are not)."""
    ns = len(ex["sn_first"])
    par = np.full(ns, -1, np.int64)
    cp, ci = ex["child_ptr"], ex["child_idx"]
    for s in range(ns):
        par[ci[cp[s]:cp[s + 1]]] = s
    return par


@dataclass
class OracleFactors:
    n: int
    l_col_ptr: np.ndarray
    l_row_idx: np.ndarray
    l_values: np.ndarray
    d_diag: np.ndarray
    d_subdiag: np.ndarray
    two_by_two: np.ndarray
    perm: np.ndarray
    scale: np.ndarray
    inertia: tuple
    n_perturbed: int
    status: int


class OracleSolver:
    """LdltSymbolic::factor + LdltSolver::solve_many restated on the CPU."""

    def __init__(self, a, sym_export: dict, dtype=None, perturb_floor: float = -1.0, panel_nb: int = 64,
                 scaling: bool = True):
        self.a = a
        vals = np.ascontiguousarray(a.values if dtype is None else a.values.astype(dtype))
        self.dtype = vals.dtype
        self.vals = vals
        st = C.c_int(0)
        s = sym_export
        self.sn_first = np.ascontiguousarray(s["sn_first"], np.int64)
        self.sn_ncol = np.ascontiguousarray(s["sn_ncol"], np.int64)
        self.cp = np.ascontiguousarray(s["child_ptr"], np.int64)
        self.ci = np.ascontiguousarray(s["child_idx"] if len(s["child_idx"]) else np.zeros(1, np.int64), np.int64)
        self.perm = np.ascontiguousarray(s["perm"], np.int64)
        self.h = lib().oracle_factor(_DT[self.dtype], a.n, _p(a.col_ptr), _p(a.row_idx),
                                     vals.ctypes.data_as(vp), _p(self.perm), len(self.sn_first), _p(self.sn_first),
                                     _p(self.sn_ncol), _p(self.cp), _p(self.ci), int(scaling), perturb_floor, -1.0,
                                     panel_nb, C.byref(st))
        self.status = st.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_free(self.h)
            self.h = None

    def factors(self) -> OracleFactors:
        n = self.a.n
        nnz = lib().oracle_factor_nnz(self.h)
        lcp = np.zeros(n + 1, np.int64)
        lri = np.zeros(max(nnz, 1), np.int64)
        lv = np.zeros(max(nnz, 1), self.dtype)
        d = np.zeros(n, self.dtype)
        ds = np.zeros(n, self.dtype)
        two = np.zeros(n, np.uint8)
        perm = np.zeros(n, np.int64)
        scale = np.zeros(n, np.float64)
        info = np.zeros(5, np.int64)
        lib().oracle_export(self.h, _p(lcp), _p(lri), lv.ctypes.data_as(vp), d.ctypes.data_as(vp),
                            ds.ctypes.data_as(vp), two.ctypes.data_as(C.POINTER(C.c_uint8)), _p(perm),
                            scale.ctypes.data_as(C.POINTER(C.c_double)), _p(info))
        return OracleFactors(n, lcp, lri[:nnz], lv[:nnz], d, ds, two.astype(bool), perm, scale,
                             (int(info[0]), int(info[1]), int(info[2])), int(info[3]), int(info[4]))

    def solve_many(self, b: np.ndarray, nrhs: int) -> np.ndarray:
        b = np.ascontiguousarray(b, self.dtype).reshape(-1)
        x = np.zeros_like(b)
        rc = lib().oracle_solve(self.h, b.ctypes.data_as(vp), nrhs, x.ctypes.data_as(vp))
        if rc != 0:
            raise RuntimeError(f"oracle solve status {rc}")
        return x.reshape(self.a.n, nrhs) if nrhs > 1 else x


def mixed_solve(lo: OracleSolver, a, b: np.ndarray, target: float):
    """MixedLdltSolver::solve_to with `lo` the f32/c32 oracle factor of cast(A)."""
    hi = np.ascontiguousarray(a.values)
    dt_hi = _DT[hi.dtype]
    b = np.ascontiguousarray(b, hi.dtype)
    x = np.zeros_like(b)
    it = np.zeros(2, np.int64)
    be = C.c_double(0)
    cert = C.c_int(0)
    rc = lib().oracle_mixed_solve(lo.h, dt_hi, a.n, _p(a.col_ptr), _p(a.row_idx), hi.ctypes.data_as(vp),
                                  b.ctypes.data_as(vp), target, x.ctypes.data_as(vp), _p(it), C.byref(be),
                                  C.byref(cert))
    if rc != 0:
        raise RuntimeError(f"oracle mixed solve status {rc}")
    return x, {"ir_iters": int(it[0]), "gmres_iters": int(it[1]), "backward_error": be.value,
               "certified": bool(cert.value)}


def backward_error(a, x: np.ndarray, b: np.ndarray) -> float:
    """Normwise ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) per column (max)."""
    A = a.to_scipy_full()
    r = b - A @ x
    anorm = float(abs(A).sum(axis=1).max())
    if x.ndim == 1:
        x, r, b = x[:, None], r[:, None], b[:, None]
    be = np.abs(r).max(axis=0) / np.maximum(anorm * np.abs(x).max(axis=0) + np.abs(b).max(axis=0), 1e-300)
    return float(be.max())
