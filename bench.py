"""Benchmark: LDL^T factor + solve at backward error <= 1e-14 on a B200.

Workload (one step): the complex-symmetric 3D 7-point Helmholtz matrix
A = -Delta_h - k^2 (1 + 0.05 i) I on a side^3 grid (default 64^3, n = 262,144),
k^2 = 0.2 lambda_max, 16 right-hand sides with U[-1, 1) real and imaginary
parts (seed 1).  Analysis (ordering + symbolic) is done once, outside the
timed region, as in the reference's methodology.
  * headline (`value`): the mixed-precision path — the numeric factor in the
    precision tier the tier network picks from the matrix's features (c32 with
    tensor-core updates on this matrix) + FP64 refinement against the
    original A (IR -> GMRES-IR) until every
    right-hand side's normwise backward error is <= 1e-14; GFLOP/s counts the
    model flops of the FP64-equivalent factor (sum_s sum_m (m^2 - 1), x4 for
    complex) per step time;
  * `fp64_gpu`: the plain FP64 GPU factor + solve (+ FP64 IR to 1e-14) on the
    same matrix, for the mixed/FP64 ratio;
  * `e2e`: the mixed path through the public Python API with host buffers
    (values + RHS copied in, solution copied out, every step).
Multi-GPU (--gpus N under torchrun): replicas — each rank factors and solves
its own copy (the path does not shard), value = N x per-rank work / max time.
`--impl reference` times the CPU oracle (C++ restatement of the reference's
CPU path) on a bounded sample on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

EPS = 2.220446049250313e-16


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--side", type=int, default=64)
    p.add_argument("--nrhs", type=int, default=16)
    p.add_argument("--target", type=float, default=1e-14)
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--workload", default="helmholtz", choices=["helmholtz", "sweep", "tiers", "batch"],
                   help="helmholtz: the 64^3 Helmholtz factor+solve step (default); sweep: the "
                        "same-pattern frequency sweep, 48^3 27-point K - w^2 M + i w C, 64 frequencies; "
                        "tiers: the learned precision tier on the held-out 80^3 27-point complex Helmholtz; "
                        "batch: 512 uneven shifted 3D Laplacians (sides 12-40) factored and solved together")
    p.add_argument("--batch-count", type=int, default=512)
    p.add_argument("--ordering", default="tuned", choices=["tuned", "amd", "metis"],
                   help="fill-reducing ordering of the helmholtz workload: tuned = the default pick of "
                        "LdltSolver::factor (nested-dissection bakeoff; MetisND on this matrix), amd, metis")
    p.add_argument("--method", default="left_looking", choices=["left_looking", "multifrontal"],
                   help="helmholtz workload: the numeric schedule of both legs (the multifrontal "
                        "method factors through contribution blocks and extend-add)")
    p.add_argument("--tiers-side", type=int, default=80)
    p.add_argument("--tier-model", default=None, help="tier network .npz (default: the package's trained one)")
    p.add_argument("--sweep-side", type=int, default=48)
    p.add_argument("--sweep-count", type=int, default=64)
    p.add_argument("--no-pivot-reuse", action="store_true",
                   help="sweep: search pivots at every frequency instead of replaying the first factor's")
    p.add_argument("--sweep-fp64-count", type=int, default=4,
                   help="frequencies (evenly spread) timed on the plain FP64 path for the ratio")
    p.add_argument("--profile-step", action="store_true",
                   help="one warm-up mixed step, then exactly one mixed step between "
                        "cudaProfilerStart/Stop (for ncu --profile-from-start off); no JSON line")
    return p.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def allmax(v: float, ws: int) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_setup(args):
    """The reference CPU path's inputs for the headline workload: the same
    Helmholtz matrix and right-hand sides, the same ordering output (the
    tuned pick: MetisND on this matrix), and the symbolic structure built by
    the oracle's own restatement of the reference's symbolic analysis from
    that ordering (oracle/symbolic.cpp).  The ordering itself comes from the
    MetisND restatement in librslab_b200 (the oracle has none), outside any
    timed region, as the analysis is in both arms."""
    from oracle.oracle import oracle_structure
    from rslab_b200 import LdltSymbolic, Ordering, matgen
    from rslab_b200.solver import amd_order, metis_order
    a = matgen.c2_matrix(args.side)
    t0 = time.perf_counter()
    full = a.to_scipy_full().tocsc()
    full.sort_indices()
    cp, ri = np.asarray(full.indptr, np.int64), np.asarray(full.indices, np.int64)
    if args.ordering == "amd":
        ordering = "AMD"
    elif args.ordering == "metis":
        ordering = "MetisND"
    else:
        _, st = LdltSymbolic.tuned(a)
        ordering = "MetisND" if st.ordering == Ordering.METIS_ND else "AMD"
    ordv = metis_order(a.n, cp, ri) if ordering == "MetisND" else amd_order(a.n, cp, ri)[0]
    ex = oracle_structure(a, ordv)
    t_an = time.perf_counter() - t0
    sn_c = ex["sn_ncol"].astype(np.float64)
    sn_r = ex["sn_nrow"].astype(np.float64)
    m = sn_r - sn_c + 1.0
    # sum_s sum_{m=r-c+1}^{r} (m^2 - 1), x4 for the complex field
    flops = 4.0 * float(np.sum((sn_r * (sn_r + 1) * (2 * sn_r + 1) - (m - 1) * m * (2 * m - 1)) / 6.0 - sn_c))
    b = matgen.uniform_rhs(a.n, args.nrhs, 1, complex_=True)
    return a, ex, b, flops, ordering, t_an


def cpu_run(a, ex, b, nrhs):
    """One FP64 factor + nrhs-column solve by the oracle in timing mode."""
    from oracle.oracle import OracleSolver
    t0 = time.perf_counter()
    o = OracleSolver(a, ex)
    x = o.solve_many(b, nrhs)
    return time.perf_counter() - t0, x


def cpu_sample(args):
    """The reported CPU baseline of the headline line: the oracle (the C++
    restatement of the reference CPU path) in timing mode (OpenBLAS products,
    level-parallel schedule, all host threads) on the full workload, one
    warm-up factor + solve and one timed."""
    from oracle.oracle import backward_error, set_parallel
    set_parallel(True)
    a, ex, b, flops, ordering, _ = cpu_setup(args)
    cpu_run(a, ex, b, args.nrhs)
    t, x = cpu_run(a, ex, b, args.nrhs)
    be = backward_error(a, x, b)
    cpu_sample.solution = x  # the oracle's FP64 solution, for the GPU arms' forward errors
    return {"value": flops / t / 1e9, "unit": "GFLOP/s", "cores": os.cpu_count(), "kind": "port",
            "seconds": t,
            "sample": f"FP64 factor + {args.nrhs}-RHS solve of the full {args.side}^3 Helmholtz workload ({ordering}, "
                      f"n={a.n}, model flops {flops:.3g}), one timed run after one warm-up; backward error "
                      f"{be:.2e}; oracle timing mode: OpenBLAS GEMMs, level-parallel supernodes, "
                      f"{os.cpu_count()} threads"}


def host_backward_error(a, x, b) -> float:
    """Normwise backward error max|b - A x| / (||A||_inf max|x| + max|b|) over
    all columns, A the symmetric matrix of the stored lower triangle (the
    certificate of MixedInfo, recomputed on the host)."""
    import scipy.sparse as sp
    n = a.n
    cp = np.asarray(a.col_ptr)
    col = np.repeat(np.arange(n), np.diff(cp))
    low = sp.csr_matrix((np.asarray(a.values), (np.asarray(a.row_idx), col)), shape=(n, n))
    full = low + low.T - sp.diags(low.diagonal())
    x2 = x.reshape(n, -1)
    b2 = np.asarray(b).reshape(n, -1)
    r = b2 - full @ x2
    anorm = float(np.abs(full).sum(axis=1).max())
    return float(np.max(np.abs(r).max(axis=0) / (anorm * np.abs(x2).max(axis=0) + np.abs(b2).max(axis=0))))


def launches_per_step(prof_mixed, sprof, minfo):
    """Kernels launched in one mixed step: the refactor's launches (counted
    by the eager profile), one c32 solve per refinement step plus the first
    (each the solve profile's count), and the FP64 refinement kernels of
    MixedLdltSolver::solve_to: ||A|| and ||b|| (2), casts around every solve
    (2 each), per check residual + two norms + best-iterate copy (4), per
    correction one axpy."""
    ir = int(minfo.ir_iters)
    solves = 1 + ir
    return int(prof_mixed["total"]["launches"] + solves * (sprof["total"]["launches"] + 2) + 2
               + (ir + 1) * 4 + ir)


def run_reference(args, ws, rank):
    """Reference arm: the reference's CPU path restated (the oracle, timing
    mode, all host threads) on the same workload as the GPU arm (rank 0 only).
    A step is one FP64 factor + solve of the full matrix (tens of seconds),
    so the arm times at most 3 steps after at most 1 warm-up and says so."""
    if rank != 0:
        return
    from oracle.oracle import backward_error, set_parallel
    set_parallel(True)
    a, ex, b, flops, ordering, t_an = cpu_setup(args)
    warm = min(max(args.warmup, 0), 1)
    steps = max(1, min(args.steps, 3))
    times, x = [], None
    for it in range(warm + steps):
        t, x = cpu_run(a, ex, b, args.nrhs)
        if it >= warm:
            times.append(t)
    t = float(np.mean(times))
    gf = flops / t / 1e9
    be = backward_error(a, x, b)
    cb = {"value": gf, "unit": "GFLOP/s", "cores": os.cpu_count(), "kind": "port", "seconds": t,
          "sample": f"the full workload: FP64 factor + {args.nrhs}-RHS solve of the {args.side}^3 Helmholtz matrix "
                    f"({ordering}), {steps} timed step(s) after {warm} warm-up (of the requested {args.steps} / "
                    f"{args.warmup}: a step is {t:.1f} s of host work); backward error {be:.2e}"}
    line = {
        "impl": "reference", "metric": "LDLT factor+solve GFLOP/s at bwd err <= 1e-14 (mixed/batched vs FP64 GPU)",
        "value": gf, "unit": "GFLOP/s", "higher_is_better": True, "n_gpus": args.gpus, "steps": steps,
        "warmup": warm, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": t * 1e3, "dtype": "c64", "data": "synthetic", "scaling": "weak", "vs_baseline": None,
        "config": {"workload": f"helmholtz3d_{args.side}^3_c64_nrhs{args.nrhs}", "n": a.n, "nnz_lower": a.nnz,
                   "nrhs": args.nrhs, "ordering": ordering, "model_flops": flops, "analysis_s": t_an,
                   "same_config": True},
        "cpu_baseline": cb,
        "e2e": {"value": gf, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def sweep_cpu_sample(side: int = 48, count: int = 4):
    """The oracle (timing mode, all host threads) on a bounded sample of the
    sweep: the full 48^3 27-point K - w^2 M + i w C matrix at `count`
    frequencies spread over the band, FP64 factor + 8-RHS solve each, on the
    oracle's own structure for the tuned ordering (MetisND here)."""
    from oracle.oracle import OracleSolver, backward_error, oracle_structure, set_parallel
    from rslab_b200 import LdltSymbolic, Ordering, matgen
    from rslab_b200.solver import amd_order, metis_order
    set_parallel(True)
    c4 = matgen.C4System(side, 3)
    om = c4.omegas(64)[np.linspace(0, 63, count).round().astype(int)]
    b = matgen.uniform_rhs(c4.n, 8, 4, complex_=True)
    a0 = c4.matrix(om[0])
    _, st = LdltSymbolic.tuned(a0)
    full = a0.to_scipy_full().tocsc()
    full.sort_indices()
    cp, ri = np.asarray(full.indptr, np.int64), np.asarray(full.indices, np.int64)
    nd = st.ordering == Ordering.METIS_ND
    ex = oracle_structure(a0, metis_order(a0.n, cp, ri) if nd else amd_order(a0.n, cp, ri)[0])
    c, r = ex["sn_ncol"].astype(np.float64), ex["sn_nrow"].astype(np.float64)
    m = r - c + 1.0
    flops = 4.0 * float(np.sum((r * (r + 1) * (2 * r + 1) - (m - 1) * m * (2 * m - 1)) / 6.0 - c))
    t = 0.0
    be = 0.0
    for w in om:
        a = c4.matrix(w)
        t0 = time.perf_counter()
        x = OracleSolver(a, ex, perturb_floor=1e-10).solve_many(b, 8)
        t += time.perf_counter() - t0
        be = max(be, backward_error(a, x, b))
    return {"value": flops * len(om) / t / 1e9, "unit": "GFLOP/s", "cores": os.cpu_count(), "kind": "port",
            "seconds": t,
            "sample": f"FP64 factor + 8-RHS solve of the {side}^3 27-point sweep matrix at {len(om)} frequencies "
                      f"({'MetisND' if nd else 'AMD'}, n={c4.n}, model flops {flops:.3g} each, static pivoting at "
                      f"1e-10); max backward error {be:.2e}; oracle timing mode, {os.cpu_count()} threads"}


def run_sweep(args, ws, rank, local):
    """Same-pattern frequency sweep: A(w) = K - w^2 M + i w C on a 48^3
    27-point grid (n = 110,592), 64 frequencies, 8 right-hand sides, each
    solved to normwise backward error <= 1e-14.  Analysis and the factor
    handle are made once outside the timed region; a step is the whole sweep
    of this rank's frequencies (round-robin over ranks, no exchange): per
    frequency a c32 refactor (captured factor graph replayed on the new
    values) and the mixed solve refined in FP64.  The plain FP64 path is
    timed on `--sweep-fp64-count` frequencies spread over the band."""
    import ctypes as C

    import torch

    from rslab_b200 import CscMatrix, LdltSymbolic, MixedLdltSolver, matgen
    from rslab_b200 import _native as N
    from rslab_b200.sweep import sweep_settings
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    c4 = matgen.C4System(args.sweep_side, 3)
    om_all = c4.omegas(args.sweep_count)
    from rslab_b200.sweep import shard_frequencies
    mine = shard_frequencies(len(om_all), rank, ws)
    nrhs = 8
    b = matgen.uniform_rhs(c4.n, nrhs, 4, complex_=True)
    st = sweep_settings()
    mats = [c4.matrix(om_all[i]) for i in mine]
    # the ordering of the default settings pick (LdltSolver::tuned): the
    # nested-dissection bakeoff adopts MetisND on this 27-point grid
    from rslab_b200 import Ordering
    _, st_t = LdltSymbolic.tuned(mats[0])
    st.ordering = st_t.ordering
    sym = LdltSymbolic.analyze_with(mats[0], st)
    info = sym.info()
    flops = 4.0 * info.flops_model
    vals_d = [torch.from_numpy(np.ascontiguousarray(a.values)).to(dev) for a in mats]
    b_d = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    x_d = torch.empty_like(b_d)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    mixed = MixedLdltSolver.factor_with(mats[0], st, sym=sym)
    stream = torch.cuda.ExternalStream(mixed.stream())
    reuse = not args.no_pivot_reuse
    # static pivot reuse: the factor above searched and recorded its pivot
    # steps; every refactor of the sweep replays them, falling back to a
    # searching refactor for a frequency that does not certify
    if reuse:
        mixed.reuse_pivots(True)
    fallbacks = [0]

    def solve_one(v):
        rc = N.lib.rslab_refactor(mixed._h, C.c_void_p(v.data_ptr()), 1)
        assert rc == 0, N.last_error()
        inf = N.MixedInfoC()
        rc = N.lib.rslab_mixed_solve(mixed._h, C.c_void_p(b_d.data_ptr()), nrhs, args.target,
                                     C.c_void_p(x_d.data_ptr()), 1, C.byref(inf))
        assert rc == 0, N.last_error()
        return inf

    def sweep_step():
        infos = []
        for v in vals_d:
            inf = solve_one(v)
            if reuse and not inf.certified:
                fallbacks[0] += 1
                N.lib.rslab_set_pivot_reuse(mixed._h, 0)
                inf = solve_one(v)
                N.lib.rslab_set_pivot_reuse(mixed._h, 1)
            infos.append((inf.certified, inf.backward_error, inf.ir_iters, inf.gmres_iters))
        return infos

    def timed(fn, strm, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        barrier(ws)
        tot, last = 0.0, None
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(strm)
            last = fn()
            e1.record(strm)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        barrier(ws)
        return tot / steps, last

    clk = ClockSampler(local)
    clk.start()
    ms_sweep, infos = timed(sweep_step, stream, args.steps, args.warmup)
    clocks = clk.stop()
    ms_sweep = allmax(ms_sweep, ws)

    # Plain FP64 factor + solve + FP64 refinement on a spread of frequencies.
    out_fp64 = None
    if not args.no_fp64 and args.sweep_fp64_count > 0:
        pick = np.unique(np.linspace(0, len(mats) - 1, args.sweep_fp64_count).round().astype(int))
        f64 = sym.factor(mats[0], st)
        s64 = torch.cuda.ExternalStream(f64.stream())
        res = []

        def fp64_some():
            for i in pick:
                rc = N.lib.rslab_refactor(f64._h, C.c_void_p(vals_d[i].data_ptr()), 1)
                assert rc == 0, N.last_error()
                rc = N.lib.rslab_solve(f64._h, C.c_void_p(b_d.data_ptr()), nrhs, C.c_void_p(x_d.data_ptr()), 1)
                assert rc == 0, N.last_error()

        ms64, _ = timed(fp64_some, s64, 1, 1)
        ms64 = allmax(ms64 / len(pick), ws)
        for i in pick[-1:]:
            res.append(host_backward_error(mats[i], x_d.cpu().numpy(), b))
        out_fp64 = {"ms_per_frequency": ms64, "frequencies_timed": int(len(pick)),
                    "ms_per_sweep_projected": ms64 * len(om_all) / ws,
                    "gflops": flops / (ms64 * 1e-3) / 1e9,
                    "backward_error_no_ir_last": res[-1] if res else None}

    # End to end through the public API with page-locked host buffers: every
    # frequency's values and the right-hand sides copied in, solutions out.
    def pinned(arr):
        t = torch.empty(arr.shape, dtype={np.complex128: torch.complex128}[arr.dtype.type], pin_memory=True)
        v = t.numpy()
        v[...] = arr
        return t, v
    keep = []
    mats_h = []
    for a in mats:
        t, v = pinned(np.ascontiguousarray(a.values))
        keep.append(t)
        mats_h.append(CscMatrix(a.n, a.col_ptr, a.row_idx, v))
    _pb, b_h = pinned(np.ascontiguousarray(b))
    _px, x_h = pinned(np.zeros_like(np.ascontiguousarray(b)))
    cert_h = 0
    t0 = time.perf_counter()
    for a_h in mats_h:
        mixed.refactor(a_h)
        x_h, inf_h = mixed.solve_to(a_h, b_h, args.target, out=x_h)
        cert_h += int(bool(inf_h.certified))
    e2e_s = allmax(time.perf_counter() - t0, ws)

    cpu_base = sweep_cpu_sample() if (rank == 0 and ws == 1 and not args.no_cpu) else None
    total_flops = flops * len(om_all)
    if rank == 0:
        line = {
            "metric": "LDLT factor+solve GFLOP/s at bwd err <= 1e-14 (mixed/batched vs FP64 GPU)",
            "value": total_flops / (ms_sweep * 1e-3) / 1e9, "unit": "GFLOP/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_sweep, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "c32 factor / f64 refinement", "data": "synthetic",
            "config": {"workload": f"freq_sweep_{args.sweep_side}^3_27pt_c32_nrhs{nrhs}_{len(om_all)}w",
                       "n": c4.n, "nnz_lower": mats[0].nnz, "frequencies": len(om_all), "nrhs": nrhs,
                       "ordering": "MetisND" if st.ordering == Ordering.METIS_ND else "AMD",
                       "static_pivot": 1e-10, "target_backward_error": args.target,
                       "pivot_reuse": reuse, "model_flops_per_frequency": flops,
                       "parallelism": f"frequencies round-robin over {ws}",
                       "l2": "flushed between steps (256 MB write)"},
            "sweep": {"ms_per_frequency": ms_sweep / len(mine),
                      "certified": int(sum(1 for c, *_ in infos if c)), "of": len(infos),
                      "max_backward_error": max(be for _, be, _, _ in infos),
                      "ir_iters_max": max(i for _, _, i, _ in infos),
                      "searching_refactors_after_failure": fallbacks[0],
                      "gmres_iters_max": max(g for *_, g in infos)},
            "fp64_gpu": out_fp64,
            "e2e": {"value": flops * len(mine) / e2e_s / 1e9 * ws, "unit": "GFLOP/s", "seconds_per_step": e2e_s,
                    "h2d_bytes_per_step": int(sum(a.values.nbytes for a in mats) + len(mats) * b.nbytes),
                    "d2h_bytes_per_step": int(len(mats) * b.nbytes), "certified": cert_h,
                    "host_buffers": "page-locked (torch pin_memory) numpy views"},
            "clocks": clocks,
            "cpu_baseline": cpu_base,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_tiers(args, ws, rank, local):
    """Learned precision tier on the held-out matrix: 27-point complex
    Helmholtz K - k2 (1 + 0.02 i) I on an 80^3 grid (n = 512,000), k2 =
    0.15 lambda_max, 4 right-hand sides, backward error <= 1e-14.  The tier
    network picks the factor's precision from the matrix's features (outside
    the timed region, with the analysis); a step is refactor + refined solve
    in that tier, plus the FP64 refactor + solve if it did not certify.  The
    plain FP64 tier is timed on the same matrix for the ratio."""
    import ctypes as C

    import torch

    from rslab_b200 import CscMatrix, LdltSymbolic, MixedLdltSolver, matgen
    from rslab_b200 import _native as N
    from rslab_b200.tiers import TIERS, TierModel, tier_features, tier_settings
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    a = matgen.c5_heldout(args.tiers_side, 6)
    nrhs = 4
    b = matgen.uniform_rhs(a.n, nrhs, 6, complex_=True)
    st = tier_settings()
    t0 = time.perf_counter()
    sym = LdltSymbolic.analyze_with(a, st)
    t_an = time.perf_counter() - t0
    info = sym.info()
    flops = 4.0 * info.flops_model
    model = TierModel.load(args.tier_model) if args.tier_model else TierModel.load()
    feats = tier_features(a, sym)
    probs = model.predict_proba(feats)[0]
    tier = int(np.argmax(probs))
    vals_d = torch.from_numpy(np.ascontiguousarray(a.values)).to(dev)
    b_d = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    x_d = torch.empty_like(b_d)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    h = MixedLdltSolver.factor_tier(a, tier, st, sym)
    h64 = MixedLdltSolver.factor_tier(a, N.TIER_FP64, st, sym) if tier != N.TIER_FP64 else h

    def one(handle):
        rc = N.lib.rslab_refactor(handle._h, C.c_void_p(vals_d.data_ptr()), 1)
        assert rc == 0, N.last_error()
        inf = N.MixedInfoC()
        rc = N.lib.rslab_mixed_solve(handle._h, C.c_void_p(b_d.data_ptr()), nrhs, args.target,
                                     C.c_void_p(x_d.data_ptr()), 1, C.byref(inf))
        assert rc == 0, N.last_error()
        return inf

    def learned_step():
        inf = one(h)
        if not inf.certified and h is not h64:
            return one(h64), True
        return inf, False

    def timed(fn, strm, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        barrier(ws)
        tot, last = 0.0, None
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(strm)
            last = fn()
            e1.record(strm)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        barrier(ws)
        return tot / steps, last

    clk = ClockSampler(local)
    clk.start()
    ms, (minfo, fell) = timed(learned_step, torch.cuda.ExternalStream(h.stream()), args.steps, args.warmup)
    clocks = clk.stop()
    ms = allmax(ms, ws)
    out64 = None
    if not args.no_fp64:
        ms64, inf64 = timed(lambda: one(h64), torch.cuda.ExternalStream(h64.stream()), max(1, args.steps // 2), 1)
        ms64 = allmax(ms64, ws)
        out64 = {"ms_per_step": ms64, "gflops": flops / (ms64 * 1e-3) / 1e9, "certified": bool(inf64.certified),
                 "backward_error": inf64.backward_error, "ir_iters": inf64.ir_iters}
    # end to end: host values and right-hand sides in page-locked memory
    def pinned(arr):
        t = torch.empty(arr.shape, dtype=torch.complex128, pin_memory=True)
        v = t.numpy()
        v[...] = arr
        return t, v
    _pa, vals_h = pinned(np.ascontiguousarray(a.values))
    _pb, b_h = pinned(np.ascontiguousarray(b))
    _px, x_h = pinned(np.zeros_like(np.ascontiguousarray(b)))
    a_h = CscMatrix(a.n, a.col_ptr, a.row_idx, vals_h)
    te = []
    for it in range(2):
        t0 = time.perf_counter()
        h.refactor(a_h)
        x_h, inf_h = h.solve_to(a_h, b_h, args.target, out=x_h)
        if not inf_h.certified and h is not h64:
            h64.refactor(a_h)
            x_h, inf_h = h64.solve_to(a_h, b_h, args.target, out=x_h)
        if it:
            te.append(time.perf_counter() - t0)
    e2e_s = allmax(float(np.mean(te)), ws)
    if rank == 0:
        line = {
            "metric": "LDLT factor+solve GFLOP/s at bwd err <= 1e-14 (mixed/batched vs FP64 GPU)",
            "value": flops / (ms * 1e-3) / 1e9 * ws, "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": f"{TIERS[tier]} factor / f64 refinement", "data": "synthetic",
            "config": {"workload": f"learned_tier_helmholtz27_{args.tiers_side}^3_c64_nrhs{nrhs}", "n": a.n,
                       "nnz_lower": a.nnz, "nrhs": nrhs, "ordering": "AMD", "static_pivot": 1e-10,
                       "target_backward_error": args.target, "model_flops": flops,
                       "factor_nnz_panels": info.panel_elems, "analysis_s": t_an,
                       "parallelism": f"replicas{ws}", "l2": "flushed between steps (256 MB write)"},
            "tier": {"chosen": TIERS[tier], "probabilities": [float(p) for p in probs],
                     "features": [float(f) for f in feats], "fell_back_to_fp64": bool(fell),
                     "certified": bool(minfo.certified), "backward_error": minfo.backward_error,
                     "ir_iters": minfo.ir_iters, "gmres_iters": minfo.gmres_iters},
            "fp64_gpu": out64,
            "e2e": {"value": flops / e2e_s / 1e9 * ws, "unit": "GFLOP/s", "seconds_per_step": e2e_s,
                    "h2d_bytes_per_step": int(a.values.nbytes + b.nbytes), "d2h_bytes_per_step": int(b.nbytes),
                    "certified": bool(inf_h.certified), "host_buffers": "page-locked (torch pin_memory) numpy views"},
            "clocks": clocks,
            "cpu_baseline": {"value": None, "unit": "GFLOP/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"not timed: {flops:.3g} model flops per factor is hours of host work"},
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_batch(args, ws, rank, local):
    """Batched uneven systems: 512 real symmetric indefinite 3D 7-point
    shifted Laplacians, cube sides U{12..40} (seed 2), shift 0.1 lambda_max,
    4 right-hand sides each (U[-1, 1), seed 2), every (system, column)
    certified at normwise backward error <= 1e-14.  One analysis handle holds
    every system (one launch per assembly-tree level and block index covers
    that level of every system); a step is the f32 refactor with tensor-core
    descendant updates + the FP64 refinement ladder.  The plain FP64 factor +
    solve of the same batch is timed for the ratio.  Multi-GPU: the systems are
    split over ranks by weight (n^2), no data exchange."""
    import ctypes as C

    import torch

    from rslab_b200 import CscMatrix, MixedLdltSolver, SolverSettings, matgen
    from rslab_b200 import _native as N
    from rslab_b200.batch import BatchSystems, analyze_batch, mixed_batch_result, shard_by_weight
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sides = matgen.c3_sides(args.batch_count, 2)
    mine = shard_by_weight([float(s) ** 6 for s in sides], ws)[rank]
    mats = [matgen.c3_matrix(sides[i]) for i in mine]
    batch = BatchSystems(mats)
    nrhs = 4
    t0 = time.perf_counter()
    sym = analyze_batch(batch)
    t_an = time.perf_counter() - t0
    info = sym.info()
    flops = info.flops_model
    a = batch.as_matrix()
    b = matgen.uniform_rhs(batch.total_n, nrhs, 2)
    st = SolverSettings()
    vals_d = torch.from_numpy(np.ascontiguousarray(a.values)).to(dev)
    b_d = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    x_d = torch.empty_like(b_d)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def timed(fn, strm, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        barrier(ws)
        tot, last = 0.0, None
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(strm)
            last = fn()
            e1.record(strm)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        barrier(ws)
        return tot / steps, last

    # the engine and launch schedule of this batch, measured on it before the
    # timed region (the analysis-time block width stays at its default)
    from rslab_b200.autotune import candidates, tune_mixed
    tuned = tune_mixed(a, b, args.target, sym=sym, cands=candidates(engines=("tensor", "fma", "fp64")), reps=2,
                       warmup=1)
    st = tuned.settings(SolverSettings())
    if tuned.fp64:
        mixed = MixedLdltSolver.factor_tier(a, N.TIER_FP64, st, sym=sym)
    else:
        mixed = MixedLdltSolver.factor_with(a, st, sym=sym)

    def mixed_step():
        rc = N.lib.rslab_refactor(mixed._h, C.c_void_p(vals_d.data_ptr()), 1)
        assert rc == 0, N.last_error()
        inf = N.MixedInfoC()
        rc = N.lib.rslab_mixed_solve(mixed._h, C.c_void_p(b_d.data_ptr()), nrhs, args.target,
                                     C.c_void_p(x_d.data_ptr()), 1, C.byref(inf))
        assert rc == 0, N.last_error()
        return inf

    clk = ClockSampler(local)
    clk.start()
    ms, minfo = timed(mixed_step, torch.cuda.ExternalStream(mixed.stream()), args.steps, args.warmup)
    clocks = clk.stop()
    ms = allmax(ms, ws)
    from rslab_b200.solver import MixedInfo
    res = mixed_batch_result(mixed, batch.count, nrhs, args.target,
                             MixedInfo(int(minfo.ir_iters), int(minfo.gmres_iters), float(minfo.backward_error),
                                       bool(minfo.certified)))
    # end to end through the public API with page-locked host buffers
    def pinned(arr):
        t = torch.empty(arr.shape, dtype=torch.float64, pin_memory=True)
        v = t.numpy()
        v[...] = arr
        return t, v
    _pa, vals_h = pinned(np.ascontiguousarray(a.values))
    _pb, b_h = pinned(np.ascontiguousarray(b))
    _px, x_h = pinned(np.zeros_like(np.ascontiguousarray(b)))
    a_h = CscMatrix(a.n, a.col_ptr, a.row_idx, vals_h)
    te = []
    for it in range(2):
        t1 = time.perf_counter()
        mixed.refactor(a_h)
        x_h, inf_h = mixed.solve_to(a_h, b_h, args.target, out=x_h)
        if it:
            te.append(time.perf_counter() - t1)
    e2e_s = allmax(float(np.mean(te)), ws)
    del mixed
    torch.cuda.synchronize()
    out64 = None
    if not args.no_fp64:
        f64 = sym.factor(a, SolverSettings())

        def fp64_step():
            rc = N.lib.rslab_refactor(f64._h, C.c_void_p(vals_d.data_ptr()), 1)
            assert rc == 0, N.last_error()
            rc = N.lib.rslab_solve(f64._h, C.c_void_p(b_d.data_ptr()), nrhs, C.c_void_p(x_d.data_ptr()), 1)
            assert rc == 0, N.last_error()

        ms64, _ = timed(fp64_step, torch.cuda.ExternalStream(f64.stream()), max(1, args.steps // 2), 1)
        ms64 = allmax(ms64, ws)
        out64 = {"ms_per_step": ms64, "gflops": flops / (ms64 * 1e-3) / 1e9 * ws,
                 "backward_error_no_ir": host_backward_error(a, x_d.cpu().numpy(), b)}
        del f64
    if rank == 0:
        line = {
            "metric": "LDLT factor+solve GFLOP/s at bwd err <= 1e-14 (mixed/batched vs FP64 GPU)",
            "value": flops / (ms * 1e-3) / 1e9 * ws, "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None,
            "dtype": ("f64 factor / f64 refinement" if tuned.fp64 else "f32 factor / f64 refinement"),
            "data": "synthetic",
            "config": {"workload": f"batch{args.batch_count}_laplacian3d_sides12-40_f64_nrhs{nrhs}",
                       "systems": batch.count, "total_n": batch.total_n, "nnz_lower": a.nnz, "nrhs": nrhs,
                       "ordering": "AMD", "target_backward_error": args.target, "model_flops": flops,
                       "supernodes": int(info.nsuper), "levels": int(info.nlevels),
                       "factor_launches": int(info.n_factor_launches), "analysis_s": t_an,
                       "parallelism": f"systems split over {ws} rank(s) by weight",
                       "l2": "flushed between steps (256 MB write)"},
            "autotune": {"chosen": {"schur_engine": tuned.chosen[0], "overlap": tuned.chosen[1],
                                    "panel_nb": tuned.chosen[2]},
                         "ms_per_candidate": tuned.table(), "tuning_s": tuned.tuning_seconds,
                         "note": "measured before the timed region: refactor + solve with host buffers"},
            "mixed": {"certified_units": int(res.certified.sum()), "units": int(res.certified.size),
                      "max_backward_error": float(res.backward_error.max()), "ir_iters": int(minfo.ir_iters),
                      "gmres_iters": int(minfo.gmres_iters)},
            "fp64_gpu": out64,
            "e2e": {"value": flops / e2e_s / 1e9 * ws, "unit": "GFLOP/s", "seconds_per_step": e2e_s,
                    "h2d_bytes_per_step": int(a.values.nbytes + b.nbytes), "d2h_bytes_per_step": int(b.nbytes),
                    "certified": bool(inf_h.certified), "host_buffers": "page-locked (torch pin_memory) numpy views"},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    ws, rank, local = dist_init(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    if args.workload == "sweep":
        run_sweep(args, ws, rank, local)
        return
    if args.workload == "tiers":
        run_tiers(args, ws, rank, local)
        return
    if args.workload == "batch":
        run_batch(args, ws, rank, local)
        return
    import torch

    from rslab_b200 import CscMatrix, LdltSymbolic, MixedLdltSolver, SolverSettings, matgen
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    a = matgen.c2_matrix(args.side)
    n, nrhs = a.n, args.nrhs
    from rslab_b200 import Ordering
    t_an = time.perf_counter()
    if args.ordering == "metis":
        sym = LdltSymbolic.analyze_with(a, SolverSettings().with_ordering(Ordering.METIS_ND))
        ordering = Ordering.METIS_ND
    elif args.ordering == "amd":
        sym = LdltSymbolic.analyze(a)
        ordering = Ordering.AMD
    else:
        sym, st_tuned = LdltSymbolic.tuned(a)
        ordering = st_tuned.ordering
    t_an = time.perf_counter() - t_an
    info = sym.info()
    ex = sym.export()
    sn_c = ex["sn_ncol"].astype(np.float64)
    sn_r = ex["sn_nrow"].astype(np.float64)
    # algorithmic bytes of one solve of nrhs columns (forward + backward panel
    # reads, right-hand sides in / out twice, D), in the factor's field
    solve_entries = float(np.sum(sn_c * (sn_c + 1) / 2 + (sn_r - sn_c) * sn_c))
    flops = 4.0 * info.flops_model  # complex: 4 real flops per complex multiply-add pair
    b = matgen.uniform_rhs(n, nrhs, 1, complex_=True)
    vals_d = torch.from_numpy(np.ascontiguousarray(a.values)).to(dev)
    b_d = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    x_d = torch.empty_like(b_d)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    st = SolverSettings(method=args.method)
    # The tier network picks the factor's precision tier from the matrix's
    # features, outside the timed region like the analysis.
    from rslab_b200.tiers import TIERS, TierModel, tier_features
    tier_feats = tier_features(a, sym)
    tier_probs = TierModel.load().predict_proba(tier_feats)[0]
    tier = int(np.argmax(tier_probs))
    mixed = MixedLdltSolver.factor_tier(a, tier, st, sym=sym)
    stream = torch.cuda.ExternalStream(mixed.stream())
    import ctypes as C

    from rslab_b200 import _native as N

    def mixed_step():
        rc = N.lib.rslab_refactor(mixed._h, C.c_void_p(vals_d.data_ptr()), 1)
        assert rc == 0, N.last_error()
        inf = N.MixedInfoC()
        rc = N.lib.rslab_mixed_solve(mixed._h, C.c_void_p(b_d.data_ptr()), nrhs, args.target,
                                     C.c_void_p(x_d.data_ptr()), 1, C.byref(inf))
        assert rc == 0, N.last_error()
        return inf

    if args.profile_step:
        mixed_step()
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStart()
        mixed_step()
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
        return

    def timed(fn, steps, warm):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        barrier(ws)
        tot = 0.0
        last = None
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            last = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        barrier(ws)
        return tot / steps, last

    clk = ClockSampler(local)
    clk.start()
    ms_mixed, minfo = timed(mixed_step, args.steps, args.warmup)
    clocks = clk.stop()
    ms_mixed = allmax(ms_mixed, ws)
    x_mixed = x_d.cpu().numpy()  # the last timed step's solution

    out_fp64 = None
    if not args.no_fp64:
        f64 = sym.factor(a, st)
        s64 = f64.stream()
        stream64 = torch.cuda.ExternalStream(s64)

        def fp64_step():
            rc = N.lib.rslab_refactor(f64._h, C.c_void_p(vals_d.data_ptr()), 1)
            assert rc == 0, N.last_error()
            rc = N.lib.rslab_solve(f64._h, C.c_void_p(b_d.data_ptr()), nrhs, C.c_void_p(x_d.data_ptr()), 1)
            assert rc == 0, N.last_error()

        stream_save = stream
        stream = stream64
        ms64, _ = timed(fp64_step, max(1, args.steps // 2), 1)
        stream = stream_save
        ms64 = allmax(ms64, ws)
        x64 = x_d.cpu().numpy()
        be64 = host_backward_error(a, x64, b)
        fi = N.FactorInfo()
        N.lib.rslab_factor_info(f64._h, C.byref(fi))
        out_fp64 = {"ms_per_step": ms64, "factor_ms": fi.factor_ms, "solve_ms": fi.solve_ms,
                    "gflops": flops / (ms64 * 1e-3) / 1e9, "backward_error_no_ir": be64,
                    "mixed_forward_error_vs_fp64": float(np.abs(x_mixed - x64).max() / np.abs(x64).max())}

    # Per-kernel-class profile of one eager refactor (events after every launch).
    from rslab_b200.solver import factor_profile, solve_profile
    prof_mixed = factor_profile(mixed._h)
    sprof_mixed = solve_profile(mixed._h, nrhs)
    prof_f64 = factor_profile(f64._h) if out_fp64 is not None else None
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak_tf = float(peaks.get("bf16_tflops", 1590.0))
    # Dominant kernel: the tensor-core descendant update, k_cmod_mm (3xTF32
    # GEMM tiles in the updater's row space).  Time from the per-launch trace
    # of the eager refactor above; algorithmic flops = the cmod model flops
    # (multiply + add of every (r >= c) update entry).  The assembly and the
    # operand split are reported beside it.
    from rslab_b200.solver import profile_trace
    factor_profile(mixed._h)
    tr = profile_trace(mixed._h)
    mm_ms = sum(ms for k, _, ms in tr if k == "cmod_mm")
    mm_n = sum(1 for k, _, _ in tr if k == "cmod_mm")
    asm_ms = sum(ms for k, _, ms in tr if k == "cmod_asm")
    split_ms = sum(ms for k, _, ms in tr if k in ("split_r", "split_c"))
    cm = prof_mixed["cmod"]
    ach = cm["flops"] / (mm_ms * 1e-3) / 1e12 if mm_ms > 0 else 0.0
    roofline = {"bound": "tensor", "kernel": "k_cmod_mm (c32, tcgen05 kind::tf32, 3xTF32 split, TMA-staged)",
                "achieved": ach, "peak": peak_tf, "unit": "TFLOP/s", "frac": ach / peak_tf,
                "traffic": None,
                "traffic_note": "not measured by this run: dram bytes per launch come from an ncu capture "
                                "of the kernel (profiles/)",
                "peak_source": ("MEASURED_PEAKS.json bf16_tflops (burst), of measured" if "bf16_tflops" in peaks
                                else "fallback 1590 TFLOP/s"),
                "launches": mm_n, "avg_launch_ms": mm_ms / max(mm_n, 1),
                "assembly_ms": asm_ms, "split_ms": split_ms,
                "tf32_pipe_frac": 3.0 * ach / (peak_tf / 2.0),
                "note": "achieved = algorithmic flops / k_cmod_mm time; the 3xTF32 split issues 3 tf32 products per "
                        "flop on a pipe with half the bf16 rate, tf32_pipe_frac = 3 x achieved / (peak / 2)"}
    if args.method != "left_looking":
        # no descendant-update tiles in this schedule: its c32 contribution-block
        # products run on the CUDA cores (k_front_cb), timed in the profile
        roofline = {"bound": None, "kernel": None,
                    "note": "multifrontal schedule: no k_cmod_mm launches; the tensor-core roofline is reported "
                            "for the default left-looking schedule"}

    # End-to-end through the public API with host buffers: the step's inputs
    # (matrix values, right-hand sides) and its result in page-locked host
    # memory, copied host->device and back inside the timed region.
    def pinned(arr):
        t = torch.empty(arr.shape, dtype={np.complex128: torch.complex128, np.float64: torch.float64}[arr.dtype.type],
                        pin_memory=True)
        v = t.numpy()
        v[...] = arr
        return t, v
    _pa, vals_h = pinned(np.ascontiguousarray(a.values))
    _pb, b_h = pinned(np.ascontiguousarray(b))
    _px, x_h = pinned(np.zeros_like(np.ascontiguousarray(b)))
    a_h = CscMatrix(a.n, a.col_ptr, a.row_idx, vals_h)
    t_e2e = []
    for it in range(1 + args.steps):
        t0 = time.perf_counter()
        mixed.refactor(a_h)
        x_h, inf_h = mixed.solve_to(a_h, b_h, args.target, out=x_h)
        dt = time.perf_counter() - t0
        if it > 0:
            t_e2e.append(dt)
    e2e_s = allmax(float(np.mean(t_e2e)), ws)
    fi = N.FactorInfo()
    N.lib.rslab_factor_info(mixed._h, C.byref(fi))
    gflops = flops / (ms_mixed * 1e-3) / 1e9 * ws
    hbm = float(peaks.get("hbm_gbs", 6650.0))

    def solve_bw(prof, esize):
        byt = 2.0 * solve_entries * esize + 4.0 * n * nrhs * esize + 2.0 * n * esize
        ms = prof["total"]["ms"]
        return {"bytes": byt, "ms": ms, "gbs": byt / (ms * 1e-3) / 1e9 if ms > 0 else None,
                "frac_of_hbm": (byt / (ms * 1e-3) / 1e9 / hbm) if ms > 0 else None,
                "hbm_peak_gbs": hbm}
    solve_gbs = {"mixed_c32": solve_bw(sprof_mixed, 8)}
    if prof_f64 is not None:
        solve_gbs["fp64_c64"] = solve_bw(solve_profile(f64._h, nrhs), 16)
    solve_gbs["note"] = ("algorithmic bytes 2 sum_s(c(c+1)/2 + (r-c)c) + 4 n nrhs + 2 n scalars per solve, "
                         "eager solve with per-launch events (no graph), of measured hbm_gbs")
    cpu_base = cpu_sample(args) if (rank == 0 and ws == 1 and not args.no_cpu) else None
    if cpu_base is not None:
        # forward errors of the GPU solutions against the oracle's FP64 solution
        # of the same system (same matrix, ordering output and right-hand sides)
        xo = np.asarray(cpu_sample.solution).reshape(x_mixed.shape)
        fe = lambda x: float(np.abs(x - xo).max() / np.abs(xo).max())
        cpu_base["mixed_forward_error_vs_oracle"] = fe(x_mixed)
        if out_fp64 is not None:
            cpu_base["fp64_forward_error_vs_oracle"] = fe(x64)
    if rank == 0:
        line = {
            "metric": "LDLT factor+solve GFLOP/s at bwd err <= 1e-14 (mixed/batched vs FP64 GPU)",
            "value": gflops, "unit": "GFLOP/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"{TIERS[tier]} factor / f64 refinement", "data": "synthetic",
            "config": {"workload": f"helmholtz3d_{args.side}^3_c64_nrhs{nrhs}", "n": n, "nnz_lower": a.nnz,
                       "nrhs": nrhs, "ordering": "MetisND" if ordering == Ordering.METIS_ND else "AMD",
                       "ordering_pick": args.ordering, "analysis_s": t_an,
                       **({"method": args.method} if args.method != "left_looking" else {}),
                       "target_backward_error": args.target,
                       "model_flops": flops, "factor_nnz_panels": info.panel_elems,
                       "parallelism": f"replicas{ws}", "l2": "flushed between steps (256 MB write)"},
            "tier": {"chosen": TIERS[tier], "probabilities": [float(p) for p in tier_probs],
                     "features": [float(f) for f in tier_feats],
                     "note": "picked by the tier network (rslab_tier_mlp_forward) before the timed region"},
            "mixed": {"certified": bool(minfo.certified), "backward_error": minfo.backward_error,
                      "ir_iters": minfo.ir_iters, "gmres_iters": minfo.gmres_iters,
                      "last_factor_ms": fi.factor_ms},
            "fp64_gpu": out_fp64,
            "e2e": {"value": flops / e2e_s / 1e9 * ws, "unit": "GFLOP/s", "seconds_per_step": e2e_s,
                    "h2d_bytes_per_step": int(a.values.nbytes + b.nbytes),
                    "d2h_bytes_per_step": int(b.nbytes), "certified": bool(inf_h.certified),
                    "host_buffers": "page-locked (torch pin_memory) numpy views"},
            "clocks": clocks,
            "roofline": roofline,
            "profile_mixed": prof_mixed,
            "profile_fp64": prof_f64,
            "solve_profile_mixed": sprof_mixed,
            "solve_gbs": solve_gbs,
            "cpu_baseline": cpu_base,
            "gpu_launches": launches_per_step(prof_mixed, sprof_mixed, minfo),
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
