"""Learned precision tier: a small network picks, per matrix, the precision
the refined factor is computed in (FP64 / FP32 / TF32x3), trained on labels
the solver makes itself by running every tier and keeping the cheapest one
that certifies; the FP64 tier is the fallback and the arbiter (a matrix whose
chosen tier does not certify is refactored in FP64).

Tiers (include/rslab_b200.h RSLAB_TIER_*), all refined in FP64 against the
original matrix by the MixedLdltSolver ladder (src/numeric/mixed.rs:140-221):
  0 fp64    the factor in the matrix's own field
  1 fp32    f32 / c32 factor, CUDA-core descendant updates
  2 tf32x3  f32 / c32 factor, 3xTF32 tensor-core descendant updates

The network (8 -> 64 -> 64 -> 3) is trained and evaluated by the library's
kernels (rslab_tier_mlp_train / _forward); this module computes features,
standardises them and moves data.  Command line (GPU):
  python -m rslab_b200.tiers label --count 2000 --out corpus.npz
  python -m rslab_b200.tiers train --corpus corpus.npz --out model.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import math
import time
from pathlib import Path
from typing import Optional

import numpy as np

from . import _native as N
from .solver import (CscMatrix, InvalidInput, LdltSymbolic, MixedLdltSolver, NumericallyRankDeficient, RslabError,
                     SolverSettings)

TIERS = ("fp64", "fp32", "tf32x3")
NFEAT = 8
FEATURES = ("log10_n", "log10_model_flops", "log10_fill_per_row", "complex", "log10_1p_median_offdiag_ratio",
            "frac_not_diag_dominant", "frac_negative_diag", "log10_norm_over_min_diag")
DATA = Path(__file__).resolve().parent / "data"


def tier_settings() -> SolverSettings:
    """Static pivoting at 1e-10 (scaled matrix), the same for every tier:
    refinement certifies the result."""
    return SolverSettings.preconditioner(1e-10)


def tier_features(a: CscMatrix, sym: LdltSymbolic) -> np.ndarray:
    """The 8 features of one matrix: size and work (n, model flops of the
    factor, fill per row), field, and local norm / growth indicators from one
    pass over the stored lower triangle (row sums of |off-diagonal| against
    |a_ii|, sign of the diagonal, ||A||_inf over the smallest |a_ii|)."""
    n = a.n
    info = sym.info()
    v = np.asarray(a.values)
    cp = np.asarray(a.col_ptr, np.int64)
    ri = np.asarray(a.row_idx, np.int64)
    cplx = np.iscomplexobj(v)
    col = np.repeat(np.arange(n, dtype=np.int64), np.diff(cp))
    dmask = ri == col
    d = np.zeros(n, v.dtype)
    d[col[dmask]] = v[dmask]
    off = ~dmask
    av = np.abs(v[off])
    rowsum = np.bincount(ri[off], av, n) + np.bincount(col[off], av, n)
    ad = np.abs(d)
    tiny = 1e-300
    ratio = rowsum / np.maximum(ad, tiny)
    anorm = float(np.max(ad + rowsum)) if n else 0.0
    f = np.array([
        math.log10(max(n, 1)),
        math.log10(max(info.flops_model * (4.0 if cplx else 1.0), 1.0)),
        math.log10(max(info.panel_elems / max(n, 1), 1.0)),
        1.0 if cplx else 0.0,
        math.log10(1.0 + float(np.median(ratio))) if n else 0.0,
        float(np.mean(ad <= rowsum)) if n else 0.0,
        float(np.mean(np.real(d) < 0)) if n else 0.0,
        min(20.0, max(0.0, math.log10(max(anorm, tiny) / max(float(ad.min()) if n else 1.0, tiny)))),
    ])
    return f


# --- running the tiers --------------------------------------------------------

def run_tier(a: CscMatrix, b: np.ndarray, tier: int, sym: LdltSymbolic, target: float = 1e-14,
             settings: Optional[SolverSettings] = None, reps: int = 1):
    """Factor handle of `tier` (outside the timing), one warm refactor +
    solve, then the best of `reps` timed refactor + solve_to(target) (host
    buffers in and out, as a caller sees it).  Returns (seconds, certified,
    backward_error, x); a factor that fails (rank deficient) counts as not
    certified with the time spent until the failure."""
    st = settings or tier_settings()
    t0 = time.perf_counter()
    try:
        s = MixedLdltSolver.factor_tier(a, tier, st, sym)
        x, info = s.solve_to(a, b, target)
    except NumericallyRankDeficient:
        return time.perf_counter() - t0, False, math.inf, None
    best = math.inf
    for _ in range(max(1, reps)):
        t0 = time.perf_counter()
        s.refactor(a)
        x, info = s.solve_to(a, b, target)
        best = min(best, time.perf_counter() - t0)
    del s
    return best, bool(info.certified), float(info.backward_error), x


def cheapest_certified(times: np.ndarray, certified: np.ndarray) -> int:
    """The label: the fastest tier that certified (FP64 when none did)."""
    t = np.where(certified, times, np.inf)
    return int(np.argmin(t)) if np.isfinite(t).any() else 0


def effective_cost(times: np.ndarray, certified: np.ndarray, tier: int) -> float:
    """What choosing `tier` costs: its time, plus the FP64 refactor when it
    does not certify."""
    return float(times[tier] + (0.0 if certified[tier] or tier == 0 else times[0]))


def sample_weight(times: np.ndarray, certified: np.ndarray) -> float:
    """Training weight: the seconds a wrong choice can cost on this matrix
    (worst minus best effective cost) + 1e-4 s, so that the weighted
    cross-entropy follows the total time of the policy (matrices whose tier
    hardly matters carry little weight)."""
    eff = np.array([effective_cost(times, certified, k) for k in range(len(TIERS))])
    return float(eff.max() - eff.min() + 1e-4)


def label_corpus(count: int = 2000, seed: int = 5, nrhs: int = 4, target: float = 1e-14, reps: int = 1,
                 log_every: int = 100, max_seconds: Optional[float] = None) -> dict:
    """Run every tier on every corpus matrix (matgen.c5_corpus) and record
    features, times, certificates and labels.  With `max_seconds`, stop after
    the first matrix that ends past that budget (the corpus is then its
    first len(labels) matrices)."""
    from . import matgen
    feats, times, cert, berr, fams, ns = [], [], [], [], [], []
    st = tier_settings()
    t_start = time.perf_counter()
    for i, (fam, a) in enumerate(matgen.c5_corpus(count, seed)):
        sym = LdltSymbolic.analyze_with(a, st)
        b = matgen.uniform_rhs(a.n, nrhs, seed * 7919 + i, complex_=np.iscomplexobj(a.values))
        row_t, row_c, row_b = [], [], []
        for k in range(len(TIERS)):
            t, c, be, _ = run_tier(a, b, k, sym, target, st, reps)
            row_t.append(t)
            row_c.append(c)
            row_b.append(be)
        feats.append(tier_features(a, sym))
        times.append(row_t)
        cert.append(row_c)
        berr.append(row_b)
        fams.append(matgen.C5_FAMILIES.index(fam))
        ns.append(a.n)
        del sym
        if log_every and (i + 1) % log_every == 0:
            print(f"labelled {i + 1}/{count} in {time.perf_counter() - t_start:.1f} s", flush=True)
        if max_seconds is not None and time.perf_counter() - t_start > max_seconds:
            print(f"time budget reached after {i + 1} matrices", flush=True)
            break
    times = np.array(times)
    cert = np.array(cert, bool)
    labels = np.array([cheapest_certified(t, c) for t, c in zip(times, cert)], np.int32)
    return {"features": np.array(feats), "times": times, "certified": cert, "backward_error": np.array(berr),
            "labels": labels, "family": np.array(fams, np.int32), "n": np.array(ns, np.int64),
            "nrhs": nrhs, "target": target, "seed": seed}


# --- the network ------------------------------------------------------------

def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class TierModel:
    """Parameters (RSLAB_TIER_MLP_PARAMS floats) + feature standardisation."""

    def __init__(self, params: np.ndarray, mu: np.ndarray, sd: np.ndarray):
        self.params = np.ascontiguousarray(params, np.float32)
        self.mu = np.asarray(mu, np.float64)
        self.sd = np.asarray(sd, np.float64)
        if self.params.shape != (N.TIER_MLP_PARAMS,):
            raise InvalidInput(f"tier network needs {N.TIER_MLP_PARAMS} parameters")

    @classmethod
    def init(cls, seed: int = 7, mu=None, sd=None) -> "TierModel":
        """He-uniform weights (bound sqrt(6 / fan_in)) from Rng(seed), zero biases."""
        from .matgen import Rng
        rng = Rng(seed)
        parts = []
        for fan_in, fan_out in ((NFEAT, 64), (64, 64), (64, len(TIERS))):
            bound = math.sqrt(6.0 / fan_in)
            parts.append((2.0 * rng.units(fan_in * fan_out) - 1.0) * bound)
            parts.append(np.zeros(fan_out))
        p = np.concatenate(parts)
        return cls(p, np.zeros(NFEAT) if mu is None else mu, np.ones(NFEAT) if sd is None else sd)

    def standardise(self, x: np.ndarray) -> np.ndarray:
        return np.ascontiguousarray((np.asarray(x, np.float64) - self.mu) / self.sd, np.float32)

    def fit(self, x: np.ndarray, y: np.ndarray, w: Optional[np.ndarray] = None, epochs: int = 200,
            lr: float = 3e-3) -> np.ndarray:
        """Set the standardisation from x, then train on the GPU; returns the
        loss before every epoch."""
        x = np.asarray(x, np.float64)
        self.mu = x.mean(axis=0)
        self.sd = np.maximum(x.std(axis=0), 1e-6)
        xs = self.standardise(x)
        yv = np.ascontiguousarray(y, np.int32)
        wv = None if w is None else np.ascontiguousarray(w, np.float32)
        curve = np.zeros(max(epochs, 1), np.float32)
        rc = N.lib.rslab_tier_mlp_train(_fp(self.params), _fp(xs), yv.ctypes.data_as(C.POINTER(C.c_int32)),
                                        None if wv is None else _fp(wv), len(yv), int(epochs), float(lr),
                                        _fp(curve), 0)
        if rc != 0:
            raise RslabError(N.last_error())
        return curve[:epochs]

    def predict_proba(self, x: np.ndarray) -> np.ndarray:
        xs = self.standardise(np.atleast_2d(x))
        probs = np.zeros((xs.shape[0], len(TIERS)), np.float32)
        rc = N.lib.rslab_tier_mlp_forward(_fp(self.params), _fp(xs), xs.shape[0], _fp(probs), 0)
        if rc != 0:
            raise RslabError(N.last_error())
        return probs

    def predict(self, x: np.ndarray) -> np.ndarray:
        return np.argmax(self.predict_proba(x), axis=1).astype(np.int32)

    def save(self, path) -> None:
        np.savez(path, params=self.params, mu=self.mu, sd=self.sd)

    @classmethod
    def load(cls, path=None) -> "TierModel":
        z = np.load(path or DATA / "tier_mlp.npz")
        return cls(z["params"], z["mu"], z["sd"])


def split(count: int, holdout_every: int = 5):
    """Deterministic train / held-out split: every 5th matrix is held out."""
    idx = np.arange(count)
    test = idx % holdout_every == holdout_every - 1
    return idx[~test], idx[test]


def policy_costs(pred: np.ndarray, times: np.ndarray, certified: np.ndarray) -> dict:
    """Total effective cost of the network's choices and of the fixed
    policies on the same matrices (seconds)."""
    m = len(pred)
    eff = np.array([[effective_cost(times[i], certified[i], k) for k in range(len(TIERS))] for i in range(m)])
    return {"network": float(eff[np.arange(m), pred].sum()), "always_fp64": float(eff[:, 0].sum()),
            "always_fp32": float(eff[:, 1].sum()), "always_tf32x3": float(eff[:, 2].sum()),
            "best_possible": float(eff.min(axis=1).sum())}


def solve_learned(a: CscMatrix, b: np.ndarray, model: Optional[TierModel] = None, target: float = 1e-14,
                  settings: Optional[SolverSettings] = None, sym: Optional[LdltSymbolic] = None):
    """Pick the tier with the network, factor and refine; if the result does
    not certify (or the low-precision factor breaks down), refactor in FP64.
    Returns (x, MixedInfo, chosen tier, fell_back)."""
    model = model or TierModel.load()
    st = settings or tier_settings()
    sym = sym or LdltSymbolic.analyze_with(a, st)
    tier = int(model.predict(tier_features(a, sym)[None])[0])
    if tier != N.TIER_FP64:
        try:
            s = MixedLdltSolver.factor_tier(a, tier, st, sym)
            x, info = s.solve_to(a, b, target)
            if info.certified:
                return x, info, tier, False
        except NumericallyRankDeficient:
            pass
    s = MixedLdltSolver.factor_tier(a, N.TIER_FP64, st, sym)
    x, info = s.solve_to(a, b, target)
    return x, info, tier, tier != N.TIER_FP64


def train_from_corpus(corpus: dict, epochs: int = 200, lr: float = 3e-3, seed: int = 7):
    """Train on the corpus's training split; returns (model, loss curve,
    held-out report).  200 full-batch epochs at 3e-3 with regret weights:
    chosen by 4-fold cross-validation of the policy cost on the training
    split (longer training fits the training matrices' timing outliers and
    costs more on unseen ones)."""
    count = len(corpus["labels"])
    tr, te = split(count)
    w = np.array([sample_weight(corpus["times"][i], corpus["certified"][i]) for i in range(count)])
    model = TierModel.init(seed)
    curve = model.fit(corpus["features"][tr], corpus["labels"][tr], w[tr], epochs, lr)
    pred = model.predict(corpus["features"][te])
    rep = policy_costs(pred, corpus["times"][te], corpus["certified"][te])
    rep["accuracy"] = float(np.mean(pred == corpus["labels"][te]))
    rep["held_out"] = int(len(te))
    rep["label_counts"] = [int(np.sum(corpus["labels"] == k)) for k in range(len(TIERS))]
    return model, curve, rep


def _main():
    ap = argparse.ArgumentParser(prog="python -m rslab_b200.tiers")
    sub = ap.add_subparsers(dest="cmd", required=True)
    p1 = sub.add_parser("label", help="run every tier on the corpus (GPU)")
    p1.add_argument("--count", type=int, default=2000)
    p1.add_argument("--seed", type=int, default=5)
    p1.add_argument("--out", required=True)
    p1.add_argument("--max-seconds", type=float, default=None)
    p2 = sub.add_parser("train", help="train the network on a labelled corpus (GPU)")
    p2.add_argument("--corpus", required=True)
    p2.add_argument("--out", required=True)
    p2.add_argument("--epochs", type=int, default=200)
    p2.add_argument("--lr", type=float, default=3e-3)
    args = ap.parse_args()
    if args.cmd == "label":
        c = label_corpus(args.count, args.seed, max_seconds=args.max_seconds)
        np.savez(args.out, **{k: np.asarray(v) for k, v in c.items()})
        print("labels per tier:", [int(np.sum(c["labels"] == k)) for k in range(len(TIERS))])
    else:
        z = np.load(args.corpus)
        corpus = {k: z[k] for k in z.files}
        model, curve, rep = train_from_corpus(corpus, args.epochs, args.lr)
        model.save(args.out)
        print(f"loss {curve[0]:.4f} -> {curve[-1]:.4f}; held-out: {rep}")


if __name__ == "__main__":
    _main()
