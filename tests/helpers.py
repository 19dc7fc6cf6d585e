"""Shared fixtures for the parity tests: golden data loaders and comparisons."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from rslab_b200 import CscMatrix

GOLDEN = Path(__file__).resolve().parent / "golden"


def amd_cases() -> dict:
    return json.loads((GOLDEN / "amd_oracle.json").read_text())


def kkt_cases():
    z = np.load(GOLDEN / "parity_kkt.npz")
    idx = json.loads(bytes(z["__index__"]).decode())
    out = []
    for e in idx:
        k = e["name"]
        a = CscMatrix.from_triplets(e["n"], z[k + "__rows"], z[k + "__cols"], z[k + "__vals"])
        out.append((e, a, np.array(z[k + "__rhs"])))
    return out


def rel_err(x: np.ndarray, y: np.ndarray) -> float:
    den = max(float(np.max(np.abs(y))) if y.size else 0.0, 1e-300)
    return float(np.max(np.abs(x - y))) / den if x.size else 0.0


def dense_from_lower(a: CscMatrix) -> np.ndarray:
    return a.to_scipy_full().toarray()
