"""Regenerate the golden fixtures under tests/golden/ from the RSLAB source tree.

Reads (never writes) the reference checkout given as argv[1]:
  * crates/rslab-amd/tests/data/amd_oracle/*.txt  — SuiteSparse AMD permutations
    and counters pinned by crates/rslab-amd/tests/oracle_match.rs:146-160,
    with the pattern generators of that test restated below;
  * tests/data/parity/<dir>/<NAME>.{mtx,json,mumps.json} — real symmetric
    indefinite KKT matrices with right-hand sides and the MUMPS inertia.
Writes amd_oracle.json and parity_kkt.npz next to this file.  The GPU box never
reads the reference tree: only these committed outputs are used by the tests.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _csc_from_pairs(n, pairs):
    s = set()
    for i, j in pairs:
        s.add((i, j))
        s.add((j, i))
    cols = [[] for _ in range(n)]
    for r, c in sorted(s):
        cols[c].append(r)
    cp, ri = [0], []
    for c in cols:
        ri += sorted(c)
        cp.append(len(ri))
    return cp, ri


def band(n, b):
    t = []
    for i in range(n):
        t.append((i, i))
        for k in range(1, b + 1):
            if i + k < n:
                t.append((i, i + k))
    return _csc_from_pairs(n, t)


def arrow(n):
    t = [(i, i) for i in range(n)] + [(0, i) for i in range(1, n)]
    return _csc_from_pairs(n, t)


def grid_2d(m, n):
    t = []
    for r in range(m):
        for c in range(n):
            k = r * n + c
            t.append((k, k))
            if r + 1 < m:
                t.append((k, (r + 1) * n + c))
            if c + 1 < n:
                t.append((k, r * n + c + 1))
    return _csc_from_pairs(m * n, t)


AMD_CASES = {
    "diag_4": lambda: band(4, 0),
    "tridiag_10": lambda: band(10, 1),
    "arrow_5": lambda: arrow(5),
    "arrow_200": lambda: arrow(200),
    "band_20_3": lambda: band(20, 3),
    "grid_7x7": lambda: grid_2d(7, 7),
    "amd_demo_24": lambda: grid_2d(6, 4),
}


def parse_oracle(path: Path) -> dict:
    out = {}
    for line in path.read_text().splitlines():
        line = line.strip()
        if not line or line.startswith("#") or ":" not in line:
            continue
        k, v = line.split(":", 1)
        out[k.strip()] = v.strip()
    return out


def read_mtx(path: Path):
    lines = [l for l in path.read_text().splitlines() if l and not l.startswith("%")]
    n, _, nz = (int(x) for x in lines[0].split())
    rows, cols, vals = [], [], []
    for l in lines[1: 1 + nz]:
        a = l.split()
        i, j, v = int(a[0]) - 1, int(a[1]) - 1, float(a[2])
        if i < j:
            i, j = j, i
        rows.append(i)
        cols.append(j)
        vals.append(v)
    return n, np.array(rows), np.array(cols), np.array(vals)


def main(ref: Path) -> None:
    amd_dir = ref / "crates/rslab-amd/tests/data/amd_oracle"
    amd = {}
    for name, gen in AMD_CASES.items():
        o = parse_oracle(amd_dir / f"{name}.txt")
        cp, ri = gen()
        amd[name] = {
            "n": int(o["n"]), "col_ptr": cp, "row_idx": ri,
            "perm": [int(x) for x in o["perm"].split()],
            "ncmpa": int(o["ncmpa"]), "n_dense": int(o["n_dense"]), "ndiv": int(o["ndiv"]),
            "nms_ldl": int(o["nms_ldl"]), "nms_lu": int(o["nms_lu"]), "lnz": int(o["lnz"]),
        }
    (HERE / "amd_oracle.json").write_text(json.dumps(amd))

    par = ref / "tests/data/parity"
    arrays = {}
    index = []
    for d in sorted(p for p in par.iterdir() if p.is_dir()):
        for mtx in sorted(d.glob("*.mtx")):
            stem = mtx.name[:-4]
            side = json.loads((d / f"{stem}.json").read_text())
            mj = d / f"{stem}.mumps.json"
            mumps = json.loads(mj.read_text()) if mj.exists() else None
            n, r, c, v = read_mtx(mtx)
            if n > 1200:
                continue
            key = stem
            arrays[f"{key}__rows"] = r
            arrays[f"{key}__cols"] = c
            arrays[f"{key}__vals"] = v
            arrays[f"{key}__rhs"] = np.array(side.get("rhs", [0.0] * n), dtype=np.float64)
            index.append({
                "name": key, "n": n,
                "inertia": side.get("inertia"),
                "mumps_inertia": mumps.get("inertia") if mumps else None,
                "mumps_status": mumps.get("factorization_status") if mumps else None,
            })
    arrays["__index__"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / "parity_kkt.npz", **arrays)
    print(f"amd cases: {len(amd)}  kkt matrices: {len(index)}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the RSLAB source tree>")
    main(Path(sys.argv[1]))
