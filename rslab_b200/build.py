"""Build the in-tree native library librslab_b200.so for sm_100a.

The product library is plain CUDA C++ (no PyTorch): the host analysis
(csrc/host/*.cpp), the kernels and the runtime (csrc/engine.cu) are compiled
with nvcc for `-gencode arch=compute_100a,code=sm_100a` and linked into one
shared object next to this file.  Run `python rslab_b200/build.py` (a plain script: importing the package
needs the library it builds).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "librslab_b200.so"
BUILD = HERE.parent / "_build" / "rslab_b200"

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xcompiler", "-ffp-contract=off",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted((CSRC / "host").glob("*.cpp")) + [CSRC / "engine.cu", CSRC / "tier_mlp.cu"]


def deps() -> list[Path]:
    out = sources()
    for pat in ("*.hpp", "*.cuh", "*.inc"):
        out += list(CSRC.rglob(pat))
    out.append(HERE.parent / "include" / "rslab_b200.h")
    return out


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in deps())


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(parents=True, exist_ok=True)
    objs = []
    nv = nvcc()
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        cmd = [nv, *NVCC_FLAGS, *(extra or []), "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd = [nv, "-x", "cu", *NVCC_FLAGS, *(extra or []), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nv, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", str(tmp), "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
    print(LIB)
