"""The C ABI library loads and exports every function include/rslab_b200.h
declares (no GPU work)."""
import re
import subprocess
from pathlib import Path

import rslab_b200._native as N

ROOT = Path(__file__).resolve().parent.parent


def declared():
    txt = (ROOT / "include" / "rslab_b200.h").read_text()
    return sorted(set(re.findall(r"\b(rslab_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (rslab_[a-z0-9_]+)$", out, flags=re.M))
    missing = [s for s in declared() if s not in exported]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(declared()) == set(N.SIGNATURES)


def test_version():
    assert N.lib.rslab_version() == 1
