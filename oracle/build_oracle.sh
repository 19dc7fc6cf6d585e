#!/usr/bin/env bash
# Build the CPU oracle (test infrastructure only) into oracle/_build/.
# -ffp-contract=off keeps every product/sum separately rounded like the
# reference's Rust code; the explicit std::fma calls mirror its `fmadd`
# (target-cpu=native builds of the reference use hardware FMA there).
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$here/_build"
g++ -O3 -std=c++17 -march=x86-64-v3 -ffp-contract=off -fopenmp -fPIC -shared \
    "$here/oracle.cpp" "$here/symbolic.cpp" -o "$here/_build/liboracle.so.tmp"
mv "$here/_build/liboracle.so.tmp" "$here/_build/liboracle.so"
echo "$here/_build/liboracle.so"
