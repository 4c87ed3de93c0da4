#!/bin/sh
# Builds the CPU oracle (test infrastructure) into oracle/_build/.
# -ffp-contract=off keeps every multiply and add separately rounded, the same
# arithmetic the CUDA side is compiled for (nvcc --fmad=false).
set -e
here="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$here/_build"
g++ -std=c++17 -O3 -march=x86-64-v3 -ffp-contract=off -fno-fast-math -fopenmp -fPIC -shared \
    -Wall -Wextra -Wno-unused-parameter \
    -o "$here/_build/librefcpu.so" "$here/refcpu.cpp" "$here/ipc_cpu.cpp"
