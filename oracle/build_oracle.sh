#!/bin/sh
# Builds the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.
# -ffp-contract=off: every C operator is one IEEE-754 operation; FMAs are
# explicit fmaf() calls, mirroring the CUDA build's --fmad=false.
set -e
here="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$here/_build"
gcc -O2 -std=c11 -fPIC -shared -fopenmp -ffp-contract=off -fno-fast-math \
    -fvisibility=hidden -o "$here/_build/liboracle.so" \
    "$here/sift_oracle.c" "$here/stitch_oracle.c" -lm
