#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure) into oracle/liboracle.so.
# IEEE float64 per operation: no -ffast-math and no FMA contraction.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
gcc -O2 -std=c11 -fPIC -shared -fopenmp -ffp-contract=off -fno-fast-math \
    -o "$here/liboracle.so" "$here/cnb_oracle.c" -lm
