#!/bin/sh
# Builds the CPU oracle (test infrastructure) into oracle/liboracle.so.
# -ffp-contract=off keeps the reference's rounding (no fused multiply-add).
set -e
cd "$(dirname "$0")"
gcc -O2 -fPIC -shared -fopenmp -ffp-contract=off -fno-fast-math -std=c11 \
    -D_GNU_SOURCE -o liboracle.so av_oracle.c -lm
