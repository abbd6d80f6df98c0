#!/bin/sh
# Builds the CPU oracle (test infrastructure) into oracle/liboracle.so.
# -ffp-contract=off keeps the FP32 mode in the kernels' operation order.
set -e
cd "$(dirname "$0")"
gcc -O3 -march=x86-64-v2 -ffp-contract=off -fno-fast-math -fopenmp -fPIC -shared -std=c11 \
    -Wall -Wextra -Wno-unused-function -o liboracle.so ettention_oracle.c -lm
