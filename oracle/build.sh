#!/bin/sh
# Builds the CPU oracle (test infrastructure only) into oracle/liboracle.so.
#   -ffp-contract=off : no fused multiply-add, matching the kernels' -fmad=false
#   liboracle_fast.so : the same source with contraction allowed, timed only
set -e
cd "$(dirname "$0")"
CC=${ORACLE_CC:-/usr/bin/gcc}
$CC -std=c11 -O3 -march=x86-64-v3 -ffp-contract=off -fno-math-errno -fopenmp -fPIC -shared \
    -Wall -Wno-unused-function -o liboracle.so oracle.c -lm
$CC -std=c11 -O3 -march=x86-64-v3 -ffp-contract=fast -fno-math-errno -fopenmp -fPIC -shared \
    -Wall -Wno-unused-function -o liboracle_fast.so oracle.c -lm
