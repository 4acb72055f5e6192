#!/bin/sh
# Builds the CPU oracle (test infrastructure only) into oracle/liboracle.so.
#   -ffp-contract=off : no fused multiply-add, matching the kernels' -fmad=false
#   liboracle_fast.so : the same source with contraction allowed, timed only
#   libworkload.so    : the seeded workload generators and the host SAH
#                       builder (the package's host-only C++ sources, no CUDA),
#                       so the CPU reference arm of the benchmark can build its
#                       scene without loading the CUDA library
set -e
cd "$(dirname "$0")"
CC=${ORACLE_CC:-/usr/bin/gcc}
CXX=${ORACLE_CXX:-/usr/bin/g++}
$CC -std=c11 -O3 -march=x86-64-v3 -ffp-contract=off -fno-math-errno -fopenmp -fPIC -shared \
    -Wall -Wno-unused-function -o liboracle.so oracle.c -lm
$CC -std=c11 -O3 -march=x86-64-v3 -ffp-contract=fast -fno-math-errno -fopenmp -fPIC -shared \
    -Wall -Wno-unused-function -o liboracle_fast.so oracle.c -lm
SRC=../strelka_b200/csrc
$CXX -std=c++17 -O3 -ffp-contract=off -fopenmp -fPIC -shared -Wall -Wno-unused-function -Wno-array-bounds \
    -I ../include -I /usr/local/cuda/include -o libworkload.so \
    $SRC/scene_gen.cpp $SRC/bvh_builder.cpp $SRC/common.cpp -lm
