#!/bin/sh
# Builds oracle/_ref/libstrelka_ref.so from the reference's own shader
# sources (TEST INFRASTRUCTURE: the checker of the oracle's restatement).
#
#   1. oracle/hlsl2cpp.py rewrites shaders/*.hlsl|*.h of the reference tree
#      (syntax only; see its docstring) into oracle/_ref/src/;
#   2. g++ compiles them over the HLSL shim oracle/ref/shim.h, with one IEEE
#      rounding per operation (-ffp-contract=off) and wrapping signed
#      arithmetic (-fwrapv, as HLSL integers wrap), linking the oracle for
#      the project's native materials.
#
# The reference tree is read where it lies (STRELKA_REFERENCE, default
# /root/reference); nothing is written outside oracle/_ref/.  Without the
# reference tree this script does nothing.
set -e
cd "$(dirname "$0")"
REF=${STRELKA_REFERENCE:-/root/reference}
if [ ! -d "$REF/shaders" ]; then
    echo "build_ref.sh: no reference tree at $REF; oracle/_ref not built" >&2
    exit 0
fi
CXX=${ORACLE_CXX:-/usr/bin/g++}
PY=${PYTHON:-python3}
mkdir -p _ref/src
$PY hlsl2cpp.py "$REF/shaders" _ref/src
FLAGS="-std=c++17 -O2 -ffp-contract=off -fno-fast-math -fwrapv -fopenmp -fPIC -Wall -Wno-unused-function \
       -Wno-unused-variable -Wno-unused-but-set-variable -Wno-pedantic -Wno-sign-compare -I _ref/src -I ref -I ../include"
$CXX $FLAGS -c ref/pt.cpp -o _ref/pt.o
$CXX $FLAGS -c ref/post.cpp -o _ref/post.o
$CXX -shared -fopenmp -o _ref/libstrelka_ref.so _ref/pt.o _ref/post.o -L. -loracle -Wl,-rpath,'$ORIGIN/..' -lm
