#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure only) into oracle/_build/.
#   liboracle64.so     FP64, sequential: the parity oracle
#   liboracle32_omp.so FP32, OpenMP over all host threads: the timed CPU baseline
#   liboracle64_omp.so FP64, OpenMP over all host threads: the oracle of the full-size
#                      accuracy fixtures (tests/golden/make_fullsize.py)
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$here/_build"
# the image exports CC=/opt/gcc/bin/gcc, which lacks libgomp; use the system gcc unless OR_CC is set
cc="${OR_CC:-/usr/bin/gcc}"
"$cc" -O2 -fPIC -shared -std=c11 -DOR_REAL=double -o "$here/_build/liboracle64.so" "$here/mpm_oracle.c" -lm
"$cc" -O3 -fPIC -shared -std=c11 -fopenmp -DOR_REAL=float -o "$here/_build/liboracle32_omp.so" "$here/mpm_oracle.c" -lm
"$cc" -O2 -fPIC -shared -std=c11 -fopenmp -DOR_REAL=double -o "$here/_build/liboracle64_omp.so" "$here/mpm_oracle.c" -lm
