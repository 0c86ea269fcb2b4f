#!/bin/bash
# Build the reference's own CPU extrapolation library from its sources, in place under the
# reference tree (read-only: objects go to oracle/_ref only).  Test infrastructure: the
# resulting oracle/_ref/extrapolation_cpu.so is used by tests as the parity anchor and by
# bench.py as the reference CPU baseline.  The reference sources are compiled unmodified;
# ref_shim/ supplies the two MKL CBLAS calls and zeroed operator new[] (see ref_shim.cpp).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${IMG2D_REFERENCE:-}"
if [ -z "$REF" ]; then
  echo "IMG2D_REFERENCE (the reference source tree) is not set; skipping oracle/_ref build" >&2
  exit 0
fi
OUT="$HERE/_ref"
if [ ! -f "$REF/cpp_src/extrapolation_cpu.cpp" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref build" >&2
  exit 0
fi
mkdir -p "$OUT"
CUDA_INC="${CUDA_HOME:-/usr/local/cuda}/include"
g++ -O3 -std=c++14 -fPIC -fopenmp -w -I"$HERE/ref_shim" -I"$CUDA_INC" -I"$REF/cpp_src" \
    -shared -Wl,-Bsymbolic -o "$OUT/extrapolation_cpu.so" \
    "$REF/cpp_src/extrapolation_cpu.cpp" "$REF/cpp_src/mkl_linalg.cpp" "$HERE/ref_shim/ref_shim.cpp"
echo "built $OUT/extrapolation_cpu.so"
