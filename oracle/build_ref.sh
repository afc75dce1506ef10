#!/usr/bin/env bash
# Builds oracle/_ref/libcrref.so: the reference's own kernels
# (include/cudaKernel.cuh + include/DPM2D.h of farceri/cudaRing, read in place
# from the reference checkout, never copied) compiled as host C++ behind
# oracle/ref_shim/shim.h, plus the host driver oracle/ref_shim/ref_driver.cpp.
# Test infrastructure only (golden fixtures, oracle pinning, CPU baseline).
#
# usage: oracle/build_ref.sh [REFERENCE_DIR]   (default $CUDARING_REFERENCE, else /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${CUDARING_REFERENCE:-/root/reference}}"
if [ ! -f "$REF/include/cudaKernel.cuh" ]; then
  echo "build_ref: reference sources not found under $REF; skipping" >&2
  exit 0
fi
CUDA_INC="${CUDA_HOME:-/usr/local/cuda}/include"
mkdir -p "$HERE/_ref"
g++ -std=c++17 -O3 -march=x86-64-v3 -fopenmp -fPIC -shared -w \
    -I"$HERE/ref_shim" -I"$HERE/ref_shim/stub" -I"$REF/include" -I"$CUDA_INC" \
    -DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_CPP -DTHRUST_HOST_SYSTEM=THRUST_HOST_SYSTEM_CPP \
    "$HERE/ref_shim/ref_driver.cpp" -o "$HERE/_ref/libcrref.so.tmp"
mv "$HERE/_ref/libcrref.so.tmp" "$HERE/_ref/libcrref.so"
echo "build_ref: wrote $HERE/_ref/libcrref.so"
