#!/usr/bin/env bash
# Builds oracle/_ref/ref_gpu_nve: the reference's own CUDA sources
# (src/DPM2D.cu, src/Simulator.cu, src/FIRE.cu, src/BumpyEllipse.cu,
# src/DPM3D.cu of farceri/cudaRing, compiled in place from the reference
# checkout, never copied) for sm_100a, linked with the timing harness
# oracle/ref_gpu/ref_gpu_nve.cu.  Flags follow the reference makefile
# (-O3 --expt-extended-lambda --expt-relaxed-constexpr, -lstdc++fs).
# Measurement infrastructure only.
#
# usage: oracle/build_ref_gpu.sh [REFERENCE_DIR]   (default $CUDARING_REFERENCE, else /root/reference)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${CUDARING_REFERENCE:-/root/reference}}"
if [ ! -f "$REF/src/DPM2D.cu" ]; then
  echo "build_ref_gpu: reference sources not found under $REF; skipping" >&2
  exit 0
fi
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
OBJ="$HERE/_ref/gpu_obj"
mkdir -p "$OBJ"
FLAGS=(-O3 -std=c++17 --expt-extended-lambda --expt-relaxed-constexpr -w
       -gencode arch=compute_100a,code=sm_100a -ccbin /usr/bin/g++ -I"$REF")
pids=()
for f in DPM2D Simulator FIRE BumpyEllipse DPM3D; do
  "$NVCC" "${FLAGS[@]}" -c "$REF/src/$f.cu" -o "$OBJ/$f.o" &
  pids+=($!)
done
"$NVCC" "${FLAGS[@]}" -c "$HERE/ref_gpu/ref_gpu_nve.cu" -o "$OBJ/ref_gpu_nve.o" &
pids+=($!)
for p in "${pids[@]}"; do wait "$p"; done
"$NVCC" -gencode arch=compute_100a,code=sm_100a -ccbin /usr/bin/g++ "$OBJ"/*.o -o "$HERE/_ref/ref_gpu_nve.tmp" -lstdc++fs
mv "$HERE/_ref/ref_gpu_nve.tmp" "$HERE/_ref/ref_gpu_nve"
rm -rf "$OBJ"
echo "build_ref_gpu: wrote $HERE/_ref/ref_gpu_nve"
