#!/usr/bin/env bash
# Builds the reference's own kernels (include/felbm_gpu/device_engine.cuh of
# matNBI/felbm_gpu, compiled unmodified) behind oracle/ref/ref_harness.cu, for
# sm_100a, into oracle/_ref/:
#   libref_kernels_f64.so  (real_t = double, the reference default build)
#   libref_kernels_f32.so  (-DFELBM_SINGLE, the reference single build)
# Test infrastructure only. Needs the reference checkout: the directory in
# $FELBM_REFERENCE, else the "reference_path" entry of the repository's
# BASELINE.json; a machine without it (the GPU box) uses the prebuilt files
# that travel with the repository snapshot.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${FELBM_REFERENCE:-}"
if [ -z "$REF" ] && [ -f "$HERE/../../BASELINE.json" ]; then
  REF="$(python3 -c 'import json,sys; print(json.load(open(sys.argv[1])).get("reference_path", ""))' \
         "$HERE/../../BASELINE.json")"
fi
if [ -z "$REF" ]; then
  echo "build_ref.sh: no reference checkout named (FELBM_REFERENCE or BASELINE.json reference_path); skipping" >&2
  exit 0
fi
OUT="$HERE/../_ref"
if [ ! -f "$REF/include/felbm_gpu/device_engine.cuh" ]; then
  echo "build_ref.sh: reference sources not found under $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
FLAGS=(-gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -ccbin g++ -shared -Xcompiler -fPIC
       -I"$REF/include" -cudart static)
nvcc "${FLAGS[@]}" -o "$OUT/libref_kernels_f64.so" "$HERE/ref_harness.cu"
nvcc "${FLAGS[@]}" -DFELBM_SINGLE -o "$OUT/libref_kernels_f32.so" "$HERE/ref_harness.cu"
echo "built $OUT/libref_kernels_f64.so $OUT/libref_kernels_f32.so"
