#!/bin/bash
# Test infrastructure: compiles the reference cuOPO3D solver from its own headers
# (reference checkout: the argument, else $CUOPO3D_REFERENCE, else /root/reference) through ref_harness.cu, once per
# grid / precision / fix set, into oracle/_ref/.  Nothing is copied from the reference;
# the headers are read where they lie.  Usage: build_ref.sh [reference_root]
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${CUOPO3D_REFERENCE:-/root/reference}}"
OUT="$HERE/../_ref"
HDR="$REF/src/headers"
if [ ! -f "$HDR/Solver3D.cuh" ]; then
    echo "reference headers not found under $HDR" >&2
    exit 3
fi
mkdir -p "$OUT"
NVCC="${NVCC:-nvcc}"
# name NX NY NT NZ NRT FP64 FIX
VARIANTS=(
    "g16_fp64fix 16 16 32 12 10 1 1"
    "g16_fp32fix 16 16 32 12 10 0 1"
    "g16_fp32asis 16 16 32 4 10 0 0"
    "g12_fp64fix 12 12 24 8 10 1 1"
    "c1_fp64fix 32 32 64 50 10 1 1"
    "c2_fp32asis 128 128 256 100 10 0 0"
    "c2_fp32fix 128 128 256 100 10 0 1"
    "c2_fp64fix 128 128 256 100 10 1 1"
)
pids=()
for v in "${VARIANTS[@]}"; do
    set -- $v
    name=$1
    bin="$OUT/ref_$name"
    if [ -x "$bin" ] && [ "$bin" -nt "$HERE/ref_harness.cu" ]; then continue; fi
    "$NVCC" -std=c++17 -O3 -DDISPERSION -DDIFFRACTION -diag-suppress 177,550,20012 \
        -I"$HDR" -DRH_NX=$2 -DRH_NY=$3 -DRH_NT=$4 -DRH_NZ=$5 -DRH_NRT=$6 -DRH_FP64=$7 \
        -DRH_FIX=$8 -gencode arch=compute_100a,code=sm_100a \
        "$HERE/ref_harness.cu" -lcufft -o "$bin" &
    pids+=($!)
done
rc=0
for p in "${pids[@]}"; do wait "$p" || rc=1; done
exit $rc
