#!/bin/bash
# Compile a program written against cuOPO3D's headers (e.g. its cuOPO3D.cu, unchanged)
# against the drop-in headers of this repository and link it to libcuopo3d.so.
#   build_dropin.sh MAIN.cu OUTPUT [extra nvcc flags, e.g. -DOPO_NT=256 -DOPO_NRT=200]
# Quoted includes resolve next to the source file first, so the program is compiled from
# a private directory where "headers/" is this repository's src/headers.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
ROOT="$(dirname "$HERE")"
MAIN="$1"; OUT="$2"; shift 2
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
[ -x "$NVCC" ] || NVCC=nvcc
[ -f "$ROOT/cuopo3d_b200/libcuopo3d.so" ] || python3 -m cuopo3d_b200.build >/dev/null
WORK="$(mktemp -d)"
trap 'rm -rf "$WORK"' EXIT
cp "$MAIN" "$WORK/main.cu"
ln -s "$HERE/headers" "$WORK/headers"
mkdir -p "$(dirname "$OUT")"
OUT_ABS="$(cd "$(dirname "$OUT")" && pwd)/$(basename "$OUT")"
(cd "$WORK" && "$NVCC" -std=c++17 -O2 -DDISPERSION -DDIFFRACTION -diag-suppress 177 "$@" -I"$ROOT/include" \
    -gencode arch=compute_100a,code=sm_100a main.cu -o "$OUT_ABS" \
    -L"$ROOT/cuopo3d_b200" -lcuopo3d -Xlinker -rpath -Xlinker "$ROOT/cuopo3d_b200")
