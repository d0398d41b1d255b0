#!/bin/bash
# Test infrastructure: compiles crystal_scalars.cpp against the reference's crystal
# headers (reference checkout: the argument, else $CUOPO3D_REFERENCE, else /root/reference) into oracle/_ref/.
# Usage: build_crystal_scalars.sh [reference_root]
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${CUOPO3D_REFERENCE:-/root/reference}}"
OUT="$HERE/../_ref"
HDR="$REF/src/headers"
if [ ! -f "$HDR/CrystalsBase/PPLN.cuh" ]; then
    echo "reference headers not found under $HDR" >&2
    exit 3
fi
mkdir -p "$OUT"
CXX="$(command -v /usr/bin/g++ || command -v g++)"
"$CXX" -std=c++17 -O2 -w -x c++ -I"$HDR" "$HERE/crystal_scalars.cpp" -o "$OUT/crystal_scalars"
