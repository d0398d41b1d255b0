#!/bin/bash
# Power / waist sweep with the argument surface of cuOPO3D's driver: builds the program
# (default ./cuOPO3D.cu, written against the cuOPO3D headers) with the drop-in headers
# and runs `./cuOPO3D <P_mW> <waist_um>` for every point, each point's .dat files moved
# into its own folder.  Grid and round trips are compile-time as in cuOPO3D; pass them
# through NVCC_FLAGS, e.g. NVCC_FLAGS="-DOPO_NT=256 -DOPO_NRT=200".
#   cuOPO3D.sh [MAIN.cu] ;  POWERS="500 1000" WAISTS="31 41" cuOPO3D.sh
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
MAIN="${1:-cuOPO3D.cu}"
POWERS="${POWERS:-500}"
WAISTS="${WAISTS:-31}"
"$HERE/build_dropin.sh" "$MAIN" ./cuOPO3D ${NVCC_FLAGS:-}
for WAIST in $WAISTS; do
    for N in $POWERS; do
        echo "Power = ${N} mW, waist = ${WAIST} um"
        OUT="waist_${WAIST}/P_${N}"
        mkdir -p "$OUT"
        ./cuOPO3D "$N" "$WAIST" | tee "$OUT/run.txt"
        shopt -s nullglob
        files=(*.dat)
        [ ${#files[@]} -gt 0 ] && mv "${files[@]}" "$OUT/"
        shopt -u nullglob
    done
done
