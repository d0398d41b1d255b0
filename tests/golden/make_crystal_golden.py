"""Regenerate tests/golden/crystal_scalars.json: the dispersion scalars of every crystal
class the reference's Crystals.cuh includes (PPLN, MgOsPPLT, MgOPPLN, ZGP), computed by
the reference's own headers (oracle/refharness/crystal_scalars.cpp, built by
oracle/refharness/build_crystal_scalars.sh in double precision).

    oracle/refharness/build_crystal_scalars.sh && python tests/golden/make_crystal_golden.py
"""
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BIN = os.path.join(ROOT, "oracle", "_ref", "crystal_scalars")


def main():
    out = subprocess.run([BIN], check=True, capture_output=True, text=True).stdout
    rows = [json.loads(line) for line in out.splitlines() if line.startswith("{")]
    with open(os.path.join(HERE, "crystal_scalars.json"), "w") as f:
        json.dump({"generator": "oracle/refharness/crystal_scalars.cpp (reference headers, double)",
                   "rows": rows}, f, indent=0)
    print(len(rows), "rows")


if __name__ == "__main__":
    main()
