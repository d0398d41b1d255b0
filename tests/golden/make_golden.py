"""Generates the golden fixtures in tests/golden/ by running the reference cuOPO3D
solver itself (its own headers compiled by oracle/refharness/build_ref.sh into
oracle/_ref/) on a B200.

Each fixture holds the harness arguments, the reference's derived scalars, its t/w
grids, slices of its pump field and its output fields.  Initial signal/idler fields
are not stored: they are regenerated from the recorded seed with the oracle's
counter-based noise (identical IEEE operations everywhere), written to files and
uploaded to the reference in place of its wall-clock-seeded noise.

Run on a machine with a B200:  python tests/golden/make_golden.py --out DIR [--only NAMES]
then copy the .npz files from DIR into tests/golden/.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

REF_DIR = os.path.join(ROOT, "oracle", "_ref")

# name, binary, (nx, ny, nt), harness args, noise (seed, sigma or "rel:x"), idler init,
# stored t-slices (None = all)
CASES = [
    ("g16_opo_fp64", "g16_fp64fix", (16, 16, 32),
     dict(mode="opo", crystal="mgosplt", LX=400, LY=400, Lcr=10000, T=27, Lambda=6.97,
          lp=0.532, ls=1.064, Rs=0.98, gdd=1.0, P=100, FWHM=2, w0=50, focal=5000,
          pump="focused-cw"),
     (11, 0.01), "copy", None),
    ("g16_single_fp64", "g16_fp64fix", (16, 16, 32),
     dict(mode="single", crystal="ppln", LX=400, LY=400, Lcr=5000, T=27, Lambda=6.97,
          lp=0.532, ls=1.064, P=2000, FWHM=2, w0=50, focal=2500, twin=20,
          pump="focused-pulsed"),
     (12, 0.05), "zero", None),
    ("g16_asis_fp32", "g16_fp32asis", (16, 16, 32),
     dict(mode="single", crystal="ppln", LX=400, LY=400, Lcr=5000, T=27, Lambda=6.97,
          lp=0.532, ls=1.064, P=2000, FWHM=2, w0=50, focal=2500, twin=20,
          pump="focused-pulsed"),
     (12, 0.05), "zero", None),
    ("g16_opo_fp32", "g16_fp32fix", (16, 16, 32),
     dict(mode="opo", crystal="mgosplt", LX=400, LY=400, Lcr=10000, T=27, Lambda=6.97,
          lp=0.532, ls=1.064, Rs=0.98, gdd=1.0, P=100, FWHM=2, w0=50, focal=5000,
          pump="focused-cw"),
     (11, 0.01), "copy", None),
    ("g12_opo_fp64", "g12_fp64fix", (12, 12, 24),
     dict(mode="opo", crystal="ppln", LX=300, LY=300, Lcr=4000, T=27, Lambda=6.97,
          lp=0.532, ls=1.064, Rs=0.9, gdd=0.5, P=200, FWHM=4, w0=40, focal=2000, twin=30,
          pump="focused-pulsed"),
     (13, 0.02), "copy", None),
    ("c1_single_fp64", "c1_fp64fix", (32, 32, 64),
     dict(mode="single", crystal="ppln", LX=400, LY=400, Lcr=5000, T=27, Lambda=6.97,
          lp=0.532, ls=1.064, dQ=14e-6, P=1, FWHM=2, w0=50, focal=2500, twin=20,
          pump="focused-pulsed"),
     (1, "rel:1e-6"), "zero", [0, 16, 32, 48]),
    # the benchmark workload: singly-resonant OPO at full size, 10 round trips of 100 steps;
    # slices at the signal / idler centre (128), where the pump leaves the crystal after
    # its group-delay walk-off in the pump frame, L (1/vp - 1/vi) = 16.4 ps (232), and
    # between them (180)
    ("c2_opo_fp64", "c2_fp64fix", (128, 128, 256),
     dict(mode="opo", crystal="ppln", LX=800, LY=800, Lcr=20000, T=27, Lambda=6.97,
          lp=0.532, ls=1.064, Rs=0.98, P=5, FWHM=2, w0=60, focal=10000, twin=40,
          pump="focused-pulsed", alpha_p=2e-7, alpha_s=2e-7, alpha_i=2e-7, resonant=2),
     (1, "rel:1e-6"), "zero", [128, 180, 232]),
]

TIMING = [
    ("c2_fp32asis", dict(mode="time_opo", crystal="ppln", LX=800, LY=800, Lcr=20000, T=27,
                         Lambda=6.97, lp=0.532, ls=1.064, Rs=0.98, gdd=1.0, P=5, FWHM=2,
                         w0=60, focal=10000, twin=40, pump="focused-pulsed",
                         alpha_s=2e-7, alpha_i=2e-7)),
    ("c2_fp32fix", None),
    ("c2_fp64fix", None),
]


def write_field(path, a):
    np.ascontiguousarray(a, dtype=np.complex128).tofile(path)


def read_field(path, shape):
    return np.fromfile(path, dtype=np.complex128).reshape(shape)


def harness_args(d):
    return [f"{k}={v}" for k, v in d.items()]


def oracle_phys_for(args, shape):
    nx, ny, nt = shape
    crystal = po.OR_PPLN if args["crystal"] == "ppln" else po.OR_MGOSPPLT
    return po.make_phys(crystal=crystal, LX=args["LX"], LY=args["LY"], Lcr=args["Lcr"],
                        T=args["T"], Lambda=args["Lambda"], lp=args["lp"], ls=args["ls"],
                        nx=nx, ny=ny, nt=nt, nz=2, P=args["P"], FWHM=args["FWHM"],
                        w0=args["w0"], focal=args["focal"], pump_mode=args["pump"],
                        t_window=args.get("twin", 0.0), dQ=args.get("dQ", -1.0))


def run_case(case, out_dir):
    name, binary, shape, args, (seed, sigma), idler, tsl = case
    nx, ny, nt = shape
    V = nx * ny * nt
    # the full fields the harness exchanges (hundreds of MB at 128 x 128 x 256) stay in a
    # temporary directory; only the fixture goes to out_dir
    with tempfile.TemporaryDirectory(prefix="golden_" + name + "_") as tmp:
        run_case_in(name, binary, shape, args, seed, sigma, idler, tsl, V, tmp, out_dir)


def run_case_in(name, binary, shape, args, seed, sigma, idler, tsl, V, tmp, out_dir):
    nx, ny, nt = shape
    if isinstance(sigma, str):
        rel = float(sigma.split(":")[1])
        api = po.Setup(oracle_phys_for(args, shape)).api_complex()
        sigma = rel * float(np.max(np.abs(api)))
    s0 = po.noise(seed, sigma, V).reshape(nt, ny, nx)
    write_field(os.path.join(tmp, "s0.bin"), s0)
    a = dict(args)
    a["init_s"] = os.path.join(tmp, "s0.bin")
    if idler == "copy":
        a["init_i"] = a["init_s"]
    a["out"] = os.path.join(tmp, "ref")
    cmd = [os.path.join(REF_DIR, "ref_" + binary)] + harness_args(a)
    t0 = time.time()
    proc = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    with open(os.path.join(out_dir, name + ".log"), "w") as f:
        f.write(proc.stdout + proc.stderr)
    if proc.returncode != 0 or "RH_DONE" not in proc.stdout:
        raise RuntimeError(f"{name}: rc={proc.returncode}\n{proc.stdout[-2000:]}\n{proc.stderr[-2000:]}")
    if a["mode"] == "opo" and "criteria: passed" not in proc.stdout:
        raise RuntimeError(f"{name}: Courant gate failed\n{proc.stdout[-2000:]}")
    sc = {}
    for line in open(a["out"] + "_scalars.txt"):
        k, v = line.split()
        sc[k] = float(v)
    fields = {k: read_field(a["out"] + f"_{k}.bin", (nt, ny, nx)) for k in ("Ap", "As", "Ai", "Api")}
    t = np.fromfile(a["out"] + "_t.bin", dtype=np.float64)
    w = np.fromfile(a["out"] + "_w.bin", dtype=np.float64)
    tidx = np.arange(nt) if tsl is None else np.array(tsl)
    meta = dict(name=name, binary=binary, shape=shape, args=args, seed=seed, sigma=sigma,
                idler=idler, seconds=time.time() - t0)
    out = dict(meta=json.dumps(meta), scalar_names=np.array(list(sc.keys())),
               scalar_values=np.array(list(sc.values())), t=t, w=w, tidx=tidx,
               Api=fields["Api"][tidx], Ap=fields["Ap"][tidx], As=fields["As"][tidx],
               Ai=fields["Ai"][tidx],
               norms=np.array([np.sum(np.abs(fields[k]) ** 2) for k in ("Ap", "As", "Ai")]),
               # energy of every t-slice of each output field, [field][t]
               tprof=np.array([np.sum(np.abs(fields[k]) ** 2, axis=(1, 2)) for k in ("Ap", "As", "Ai")]))
    np.savez_compressed(os.path.join(out_dir, name + ".npz"), **out)
    print(f"{name}: ok in {meta['seconds']:.1f}s nsteps={sc['nsteps']:.0f} "
          f"|As|^2={out['norms'][1]:.6e}", flush=True)


def run_timing(out_dir, steps, warmup):
    base = None
    res = []
    for binary, args in TIMING:
        if args is not None:
            base = args
        a = dict(base, steps=steps, warmup=warmup)
        cmd = [os.path.join(REF_DIR, "ref_" + binary)] + harness_args(a)
        proc = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        line = [ln for ln in proc.stdout.splitlines() if ln.startswith("{\"rh_time_opo\"")]
        rec = json.loads(line[-1]) if line else dict(error=proc.stderr[-500:], rc=proc.returncode)
        rec["binary"] = binary
        res.append(rec)
        print(json.dumps(rec), flush=True)
    with open(os.path.join(out_dir, "ref_timing.json"), "w") as f:
        json.dump(res, f, indent=1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory for the new .npz fixtures")
    ap.add_argument("--only", default="")
    ap.add_argument("--timing", action="store_true")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    for case in CASES:
        if a.only and case[0] not in a.only.split(","):
            continue
        run_case(case, a.out)
    if a.timing:
        run_timing(a.out, a.steps, a.warmup)


if __name__ == "__main__":
    main()
