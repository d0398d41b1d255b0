"""Profiling driver: the bench workload (128 x 128 x 256 grid, 100 z-steps, one cavity
round trip per step) with a pinned kernel configuration, so that an ncu launch list has
a fixed launch order: 4 field-conversion kernels (fields uploaded from FP64 host
arrays), then per round trip n t-passes, n x- and y-passes, the closing t-pass and the
free-space x'/y' passes (3n + 3 launches; with --plane K the x and y passes are one plane pass: 2n + 2).

    python -m cuopo3d_b200.profile_workload --precision fp32 --round-trips 1
"""
import argparse

import numpy as np

import cuopo3d_b200 as co

TUNED = {
    "fp32": {"t": dict(threads=128, tile=2048, r1=4), "x": dict(threads=128, tile=2048, r1=8),
             "y": dict(threads=128, tile=2048, r1=16)},
    "fp64": {"t": dict(threads=128, tile=1024, r1=4), "x": dict(threads=160, tile=1024, r1=8),
             "y": dict(threads=288, tile=2048, r1=8)},
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="fp32", choices=("fp32", "fp64"))
    ap.add_argument("--round-trips", type=int, default=1)
    ap.add_argument("--plane", type=int, default=0,
                    help="fused (x, y) plane pass cluster size; 0 runs the separate x and y passes")
    a = ap.parse_args()
    prec = co.FP64 if a.precision == "fp64" else co.FP32
    cfg = co.make_config(nx=128, ny=128, nt=256, nz=100, LX=800.0, LY=800.0, Lcr=20000.0, t_window=40.0,
                         P=5.0, w0=60.0, FWHM=2.0, focal=10000.0, Rs=0.98, alpha=(2e-7, 2e-7, 2e-7),
                         pump_mode="focused-pulsed", total_rt=200, resonant=2, precision=prec)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning(TUNED[a.precision])
    sim.set_plane_pass(a.plane)
    api = co.pump_field(cfg)
    s0 = co.noise(1, 1e-6 * float(np.max(np.abs(api))), api.size).reshape(api.shape)
    for which, arr in ((co.FIELD_API, api), (co.FIELD_AP, api), (co.FIELD_AS, s0),
                       (co.FIELD_AI, np.zeros_like(s0))):
        sim.set_field(which, arr)
    sim.run_round_trips(a.round_trips)
    sim.synchronize()
    print("ok", sim.kernel_launches, sim.tuning)


if __name__ == "__main__":
    main()
