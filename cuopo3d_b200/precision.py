"""Accuracy of the FP32 precision form against the FP64 plain form, per round trip.

The FP64 plain form of this library reproduces the FP64 oracle and the reference's own
FP64 build to <= 1e-10 (tests/test_gpu_parity.py), so it stands in for the FP64 oracle
at sizes and round-trip counts the CPU oracle cannot reach (one 128x128x256 round trip
of the oracle takes minutes on the host cores).  Both forms start from the same fields
and run in lockstep; at each checkpoint the fields are read back and compared.

Reference: the round-trip loop whose rounding accumulates is Solver3D.cuh:964-1023
(runOPO); output power as the reference tallies it, Solver3D.cuh:508-545.
"""
import numpy as np

from . import FIELD_AI, FIELD_AP, FIELD_API, FIELD_AS, FP32, FP64, Simulation, derive, make_config, noise, \
    pump_field, time_freq


def rel_l2(a, b):
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a))


def _solver(precision, kw, tuning, autotune):
    cfg = make_config(precision=precision, **kw)
    params, _ = derive(cfg)
    _, w = time_freq(cfg.nt, params.t_window)
    sim = Simulation(params, w)
    if tuning is not None:
        sim.set_tuning(tuning)
    elif autotune:
        sim.autotune()
    return cfg, params, sim


def error_vs_round_trip(kw, checkpoints, seed=1, noise_rel=1e-6, tuning32=None, tuning64=None, autotune=True):
    """FP32 against FP64 on configuration `kw` (make_config keywords) at each round trip
    in `checkpoints` (ascending).  The pump is the configuration's analytic pump, the
    signal seeded complex Gaussian noise at `noise_rel` of the pump's peak amplitude, the
    idler zero.  Returns a list of dicts: round trip, relative L2 field error of pump,
    signal and idler, and the relative error of the output signal power (FP64 tallies of
    sum |As|^2)."""
    cfg64, p64, s64 = _solver(FP64, kw, tuning64, autotune)
    _, _, s32 = _solver(FP32, kw, tuning32, autotune)
    api = pump_field(cfg64)
    s0 = noise(seed, noise_rel * float(np.max(np.abs(api))), api.size).reshape(api.shape)
    for sim in (s64, s32):
        for which, arr in ((FIELD_API, api), (FIELD_AP, api), (FIELD_AS, s0), (FIELD_AI, np.zeros_like(s0))):
            sim.set_field(which, arr)
    out, done = [], 0
    try:
        for rt in checkpoints:
            if rt > done:
                s64.run_round_trips(rt - done)
                s32.run_round_trips(rt - done)
                done = rt
            rec = {"round_trip": rt}
            for which, name in ((FIELD_AP, "pump"), (FIELD_AS, "signal"), (FIELD_AI, "idler")):
                rec[f"{name}_rel_l2"] = rel_l2(s32.get_field(which), s64.get_field(which))
            ps64, ps32 = s64.field_sums()[1], s32.field_sums()[1]
            rec["signal_power_rel"] = abs(ps32 / ps64 - 1) if ps64 > 0 else float("nan")
            rec["signal_power_fp64"] = ps64
            out.append(rec)
    finally:
        s64.close()
        s32.close()
    return out


def error_of_request(cfg_kw, seed, sigma, round_trips, tuning32=None):
    """Field and output-power error of one served or batched instance: the FP32 precision
    form against the FP64 plain form, both initialised on the device the way the batch
    and the serving loop do it (pump, seeded signal noise `sigma`, idler zero) and run
    for `round_trips`.  A batched or served FP32 result equals the standalone FP32 run
    bit for bit (tests/test_batch.py, tests/test_serve.py), so this is its error."""
    recs = {}
    for prec in (FP64, FP32):
        cfg = make_config(precision=prec, **cfg_kw)
        params, _ = derive(cfg)
        _, w = time_freq(cfg.nt, params.t_window)
        sim = Simulation(params, w)
        try:
            if prec == FP32 and tuning32 is not None:
                sim.set_tuning(tuning32)
                sim.set_plane_pass(0)
            sim.init_fields(cfg, seed, sigma)
            sim.run_round_trips(round_trips)
            recs[prec] = ([sim.get_field(k) for k in (FIELD_AP, FIELD_AS, FIELD_AI)], sim.field_sums())
        finally:
            sim.close()
    (f64, p64), (f32, p32) = recs[FP64], recs[FP32]
    out = {"round_trips": round_trips}
    for k, name in enumerate(("pump", "signal", "idler")):
        out[f"{name}_rel_l2"] = rel_l2(f32[k], f64[k])
    out["signal_power_rel"] = abs(p32[1] / p64[1] - 1) if p64[1] > 0 else float("nan")
    return out
