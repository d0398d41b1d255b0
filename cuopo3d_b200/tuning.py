"""Kernel configuration of a batch, tuned for its own instance mix.

A batch runs every instance with one kernel variant per pass (threads, tile elements,
first-stage radix; opo_batch_create), so the best choice depends on the mix, not on
any single grid.  The candidates are the single-instance autotuner's choices for each
distinct grid of the mix (opo_autotune, cached per grid), and for a choice with the
line-specialised t-pass also the same choice with the generic t-pass of its fallback
radix (the batched kernels run the line body per instance, and a mix of time axes may
prefer the generic one); each candidate that every instance of the mix accepts is timed
on the whole mix for a few batched round trips, and the fastest is kept.  The reference has no batching and compile-time block sizes
(DtypesConsts.cuh:48-50).
"""
import time

from . import FP64, LINE, Batch, OpoError, Simulation, derive, time_freq


def generic_t(precision, tuning):
    """`tuning` with its line-specialised t-pass replaced by the generic t-pass of the
    line setting's fallback radix (FP32: its radix, FP64: 4)."""
    t = dict(tuning["t"])
    if not t["r1"] & LINE:
        return tuning
    t["r1"] = 4 if precision == FP64 else t["r1"] - LINE
    return {**tuning, "t": t}


def grid_tunings(precision, cfgs):
    """{(nx, ny, nt): tuning} of the single-instance autotuner for every distinct grid."""
    out = {}
    for cfg in cfgs:
        key = (cfg.nx, cfg.ny, cfg.nt)
        if key in out:
            continue
        params, _ = derive(cfg)
        _, w = time_freq(cfg.nt, params.t_window)
        sim = Simulation(params, w)
        try:
            out[key] = sim.autotune()
        finally:
            sim.close()
    return out


def time_batch(precision, cfgs, tuning, hbm_budget, seeds, sigma=1e-3, round_trips=2):
    """Seconds per batched round trip of the mix under `tuning`, or None when an instance
    of the mix does not accept it (a first-stage radix its grid cannot take)."""
    b = Batch(precision, len(cfgs), hbm_budget, tuning=tuning)
    try:
        for cfg, seed in zip(cfgs, seeds):
            try:
                slot = b.add(cfg)
            except OpoError:
                return None
            b.init_fields(slot, cfg, seed, sigma)
        b.run_round_trips(1)
        b.synchronize()
        t0 = time.perf_counter()
        b.run_round_trips(round_trips)
        b.synchronize()
        return (time.perf_counter() - t0) / round_trips
    finally:
        b.close()


def tune_batch(precision, cfgs, hbm_budget, seeds=None, round_trips=2):
    """(best tuning, [(tuning, seconds per round trip or None)]) for the instance mix
    `cfgs` (OpoConfig list, all with the same number of z-steps)."""
    seeds = seeds if seeds is not None else [1000 + k for k in range(len(cfgs))]
    cands = []
    for t in grid_tunings(precision, cfgs).values():
        for c in (t, generic_t(precision, t)):
            if c not in cands:
                cands.append(c)
    timed = [(t, time_batch(precision, cfgs, t, hbm_budget, seeds, round_trips=round_trips)) for t in cands]
    ok = [(t, s) for t, s in timed if s is not None]
    if not ok:
        raise OpoError(1, "no candidate configuration accepts every instance of the mix")
    best = min(ok, key=lambda ts: ts[1])[0]
    return best, timed

