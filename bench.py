"""Benchmark of the split-step OPO solver on B200 GPUs (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the singly-resonant OPO at full size -- PPLN 20 mm, 128 x 128 x 256 grid over
800 um / 40 ps, 100 z-slices (100 split steps per crystal pass), GVD and group-velocity
mismatch on, absorption 0.002/cm, signal mirror R = 0.98, detuning 0, 60 um / 5 W / 2 ps
Gaussian pump, noise-seeded signal, FP64 fields.  One step = one cavity round trip
(100 z-steps of 4,194,304 voxels).  The metric is voxel-steps/s (one voxel of all three
fields advanced through one full split step).
  value      device-timed (CUDA events on the solver's stream), inputs resident in HBM
  e2e        through the C-ABI with host buffers, one solver: every step uploads its
             three input fields from pinned host memory, runs one round trip and reads
             its three output fields back to pinned host memory, all inside the timed
             region (e2e_pipelined: two solvers alternate so one's copies overlap the
             other's round trip, the way a sweep drives the library)
Extra legs on rank 0 (N = 1): the FP32 precision form, the batched form (64 uneven
instances, FP32 and FP64, kernel configuration tuned for the mix), the served form (a
Poisson stream with 50-500 round trips per request, FP32 and FP64, p50/p99 latency and
the FP32 results' error against FP64), the FP32 error per round trip on the batched
form's grids, and the FP64 CPU oracle as the reported CPU baseline.

Multi-GPU: every rank runs its own independent instance (weak scaling, no collective on
the data path); value = all ranks' voxel-steps / the slowest rank's time.  The batched
mix (64 instances per rank) is sharded over the ranks by longest-processing-time first.

`--impl reference` times the reference's own cuFFT pipeline (its headers compiled by
oracle/refharness into oracle/_ref/, unmodified code path, FP32 as shipped) on the same
GPU for --steps round trips after --warmup; without that build it times the FP64 CPU
oracle on the host cores instead.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "voxel-steps/s, HBM GB/s vs ref cuFFT build; sweep p50/p99 at ≤1e-5 rel err"
UNIT = "voxel-steps/s"
WORKLOAD = dict(nx=128, ny=128, nt=256, nz=100, LX=800.0, LY=800.0, Lcr=20000.0, t_window=40.0,
                P=5.0, w0=60.0, FWHM=2.0, focal=10000.0, Rs=0.98, Ri=0.98,
                alpha=(2e-7, 2e-7, 2e-7), pump_mode="focused-pulsed", gdd_gamma=0.0,
                detuning=0.0, total_rt=200, resonant=2)
WORKLOAD_NAME = ("singly-resonant OPO, PPLN 20 mm, 128x128x256 over 800 um / 40 ps, 100 z-steps, "
                 "5 W 60 um 2 ps pump, R=0.98, one cavity round trip per step")
V = 128 * 128 * 256
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0
# batched and served instances: 20 mm PPLN, 100 slices, 800 um / 40 ps windows
FORM_BASE = dict(nz=100, LX=800.0, LY=800.0, Lcr=20000.0, t_window=40.0, FWHM=2.0, focal=10000.0, Rs=0.98,
                 alpha=(2e-7, 2e-7, 2e-7), zloop_f32=1, pump_mode="focused-pulsed")


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def ncu_traffic(kernel, precision):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d[f"{kernel}_{precision}"]["bytes_per_launch"]
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in getattr(self, "lines", []):
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return rank, world, local


def barrier_sync(world):
    import torch
    from cuopo3d_b200 import shard
    torch.cuda.synchronize()
    shard.barrier()
    torch.cuda.synchronize()


def max_over_ranks(x, world):
    from cuopo3d_b200 import shard
    return shard.reduce_scalar(x, "max")


def sum_over_ranks(x, world):
    from cuopo3d_b200 import shard
    return shard.reduce_scalar(x, "sum")


def make_instance(co, precision, seed):
    cfg = co.make_config(precision=precision, **WORKLOAD)
    params, sc = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.autotune()  # picks kernel variants and tiles per pass (cached per grid); untimed
    api = co.pump_field(cfg)
    s0 = co.noise(seed, 1e-6 * float(np.max(np.abs(api))), api.size).reshape(api.shape)
    return cfg, params, sim, api, s0


def upload(co, sim, api, s0):
    for which, arr in ((co.FIELD_API, api), (co.FIELD_AP, api), (co.FIELD_AS, s0),
                       (co.FIELD_AI, np.zeros_like(s0))):
        sim.set_field(which, arr)


def time_device(sim, steps, world, tag):
    """K round trips between events on the solver's stream; max over ranks (ms).  The
    region is an NVTX range named timed_<tag>, so a profiler can select its launches."""
    import torch
    stream = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier_sync(world)
    sim.synchronize()
    torch.cuda.nvtx.range_push(f"timed_{tag}")
    e0.record(stream)
    sim.run_round_trips(steps)
    e1.record(stream)
    sim.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier_sync(world)
    return max_over_ranks(e0.elapsed_time(e1), world)


class HostIO:
    """Pinned host buffers of one step's inputs (Api, As, Ai) and outputs (Ap, As, Ai),
    complex128, moved through the C-ABI (opo_set_field / opo_get_field with host memory)."""

    def __init__(self, co, api, s0):
        import torch
        self.co = co
        self.inp = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128).reshape(-1)).pin_memory()
                    for a in (api, s0, np.zeros_like(s0))]
        self.out = [torch.empty(V, dtype=torch.complex128).pin_memory() for _ in range(3)]

    def h2d_bytes(self):
        return sum(t.numel() * 16 for t in self.inp)

    def d2h_bytes(self):
        return sum(t.numel() * 16 for t in self.out)

    def put(self, sim):
        co = self.co
        for which, t in zip((co.FIELD_API, co.FIELD_AS, co.FIELD_AI), self.inp):
            rc = co.lib().opo_set_field(sim.handle, which, ctypes.c_void_p(t.data_ptr()), co.MEM_HOST, co.FP64)
            assert rc == 0, rc

    def get(self, sim, out=None):
        co = self.co
        for which, t in zip((co.FIELD_AP, co.FIELD_AS, co.FIELD_AI), out or self.out):
            rc = co.lib().opo_get_field(sim.handle, which, ctypes.c_void_p(t.data_ptr()), co.MEM_HOST, co.FP64)
            assert rc == 0, rc


def e2e_streamed(co, sim, api, s0, steps, world, nsteps):
    """One solver through the streamed C-ABI (opo_stream_put / run / get): every step
    uploads its inputs (Api, As, Ai) from pinned host memory in the solver's precision,
    runs one round trip and downloads its results (Ap, As, Ai); the uploads of step k+1
    and the downloads of step k run on copy streams during the round trips.  Returns
    (voxel-steps/s, bytes up per step, bytes down per step)."""
    import torch
    dt = torch.complex128 if sim.params.precision == co.FP64 else torch.complex64
    inp = [torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to(dt).pin_memory()
           for a in (api, s0, np.zeros_like(s0))]
    outs = [[torch.empty(V, dtype=dt).pin_memory() for _ in range(3)] for _ in range(2)]
    ins_w, outs_w = (co.FIELD_API, co.FIELD_AS, co.FIELD_AI), (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)

    def step(k):
        for which, t in zip(ins_w, inp):
            sim.stream_put(which, t.data_ptr())
        sim.stream_run(1)
        for which, t in zip(outs_w, outs[k % 2]):
            sim.stream_get(which, t.data_ptr())

    step(0)
    sim.stream_wait()
    barrier_sync(world)
    t0 = time.perf_counter()
    for k in range(steps):
        step(k)
    sim.stream_wait()
    barrier_sync(world)
    dt_s = max_over_ranks(time.perf_counter() - t0, world)
    esz = inp[0].element_size()
    return sum_over_ranks(float(V) * nsteps * steps, world) / dt_s, 3 * V * esz, 3 * V * esz


def e2e_single(co, sim, io, steps, world, nsteps):
    """One solver: every step uploads its inputs, runs one round trip, reads its outputs
    (opo_get_field into host memory waits for the solver's stream)."""
    io.put(sim)
    sim.run_round_trips(1)
    io.get(sim)
    barrier_sync(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        io.put(sim)
        sim.run_round_trips(1)
        io.get(sim)
    barrier_sync(world)
    dt = max_over_ranks(time.perf_counter() - t0, world)
    return sum_over_ranks(float(V) * nsteps * steps, world) / dt


def e2e_pipelined(co, params, sim, io, steps, world, nsteps):
    """Two solvers alternate (step k on solver k % 2): step k+1's uploads and round trip
    are enqueued before step k's outputs are read, so one solver's host copies run on the
    copy engines while the other's round trip runs on the SMs."""
    import torch
    _, w = co.time_freq(params.nt, params.t_window)
    sim2 = co.Simulation(params, w)
    sim2.autotune()  # cached: the same configuration as sim
    sims = (sim, sim2)
    outs = [io.out, [torch.empty(V, dtype=torch.complex128).pin_memory() for _ in range(3)]]

    def enqueue(k):
        io.put(sims[k % 2])
        sims[k % 2].run_round_trips(1)

    def collect(k):
        io.get(sims[k % 2], outs[k % 2])

    enqueue(0)
    enqueue(1)
    collect(0)
    collect(1)
    barrier_sync(world)
    t0 = time.perf_counter()
    enqueue(0)
    for k in range(steps):
        if k + 1 < steps:
            enqueue(k + 1)
        collect(k)
    barrier_sync(world)
    dt = max_over_ranks(time.perf_counter() - t0, world)
    sim2.close()
    return sum_over_ranks(float(V) * nsteps * steps, world) / dt


def run_ours(args):
    import cuopo3d_b200 as co
    rank, world, local = dist_setup(args.gpus)
    out = {}
    hbm, hbm_kind = hbm_peak()
    e2e_steps = max(4, args.steps // 2)
    for prec, tag, bpv in ((co.FP64, "fp64", 96), (co.FP32, "fp32", 48)):
        cfg, params, sim, api, s0 = make_instance(co, prec, seed=1 + rank)
        nsteps = params.n_steps
        upload(co, sim, api, s0)
        sim.run_round_trips(args.warmup)
        sim.synchronize()
        l0 = sim.kernel_launches
        with ClockSampler(local) as clk:
            ms = time_device(sim, args.steps, world, tag)
        launches = sim.kernel_launches - l0
        vsteps = float(V) * nsteps * args.steps
        total_vsteps = sum_over_ranks(vsteps, world)
        value = total_vsteps / (ms * 1e-3)
        # Per-pass durations: the same round trips launched pass by pass between CUDA
        # events on the solver stream (no graph replay), after the timed region.
        sim.set_pass_timing(True)
        sim.pass_times()
        sim.run_round_trips(max(2, min(args.steps, 5)))
        pt = sim.pass_times()
        sim.set_pass_timing(False)
        passes = {}
        for k in ("t", "x", "y"):
            tot, n = pt[k]
            if n:
                avg_us = tot / n * 1e3
                passes[k] = {"avg_us": round(avg_us, 2), "launches": n,
                             "alg_GBps": round(V * bpv / (avg_us * 1e-6) / 1e9, 1)}
        io = HostIO(co, api, s0)
        e2e_s, up_b, down_b = e2e_streamed(co, sim, api, s0, e2e_steps, world, nsteps)
        e2e = e2e_single(co, sim, io, e2e_steps, world, nsteps)
        e2e_pipe = e2e_pipelined(co, params, sim, io, e2e_steps, world, nsteps)
        out[tag] = dict(value=value, ms_per_step=ms / args.steps, launches=launches, passes=passes,
                        tuning=sim.tuning, clocks=clk.summary(), nsteps=nsteps,
                        e2e=dict(value=e2e_s, unit=UNIT, h2d_bytes_per_step=up_b, d2h_bytes_per_step=down_b,
                                 solvers=1, steps=e2e_steps,
                                 form="streamed: opo_stream_put / opo_stream_run / opo_stream_get, host data "
                                      "in the solver's precision, copies overlapping the round trips"),
                        e2e_blocking=dict(value=e2e, unit=UNIT, h2d_bytes_per_step=io.h2d_bytes(),
                                          d2h_bytes_per_step=io.d2h_bytes(), solvers=1, steps=e2e_steps,
                                          form="opo_set_field / opo_run_round_trips / opo_get_field from complex128 "
                                               "host buffers, each step waiting for its results"),
                        e2e_pipelined=dict(value=e2e_pipe, unit=UNIT, h2d_bytes_per_step=io.h2d_bytes(),
                                           d2h_bytes_per_step=io.d2h_bytes(), solvers=2, steps=e2e_steps))
        sim.close()
    legs = {}
    if world > 1 and not args.no_forms:
        legs["batched_sharded"] = batched_sharded_leg(co, rank, world, args.batched_instances)
    if rank == 0:
        main = out["fp64"]
        t = main["passes"].get("t")
        achieved = V * 96 / (t["avg_us"] * 1e-6) / 1e9 if t else None
        # The t-pass's second bound, the FP64 pipe: 558 flops per voxel (two RK4 half steps
        # of 150 flops, three 256-point transform pairs at 5 N log2 N each way plus the phase
        # multiply, 86 flops per field) against the device's measured FMA throughput.
        fp64_peak = co.fp64_peak()
        flops_t = V * 558.0
        ach_tf = flops_t / (t["avg_us"] * 1e-6) / 1e12 if t else None
        t_kernel = ("tpass_line_kernel<double2, 256, 16, 128>" if main["tuning"]["t"]["r1"] & 256
                    else "tpass_kernel<double2>")
        line = {
            "metric": METRIC, "value": main["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": main["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded noise signal, analytic pump)",
            "config": {"workload": WORKLOAD_NAME, "grid": [128, 128, 256], "z_steps": main["nsteps"],
                       "round_trips_per_step": 1, "precision": "fp64 complex128",
                       "global_batch": world, "parallelism": f"independent instances x{world}",
                       "l2": "inputs larger than L2 (FP64 state 201 MB + pump 67 MB > 126 MB)"},
            "e2e": main["e2e"],
            "e2e_blocking": main["e2e_blocking"],
            "e2e_pipelined": main["e2e_pipelined"],
            "gpu_launches": main["launches"],
            "clocks": main["clocks"],
            "roofline": {"bound": "hbm", "kernel": f"{t_kernel} (RK4 x2 + t-axis FFT pair)",
                         "achieved": achieved, "peak": hbm,
                         "peak_kind": f"{hbm_kind} (MEASURED_PEAKS.json hbm_gbs)" if hbm_kind == "measured" else "fallback",
                         "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                         "traffic": ncu_traffic("tpass", "fp64"),
                         "alg_bytes_per_launch": V * 96},
            "roofline_fp64_pipe": {"bound": "fp64", "kernel": t_kernel, "achieved": ach_tf,
                                   "peak": fp64_peak, "peak_kind": "measured (opo_fp64_peak: FMA chains)",
                                   "unit": "TFLOP/s", "frac": (ach_tf / fp64_peak) if ach_tf else None,
                                   "alg_flops_per_launch": flops_t},
            "passes_fp64": main["passes"],
            "tuning_fp64": main["tuning"],
            "fp32": {k: out["fp32"][k] for k in ("value", "ms_per_step", "passes", "e2e", "e2e_blocking",
                                                  "e2e_pipelined", "clocks", "tuning")},
        }
        line.update(legs)
        if world == 1 and not args.no_forms:
            line["batched"] = batched_leg(co, co.FP32, args.batched_instances)
            line["batched_fp64"] = batched_leg(co, co.FP64, args.batched_instances)
            line["served"] = served_leg(co, co.FP32, args.served_requests, line["batched"]["value"])
            line["served_fp64"] = served_leg(co, co.FP64, args.served_requests_fp64, line["batched_fp64"]["value"])
            line["precision"] = precision_leg(co)
        if world == 1 and args.writer:
            line["writer"] = writer_leg(co)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def c4_mix(n_inst, seed=2024, precision=None):
    """The batched form's instance mix: N x N x NT with N in {32, 64, 128} and NT in
    {64, 128, 256}, P log-uniform 0.5-20 W, waist U[30, 100] um, detuning U[-pi, pi],
    200 round trips each; list of make_config keyword dicts."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_inst):
        N = int(rng.choice([32, 64, 128]))
        NT = int(rng.choice([64, 128, 256]))
        out.append(dict(FORM_BASE, nx=N, ny=N, nt=NT, P=float(np.exp(rng.uniform(np.log(0.5), np.log(20.0)))),
                        w0=float(rng.uniform(30, 100)), detuning=float(rng.uniform(-np.pi, np.pi)), total_rt=200))
    return out


def run_batch(co, precision, kws, tuning, seeds, warm=1, steps=3):
    """Device time per batched round trip (ms) of the instances kws; kernel launches per
    round trip."""
    import torch
    b = co.Batch(precision, len(kws), 150 << 30, tuning=tuning)
    for kw, seed in zip(kws, seeds):
        cfg = co.make_config(precision=precision, **kw)
        slot = b.add(cfg)
        b.init_fields(slot, cfg, seed, 1e-3)
    b.run_round_trips(warm)
    b.synchronize()
    stream = torch.cuda.ExternalStream(b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = b.stats()["launches"]
    e0.record(stream)
    b.run_round_trips(steps)
    e1.record(stream)
    b.synchronize()
    ms = e0.elapsed_time(e1)
    launches = b.stats()["launches"] - l0
    b.close()
    return ms / steps, launches / steps


def batched_leg(co, precision, n_inst=64, steps=3):
    """Batched form: n_inst instances of the C4 mix in one persistent launch per pass,
    round trips replayed as CUDA graphs, kernel configuration tuned for this mix
    (cuopo3d_b200.tuning.tune_batch)."""
    from cuopo3d_b200.tuning import tune_batch
    kws = c4_mix(n_inst)
    seeds = [1000 + k for k in range(n_inst)]
    cfgs = [co.make_config(precision=precision, **kw) for kw in kws]
    t0 = time.perf_counter()
    tuning, timed = tune_batch(precision, cfgs, 150 << 30, seeds)
    tune_s = time.perf_counter() - t0
    ms, launches = run_batch(co, precision, kws, tuning, seeds, steps=steps)
    vox = sum(kw["nx"] * kw["ny"] * kw["nt"] for kw in kws)
    return {"value": vox * 100.0 / (ms * 1e-3), "unit": UNIT, "instances": n_inst, "voxels": vox,
            "round_trips_timed": steps, "ms_per_round_trip": ms, "launches_per_round_trip": launches,
            "precision": "fp32" if precision == co.FP32 else "fp64", "tuning": tuning,
            "tuning_candidates": [[t, s] for t, s in timed], "tuning_s": round(tune_s, 1),
            "workload": f"{n_inst} instances, N in {{32,64,128}}, NT in {{64,128,256}}, P 0.5-20 W, "
                        "w0 30-100 um, detuning U[-pi,pi], 20 mm PPLN, 100 slices"}


def batched_sharded_leg(co, rank, world, per_rank=64, steps=3):
    """The C4 mix with per_rank x world instances, sharded over the ranks by
    longest-processing-time first (cost = voxels); every rank runs its share as one
    batch; value = all instances' voxel-steps / the slowest rank's device time."""
    from cuopo3d_b200 import shard
    kws = c4_mix(per_rank * world, seed=4048)
    costs = [kw["nx"] * kw["ny"] * kw["nt"] for kw in kws]
    mine = shard.local_indices(costs, rank, world)
    tuning = {"t": dict(threads=128, tile=2048, r1=8), "x": dict(threads=128, tile=2048, r1=8),
              "y": dict(threads=128, tile=2048, r1=16)}
    barrier_sync(world)
    ms, _ = run_batch(co, co.FP32, [kws[k] for k in mine], tuning, [1000 + k for k in mine], steps=steps)
    slowest = max_over_ranks(ms, world)
    vox = sum(costs)
    return {"value": vox * 100.0 / (slowest * 1e-3), "unit": UNIT, "instances": len(kws), "ranks": world,
            "ms_per_round_trip_slowest_rank": slowest, "precision": "fp32", "sharding": "LPT by voxels"}


def c5_requests(co, precision, n_req, rate_per_s, seed=7):
    """n_req Poisson arrivals at rate_per_s, grids from {64^2x128, 128^2x256, 96^2x192},
    P log-uniform 0.5-20 W, waist U[30, 100] um, 50-500 round trips, retired early when the
    signal power changes by less than 1e-6 over a round trip."""
    rng = np.random.default_rng(seed)
    grids = [(64, 128), (128, 256), (96, 192)]
    reqs, kws, t = [], [], 0.0
    for k in range(n_req):
        t += float(rng.exponential(1.0 / rate_per_s))
        N, NT = grids[int(rng.integers(0, 3))]
        kw = dict(FORM_BASE, nx=N, ny=N, nt=NT, P=float(np.exp(rng.uniform(np.log(0.5), np.log(20.0)))),
                  w0=float(rng.uniform(30, 100)), total_rt=int(rng.integers(50, 501)))
        kws.append(kw)
        reqs.append(dict(cfg=co.make_config(precision=precision, **kw), arrival_s=t, seed=5000 + k,
                         noise_sigma=1e-3, tol=1e-6))
    return reqs, kws


def served_leg(co, precision, n_req, batched_value, error_sample=2):
    """Served form, a bounded sample of the request stream: n_req requests of the C5
    distribution arriving at ~85 % of the batched throughput's capacity, 150 GB budget,
    kernel configuration tuned for the request grids.  For FP32, the field and output-power
    error of the error_sample shortest requests against FP64 (the same request run alone in
    each precision; a served result equals its standalone run bit for bit)."""
    from cuopo3d_b200.precision import error_of_request
    from cuopo3d_b200.tuning import tune_batch
    mean_vox = (64 * 64 * 128 + 128 * 128 * 256 + 96 * 96 * 192) / 3.0
    rate = 0.85 * batched_value / (mean_vox * 100 * 275)  # mean request: 275 round trips
    reqs, kws = c5_requests(co, precision, n_req, rate)
    mix = [co.make_config(precision=precision, **dict(FORM_BASE, nx=N, ny=N, nt=NT, P=5.0, w0=60.0))
           for N, NT in ((64, 128), (128, 256), (96, 192)) for _ in range(2)]
    tuning, _ = tune_batch(precision, mix, 150 << 30)
    res, st = co.serve(reqs, precision, capacity=1024, hbm_budget=150 << 30, realtime=True, tuning=tuning)
    ok = [r for r in res if r["status"] == co.OPO_OK]
    leg = {"p50_latency_s": st["p50_latency_s"], "p99_latency_s": st["p99_latency_s"],
           "value": st["voxel_steps_per_s"], "unit": UNIT, "requests": n_req, "completed": len(ok),
           "arrival_rate_per_s": rate, "wall_s": st["wall_s"], "max_resident": st["max_resident"],
           "round_trips_mean": float(np.mean([r["round_trips"] for r in res])),
           "retired_steady": sum(1 for r, q in zip(res, kws) if r["status"] == co.OPO_OK and
                                 r["round_trips"] < q["total_rt"]),
           "precision": "fp32" if precision == co.FP32 else "fp64", "tuning": tuning,
           "workload": f"{n_req} Poisson requests (a sample of the 2000-request stream), grids "
                       "{64^2x128, 128^2x256, 96^2x192}, P 0.5-20 W, w0 30-100 um, 50-500 round trips, "
                       "early retirement at |dPs/Ps| < 1e-6, 150 GB budget"}
    if precision == co.FP32 and error_sample:
        order = sorted(range(n_req), key=lambda k: res[k]["round_trips"] * kws[k]["nx"] ** 2 * kws[k]["nt"])
        # the batch kernels run a warp-specialised CTA size as its consumer size
        solo = {k: dict(v, threads={160: 128, 288: 256}.get(v["threads"], v["threads"])) for k, v in tuning.items()}
        errs = []
        for k in order[:error_sample]:
            kw = dict(kws[k])
            e = error_of_request(kw, 5000 + k, 1e-3, res[k]["round_trips"], tuning32=solo)
            e["grid"] = [kw["nx"], kw["ny"], kw["nt"]]
            errs.append(e)
        leg["error_vs_fp64"] = errs
    return leg


def precision_leg(co, checkpoints=(1, 10, 50, 200)):
    """FP32 against FP64 per round trip on grids of the batched form (N^2 x NT), the
    bench workload's physics: relative L2 field error and output-power error."""
    from cuopo3d_b200.precision import error_vs_round_trip
    out = []
    for N, NT in ((32, 64), (64, 128), (128, 256)):
        kw = dict(WORKLOAD, nx=N, ny=N, nt=NT)
        for r in error_vs_round_trip(kw, list(checkpoints)):
            r["grid"] = [N, N, NT]
            out.append(r)
    return {"reference": "the FP64 plain form (<= 1e-10 from the FP64 oracle and the reference's FP64 build)",
            "points": out}


def writer_leg(co, nx=128, ny=128, nt=2048):
    """The output writer (opo_save_fields) on one FP32 field of nx x ny x nt: the reference
    main's text dumps (nt slice files + nx ny trace files, "_r"/"_i" pairs) and the one-file
    binary form, into a temporary directory that is removed afterwards."""
    import shutil
    import tempfile
    cfg = co.make_config(**dict(FORM_BASE, nx=nx, ny=ny, nt=nt, P=5.0, w0=60.0, precision=co.FP32))
    params, _ = co.derive(cfg)
    _, w = co.time_freq(nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.init_fields(cfg, 1, 1e-3)
    sim.synchronize()
    out = {"grid": [nx, ny, nt], "precision": "fp32"}
    d = tempfile.mkdtemp(prefix="opo_writer_")
    try:
        t0 = time.perf_counter()
        sim.save_fields(co.FIELD_AS, os.path.join(d, "As"), binary=True)
        out["binary_s"] = time.perf_counter() - t0
        out["binary_bytes"] = os.path.getsize(os.path.join(d, "As.bin"))
        t0 = time.perf_counter()
        sim.save_fields(co.FIELD_AS, os.path.join(d, "OutputSignalPower_slice"), os.path.join(d, "As_temporal_x_"))
        out["text_s"] = time.perf_counter() - t0
        names = os.listdir(d)
        out["text_files"] = len(names) - 1
        out["text_bytes"] = sum(os.path.getsize(os.path.join(d, n)) for n in names) - out["binary_bytes"]
    finally:
        shutil.rmtree(d, ignore_errors=True)
        sim.close()
    out["host_threads"] = min(16, os.cpu_count() or 1)
    return out


def cpu_baseline(z_steps=10):
    """The FP64 CPU oracle (test infrastructure, used here only as the reported CPU
    baseline) on all host cores: z_steps split steps of the same C2 grid."""
    from oracle import pyoracle as po
    cores = os.cpu_count() or 1
    po.set_threads(cores)
    kw = dict(WORKLOAD)
    kw.pop("resonant")
    ph = po.make_phys(n_steps=z_steps, **{k: v for k, v in kw.items()})
    st = po.Setup(ph)
    api = st.api_complex()
    s0 = po.noise(1, 1e-6, api.size).reshape(api.shape)
    t0 = time.perf_counter()
    po.single_pass(st, api, s0, np.zeros_like(s0))
    dt = time.perf_counter() - t0
    return {"value": V * z_steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{z_steps} split steps (RK4 x2, dispersion, diffraction) of the 128x128x256 "
                      f"grid in FP64, {dt:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_c2_fp32asis")
    steps, warm = max(1, args.steps), max(0, args.warmup)
    if os.path.exists(binary):
        a = dict(mode="time_opo", crystal="ppln", LX=800, LY=800, Lcr=20000, T=27, Lambda=6.97,
                 lp=0.532, ls=1.064, Rs=0.98, gdd=0.0, P=5, FWHM=2, w0=60, focal=10000, twin=40,
                 pump="focused-pulsed", alpha_p=2e-7, alpha_s=2e-7, alpha_i=2e-7, resonant=2, steps=steps,
                 warmup=warm)
        cmd = [binary] + [f"{k}={v}" for k, v in a.items()]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=1700)
        rec = None
        for ln in p.stdout.splitlines():
            if ln.startswith("{\"rh_time_opo\""):
                rec = json.loads(ln)
        if rec is None:
            print(json.dumps({"impl": "reference", "unavailable": f"reference build failed rc={p.returncode}"}))
            return
        value = rec["voxel_steps_per_s"]
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": steps,
                "warmup": warm, "ms_per_step": rec["ms_per_round_trip"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "impl": "reference",
                "data": "synthetic (zero-initialised fields, analytic pump)",
                "config": {"workload": WORKLOAD_NAME, "grid": [128, 128, 256], "z_steps": rec["nsteps"],
                           "precision": "fp32 complex64 (as shipped)",
                           "build": "reference headers unmodified, grid constants 128x128x256 NZ=100, "
                                    "nvcc -O3 sm_100a, cuFFT; run as its round-trip member sequence"},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": 0, "kind": "reference",
                                 "sample": f"{steps} cavity round trips of the reference's own cuFFT "
                                           "pipeline on the B200 (the reference has no CPU path)"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    cb = cpu_baseline()
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": 0, "steps": 1, "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "impl": "reference", "data": "synthetic", "config": {"workload": WORKLOAD_NAME},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Pinned kernel configurations of the bench workload (the autotuner's choices on a B200),
# for profiling runs whose launch order must not depend on a timing-based choice.
PINNED_TUNING = {
    # t: the line-specialised t-pass (its fallback radix + the line flag 256)
    "fp32": {"t": dict(threads=128, tile=2048, r1=16 + 256), "x": dict(threads=128, tile=2048, r1=8),
             "y": dict(threads=128, tile=2048, r1=16)},
    "fp64": {"t": dict(threads=128, tile=1024, r1=4 + 256), "x": dict(threads=160, tile=1024, r1=8),
             "y": dict(threads=160, tile=1024, r1=8)},
}


def profile_workload(precision, round_trips, plane=0, grid=None):
    """The bench workload with a pinned kernel configuration and no timing, for profilers:
    4 field-conversion kernels (fields uploaded from FP64 host arrays), then per round trip
    n t-passes, n x- and y-passes, the closing t-pass and the free-space x'/y' passes
    (3n + 3 launches; with plane = K the x and y passes are one plane pass: 2n + 2)."""
    import cuopo3d_b200 as co
    prec = co.FP64 if precision == "fp64" else co.FP32
    kw = dict(WORKLOAD)
    if grid:  # a smaller grid of the same physics (tile geometry as long as nx >= the tile's pixels)
        kw.update(nx=grid[0], ny=grid[1], nt=grid[2])
    cfg = co.make_config(precision=prec, **kw)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning(PINNED_TUNING[precision])
    sim.set_plane_pass(plane)
    api = co.pump_field(cfg)
    s0 = co.noise(1, 1e-6 * float(np.max(np.abs(api))), api.size).reshape(api.shape)
    upload(co, sim, api, s0)
    sim.run_round_trips(round_trips)
    sim.synchronize()
    print("ok", sim.kernel_launches, sim.tuning)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile-passes", choices=("fp32", "fp64"),
                    help="run the workload with the pinned kernel configuration, untimed (for profilers)")
    ap.add_argument("--round-trips", type=int, default=1, help="round trips of --profile-passes")
    ap.add_argument("--plane", type=int, default=0, help="--profile-passes: plane-pass cluster size (0: x and y)")
    ap.add_argument("--profile-grid", type=int, nargs=3, metavar=("NX", "NY", "NT"),
                    help="--profile-passes: grid (default: the workload's 128 128 256)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched, served and precision legs")
    ap.add_argument("--batched-instances", type=int, default=64, help="instances of the batched leg (per rank)")
    ap.add_argument("--served-requests", type=int, default=12, help="requests of the FP32 served leg's sample")
    ap.add_argument("--served-requests-fp64", type=int, default=6, help="requests of the FP64 served leg's sample")
    ap.add_argument("--writer", action="store_true", help="time the output writer on a 128x128x2048 field")
    args = ap.parse_args()
    if args.profile_passes:
        profile_workload(args.profile_passes, args.round_trips, args.plane, args.profile_grid)
        return
    args.warmup = max(3, args.warmup) if args.impl == "ours" else args.warmup
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
