"""Benchmark of the split-step OPO solver on B200 GPUs (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the singly-resonant OPO at full size -- PPLN 20 mm, 128 x 128 x 256 grid over
800 um / 40 ps, 100 z-slices (100 split steps per crystal pass), GVD and group-velocity
mismatch on, absorption 0.002/cm, signal mirror R = 0.98, detuning 0, 60 um / 5 W / 2 ps
Gaussian pump, noise-seeded signal, FP64 fields.  One step = one cavity round trip
(100 z-steps of 4,194,304 voxels).  The metric is voxel-steps/s (one voxel of all three
fields advanced through one full split step); `value` is device-timed with inputs
resident; `e2e` runs every step through the C-ABI from pinned host buffers (inputs up, one
round trip, signal down), two solvers alternating so that host copies overlap compute.

Multi-GPU: every rank runs its own independent instance (weak scaling, no collective on
the data path); value = all ranks' voxel-steps / the slowest rank's time.

`--impl reference` times the reference's own cuFFT pipeline (its headers compiled by
oracle/refharness into oracle/_ref/, unmodified code path, FP32 as shipped) on the same
GPU; without that build it times the FP64 CPU oracle on the host cores instead.
"""
import argparse
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
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


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


def run_ours(args):
    import torch
    import cuopo3d_b200 as co
    rank, world, local = dist_setup(args.gpus)
    V = 128 * 128 * 256
    out = {}
    hbm, hbm_kind = hbm_peak()
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
        # End to end through the C-ABI: every step uploads its three input fields from pinned
        # host memory, runs one round trip and reads its signal back to pinned host memory.
        # Two solvers alternate (step k on solver k % 2): step k+1's uploads and round trip
        # are enqueued before step k's result is read, so one solver's host copies run on
        # the copy engines while the other's round trip runs on the SMs.
        pin = {k: torch.from_numpy(np.ascontiguousarray(a, dtype=np.complex128).reshape(-1)).pin_memory()
               for k, a in (("api", api), ("s", s0), ("i", np.zeros_like(s0)))}
        _, w2 = co.time_freq(cfg.nt, params.t_window)
        sim2 = co.Simulation(params, w2)
        sim2.autotune()  # cached: the same configuration as sim
        upload(co, sim2, api, s0)
        sims = (sim, sim2)
        res = [torch.empty(V, dtype=torch.complex128).pin_memory() for _ in sims]
        lib = co.lib()
        import ctypes

        def enqueue(k):
            h = sims[k % 2].handle
            for which, t in ((co.FIELD_API, pin["api"]), (co.FIELD_AS, pin["s"]), (co.FIELD_AI, pin["i"])):
                rc = lib.opo_set_field(h, which, ctypes.c_void_p(t.data_ptr()), co.MEM_HOST, co.FP64)
                assert rc == 0
            sims[k % 2].run_round_trips(1)

        def collect(k):
            rc = lib.opo_get_field(sims[k % 2].handle, co.FIELD_AS, ctypes.c_void_p(res[k % 2].data_ptr()),
                                   co.MEM_HOST, co.FP64)
            assert rc == 0

        enqueue(0)
        enqueue(1)
        collect(0)
        collect(1)
        e2e_steps = max(4, args.steps // 2)
        barrier_sync(world)
        t0 = time.perf_counter()
        enqueue(0)
        for k in range(e2e_steps):
            if k + 1 < e2e_steps:
                enqueue(k + 1)
            collect(k)
        barrier_sync(world)
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
        e2e_value = sum_over_ranks(float(V) * nsteps * e2e_steps, world) / e2e_s
        sim2.close()
        out[tag] = dict(value=value, ms_per_step=ms / args.steps, launches=launches, passes=passes,
                        tuning=sim.tuning,
                        clocks=clk.summary(), nsteps=nsteps,
                        e2e=dict(value=e2e_value, unit=UNIT, h2d_bytes_per_step=3 * V * 16,
                                 d2h_bytes_per_step=V * 16))
        sim.close()
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
            "gpu_launches": main["launches"],
            "clocks": main["clocks"],
            "roofline": {"bound": "hbm", "kernel": "tpass_kernel<double2> (RK4 x2 + t-axis FFT pair)",
                         "achieved": achieved, "peak": hbm,
                         "peak_kind": f"{hbm_kind} (MEASURED_PEAKS.json hbm_gbs)" if hbm_kind == "measured" else "fallback",
                         "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                         "traffic": ncu_traffic("tpass", "fp64"),
                         "alg_bytes_per_launch": V * 96},
            "roofline_fp64_pipe": {"bound": "fp64", "kernel": "tpass_kernel<double2>", "achieved": ach_tf,
                                   "peak": fp64_peak, "peak_kind": "measured (opo_fp64_peak: FMA chains)",
                                   "unit": "TFLOP/s", "frac": (ach_tf / fp64_peak) if ach_tf else None,
                                   "alg_flops_per_launch": flops_t},
            "passes_fp64": main["passes"],
            "tuning_fp64": main["tuning"],
            "fp32": {"value": out["fp32"]["value"], "ms_per_step": out["fp32"]["ms_per_step"],
                     "passes": out["fp32"]["passes"], "e2e": out["fp32"]["e2e"],
                     "clocks": out["fp32"]["clocks"], "tuning": out["fp32"]["tuning"]},
        }
        if not args.no_forms:
            tun = out["fp32"]["tuning"]
            line["batched"] = batched_leg(co, tun, n_inst=args.batched_instances)
            # arrival rate at ~85 % of capacity: throughput / mean work of a request
            mean_vox = (64 * 64 * 128 + 128 * 128 * 256 + 96 * 96 * 192) / 3.0
            rate = 0.85 * line["batched"]["value"] / (mean_vox * 100 * 15)
            line["served"] = served_leg(co, tun, rate, n_req=args.served_requests)
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def batched_leg(co, tuning, n_inst=64, warm=1, steps=3, seed=2024):
    """Batched form: n_inst instances with grids drawn from N in {32, 64, 128} and
    NT in {64, 128, 256}, P log-uniform 0.5-20 W, waist U[30, 100] um, detuning U[-pi, pi],
    20 mm PPLN, 100 slices, FP32; one persistent launch per pass for all of them."""
    import torch
    rng = np.random.default_rng(seed)
    b = co.Batch(co.FP32, n_inst, 150 << 30, tuning=tuning)
    vox = 0
    for k in range(n_inst):
        N = int(rng.choice([32, 64, 128]))
        NT = int(rng.choice([64, 128, 256]))
        cfg = co.make_config(nx=N, ny=N, nt=NT, nz=100, LX=800.0, LY=800.0, Lcr=20000.0, t_window=40.0,
                             P=float(np.exp(rng.uniform(np.log(0.5), np.log(20.0)))),
                             w0=float(rng.uniform(30, 100)), detuning=float(rng.uniform(-np.pi, np.pi)),
                             FWHM=2.0, focal=10000.0, Rs=0.98, alpha=(2e-7, 2e-7, 2e-7), zloop_f32=1,
                             pump_mode="focused-pulsed", total_rt=200, precision=co.FP32)
        slot = b.add(cfg)
        b.init_fields(slot, cfg, 1000 + k, 1e-3)
        vox += N * N * NT
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
    return {"value": vox * 100.0 * steps / (ms * 1e-3), "unit": UNIT, "instances": n_inst,
            "voxels": vox, "round_trips_timed": steps, "ms_per_round_trip": ms / steps,
            "launches_per_round_trip": launches / steps, "precision": "fp32",
            "workload": f"{n_inst} instances, N in {{32,64,128}}, NT in {{64,128,256}}, 20 mm PPLN, 100 slices"}


def served_leg(co, tuning, rate_per_s, n_req=40, seed=7):
    """Served form, bounded sample of the request stream: n_req Poisson arrivals at
    rate_per_s, grids from {64^2x128, 128^2x256, 96^2x192}, P log-uniform 0.5-20 W,
    waist U[30, 100] um, 5-25 round trips (retired early when the signal power changes by
    less than 1e-6 over a round trip), 150 GB budget, FP32."""
    rng = np.random.default_rng(seed)
    grids = [(64, 128), (128, 256), (96, 192)]
    reqs, t = [], 0.0
    for k in range(n_req):
        t += float(rng.exponential(1.0 / rate_per_s))
        N, NT = grids[int(rng.integers(0, 3))]
        cfg = co.make_config(nx=N, ny=N, nt=NT, nz=100, LX=800.0, LY=800.0, Lcr=20000.0, t_window=40.0,
                             P=float(np.exp(rng.uniform(np.log(0.5), np.log(20.0)))),
                             w0=float(rng.uniform(30, 100)), FWHM=2.0, focal=10000.0, Rs=0.98,
                             alpha=(2e-7, 2e-7, 2e-7), zloop_f32=1, pump_mode="focused-pulsed",
                             total_rt=int(rng.integers(5, 26)), precision=co.FP32)
        reqs.append(dict(cfg=cfg, arrival_s=t, seed=5000 + k, noise_sigma=1e-3, tol=1e-6))
    res, st = co.serve(reqs, co.FP32, capacity=1024, hbm_budget=150 << 30, realtime=True, tuning=tuning)
    ok = sum(1 for r in res if r["status"] == co.OPO_OK)
    return {"p50_latency_s": st["p50_latency_s"], "p99_latency_s": st["p99_latency_s"],
            "value": st["voxel_steps_per_s"], "unit": UNIT, "requests": n_req, "completed": ok,
            "arrival_rate_per_s": rate_per_s, "wall_s": st["wall_s"], "max_resident": st["max_resident"],
            "precision": "fp32",
            "workload": "Poisson stream, grids {64^2x128, 128^2x256, 96^2x192}, 5-25 round trips, "
                        "early retirement at |dPs/Ps| < 1e-6, 150 GB budget"}


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
    V = 128 * 128 * 256
    return {"value": V * z_steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{z_steps} split steps (RK4 x2, dispersion, diffraction) of the 128x128x256 "
                      f"grid in FP64, {dt:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    binary = os.path.join(ROOT, "oracle", "_ref", "ref_c2_fp32asis")
    steps = max(1, min(args.steps, 5))
    warm = max(1, min(args.warmup, 1))
    if os.path.exists(binary):
        a = dict(mode="time_opo", crystal="ppln", LX=800, LY=800, Lcr=20000, T=27, Lambda=6.97,
                 lp=0.532, ls=1.064, Rs=0.98, gdd=0.0, P=5, FWHM=2, w0=60, focal=10000, twin=40,
                 pump="focused-pulsed", alpha_p=2e-7, alpha_s=2e-7, alpha_i=2e-7, steps=steps,
                 warmup=warm)
        cmd = [binary] + [f"{k}={v}" for k, v in a.items()]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=1200)
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and served legs")
    ap.add_argument("--batched-instances", type=int, default=64, help="instances of the batched leg")
    ap.add_argument("--served-requests", type=int, default=40, help="requests of the served leg's sample")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup) if args.impl == "ours" else args.warmup
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
