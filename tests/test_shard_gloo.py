"""Multi-rank path on CPU: gloo ranks shard independent OPO instances (no data-path
collective), reduce the slowest time and the total work, and gather the results on
rank 0.  The instances are real: every rank runs its share through the FP64 oracle (the
GPU library is not available on CPU ranks), and the gathered results must equal a
one-rank run of the same instances bit for bit."""
import os
import socket
import time

import numpy as np
import pytest
import torch.multiprocessing as mp

from cuopo3d_b200 import shard

# small instances with uneven grids and pumps: (nx, ny, nt, P, seed, round trips)
SPECS = [(8, 8, 16, 300.0, 1, 2), (16, 8, 16, 150.0, 2, 1), (8, 8, 32, 500.0, 3, 3), (12, 12, 24, 80.0, 4, 2),
         (8, 16, 16, 220.0, 5, 1), (16, 16, 32, 400.0, 6, 2), (8, 8, 16, 60.0, 7, 3)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def run_instance(spec):
    """One OPO instance through the FP64 oracle: powers and a field checksum after its
    round trips."""
    from oracle import pyoracle as po
    nx, ny, nt, P, seed, nrt = spec
    st = po.Setup(po.make_phys(nx=nx, ny=ny, nt=nt, nz=3, LX=300.0, LY=300.0, Lcr=3000.0, P=P, w0=40.0, FWHM=3.0,
                               t_window=25.0, pump_mode="focused-pulsed", total_rt=nrt))
    api = st.api_complex()
    s0 = po.noise(seed, 0.02, api.size).reshape(api.shape)
    ap, as_, ai = po.round_trips(st, api, api, s0, np.zeros_like(s0), nrt)
    return {"power": [float(np.sum(np.abs(f) ** 2)) for f in (ap, as_, ai)],
            "checksum": complex(np.sum(as_ * np.arange(as_.size).reshape(as_.shape)))}


class _Cfg:
    """Stand-in for OpoConfig with the fields request_cost reads."""

    def __init__(self, spec):
        self.nx, self.ny, self.nt, _, _, self.total_rt = spec


def serve_share(specs_by_index):
    """A rank's share of the served form: each request run to its round-trip bound (the
    oracle stands in for the GPU batch), with the per-request result fields of
    cuopo3d_b200.serve."""
    def run(reqs):
        t0 = time.perf_counter()
        res, vs = [], 0.0
        for r in reqs:
            spec = specs_by_index[r["index"]]
            out = run_instance(spec)
            res.append({"status": 0, "round_trips": spec[5], "latency_s": time.perf_counter() - t0,
                        "power": out["power"]})
            vs += spec[0] * spec[1] * spec[2] * 3 * spec[5]
        return res, {"wall_s": time.perf_counter() - t0, "voxel_steps": vs}
    return run


def _worker(rank, world, port, outdir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        costs = [s[0] * s[1] * s[2] * s[5] for s in SPECS]
        res = shard.sweep(costs, lambda k: dict(run_instance(SPECS[k]), rank=rank), rank, world)
        slowest = shard.reduce_scalar(1.0 + rank, "max")
        total = shard.reduce_scalar(sum(costs[k] for k in shard.local_indices(costs, rank, world)), "sum")
        reqs = [{"cfg": _Cfg(s), "index": k} for k, s in enumerate(SPECS)]
        served, st = shard.serve_sharded(reqs, serve_share(SPECS), rank, world)
        shard.barrier()
        with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as f:
            f.write(repr((res, slowest, total, served, st)))
    finally:
        dist.destroy_process_group()


def test_assign_balances_and_covers():
    costs = [4.19e6, 5.2e5, 1.77e6, 4.19e6, 5.2e5, 1.77e6, 1.0e5]
    owner = shard.assign(costs, 2)
    assert sorted(shard.local_indices(costs, 0, 2) + shard.local_indices(costs, 1, 2)) == list(range(7))
    loads = [sum(c for c, r in zip(costs, owner) if r == k) for k in range(2)]
    assert max(loads) / min(loads) < 1.2


def test_two_gloo_ranks_run_real_instances(tmp_path):
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    res0, slowest0, total0, served0, st0 = eval(open(tmp_path / "rank0.txt").read())
    res1, slowest1, total1, served1, st1 = eval(open(tmp_path / "rank1.txt").read())
    assert res1 is None and served1 is None
    assert sorted(res0) == list(range(len(SPECS)))
    assert {res0[k]["rank"] for k in res0} == {0, 1}  # both ranks ran instances
    one_rank = [run_instance(s) for s in SPECS]
    for k, ref in enumerate(one_rank):
        assert res0[k]["power"] == ref["power"] and res0[k]["checksum"] == ref["checksum"]
    assert slowest0 == slowest1 == 2.0
    assert total0 == total1 == pytest.approx(sum(s[0] * s[1] * s[2] * s[5] for s in SPECS))
    # served form over two ranks: results in request order, equal to the one-rank run
    assert [r["power"] for r in served0] == [ref["power"] for ref in one_rank]
    assert st0["completed"] == len(SPECS) and st0["ranks"] == 2
    assert st0["voxel_steps"] == pytest.approx(sum(s[0] * s[1] * s[2] * 3 * s[5] for s in SPECS))
    assert st0["p99_latency_s"] >= st0["p50_latency_s"] > 0
