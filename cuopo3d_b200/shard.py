"""Multi-GPU sharding of independent OPO instances (sweep points, requests).

Instances never exchange data, so ranks share no collective on the data path: each
rank runs its own share (one process per GPU), and only scalars cross ranks -- the
slowest rank's time, the total voxel-steps, and the per-instance results gathered on
rank 0.  Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU).
"""
import heapq


def assign(costs, world):
    """Rank of each instance: longest-processing-time-first over `world` ranks, so
    that the largest instances are spread first and the loads stay balanced."""
    order = sorted(range(len(costs)), key=lambda k: -costs[k])
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * len(costs)
    for k in order:
        load, r = heapq.heappop(heap)
        owner[k] = r
        heapq.heappush(heap, (load + float(costs[k]), r))
    return owner


def local_indices(costs, rank, world):
    owner = assign(costs, world)
    return [k for k, r in enumerate(owner) if r == rank]


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def _device_for(dist):
    import torch
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def reduce_scalar(x, op="max"):
    """x reduced over ranks (max or sum); x itself on a single process."""
    dist = _dist()
    if dist is None or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def barrier():
    dist = _dist()
    if dist is not None and dist.get_world_size() > 1:
        dist.barrier()


def _gather_dict(mine, rank, world):
    dist = _dist()
    if dist is None or world == 1:
        return mine
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0)
    if rank != 0:
        return None
    out = {}
    for part in gathered:
        out.update(part)
    return out


def sweep(costs, run_one, rank=0, world=1):
    """Run instance k (run_one(k) -> picklable result) for every k this rank owns and
    gather {k: result} of all ranks on rank 0 (None elsewhere)."""
    mine = {k: run_one(k) for k in local_indices(costs, rank, world)}
    return _gather_dict(mine, rank, world)


def request_cost(req):
    """Work of a served request: voxels x its round-trip bound (the z-steps of the
    instances that share a batch are equal)."""
    c = req["cfg"]
    return float(c.nx) * c.ny * c.nt * max(1, c.total_rt)


def _percentile(v, q):
    if not v:
        return 0.0
    v = sorted(v)
    pos = q * (len(v) - 1)
    lo = int(pos)
    hi = min(lo + 1, len(v) - 1)
    return v[lo] + (pos - lo) * (v[hi] - v[lo])


def serve_sharded(requests, run_share, rank=0, world=1):
    """The served form on `world` GPUs: requests are assigned to ranks by
    longest-processing-time first on request_cost, each rank serves its share with
    run_share(list of requests) -> (results, stats) (cuopo3d_b200.serve on its own GPU,
    continuous batching within the rank), and rank 0 gets the results in request order
    and the job's stats: wall = the slowest rank's, voxel-steps summed, p50 / p99 over
    all requests' latencies.  No data crosses ranks but the results."""
    costs = [request_cost(r) for r in requests]
    mine = local_indices(costs, rank, world)
    res, st = run_share([requests[k] for k in mine]) if mine else ([], {"wall_s": 0.0, "voxel_steps": 0.0})
    wall = reduce_scalar(st.get("wall_s", 0.0), "max")
    vsteps = reduce_scalar(st.get("voxel_steps", 0.0), "sum")
    allres = _gather_dict({k: r for k, r in zip(mine, res)}, rank, world)
    if allres is None:
        return None, None
    ordered = [allres[k] for k in range(len(requests))]
    lat = [r["latency_s"] for r in ordered if r["status"] == 0]
    stats = {"p50_latency_s": _percentile(lat, 0.5), "p99_latency_s": _percentile(lat, 0.99), "wall_s": wall,
             "voxel_steps": vsteps, "voxel_steps_per_s": vsteps / wall if wall > 0 else 0.0,
             "completed": len(lat), "ranks": world}
    return ordered, stats
