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


def sweep(costs, run_one, rank=0, world=1):
    """Run instance k (run_one(k) -> picklable result) for every k this rank owns and
    gather {k: result} of all ranks on rank 0 (None elsewhere)."""
    mine = {k: run_one(k) for k in local_indices(costs, rank, world)}
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
