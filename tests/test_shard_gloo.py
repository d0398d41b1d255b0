"""Multi-rank path on CPU: two gloo ranks shard independent instances (no data-path
collective), reduce the slowest time and the total work, and gather results on rank 0."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from cuopo3d_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, costs, outdir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = shard.sweep(costs, lambda k: {"k": k, "rank": rank, "value": k * k}, rank, world)
        slowest = shard.reduce_scalar(1.0 + rank, "max")
        total = shard.reduce_scalar(sum(costs[k] for k in shard.local_indices(costs, rank, world)), "sum")
        shard.barrier()
        with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as f:
            f.write(repr((res, slowest, total)))
    finally:
        dist.destroy_process_group()


def test_assign_balances_and_covers():
    costs = [4.19e6, 5.2e5, 1.77e6, 4.19e6, 5.2e5, 1.77e6, 1.0e5]
    owner = shard.assign(costs, 2)
    assert sorted(shard.local_indices(costs, 0, 2) + shard.local_indices(costs, 1, 2)) == list(range(7))
    loads = [sum(c for c, r in zip(costs, owner) if r == k) for k in range(2)]
    assert max(loads) / min(loads) < 1.2


def test_two_gloo_ranks(tmp_path):
    costs = [3.0, 1.0, 2.0, 5.0, 1.5, 0.5, 4.0]
    mp.spawn(_worker, args=(2, _free_port(), costs, str(tmp_path)), nprocs=2, join=True)
    res0, slowest0, total0 = eval(open(tmp_path / "rank0.txt").read())
    res1, slowest1, total1 = eval(open(tmp_path / "rank1.txt").read())
    assert res1 is None
    assert sorted(res0) == list(range(len(costs)))
    assert all(res0[k]["value"] == k * k for k in res0)
    assert {res0[k]["rank"] for k in res0} == {0, 1}
    assert slowest0 == slowest1 == 2.0
    assert total0 == total1 == pytest.approx(sum(costs))
