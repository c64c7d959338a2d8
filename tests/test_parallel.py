"""The several-GPU logic on the host: the partition of a batch of independent
models over ranks, and the max-over-ranks timing, run as two gloo processes
on the CPU (no GPU involved)."""
import os
import socket

import numpy as np
import pytest

import helpers
from helpers import meshes
from dnlPython import parallel


def test_shards_cover_every_instance_once_and_balance():
    descs = meshes.taylor_batch(n=64, seed=3)
    costs = [parallel.instance_cost(d) for d in descs]
    for world in (1, 2, 3, 8):
        parts = parallel.shard_instances(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(descs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # longest-processing-time bound: no rank above the mean by more than the largest instance
        assert max(loads) <= np.mean(loads) + max(costs) + 1e-6
    assert parallel.shard_instances(costs, 4) == parallel.shard_instances(costs, 4)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        descs = meshes.taylor_batch(n=16, seed=9, elems=(300, 3000))
        costs = [parallel.instance_cost(d) for d in descs]
        mine = parallel.shard_instances(costs, world)[rank]
        work = sum(descs[i].n_elems for i in mine)
        total = parallel.reduce_sum(work, dist)
        slowest = parallel.reduce_max(1.0 + rank, dist)
        records = parallel.gather_records({i: {"elements": descs[i].n_elems, "rank": rank} for i in mine}, dist)
        out.put((rank, mine, total, slowest, records))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_a_batch():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    descs = meshes.taylor_batch(n=16, seed=9, elems=(300, 3000))
    assert sorted(res[0][1] + res[1][1]) == list(range(16)) and not set(res[0][1]) & set(res[1][1])
    assert res[0][2] == res[1][2] == sum(d.n_elems for d in descs)
    assert res[0][3] == res[1][3] == 2.0
    # every rank ends with every instance's record, each from the rank that ran it
    for r in res:
        assert sorted(r[4]) == list(range(16))
        assert all(r[4][i]["elements"] == descs[i].n_elems for i in range(16))
        assert all(r[4][i]["rank"] == (0 if i in res[0][1] else 1) for i in range(16))

