"""The multi-rank host logic on CPU with world_size 2 over gloo: the bench's
max/sum reductions over ranks and the ensemble's bin-packing of replicas over
GPUs (every replica on exactly one rank, loads balanced)."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "md-bench_b200")]
    import datetime

    import bench
    import workloads as W
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        secs = 1.5 + rank
        mx = bench.reduce_scalar(torch, dist, secs, "max", "cpu")
        sm = bench.reduce_scalar(torch, dist, 10.0 * (rank + 1), "sum", "cpu")
        sizes = [4 * n ** 3 for n, _, _ in W.c4_replicas(256)]
        mine = W.assign_replicas(sizes, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, mine)
        loads = [sum(sizes[i] for i in g) for g in got]
        q.put((rank, mx, sm, sorted(i for g in got for i in g), loads, max(sizes)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_rank_reductions_and_replica_packing():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=150) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm, allidx, loads, biggest in res:
        assert mx == 2.5 and sm == 30.0
        assert allidx == list(range(256))
        assert max(loads) - min(loads) <= biggest
