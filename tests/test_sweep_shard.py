"""CPU tests of the multi-GPU host logic of the batched sweep: every rank
takes its shard of the solves (workloads.sweep_shard, no data exchange) and
the job time is the maximum over ranks; world size 2 over gloo."""
import os
import socket

import pytest

from mpdpft_b200 import workloads as W


def test_sweep_shard_partition():
    count = 256
    loads = {}
    for world in (1, 2, 4, 8):
        shards = [W.sweep_shard(count, r, world) for r in range(world)]
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(count))
        load = [sum(W.sweep_steps(i) ** 2 for i in sh) for sh in shards]
        loads[world] = load
        assert max(load) <= sum(load) / world + 512 ** 2  # LPT: within one largest solve
    assert loads[1][0] == sum(W.sweep_steps(i) ** 2 for i in range(count))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = W.sweep_shard(64, rank, world)
        got = [None] * world
        dist.all_gather_object(got, mine)
        t = torch.tensor([1.0 + rank], dtype=torch.float64)  # this rank's time
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, got, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_sweep_shard_gloo_two_ranks():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, tmax in out:
        flat = sorted(i for sh in got for i in sh)
        assert flat == list(range(64))
        assert not set(got[0]) & set(got[1])
        assert tmax == 2.0
