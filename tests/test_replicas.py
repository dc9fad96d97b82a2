"""Multi-GPU replica logic on CPU: two gloo ranks (spawned processes) agree on
the item assignment without communicating, and the timing reduction returns
the max over ranks."""
import os
import socket

import pytest

from kahip_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, _ = replicas.rank_env()
        mine = replicas.shard_items(sizes, r, w)
        t = replicas.max_over_ranks(10.0 * (rank + 1))
        dist.barrier()
        out.put((rank, mine, t, replicas.member_seed(7, r, w)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    sizes = [5, 100, 3, 3, 77, 50, 50, 1, 0, 64]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0, s0), (r1, m1, t1, s1) = res
    assert sorted(m0 + m1) == list(range(len(sizes))) and not set(m0) & set(m1)
    assert t0 == t1 == 20.0
    assert s0 != s1
    w0, w1 = sum(sizes[i] for i in m0), sum(sizes[i] for i in m1)
    assert abs(w0 - w1) <= max(sizes)


def test_single_process_defaults():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.shard_items([4, 2, 9], 0, 1) == [0, 1, 2]
    assert replicas.member_seed(3, 1, 4) == 13
