"""Host logic of the multi-GPU path, on CPU with the gloo backend and
world size 2: batch sharding (uniform and cost-balanced uneven) and the
max-over-ranks timing reduction that bench.py uses."""
import os
import socket

import numpy as np
import pytest


def test_shard_range_partitions_batch():
    from eigeng_b200.multi import shard_range
    for L in (1, 7, 8, 4096, 10001):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                s, c = shard_range(L, r, world)
                seen.extend(range(s, s + c))
            assert seen == list(range(L))


def test_shard_uneven_balances_cost():
    from eigeng_b200.multi import shard_uneven
    rng = np.random.default_rng(0)
    ns = rng.integers(8, 513, size=1000)
    for world in (2, 4, 8):
        parts = shard_uneven(ns, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(ns)))
        loads = [sum(int(ns[i]) ** 3 for i in p) for p in parts]
        assert max(loads) / min(loads) < 1.05


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from eigeng_b200.multi import max_over_ranks, shard_range
    start, count = shard_range(11, rank, world)
    m = max_over_ranks(10.0 + rank * 5.0)
    out.put((rank, start, count, m))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import multiprocessing as mp
    import sys
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "eigeng-batched_b200"))
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1:] == (0, 6, 15.0) and res[1][1:] == (6, 5, 15.0)
