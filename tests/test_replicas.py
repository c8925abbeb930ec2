"""Replicas-only multi-process path on CPU (gloo, world size 2): shards are
disjoint and cover every system, and the host-side reductions reassemble the
single-process result exactly (systems are independent)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from wind_b200 import replicas


@pytest.mark.parametrize("nsys,world", [(10, 2), (7, 3), (1, 2), (0, 2), (65536, 8)])
def test_shards_partition(nsys, world):
    seen = []
    for r in range(world):
        b, e = replicas.shard_range(nsys, r, world)
        seen.extend(range(b, e))
        assert e - b in (nsys // world, nsys // world + 1)
    assert seen == list(range(nsys))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from oracle import pyoracle as O
    from wind_b200 import networks as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    wl = W.workload_katz96(40, seed=5)
    mine = replicas.shard(wl, rank, world)
    y = mine.y0.copy()
    tot, _, _ = O.restated(mine.net, y, 0.0, 1e11, 1e-6, 1e-5, "sie", "device")
    full = replicas.gather_states(y, wl.net.nsys, rank, world, dist)
    total = replicas.reduce_sum(tot, dist)
    tmax = replicas.reduce_max(float(rank + 1), dist)
    if rank == 0:
        q.put((full, total, tmax))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_replicas_match_single_process():
    from oracle import pyoracle as O
    from wind_b200 import networks as W
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, total, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    wl = W.workload_katz96(40, seed=5)
    y = wl.y0.copy()
    tot1, _, _ = O.restated(wl.net, y, 0.0, 1e11, 1e-6, 1e-5, "sie", "device")
    assert np.array_equal(full, y)
    assert total == tot1
    assert tmax == 2.0
