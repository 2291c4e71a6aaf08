"""Multi-process paths on CPU (gloo, world size 2): shard assignment, the final
gather of per-design results in global order, and the gradient average of
data-parallel surrogate training. No GPU: the per-design work is the oracle."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from diffractiveopticalelement_b200.sharding import (allreduce_mean_, design_cost, gather_results, my_shard,
                                                     shard_by_cost)


def test_shard_by_cost_is_contiguous_and_balanced():
    rng = np.random.default_rng(0)
    sizes = rng.choice([128, 256, 512, 1024], size=512, p=[0.4, 0.3, 0.2, 0.1])
    costs = [design_cost(int(n), 200) for n in sizes]
    for world in (1, 2, 3, 4, 8):
        sh = shard_by_cost(costs, world)
        assert sh[0][0] == 0 and sh[-1][1] == len(costs)
        assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
        loads = [sum(costs[a:b]) for a, b in sh]
        # every boundary is within one unit of its ideal position
        assert max(loads) - sum(costs) / world <= max(costs) + 1e-6
    assert shard_by_cost([], 3) == [(0, 0)] * 3
    assert shard_by_cost([1.0], 4)[0] in [(0, 1), (0, 0)]
    with pytest.raises(ValueError):
        shard_by_cost([1, -1], 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        n, D = 32, 6
        costs = [design_cost(n, 3)] * D
        a, b = my_shard(costs, rank, world)
        ill = O.disc_mask(n, n, 8e-6, 8e-6, 0.45 * n * 8e-6, 16e-6)
        res = []
        for k in range(a, b):
            i = np.arange(n)
            X, Y = np.meshgrid(i, i)
            t = (np.hypot(X - n / 2, Y - n / 2) <= 4 + k).astype(float).ravel()
            r = O.design("wgs", ill, O.prepare_target(t, ill), nx=n, ny=n, dx=8e-6, iterations=3,
                         init_phase=O.random_phase(n, n, 10 + k))
            res.append([r["rmse"], r["error"][-1]])
        local = torch.tensor(np.array(res).reshape(-1, 2), dtype=torch.float64)
        counts = [e - s for s, e in (my_shard(costs, q, world) for q in range(world))]
        full = gather_results(local, rank, world, counts)
        g = torch.full((5,), float(rank + 1), dtype=torch.float32)
        allreduce_mean_(g, world)
        if rank == 0:
            out.put((full.numpy(), g.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_and_gradient_average():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    full, g = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # the same six designs in one process
    from oracle import oracle as O
    n = 32
    ill = O.disc_mask(n, n, 8e-6, 8e-6, 0.45 * n * 8e-6, 16e-6)
    want = []
    for k in range(6):
        i = np.arange(n)
        X, Y = np.meshgrid(i, i)
        t = (np.hypot(X - n / 2, Y - n / 2) <= 4 + k).astype(float).ravel()
        r = O.design("wgs", ill, O.prepare_target(t, ill), nx=n, ny=n, dx=8e-6, iterations=3,
                     init_phase=O.random_phase(n, n, 10 + k))
        want.append([r["rmse"], r["error"][-1]])
    assert np.array_equal(full, np.array(want))
    assert np.allclose(g, 1.5)
