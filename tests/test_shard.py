"""Job sharding for batched / serving workloads (CPU; world_size 2 over gloo)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_assign_is_a_partition_and_balanced():
    from gpuintersector import shard

    rng = np.random.default_rng(4)
    tris = np.exp(rng.uniform(np.log(1e3), np.log(2e5), size=(4096, 2)))
    costs = [shard.job_cost(a, b) for a, b in tris]
    for world in (1, 2, 3, 8):
        parts = shard.assign(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        ld = shard.loads(costs, parts)
        # LPT bound: max load <= mean + largest job
        assert max(ld) <= sum(costs) / world + max(costs) + 1e-6
    assert shard.assign([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.assign([1.0], 0)


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist
    from gpuintersector import shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # a stand-in executor: the result of a job is a function of its index and the rank
        res = shard.run_sharded(costs, lambda idx: {i: (i * i, rank) for i in idx}, rank, world, dist)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_run_sharded_gloo_world2():
    import torch.multiprocessing as mp
    from gpuintersector import shard

    costs = [float(c) for c in np.random.default_rng(1).integers(1, 100, 37)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[1] is None
    merged = out[0]
    parts = shard.assign(costs, 2)
    assert sorted(merged) == list(range(len(costs)))
    for r, part in enumerate(parts):
        for i in part:
            assert merged[i] == (i * i, r)
