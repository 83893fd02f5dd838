"""Multi-rank host logic on CPU (gloo, world size 2): the LPT partition of
ensemble instances and the max-over-ranks timing reduction used by
bench.py --gpus N."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from quac_b200.replicas import lpt_partition, max_over_ranks


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(4)
    costs = (2 * rng.integers(5, 41, size=4096)) ** 2
    parts = lpt_partition(costs, 4)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(4096))
    loads = [costs[p].sum() for p in map(np.array, parts)]
    assert max(loads) - min(loads) <= costs.max()


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = max_over_ranks([10.0 * (rank + 1), -rank])
        parts = lpt_partition([9, 7, 5, 3, 1], world)
        dist.barrier()
        q.put((rank, got, parts[rank]))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] == [20.0, 0.0] and res[1][1] == [20.0, 0.0]
    assert sorted(res[0][2] + res[1][2]) == [0, 1, 2, 3, 4]


def test_config4_ensemble_shards():
    """The sharded ensemble of bench.py --gpus N: the 4096 driven-JC
    instances split over 2, 4 and 8 ranks, each instance once, the D^2
    loads within one instance of each other."""
    from quac_b200 import systems as Sy
    params = Sy.driven_jc_ensemble_params(4096)
    costs = np.array([(2 * p["nc"]) ** 2 for p in params])
    for world in (2, 4, 8):
        parts = lpt_partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(4096))
        loads = [costs[np.array(p)].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max()
        assert all(costs[p[k]] >= costs[p[k + 1]] for p in parts for k in range(len(p) - 1))
