"""Host logic of the multi-GPU path: one process per GPU, independent work
per rank (replicas of one system, or a share of an ensemble), no collective
on the data path.

The only collectives are the timing reduction (max over ranks) and
barriers, which work on any torch.distributed backend (NCCL on GPUs, gloo in
the CPU tests).
"""
import heapq


def lpt_partition(costs, world):
    """Longest-processing-time-first assignment of independent items
    (cost = D^2 for ensemble instances) to `world` ranks.  Returns one list
    of item indices per rank, each in decreasing cost order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return out


def max_over_ranks(values, device=None):
    """Element-wise maximum of a list of floats over all ranks (identity
    without an initialised process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]
