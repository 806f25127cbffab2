"""Placement of independent embedding jobs on the GPUs of one node (one process per GPU).

Embeddings do not interact, so several GPUs run replicas: each rank takes a disjoint share of
the jobs and no collective touches the data path. The only collectives are the timing
reduction (the slowest rank's device time) and the result gather of the harness, both on the
host side of the work. Launch: one process per GPU under torch.distributed (NCCL on GPUs,
gloo on CPU); RANK / WORLD_SIZE / LOCAL_RANK come from the environment.
"""
import math
import os


def rank_world():
    """(rank, world, local_rank) from the launcher's environment (1 process when absent)."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def job_cost(n_points, n_iter=1000):
    """Relative cost of one embedding job: the per-iteration work is O(N) with an O(N log N)
    tree rebuild; the constant does not matter for the placement."""
    n = max(int(n_points), 2)
    return float(n_iter) * n * (1.0 + 0.05 * math.log2(n))


def shard(costs, world):
    """Deterministic longest-first placement of jobs on `world` ranks.

    Jobs are taken in decreasing cost (ties by index) and each goes to the rank with the least
    load so far (ties by rank). Returns one sorted list of job indices per rank; the lists
    partition range(len(costs)).
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += float(costs[i])
        out[r].append(i)
    return [sorted(x) for x in out]


def max_over_ranks(values, device=None):
    """Element-wise maximum of a list of floats over all ranks of the default process group
    (identity without one). Every rank must call it with the same length."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()
