"""Host-side sharding of render work over ranks (one process per GPU).

The path has no data exchange: jobs (and requests) are independent, so N
GPUs run N independent wavefronts. What the ranks share is the assignment of
jobs to ranks, which every rank computes identically from the same job list,
and the final reduction of timings and counters. Nothing here touches a
device buffer; the reductions use whatever backend the process group has
(NCCL between GPUs, gloo on CPU).
"""
import heapq


def job_cost(rays, spp, depth):
    """Estimated intersect queries of a job: rays x spp x (1 + depth / 2)."""
    return float(rays) * spp * (1.0 + 0.5 * depth)


def assign_jobs(costs, world):
    """Longest-processing-time-first assignment of jobs to `world` ranks.

    Jobs are taken in decreasing cost (ties by index) and each goes to the
    rank with the least assigned cost (ties by rank). Deterministic, so every
    rank computes the same table. Returns one list of job indices per rank,
    each in increasing index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(x) for x in out]


def _reduce(x, op, world, device):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def allreduce_max(x, world, device="cuda"):
    """Maximum of x over the ranks (each rank passes its own value)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX if world > 1 else None, world, device)


def allreduce_sum(x, world, device="cuda"):
    """Sum of x over the ranks."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM if world > 1 else None, world, device)
