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


# --- One frame's samples over the ranks ------------------------------------
# The random stream of a path is keyed by (ray, the frame's sample index,
# bounce), and a render of samples [f, f + n) of a frame (first_sample = f)
# traces exactly the paths of those samples of one whole-frame render. So a
# frame can be split by samples over N GPUs with one exchange step: the sum
# of the per-ray radiance accumulators (w*h*ss^2 * 3 floats), after which
# any rank resolves the image.

def spp_slices(spp, world):
    """Samples [0, spp) in `world` contiguous slices, the first spp % world
    ranks taking one more: a list of (first_sample, count) per rank (count 0
    for a rank with nothing to render)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if spp < 1:
        raise ValueError("spp must be >= 1")
    base, extra = divmod(int(spp), world)
    out, first = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((first, n))
        first += n
    return out


def split_spp_accum(render_slice, spp, rays, rank, world, device="cuda"):
    """This rank's slice of a frame's samples, summed over the ranks.

    render_slice(first, count) renders samples [first, first + count) and
    returns their (rays, 3) float32 accumulator; it is not called for an
    empty slice. The accumulators are added with one all-reduce over the
    process group (NCCL between GPUs, gloo on CPU); every rank returns the
    frame's (rays, 3) sum."""
    import numpy as np
    first, count = spp_slices(spp, world)[rank]
    acc = (np.asarray(render_slice(first, count), np.float32).reshape(rays, 3)
           if count > 0 else np.zeros((rays, 3), np.float32))
    if world == 1:
        return acc
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(acc)).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def render_split_spp(scene, camera, params, rank, world, device="cuda"):
    """One frame (hpt_render_params `params`) with its samples split over the
    ranks: each rank renders its slice on its own GPU (`scene` lives there),
    the accumulators are summed with one all-reduce and the image is resolved
    from the sum. Returns (rgba, accum) of the whole frame on every rank.
    The sum equals one render of all the samples up to float32 rounding of
    the per-ray accumulators (the renders add radiance in 2^-32 fixed point
    and hand out float32 sums)."""
    import ctypes

    import hptracing_b200 as H
    rays = (params.sample_x * params.supersample_x * params.sample_y * params.supersample_y)

    def render_slice(first, count):
        p = H.RenderParams()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(params), ctypes.sizeof(p))
        p.sample = count
        p.first_sample = params.first_sample + first
        return scene.render(camera, p, want_accum=True)[1]

    acc = split_spp_accum(render_slice, params.sample, rays, rank, world, device)
    rgba = H.resolve(acc, params.sample_x, params.sample_y, params.supersample_x,
                     params.supersample_y, params.sample, params.brightness)
    return rgba, acc
