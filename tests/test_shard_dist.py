"""Sharding of render work over ranks: the assignment table and the
reductions, run as two gloo ranks on the CPU (no GPU)."""
import os
import socket

import pytest

from hptracing_b200 import shard


def test_assignment_is_balanced_complete_and_deterministic():
    costs = [shard.job_cost(r * r, spp, d) for r, spp, d in
             [(1024, 64, 10), (512, 64, 10), (128, 1, 3), (256, 16, 5), (512, 4, 8),
              (1024, 1, 3), (128, 64, 9), (256, 4, 4), (512, 16, 6), (128, 16, 7)]]
    for world in (1, 2, 3, 4, 8):
        table = shard.assign_jobs(costs, world)
        assert len(table) == world
        flat = sorted(i for part in table for i in part)
        assert flat == list(range(len(costs)))
        assert table == shard.assign_jobs(list(costs), world)
        loads = [sum(costs[i] for i in part) for part in table]
        # LPT bound: no rank carries more than the mean plus the largest job.
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-6
    # More ranks than jobs: the extra ranks get nothing.
    assert shard.assign_jobs([3.0, 1.0], 4) == [[0], [1], [], []]
    with pytest.raises(ValueError):
        shard.assign_jobs([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [float(c) for c in (9, 1, 7, 3, 5, 2, 8)]
        table = shard.assign_jobs(costs, world)
        mine = table[rank]
        done = sum(costs[i] for i in mine)           # the "work" this rank did
        slowest = shard.allreduce_max(done, world, device="cpu")
        total = shard.allreduce_sum(done, world, device="cpu")
        count = shard.allreduce_sum(len(mine), world, device="cpu")
        out.put((rank, table, slowest, total, count))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_table_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, m0, s0, c0), (r1, t1, m1, s1, c1) = res
    assert (r0, r1) == (0, 1) and t0 == t1
    costs = [9, 1, 7, 3, 5, 2, 8]
    loads = [sum(costs[i] for i in part) for part in t0]
    assert m0 == m1 == max(loads)
    assert s0 == s1 == sum(costs)
    assert c0 == c1 == len(costs)


def test_spp_slices_partition_the_samples():
    for spp in (1, 2, 7, 64, 257):
        for world in (1, 2, 3, 4, 8):
            sl = shard.spp_slices(spp, world)
            assert len(sl) == world
            # contiguous, in rank order, covering [0, spp) exactly
            assert sl[0][0] == 0
            for (f0, n0), (f1, _) in zip(sl, sl[1:]):
                assert f1 == f0 + n0
            assert sum(n for _, n in sl) == spp
            assert max(n for _, n in sl) - min(n for _, n in sl) <= 1
    with pytest.raises(ValueError):
        shard.spp_slices(4, 0)
    with pytest.raises(ValueError):
        shard.spp_slices(0, 2)


RAYS = 40
SPP = 7


def _fake_slice(first, count):
    """Stand-in for a render of samples [first, first + count): per ray and
    sample an integer-valued radiance, so float sums are exact in any order."""
    import numpy as np
    acc = np.zeros((RAYS, 3), np.float32)
    for s in range(first, first + count):
        acc += (np.arange(RAYS * 3, dtype=np.float32).reshape(RAYS, 3) * (s + 1)) % 97
    return acc


def _split_rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        calls = []

        def render(first, count):
            calls.append((first, count))
            return _fake_slice(first, count)

        acc = shard.split_spp_accum(render, SPP, RAYS, rank, world, device="cpu")
        out.put((rank, calls, acc.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_one_frames_samples():
    """Each rank renders only its slice of the samples; after the one
    all-reduce both hold the accumulator of all the samples."""
    import numpy as np
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((r, c, a) for r, c, a in (out.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, c0, a0), (r1, c1, a1) = res
    assert c0 == [(0, 4)] and c1 == [(4, 3)]
    whole = _fake_slice(0, SPP)
    assert np.array_equal(np.asarray(a0, np.float32), whole)
    assert np.array_equal(np.asarray(a1, np.float32), whole)
