"""Serving loop (hpt_server), CUDA-graph replay and the autotuner on the GPU.

The engine draws every random number from a stream keyed by (request seed,
ray, sample, bounce) and sums radiance in 2^-32 fixed point, so a request's
result does not depend on what else shares the wavefront: the tolerance of
the alone-vs-mix comparison is zero (bit-identical accumulators)."""
import os
import tempfile

import numpy as np
import pytest

import hptracing_b200 as H
from tests import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes(built):
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    room = H.Scene(*S.make_scene(0))
    spheres = H.Scene(*S.make_scene(1, seed=1, texture_size=64))
    return room, spheres


# (scene index, camera, w, h, ss, spp, depth, background, seed)
REQUESTS = [
    (0, S.ROOM_CAM, 64, 48, 1, 4, 6, (0, 0, 0), 101),
    (1, S.ROOM_CAM, 96, 64, 1, 2, 5, (0.1, 0.1, 0.1), 102),
    (0, S.PANO_CAM, 128, 64, 1, 3, 6, (0.2, 0.3, 0.4), 103),
    (1, S.ROOM_CAM, 32, 32, 2, 8, 8, (0, 0, 0), 104),
    (0, S.ROOM_CAM, 48, 48, 1, 16, 4, (0, 0, 0), 105),
    (1, S.PANO_CAM, 64, 32, 1, 1, 6, (0, 0, 0.5), 106),
]


def _params(req):
    _, _, w, h, ss, spp, depth, bg, seed = req
    return H.make_params(w, h, ss, ss, bg, spp, depth, 0, 1.0, seed)


def _alone(scenes, req):
    rgba, acc = scenes[req[0]].render(S.hp_camera(req[1]), _params(req), want_accum=True)
    return rgba, acc


def _drain(server, ids, reqs, max_pumps=20000):
    out = {}
    for _ in range(max_pumps):
        server.pump(2)
        for rid, req in zip(ids, reqs):
            if rid in out:
                continue
            p = _params(req)
            rgba = np.zeros((p.sample_y, p.sample_x, 4), np.uint8)
            acc = np.zeros((p.sample_x * p.supersample_x * p.sample_y * p.supersample_y, 3),
                           np.float32)
            st, info = server.poll(rid, rgba, acc)
            if st == 0:
                out[rid] = (rgba, acc, info)
        if len(out) == len(ids):
            return out
    raise AssertionError("server did not finish: %d of %d" % (len(out), len(ids)))


@pytest.mark.parametrize("capacity,large_pct", [(1 << 16, 0), (1 << 14, 25)])
def test_results_alone_equal_results_in_the_mix(scenes, capacity, large_pct):
    # With capacity 2^14 most requests exceed one wavefront and run capped at
    # 25 % of it in flight: scheduling changes, results must not.
    server = H.Server(max_jobs=8, memory_budget=1 << 30, capacity=capacity,
                      large_inflight_pct=large_pct)
    slots = [server.add_scene(s) for s in scenes]
    # Staggered arrivals: half submitted up front, the rest while the first
    # half runs (continuous batching into freed slots).
    ids = []
    for req in REQUESTS[:3]:
        ids.append(server.submit(slots[req[0]], S.hp_camera(req[1]), _params(req)))
    server.pump(3)
    for req in REQUESTS[3:]:
        ids.append(server.submit(slots[req[0]], S.hp_camera(req[1]), _params(req)))
    out = _drain(server, ids, REQUESTS)
    for rid, req in zip(ids, REQUESTS):
        rgba, acc, info = out[rid]
        a_rgba, a_acc = _alone(scenes, req)
        assert np.array_equal(acc, a_acc), req
        assert np.array_equal(rgba, a_rgba), req
        assert info["state"] == 2 and info["samples_done"] == req[5]
        assert info["submit_ms"] <= info["admit_ms"] <= info["done_ms"]
        assert info["intersect_queries"] > 0
    st = server.stats()
    assert st["paths"] == len(REQUESTS) and st["error_flags"] == 0
    assert server.pending() == 0
    server.close()


def test_admission_respects_the_memory_budget(scenes):
    # Budget for about two of these requests at a time.
    req = (0, S.ROOM_CAM, 64, 64, 1, 2, 5, (0, 0, 0), 7)
    fp = 64 * 64 * (24 + 4 + 32 + 12) + 64 * 64 * 4 + 64
    server = H.Server(max_jobs=8, memory_budget=2 * fp + 100, capacity=1 << 14)
    slot = server.add_scene(scenes[0])
    reqs = [req[:-1] + (7 + k,) for k in range(5)]
    ids = [server.submit(slot, S.hp_camera(r[1]), _params(r)) for r in reqs]
    server.pump(1)
    running = sum(server.poll(i)[1]["state"] == 1 for i in ids)
    assert 1 <= running <= 2
    out = _drain(server, ids, reqs)
    for rid, r in zip(ids, reqs):
        assert np.array_equal(out[rid][1], _alone(scenes, r)[1])
    assert sorted(server.completed()) == sorted(ids)
    assert server.completed() == []
    # A request larger than the whole budget is refused at submission.
    big = H.make_params(1024, 1024, 1, 1, (0, 0, 0), 1, 5, 0, 1.0, 1)
    with pytest.raises(H.HptError) as e:
        server.submit(slot, S.hp_camera(S.ROOM_CAM), big)
    assert e.value.status == 4
    server.close()


def test_progressive_previews_and_cancel(scenes):
    server = H.Server(max_jobs=4, memory_budget=1 << 30, capacity=1 << 12, progressive=1)
    slot = server.add_scene(scenes[1])
    req = (1, S.ROOM_CAM, 64, 64, 1, 32, 6, (0, 0, 0), 55)
    rid = server.submit(slot, S.hp_camera(req[1]), _params(req))
    victim = server.submit(slot, S.hp_camera(req[1]), _params(req[:-1] + (56,)))
    server.cancel(victim)
    previews = []
    for _ in range(10000):
        server.pump(1)
        rgba = np.zeros((64, 64, 4), np.uint8)
        st, info = server.poll(rid, rgba)
        if st == 0:
            break
        assert st == 9  # busy
        if info["samples_done"] > 0:
            previews.append(rgba.copy())
    assert previews, "no progressive preview was produced"
    with pytest.raises(H.HptError) as e:
        server.poll(victim)
    assert e.value.status in (6, 8)
    final_rgba = _alone(scenes, req)[0]
    assert np.abs(previews[-1].astype(int) - final_rgba.astype(int)).mean() < 40
    server.close()


def test_graph_replay_equals_eager(scenes):
    room = scenes[0]
    t0 = room.tuning()
    p = H.make_params(64, 64, 1, 1, (0, 0, 0), 8, 6, 0, 1.0, 9)
    eager = room.render(S.hp_camera(S.ROOM_CAM), p, want_accum=True)[1]
    t = room.tuning()
    t.use_graph = 1
    t.capacity = 1 << 13
    room.set_tuning(t)
    try:
        a = room.render(S.hp_camera(S.ROOM_CAM), p, want_accum=True)[1]
        b = room.render(S.hp_camera(S.ROOM_CAM), p, want_accum=True)[1]
    finally:
        room.set_tuning(t0)
    assert np.array_equal(a, eager) and np.array_equal(b, eager)


def test_graph_replay_follows_a_change_of_scene(scenes):
    """A batch engine that replays a captured graph bakes the one scene of
    its jobs into the graph's kernel parameters; running it next on another
    scene must re-capture, not replay the first scene's pointers."""
    room, spheres = scenes
    p = H.make_params(48, 48, 1, 1, (0, 0, 0), 4, 6, 0, 1.0, 5)
    want = [g.render(S.hp_camera(S.ROOM_CAM), p, want_accum=True)[1] for g in (room, spheres)]
    t = room.tuning()
    t.use_graph = 1
    t.capacity = 1 << 13
    batch = H.Batch()
    batch.set_tuning(t)
    try:
        for _ in range(2):
            for g, w in zip((room, spheres), want):
                batch.add(g, S.hp_camera(S.ROOM_CAM), p, want_accum=True)
                assert np.array_equal(batch.run()[0][1], w)
    finally:
        batch.close()


def test_autotune_picks_a_valid_tuning_and_caches_it(scenes):
    spheres = scenes[1]
    t0 = spheres.tuning()
    p = H.make_params(96, 96, 1, 1, (0, 0, 0), 2, 5, 0, 1.0, 3)
    want = spheres.render(S.hp_camera(S.ROOM_CAM), p, want_accum=True)[1]
    with tempfile.TemporaryDirectory() as d:
        cache = os.path.join(d, "tune.txt")
        try:
            best = spheres.autotune(S.hp_camera(S.ROOM_CAM), p, cache)
            assert best.isect_block in (128, 256) and 1 <= best.refill_chunk <= 32
            assert os.path.exists(cache) and open(cache).read().count("\n") == 1
            again = spheres.autotune(S.hp_camera(S.ROOM_CAM), p, cache)  # cache hit
            assert open(cache).read().count("\n") == 1
            assert (again.capacity, again.isect_block, again.refill_chunk, again.smem_nodes) == \
                (best.capacity, best.isect_block, best.refill_chunk, best.smem_nodes)
            got = spheres.render(S.hp_camera(S.ROOM_CAM), p, want_accum=True)[1]
        finally:
            spheres.set_tuning(t0)
    assert np.array_equal(got, want)


def test_primary_pass_in_parts_keeps_results(scenes):
    """A large request (more paths than the wavefront) has its primary pass
    traced in parts over several pumps, at most its in-flight share of the
    wavefront in rays per pump for all large requests together, while the
    smaller requests admitted meanwhile run. Capacity 2^12 with a 25 %
    share makes that 1,024 rays per pump: the 128x96 panorama (3 spp), the
    80x64 request and the 4x4 supersampled 24x16 one take 23 pumps in all,
    the two small ones are traced whole. All must equal the same requests
    rendered alone."""
    reqs = [
        (0, S.PANO_CAM, 128, 96, 1, 3, 6, (0.2, 0.3, 0.4), 401),
        (1, S.ROOM_CAM, 32, 32, 1, 2, 5, (0, 0, 0), 402),
        (1, S.ROOM_CAM, 80, 64, 1, 1, 6, (0.1, 0.1, 0.1), 403),
        (0, S.ROOM_CAM, 24, 16, 4, 2, 6, (0, 0, 0), 404),
        (0, S.ROOM_CAM, 16, 16, 1, 4, 6, (0, 0, 0), 405),
    ]
    server = H.Server(max_jobs=8, memory_budget=1 << 30, capacity=1 << 12, large_inflight_pct=25)
    slots = [server.add_scene(s) for s in scenes]
    ids = [server.submit(slots[r[0]], S.hp_camera(r[1]), _params(r)) for r in reqs[:3]]
    server.pump(1)
    ids += [server.submit(slots[r[0]], S.hp_camera(r[1]), _params(r)) for r in reqs[3:]]
    out = _drain(server, ids, reqs)
    for rid, req in zip(ids, reqs):
        rgba, acc, info = out[rid]
        a_rgba, a_acc = _alone(scenes, req)
        assert np.array_equal(acc, a_acc), req
        assert np.array_equal(rgba, a_rgba), req
        assert info["intersect_queries"] > 0
    assert server.stats()["error_flags"] == 0
    server.close()


def test_overload_policy_sheds_late_requests_and_keeps_results(scenes):
    """deadline_ms: latency-bound requests (<= capacity paths) are admitted
    when predicted to finish in time and shed once they cannot. A burst of
    64 requests with a 1 ms deadline: the first runs (it measures the
    scene's service time), the others are shed (HPT_ERR_CANCELLED, counted
    by hpt_server_shed), and every request that does complete is
    bit-identical to the same request rendered alone. Without the policy
    nothing is shed."""
    req = (1, S.ROOM_CAM, 96, 64, 1, 4, 6, (0, 0, 0), 300)
    _, ref = _alone(scenes, req)
    for deadline, expect_shed in ((1, True), (0, False)):
        server = H.Server(max_jobs=8, memory_budget=1 << 30, capacity=1 << 16,
                          deadline_ms=deadline)
        slots = [server.add_scene(s) for s in scenes]
        p = _params(req)
        ids = [server.submit(slots[1], S.hp_camera(S.ROOM_CAM), p) for _ in range(64)]
        done, shed = 0, 0
        pending = set(ids)
        for _ in range(200000):
            if not pending:
                break
            server.pump(2)
            for rid in list(pending):
                acc = np.zeros((p.sample_x * p.sample_y, 3), np.float32)
                try:
                    st, _ = server.poll(rid, None, acc)
                except H.HptError as e:
                    assert e.status == 8 and "shed" in str(e), str(e)
                    shed += 1
                    pending.discard(rid)
                    continue
                if st == 0:
                    assert np.array_equal(acc, ref)
                    done += 1
                    pending.discard(rid)
        assert not pending
        assert server.shed() == shed
        print("deadline %d ms: %d done, %d shed" % (deadline, done, shed))
        if expect_shed:
            assert shed > 0 and done > 0
        else:
            assert shed == 0 and done == 64
        server.close()
