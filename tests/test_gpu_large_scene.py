"""The large scene (terrain: 1024x1024-vertex heightfield + 16 columns,
2.4M triangles, eight 2048^2 textures) on the GPU.

At full size the oracle still intersects a few ten thousand rays in
seconds, so closest hits are compared bit for bit there; whole renders are
compared with the oracle on a reduced terrain (256^2 heightfield, 450k
triangles) and checked at full size through properties that do not depend
on size: determinism, batch == alone, no device check or step cap firing."""
import numpy as np
import pytest

import hptracing_b200 as H
import oracle as O
from tests import scenes as S

pytestmark = pytest.mark.gpu

CAM = S.terrain_cam(16 / 9)


def _terrain(n):
    mesh = H.Mesh.generate(2, seed=2, heightfield_n=n, texture_size=256)
    nodes, leaf = H.build_kdtree(mesh.points, mesh.triangles)
    return mesh, nodes, leaf


@pytest.fixture(scope="module")
def full(built):
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    mesh, nodes, leaf = _terrain(1024)
    assert len(mesh.triangles) > 2_000_000
    return mesh, H.Scene(mesh, nodes, leaf), O.CpuScene(mesh, nodes, leaf)


@pytest.fixture(scope="module")
def small(built):
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    mesh, nodes, leaf = _terrain(256)
    return mesh, H.Scene(mesh, nodes, leaf), O.CpuScene(mesh, nodes, leaf)


def _same_hits(ref, got):
    ok = ref["overflow"] == 0
    assert ok.mean() > 0.999
    for k in ("tri", "t", "u", "v"):
        a, b = np.asarray(ref[k])[ok], np.asarray(got[k])[ok]
        bad = np.flatnonzero(a.view(np.int32) != b.view(np.int32))
        assert bad.size == 0, (k, bad[:5])


def test_full_size_closest_hits_bitexact(full):
    mesh, gpu, cpu = full
    o1, d1 = O.raygen(CAM, 480, 270, 1, 1)
    rng = np.random.default_rng(17)
    lo, hi = mesh.points[:, :3].min(0), mesh.points[:, :3].max(0)
    o2 = rng.uniform(lo - 0.1, hi + 0.1, (20000, 3)).astype(np.float32)
    d2 = rng.normal(size=(20000, 3)).astype(np.float32)
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    for o, d in ((o1, d1), (o2, d2)):
        ref = cpu.intersect(o, d)
        tri, t, u, v = gpu.intersect(o, d)
        got = dict(tri=tri, t=t, u=u, v=v)
        _same_hits(ref, got)
    assert (got["tri"] >= 0).mean() > 0.3


def test_reduced_terrain_render_matches_counter_oracle(small):
    _, gpu, cpu = small
    w, h, spp, depth, bg = 160, 90, 4, 6, (0.2, 0.2, 0.2)
    p = H.make_params(w, h, 1, 1, bg, spp, depth, 0, 1.0, 3)
    _, acc = gpu.render(S.hp_camera(CAM), p, want_accum=True)
    st = gpu.stats()
    ref, _, counts = cpu.render(CAM, w, h, 1, 1, bg, spp, depth, 0, seed=3, rng_mode=1)
    rel = np.abs(acc - ref) / (np.abs(ref) + 1e-3)
    bad = (rel > 1e-3).any(axis=1).mean()
    print("terrain: rays off by >1e-3: %.4f; queries gpu %d oracle %d"
          % (bad, st["intersect_queries"], counts[0]))
    assert bad < 0.02
    assert abs(acc.sum() - ref.sum()) / ref.sum() < 0.01
    assert abs(st["intersect_queries"] - counts[0]) / counts[0] < 0.01
    assert st["error_flags"] == 0


def test_full_size_render_properties(full, small):
    _, gpu, _ = full
    _, g_small, _ = small
    p = H.make_params(480, 270, 1, 1, (0.2, 0.2, 0.2), 2, 8, 0, 1.0, 11)
    _, a = gpu.render(S.hp_camera(CAM), p, want_accum=True)
    st = gpu.stats()
    _, b = gpu.render(S.hp_camera(CAM), p, want_accum=True)
    assert np.array_equal(a, b)
    assert st["error_flags"] == 0 and np.isfinite(a).all()
    assert st["intersect_queries"] > 480 * 270 * 2
    batch = H.Batch()
    batch.add(gpu, S.hp_camera(CAM), p, want_accum=True)
    q = H.make_params(96, 54, 1, 1, (0, 0, 0), 3, 5, 0, 1.0, 4)
    batch.add(g_small, S.hp_camera(CAM), q, want_accum=True)
    out = batch.run()
    assert np.array_equal(out[0][1], a)
    assert np.array_equal(out[1][1], g_small.render(S.hp_camera(CAM), q, want_accum=True)[1])
