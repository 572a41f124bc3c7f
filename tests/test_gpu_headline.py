"""Parity at the benchmarked configuration: the spheres frame exactly as
bench.py renders it (box room + 64 UV spheres, 61,476 triangles, four
1024^2 value-noise textures; 512x512, 64 spp, depth 8).

Ray batches of 2^20 rays each, against the oracle through the C ABI:
  camera     the camera's primary rays (1024 x 1024 raster)
  random     origins uniform in the scene box grown by 10 %, directions
             uniform on the sphere
  secondary  the rays the oracle itself sends to intersect after two
             shading passes from the camera rays (s1_run + s2_*_run)
Closest hits (triangle id, t, u, v) must be bit-exact. Counted and printed
per batch: rays past the reference's 512-leaf gather cap (not compared)
and shared-edge ties (another triangle at the bit-identical t); none occur
on these batches. Shading runs on the hits with the full 1024^2 textures.
Whole frames: the counter-mode oracle at reduced resolution, and the image
against the reference's own estimator (per-lane LCG) within per-pixel
3 sigma Monte Carlo error and a stated relMSE bar."""
import os

import numpy as np
import pytest

import hptracing_b200 as H
import oracle as O
from tests import scenes as S

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)
N = 1 << 20
BENCH_DEPTH = 8


@pytest.fixture(scope="module")
def c1(built):
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    mesh, nodes, leaf = S.make_scene(1, seed=1)  # bench.py's scene, 1024^2 textures
    assert len(mesh.triangles) == 61476
    assert mesh.texture_dims.tolist() == [[1024, 1024]] * 4
    return mesh, H.Scene(mesh, nodes, leaf), O.CpuScene(mesh, nodes, leaf)


@pytest.fixture(scope="module")
def batches(c1):
    mesh, _, cpu = c1
    cam = O.raygen(S.ROOM_CAM, 1024, 1024, 1, 1)
    rnd = S.aabb_random_rays(mesh, N, seed=0x48505401)
    parts = [S.oracle_bounce_rays(cpu, cam[0], cam[1], 2, seed=s, threads=THREADS)
             for s in (1, 2)]
    sec = (np.concatenate([p[0] for p in parts])[:N], np.concatenate([p[1] for p in parts])[:N])
    assert len(sec[0]) == N
    return {"camera": cam, "random": rnd, "secondary": sec}


@pytest.mark.parametrize("kind", ["camera", "random", "secondary"])
def test_headline_closest_hits_2pow20(c1, batches, kind):
    _, gpu, cpu = c1
    o, d = batches[kind]
    tri, t, u, v = gpu.intersect(o, d)
    ref = cpu.intersect(o, d, threads=THREADS)
    c = S.hit_parity(ref, tri, t, u, v)
    print("C1 %s: %d rays, %d hits, cap cases %d, shared-edge ties %d, other differences %d"
          % (kind, c["rays"], c["hits"], c["cap"], c["ties"], c["other"]))
    assert c["rays"] == N
    assert c["other"] == 0, c["first_other"]
    assert c["cap"] == 0 and c["ties"] == 0


def test_headline_fp32_vs_fp64(c1, batches):
    """States the FP32 error of the closest hits against an FP64 brute force
    over all 61,476 triangles (a 16k-ray subset of the random batch)."""
    _, gpu, cpu = c1
    o, d = (x[:16384] for x in batches["random"])
    tri, t, _, _ = gpu.intersect(o, d)
    btri, bt = cpu.brute_f64(o, d, threads=THREADS)
    agree = ((tri >= 0) == (btri >= 0)).mean()
    both = (tri >= 0) & (btri >= 0)
    rel = np.abs(t[both] - bt[both]) / np.maximum(bt[both], 1e-6)
    other = (tri != btri)[both]
    print("C1 fp32 vs fp64: hit/miss agreement %.6f, same triangle %.6f, rel t error "
          "p50 %.3g p99 %.3g max %.3g" % (agree, 1 - other.mean(), np.median(rel),
                                           np.percentile(rel, 99), rel.max()))
    assert agree > 0.9999
    assert np.percentile(rel, 99) < 1e-5
    if other.any():
        assert rel[other].max() < 1e-5


@pytest.mark.parametrize("kind", ["camera", "secondary"])
def test_headline_shade_full_textures(c1, batches, kind):
    """s1_run on every hit of a batch with the 1024^2 textures, then the
    next directions: shading bit-exact; next-dir light branch bit-exact; the
    other branches use acos / sin / cos / pow / asin, whose last bits differ
    between CUDA and the host library: >= 99.99 % of the rays within 2e-5 and
    all within 1e-3 (refraction close to the critical angle amplifies an
    ulp: sqrt(1 - x^2) has slope x / sqrt(1 - x^2) there)."""
    _, gpu, cpu = c1
    o, d = batches[kind]
    ref = cpu.intersect(o, d, threads=THREADS)
    h = np.flatnonzero(ref["tri"] >= 0)
    rng = np.random.default_rng(0x5EED)
    st = rng.uniform(0.0, 1.0, (len(h), 3)).astype(np.float32)
    seeds = rng.integers(0, 2 ** 48, len(h), dtype=np.int64)
    o, d, tri, t = o[h], d[h], ref["tri"][h], ref["t"][h]
    g = gpu.shade(o, d, st, tri, t, seeds.astype(np.uint64), 0)
    r = cpu.shade(o, d, st, tri, t, seeds, 0)
    alive = r["branch"] >= 0
    for k in ("contrib", "branch"):
        assert np.array_equal(g[k], r[k]), k
    for k in ("hit_p", "normal", "strength", "param"):
        assert np.array_equal(g[k][alive], r[k][alive]), k
    assert np.array_equal(g["seeds"].astype(np.int64)[alive], r["seeds"][alive])
    mats = cpu.triangles[tri, 3]
    textured = cpu.materials["diffuse_texture_id"][mats] >= 0
    print("C1 %s shading: %d hits, %d on textured materials, branches %s"
          % (kind, len(h), int(textured.sum()), np.bincount(r["branch"] + 1).tolist()))
    assert textured.sum() > 10000
    a = np.flatnonzero(alive)
    args = (r["branch"][a], d[a], r["hit_p"][a], r["normal"][a], r["strength"][a], r["param"][a])
    gn = gpu.next_dir(*args, r["seeds"][a].astype(np.uint64))
    cn = cpu.next_dir(*args, r["seeds"][a])
    light = r["branch"][a] == 3
    for k in ("origins", "directions", "strength", "alive"):
        assert np.array_equal(gn[k][light], cn[k][light]), k
    for k in ("origins", "directions", "strength"):
        err = np.abs(gn[k][~light] - cn[k][~light]) / np.maximum(np.abs(cn[k][~light]), 1.0)
        within = (err < 2e-5).all(axis=1).mean()
        print("next-dir %s: within 2e-5 %.6f, max %.3g" % (k, within, err.max()))
        assert within >= 0.9999 and err.max() < 1e-3, (k, within, err.max())
    assert (gn["alive"] == cn["alive"]).mean() > 0.9999
    assert np.array_equal(gn["seeds"].astype(np.int64), cn["seeds"])


def test_headline_frame_matches_counter_oracle(c1):
    """The benchmarked frame at reduced resolution (64 x 64, 8 spp, depth 8):
    per-ray radiance against the oracle driven by the same random streams."""
    _, gpu, cpu = c1
    w = h = 64
    spp = 8
    p = H.make_params(w, h, 1, 1, (0, 0, 0), spp, BENCH_DEPTH, 0, 1.0, 1000)
    _, acc = gpu.render(S.hp_camera(S.ROOM_CAM), p, want_accum=True)
    st = gpu.stats()
    ref, _, counts = cpu.render(S.ROOM_CAM, w, h, 1, 1, (0, 0, 0), spp, BENCH_DEPTH, 0,
                                seed=1000, rng_mode=1, threads=THREADS)
    rel = np.abs(acc - ref) / (np.abs(ref) + 1e-3)
    bad = (rel > 1e-3).any(axis=1).mean()
    print("C1 frame: rays off by >1e-3: %.4f; queries gpu %d oracle %d"
          % (bad, st["intersect_queries"], counts[0]))
    assert bad < 0.02
    assert abs(acc.sum() - ref.sum()) / ref.sum() < 0.01
    assert abs(st["intersect_queries"] - counts[0]) / counts[0] < 0.01
    assert st["error_flags"] == 0


def test_headline_image_vs_reference_estimator(c1):
    """The benchmarked frame's image (its camera at 32 x 32, depth 8)
    against the reference's own estimator (per-lane LCG, as
    TraceRunner::run draws it): GPU 1024 spp vs reference 512 spp.
    Glass and mirror spheres make the estimator heavy-tailed, so the
    per-sample variance under-covers: two runs of the reference estimator
    itself (1024 vs 512 spp, other seeds) put 93.0 % of ray means within
    3 sigma, relMSE 1.07x the predicted value, totals 1.3 % apart; the
    counter-mode oracle (the GPU's random streams) gives 93.9 %, 1.07x,
    0.9 %. Bars: >= 90 % within 3 sigma, relMSE <= 1.5x predicted, totals
    within 2 %."""
    _, gpu, cpu = c1
    w = h = 32
    spp_g, spp_o = 1024, 512
    p = H.make_params(w, h, 1, 1, (0, 0, 0), spp_g, BENCH_DEPTH, 0, 1.0, 5)
    _, acc = gpu.render(S.hp_camera(S.ROOM_CAM), p, want_accum=True)
    ref, ref2, _ = cpu.render(S.ROOM_CAM, w, h, 1, 1, (0, 0, 0), spp_o, BENCH_DEPTH, 0, seed=9,
                              rng_mode=0, threads=THREADS)
    mg, mo = acc / spp_g, ref / spp_o
    var = np.maximum(ref2 / spp_o - mo * mo, 0.0)
    sigma = np.sqrt(var / spp_g + var / spp_o) + 1e-5 * np.abs(mo) + 1e-6
    frac = (np.abs(mg - mo) / sigma <= 3).mean()
    relmse = np.mean((mg - mo) ** 2 / (mo ** 2 + 1e-2))
    expected = np.mean((var / spp_g + var / spp_o) / (mo ** 2 + 1e-2))
    total = abs(mg.sum() - mo.sum()) / mo.sum()
    print("C1 image vs reference estimator: within 3 sigma %.4f, relMSE %.4g (predicted %.4g), "
          "totals %.4g" % (frac, relmse, expected, total))
    assert frac >= 0.90
    assert relmse <= 1.5 * expected
    assert total < 0.02
