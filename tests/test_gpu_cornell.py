"""A scene file of the reference on the GPU: the embree Cornell box
(scene/simple-cornell-box/cornell_box.obj, 36 triangles, a glass block),
travelling as the golden fixture tests/golden/cornell_box.npz that
make_golden.py wrote from the reference's own loader, SAH builder and
kernels (the GPU host has no copy of the reference).

The camera is the embree scene's viewpoint; depth 5 and 50 samples are the
Readme's low-sample render (Readme.md:53-55, 500 x 500).

The scene spans 556 units, and the reference starts each next ray at
hit + 1e-5 * dir (kernel.cl:413-557): above 256 a float32 coordinate has an
ulp of 3e-5, so the offset rounds away and the next ray starts exactly on the
surface it left, where a re-hit depends on the last bits of its direction.
Paths are therefore chaotic: a transcendental's last bit (CUDA vs the host
library) or a one-ulp move of the camera changes a path from there on. The
whole-render comparisons with the oracle are calibrated against that: the
GPU must differ from the oracle no more than the oracle differs from itself
when the camera moves by one ulp."""
import os

import numpy as np
import pytest

import hptracing_b200 as H
import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cornell_box.npz")
THREADS = max(1, os.cpu_count() or 1)


@pytest.fixture(scope="module")
def cornell(built):
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    f = dict(np.load(GOLD))
    mesh = H.Mesh(f["points"], f["triangles"], f["materials"], f["normals"], f["texcoords"],
                  f["lights"])
    c = f["camera"]
    cam = dict(view_p=tuple(c[0:3]), top_dir=tuple(c[3:6]), right_dir=tuple(c[6:9]),
               width=float(c[9]), height=float(c[10]))
    return f, cam, H.Scene(mesh, f["nodes"], f["leaf_data"]), O.CpuScene(mesh, f["nodes"],
                                                                          f["leaf_data"])


def _shifted(cam):
    """The camera with view_p.x moved up by one float32 ulp."""
    v = np.asarray(cam["view_p"], np.float32).copy()
    v[0] = np.nextafter(v[0], np.float32(np.inf))
    out = dict(cam)
    out["view_p"] = tuple(float(x) for x in v)
    return out


def _off(a, b):
    """Fraction of rays whose radiance differs by more than 1e-3 relative."""
    return (np.abs(a - b) / (np.abs(b) + 1e-3) > 1e-3).any(axis=1).mean()


def _hp(cam):
    return H.make_camera(cam["view_p"], cam["top_dir"], cam["right_dir"], cam["width"],
                         cam["height"])


def test_cornell_closest_hits_readme_raster(cornell):
    """The 500 x 500 camera rays of the Readme render plus rays from inside
    the box: closest hits bit-exact against the oracle."""
    f, cam, gpu, cpu = cornell
    o, d = O.raygen(cam, 500, 500, 1, 1)
    rng = np.random.default_rng(31)
    lo, hi = f["points"][:, :3].min(0), f["points"][:, :3].max(0)
    o2 = rng.uniform(lo, hi, (200000, 3)).astype(np.float32)
    d2 = rng.normal(size=(200000, 3))
    d2 = (d2 / np.linalg.norm(d2, axis=1, keepdims=True)).astype(np.float32)
    for oo, dd in ((o, d), (o2, d2)):
        tri, t, u, v = gpu.intersect(oo, dd)
        ref = cpu.intersect(oo, dd, threads=THREADS)
        assert (ref["overflow"] == 0).all()
        for k, x in (("tri", tri), ("t", t), ("u", u), ("v", v)):
            assert np.array_equal(ref[k].view(np.int32), x.view(np.int32)), k
        assert (tri >= 0).mean() > 0.5


def test_cornell_readme_render_matches_counter_oracle(cornell):
    """Readme settings (50 samples, depth 5) on a 100 x 100 raster: per-ray
    radiance against the oracle driven by the GPU's random streams, no more
    rays off than a one-ulp camera move gives the oracle itself (37 % when
    measured; the GPU: 13 %), totals and query counts within 1 %."""
    _, cam, gpu, cpu = cornell
    w, spp, depth = 100, 50, 5
    p = H.make_params(w, w, 1, 1, (0, 0, 0), spp, depth, 0, 1.0, 50)
    _, acc = gpu.render(_hp(cam), p, want_accum=True)
    st = gpu.stats()
    ref, _, counts = cpu.render(cam, w, w, 1, 1, (0, 0, 0), spp, depth, 0, seed=50, rng_mode=1,
                                threads=THREADS)
    moved, _, _ = cpu.render(_shifted(cam), w, w, 1, 1, (0, 0, 0), spp, depth, 0, seed=50,
                             rng_mode=1, threads=THREADS)
    bad, self_bad = _off(acc, ref), _off(moved, ref)
    print("Cornell: rays off by >1e-3: %.4f (oracle vs its one-ulp camera move: %.4f); "
          "queries gpu %d oracle %d" % (bad, self_bad, st["intersect_queries"], counts[0]))
    assert bad <= self_bad
    assert abs(acc.sum() - ref.sum()) / ref.sum() < 0.01
    assert abs(st["intersect_queries"] - counts[0]) / counts[0] < 0.01
    assert st["error_flags"] == 0


def test_cornell_image_vs_reference_kernels(cornell):
    """The GPU's estimate (1024 spp) against the reference kernels' own
    estimate stored in the fixture (256 spp, same camera and depth).
    At this scale the reference's image depends on the last bits of its
    math library: a next ray that starts on the surface it left re-hits it
    or not according to those bits. Two runs of the reference estimator
    (1024 vs 256 spp) put 94.1 % of ray means within 3 sigma, relMSE 1.32x
    the value the per-sample variances predict, totals 0.2 % apart; the
    oracle with every acos / asin / sin / cos / pow result moved one ulp
    toward zero (an equally valid library) gives relMSE 12.3x, totals
    0.3-0.4 %. CUDA's library is another such library. Bars: >= 90 % within
    3 sigma, relMSE below the one-ulp library's 12.3x, totals within 1 %.
    The unit-scale copy of the box below carries the tight bars."""
    f, cam, gpu, _ = cornell
    w, spp_o, depth = int(f["res"]), int(f["spp"]), int(f["depth"])
    spp_g = 1024
    p = H.make_params(w, w, 1, 1, (0, 0, 0), spp_g, depth, 0, 1.0, 3)
    _, acc = gpu.render(_hp(cam), p, want_accum=True)
    ref, ref2 = f["ref_accum"], f["ref_accum_sq"]
    mg, mo = acc / spp_g, ref / spp_o
    var = np.maximum(ref2 / spp_o - mo * mo, 0.0)
    sigma = np.sqrt(var / spp_g + var / spp_o) + 1e-5 * np.abs(mo) + 1e-6
    frac = (np.abs(mg - mo) / sigma <= 3).mean()
    relmse = np.mean((mg - mo) ** 2 / (mo ** 2 + 1e-2))
    expected = np.mean((var / spp_g + var / spp_o) / (mo ** 2 + 1e-2))
    total = abs(mg.sum() - mo.sum()) / mo.sum()
    print("Cornell vs reference kernels: within 3 sigma %.4f, relMSE %.4g (predicted %.4g), "
          "totals %.4g" % (frac, relmse, expected, total))
    assert frac >= 0.90
    assert relmse <= 12.3 * expected
    assert total < 0.01


@pytest.fixture(scope="module")
def cornell_unit(built):
    """The same box scaled by 1/556 (one unit across): the reference's 1e-5
    origin offset is far above an ulp there, so paths are not chaotic (a
    one-ulp camera move changes 0.27 % of the oracle's rays, against 37 %
    at full scale). The KD-tree is rebuilt by the SAH builder, which gives
    the reference builder's tree bit for bit."""
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    f = dict(np.load(GOLD))
    k = np.float32(1.0 / 556.0)
    pts = f["points"].copy()
    pts[:, :3] *= k
    mesh = H.Mesh(pts, f["triangles"], f["materials"], f["normals"], f["texcoords"])
    mesh.rebuild_lights()
    nodes, leaf = H.build_kdtree(mesh.points, mesh.triangles)
    c = f["camera"]
    cam = dict(view_p=tuple(float(np.float32(x) * k) for x in c[0:3]),
               top_dir=tuple(float(x) for x in c[3:6]), right_dir=tuple(float(x) for x in c[6:9]),
               width=float(c[9]), height=float(c[10]))
    return cam, H.Scene(mesh, nodes, leaf), O.CpuScene(mesh, nodes, leaf)


def test_cornell_unit_scale_matches_counter_oracle(cornell_unit):
    """Readme settings (50 spp, depth 5), 100 x 100: per-ray radiance against
    the oracle driven by the GPU's random streams: <= 2 % of rays off by
    more than 1e-3, totals and query counts within 1 %."""
    cam, gpu, cpu = cornell_unit
    p = H.make_params(100, 100, 1, 1, (0, 0, 0), 50, 5, 0, 1.0, 50)
    _, acc = gpu.render(_hp(cam), p, want_accum=True)
    st = gpu.stats()
    ref, _, counts = cpu.render(cam, 100, 100, 1, 1, (0, 0, 0), 50, 5, 0, seed=50, rng_mode=1,
                                threads=THREADS)
    bad = _off(acc, ref)
    print("Cornell unit scale: rays off by >1e-3: %.4f; queries gpu %d oracle %d"
          % (bad, st["intersect_queries"], counts[0]))
    assert bad < 0.02
    assert abs(acc.sum() - ref.sum()) / ref.sum() < 0.01
    assert abs(st["intersect_queries"] - counts[0]) / counts[0] < 0.01
    assert st["error_flags"] == 0


def test_cornell_unit_scale_vs_reference_estimator(cornell_unit):
    """GPU 1024 spp against the reference's own estimator (per-lane LCG,
    256 spp, computed here). Calibration on this scene: the counter-mode
    oracle and a second reference run give 97.3-97.4 % within 3 sigma,
    relMSE 1.38-1.41x predicted, totals 0.2-0.3 % apart. Bars: >= 95 %,
    relMSE <= 1.6x predicted, totals within 1 %."""
    cam, gpu, cpu = cornell_unit
    p = H.make_params(100, 100, 1, 1, (0, 0, 0), 1024, 5, 0, 1.0, 3)
    _, acc = gpu.render(_hp(cam), p, want_accum=True)
    ref, ref2, _ = cpu.render(cam, 100, 100, 1, 1, (0, 0, 0), 256, 5, 0, seed=9, rng_mode=0,
                              threads=THREADS)
    mg, mo = acc / 1024, ref / 256
    var = np.maximum(ref2 / 256 - mo * mo, 0.0)
    sigma = np.sqrt(var / 1024 + var / 256) + 1e-5 * np.abs(mo) + 1e-6
    frac = (np.abs(mg - mo) / sigma <= 3).mean()
    relmse = np.mean((mg - mo) ** 2 / (mo ** 2 + 1e-2))
    expected = np.mean((var / 1024 + var / 256) / (mo ** 2 + 1e-2))
    total = abs(mg.sum() - mo.sum()) / mo.sum()
    print("Cornell unit scale vs reference estimator: within 3 sigma %.4f, relMSE %.4g "
          "(predicted %.4g), totals %.4g" % (frac, relmse, expected, total))
    assert frac >= 0.95
    assert relmse <= 1.6 * expected
    assert total < 0.01


def test_cornell_readme_full_render(cornell):
    """The Readme's low-sample render itself (500 x 500, 50 spp, depth 5)
    through the drop-in TraceRunner mirror (hp::TraceRunner(scene) +
    run(...), trace_runner.h:51-65): the RGBA image against the oracle's
    render of the same frame with the same random streams, tone-mapped by
    the oracle's get_image: at least as many pixels within 1/255 as between
    the oracle and its one-ulp camera move (71 % when measured; the GPU:
    91 %), and the image mean within 0.5 % (the move: 0.4 %)."""
    f, cam, _, cpu = cornell

    class KDTreeLike:
        mesh = H.Mesh(f["points"], f["triangles"], f["materials"], f["normals"], f["texcoords"],
                      f["lights"])

        def getData(self):
            return f["nodes"], f["leaf_data"]

    runner = H.TraceRunner(KDTreeLike())
    pixels = np.zeros(500 * 500 * 4, np.uint8)
    runner.run(pixels, cam["view_p"], cam["top_dir"], cam["right_dir"], cam["width"],
               cam["height"], 500, 500, 1, 1, (0, 0, 0), 50, 5, 0, 1.0, 50)
    st = runner.scene.stats()
    acc, _, counts = cpu.render(cam, 500, 500, 1, 1, (0, 0, 0), 50, 5, 0, seed=50, rng_mode=1,
                                threads=THREADS)
    img = pixels.reshape(500, 500, 4).astype(np.int32)
    ref = O.resolve(acc, 500, 500, 1, 1, 50).astype(np.int32)
    moved, _, _ = cpu.render(_shifted(cam), 500, 500, 1, 1, (0, 0, 0), 50, 5, 0, seed=50,
                             rng_mode=1, threads=THREADS)
    mimg = O.resolve(moved, 500, 500, 1, 1, 50).astype(np.int32)
    close = (np.abs(img - ref).max(axis=2) <= 1).mean()
    self_close = (np.abs(mimg - ref).max(axis=2) <= 1).mean()
    print("Readme render: %.1f ms on the GPU, %d queries (oracle %d); pixels within 1/255 %.4f "
          "(oracle vs its one-ulp camera move %.4f), mean %.3f vs %.3f"
          % (st["ms_total"], st["intersect_queries"], counts[0], close, self_close,
             img[:, :, :3].mean(), ref[:, :, :3].mean()))
    assert st["error_flags"] == 0
    assert close >= self_close
    assert abs(img[:, :, :3].mean() - ref[:, :, :3].mean()) / ref[:, :, :3].mean() < 0.005
