"""CPU tests: the oracle and the host-side producers against the reference.

Pins, in order of strength:
  1. golden vectors produced by the reference's own code/tests (tests/golden,
     generated by tests/golden/make_golden.py) - always run;
  2. the reference's own sources compiled here (oracle/_ref) - run when the
     reference checker was built;
  3. the reference's known-answer tests (box test, Cornell light table).
"""
import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

import hptracing_b200 as H
import oracle as O
from oracle import build as obuild
from oracle import objio
from tests import scenes as S

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF = obuild.reference_root() or "<reference sources absent>"
CORNELL = os.path.join(REF, "scene", "simple-cornell-box", "cornell_box.obj")


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def tree_hash(nodes, leaf):
    return sha(nodes["box_start"][:, :3], nodes["box_end"][:, :3], nodes["child"],
               nodes["parent"], nodes["sibling"], nodes["data"], leaf)


def test_box_intersect_known_answers(built):
    """SceneCLTest.box_intersect (tests/src/test_scene_cl.cpp:91-116)."""
    cases = json.load(open(os.path.join(GOLD, "box_intersect.json")))
    assert len(cases) == 7
    for c in cases:
        assert O.box_intersect(c["box_start"], c["box_end"], c["start_p"], c["dir"]) == \
            c["expected"], c


def test_cornell_light_table_golden(built):
    """SceneCLTest.load (test_scene_cl.cpp:19-27): 256 entries, 127 pick s[1]==14."""
    g = json.load(open(os.path.join(GOLD, "cornell_lights.json")))
    lights = np.asarray(g["lights"], np.int32)
    assert lights.shape == (256, 4)
    assert g["count_s1_eq_14"] == 127 == int((lights[:, 1] == 14).sum())
    if not os.path.exists(CORNELL):
        pytest.skip("reference scene not mounted")
    m = H.Mesh.load_obj(CORNELL, os.path.dirname(CORNELL) + "/")
    assert np.array_equal(m.lights, lights)
    assert sha(m.points[:, :3]) == g["points_xyz_sha"]
    nodes, leaf = H.build_kdtree(m.points, m.triangles)
    assert tree_hash(nodes, leaf) == g["tree_sha"]


@pytest.mark.parametrize("name", ["room", "spheres_small", "terrain_small", "room_tess"])
def test_kdtree_matches_reference_hash(built, name):
    """The SAH builder reproduces hp::KDTree::getData() bit for bit."""
    g = json.load(open(os.path.join(GOLD, "kdtree_hashes.json")))[name]
    mesh = H.Mesh.generate(**g["kw"])
    with tempfile.TemporaryDirectory() as d:
        path = objio.write_obj(mesh, d, name)
        text = open(path, "rb").read() + open(path[:-4] + ".mtl", "rb").read()
        assert hashlib.sha256(text).hexdigest() == g["obj_sha"]
        loaded = H.Mesh.load_obj(path, d + "/")
    nodes, leaf = H.build_kdtree(loaded.points, loaded.triangles)
    assert len(nodes) == g["nodes"]
    assert tree_hash(nodes, leaf) == g["tree_sha"]
    assert sha(loaded.lights) == g["lights_sha"]


def test_kdtree_threads_do_not_change_result(built):
    mesh = H.Mesh.generate(3, seed=3, family=2, target_triangles=60000, texture_size=8)
    a = H.build_kdtree(mesh.points, mesh.triangles, threads=1)
    b = H.build_kdtree(mesh.points, mesh.triangles, threads=8)
    assert tree_hash(*a) == tree_hash(*b)


REF_SCENES = ["simple-cornell-box/cornell_box.obj", "geometries/geometries.obj",
              "cornell-box-orig/CornellBox-Sphere.obj", "cornell-box-orig/CornellBox-Glossy.obj",
              "cornell-box/untitled.obj"]


def _strip_textures(obj, d):
    base = os.path.dirname(obj)
    for f in os.listdir(base):
        if f.endswith(".mtl"):
            txt = open(os.path.join(base, f)).read().splitlines()
            open(os.path.join(d, f), "w").write(
                "\n".join(x for x in txt if not x.strip().startswith("map_")) + "\n")
    dst = os.path.join(d, os.path.basename(obj))
    open(dst, "w").write(open(obj).read())
    return dst


@pytest.mark.parametrize("rel", REF_SCENES)
def test_loader_and_builder_match_reference_sources(built, rel):
    """Our OBJ/MTL reader, light table and SAH tree vs the reference's own
    hp::KDTree compiled from its sources (texture maps dropped: the
    reference decodes PNG/JPG through ImageMagick, absent here)."""
    if O.refscene_lib() is None or not os.path.exists(os.path.join(REF, "scene", rel)):
        pytest.skip("reference sources not available")
    with tempfile.TemporaryDirectory() as d:
        obj = _strip_textures(os.path.join(REF, "scene", rel), d)
        m = H.Mesh.load_obj(obj, d + "/")
        r = O.ref_load_scene(obj, d + "/")
    for k in ("points", "normals"):
        assert np.array_equal(getattr(m, k)[:, :3], r[k][:, :3]), k
    for k in ("texcoords", "triangles", "lights"):
        assert np.array_equal(getattr(m, k), r[k]), k
    assert m.materials.tobytes() == r["materials"].tobytes()
    nodes, leaf = H.build_kdtree(m.points, m.triangles)
    assert tree_hash(nodes, leaf) == tree_hash(r["nodes"], r["leaf_data"])


@pytest.fixture(scope="module")
def room(built):
    mesh, nodes, leaf = S.make_scene(0)
    return mesh, O.CpuScene(mesh, nodes, leaf)


def test_oracle_stages_match_golden(room):
    """The oracle restatement reproduces the reference kernels' outputs
    recorded in tests/golden/stages_room.npz bit for bit."""
    mesh, cs = room
    g = np.load(os.path.join(GOLD, "stages_room.npz"))
    o, d = O.raygen(S.ROOM_CAM, 24, 16, 2, 2)
    assert np.array_equal(o, g["cam_o"]) and np.array_equal(d, g["cam_d"])
    po, pd = O.raygen(S.PANO_CAM, 24, 12, 1, 1)
    assert np.array_equal(po, g["pano_o"]) and np.array_equal(pd, g["pano_d"])
    r = cs.intersect(g["ray_o"], g["ray_d"], threads=1)
    hit = r["tri"] >= 0
    assert np.array_equal(hit.astype(np.int32), g["hit"])
    assert np.array_equal(mesh.triangles[r["tri"][hit]], g["geometry"][hit])
    assert np.array_equal(r["t"][hit], g["t"][hit])
    h = g["shade_idx"]
    sh = cs.shade(g["ray_o"][h], g["ray_d"][h], g["shade_in_strength"], g["shade_tri"],
                  g["t"][h], g["shade_in_seeds"])
    alive = sh["branch"] >= 0
    for k in ("contrib", "branch"):
        assert np.array_equal(sh[k], g["shade_" + k]), k
    for k in ("hit_p", "normal", "strength", "param", "seeds"):
        assert np.array_equal(sh[k][alive], g["shade_" + k][alive]), k
    a = g["next_idx"]
    nx = cs.next_dir(g["shade_branch"][a], g["ray_d"][h][a], g["shade_hit_p"][a],
                     g["shade_normal"][a], g["shade_strength"][a], g["shade_param"][a],
                     g["shade_seeds"][a])
    for k in ("origins", "directions", "strength", "alive", "seeds"):
        assert np.array_equal(nx[k], g["next_" + k]), k
    img = O.resolve(g["resolve_accum"], 24, 16, 2, 2, 5, 1.2)
    assert np.array_equal(img, g["resolve_rgba"])


def test_oracle_render_matches_golden(room):
    """TraceRunner::run restatement == the reference kernels' render."""
    _, cs = room
    g = np.load(os.path.join(GOLD, "render_room.npz"))
    acc, _, counts = cs.render(S.ROOM_CAM, 16, 12, 2, 2, (0.1, 0.2, 0.3), sample=3, depth=4,
                               seed=11, rng_mode=0, threads=1)
    assert np.array_equal(acc, g["accum"])
    assert counts[0] == g["counts"][0] and counts[1] == g["counts"][1]
    assert np.array_equal(O.resolve(acc, 16, 12, 2, 2, 3, 1.0), g["rgba"])


def _need_refcl():
    if O.refcl_lib() is None:
        pytest.skip("reference kernels not built")


@pytest.mark.parametrize("config,kw", [(0, {}), (3, dict(family=1, target_triangles=8000,
                                                          texture_size=32)),
                                       (3, dict(family=2, target_triangles=20000,
                                                texture_size=32))])
def test_oracle_matches_reference_kernels(built, config, kw):
    """Stage by stage, on seeded rays, against kernel.cl compiled as C++."""
    _need_refcl()
    import ctypes as C
    mesh, nodes, leaf = S.make_scene(config, seed=2, **kw)
    cs = O.CpuScene(mesh, nodes, leaf)
    o, d = S.random_rays(20000, seed=7)
    r = cs.intersect(o, d)
    n = len(o)
    geo = np.zeros((n, 4), np.int32)
    t = np.zeros(n, np.float32)
    hit = np.zeros(n, np.int32)
    O.refcl_lib().refcl_intersect(C.byref(cs.c), n, o.ctypes.data, d.ctypes.data,
                                  geo.ctypes.data, t.ctypes.data, hit.ctypes.data, 8)
    h = r["tri"] >= 0
    assert np.array_equal(h, hit.astype(bool))
    assert np.array_equal(mesh.triangles[r["tri"][h]], geo[h])
    assert np.array_equal(r["t"][h], t[h])
    idx = np.nonzero(h)[0]
    rng = np.random.default_rng(1)
    st = rng.uniform(0, 1, (len(idx), 3)).astype(np.float32)
    seeds = rng.integers(0, 2 ** 48, len(idx), dtype=np.int64)
    a = cs.shade(o[idx], d[idx], st, r["tri"][idx], r["t"][idx], seeds)
    b = cs.shade(o[idx], d[idx], st, r["tri"][idx], r["t"][idx], seeds, impl="ref")
    alive = a["branch"] >= 0
    for k in ("contrib", "branch"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("hit_p", "normal", "strength", "param", "seeds"):
        assert np.array_equal(a[k][alive], b[k][alive]), k
    sel = np.nonzero(alive)[0]
    args = (a["branch"][sel], d[idx][sel], a["hit_p"][sel], a["normal"][sel],
            a["strength"][sel], a["param"][sel], a["seeds"][sel])
    x = cs.next_dir(*args)
    y = cs.next_dir(*args, impl="ref")
    for k in x:
        assert np.array_equal(x[k], y[k]), k


def test_oracle_render_matches_reference_kernels(built):
    _need_refcl()
    mesh, nodes, leaf = S.make_scene(3, seed=4, family=1, target_triangles=6000,
                                     texture_size=32)
    cs = O.CpuScene(mesh, nodes, leaf)
    for cam, bg, dd in ((S.ROOM_CAM, (0, 0, 0), 0), (S.PANO_CAM, (0.2, 0.1, 0.0), 1)):
        w, h = (20, 16) if cam["height"] > 0 else (24, 12)
        a, _, ca = cs.render(cam, w, h, 1, 1, bg, 3, 6, dd, seed=5, rng_mode=0, threads=1)
        b, _, cb = cs.refcl_render(cam, w, h, 1, 1, bg, 3, 6, dd, 1.0, seed=5, threads=1)
        assert np.array_equal(a, b)
        assert ca[0] == cb[0] and ca[1] == cb[1]


def test_kdtree_traversal_vs_bruteforce(room):
    """SceneCLTest.kdtree_intersect (test_scene_cl.cpp:220-232): rope
    traversal vs brute force within 0.1 (-1 for a miss), on a 100 x 100 grid
    of +z rays. The grid avoids x / y values of scene vertices: a ray with a
    zero direction component that lies exactly in a node's face plane gets
    0/0 = NaN slab distances in _box_intersect (kernel.cl:51-83) and is
    rejected by both neighbouring boxes - a reference behaviour the oracle
    and the GPU reproduce, but brute force does not share."""
    _, cs = room
    i, j = np.meshgrid(np.arange(100), np.arange(100))
    o = np.stack([(i.ravel() + 0.37) / 100.0, (j.ravel() + 0.29) / 100.0,
                  np.full(10000, -5.0)], 1)
    d = np.tile(np.array([[0, 0, 1.0]]), (10000, 1))
    r = cs.intersect(o, d)
    btri, bt = cs.brute_f64(o, d)
    t_kd = np.where(r["tri"] >= 0, r["t"], -1.0)
    t_bf = np.where(btri >= 0, bt, -1.0)
    assert np.abs(t_kd - t_bf).max() < 0.1
