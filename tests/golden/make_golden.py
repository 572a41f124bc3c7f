"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run where the reference sources are present (REFERENCE_ROOT, or the mount
oracle.build.reference_root() finds) after `python -m oracle.build` has
built oracle/_ref/:

    python tests/golden/make_golden.py

Fixtures (all outputs of the reference's own code or tests):
  box_intersect.json   the 7 known-answer cases of SceneCLTest.box_intersect
                       (tests/src/test_scene_cl.cpp:91-116), parsed from the
                       test source
  cornell_lights.json  hp::Scene's light table for the embree Cornell box
                       (scene/simple-cornell-box/cornell_box.obj), checked by
                       SceneCLTest.load (test_scene_cl.cpp:19-27): 256
                       entries, 127 with s[1] == 14
  kdtree_hashes.json   sha256 of hp::KDTree::getData() for seeded synthetic
                       scenes written out as OBJ files, plus the OBJ text hash
  stages_room.npz      inputs and outputs of the reference kernels
                       (kernel.cl compiled as C++) on the box-room scene:
                       raygen, kdtree_intersect, s1_run, s2_*_run, get_image
  render_room.npz      a small TraceRunner::run-equivalent render
  cornell_box.npz      the embree Cornell box (scene/simple-cornell-box/
                       cornell_box.obj) as the reference's own loader and
                       SAH builder produce it (hp::KDTree: points, normals,
                       texcoords, triangles, materials, lights, getData()),
                       plus the reference kernels' estimate of its image
                       (kernel.cl compiled as C++, one host thread, per-lane
                       LCG as TraceRunner::run draws it) with per-ray sums
                       of squares from the oracle's bit-identical run

    python tests/golden/make_golden.py [--only cornell]
"""
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import hptracing_b200 as H  # noqa: E402
import oracle as O  # noqa: E402
from tests import scenes as S  # noqa: E402
from oracle import objio  # noqa: E402

from oracle import build as obuild  # noqa: E402

REF = obuild.reference_root()
if REF is None:
    raise SystemExit("reference sources not found: set REFERENCE_ROOT")


def parse_box_cases():
    """Reads the (box, start, dir, expected) sequence of the reference test."""
    src = open(os.path.join(REF, "tests", "src", "test_scene_cl.cpp")).read()
    body = src[src.index("TEST(SceneCLTest, box_intersect)"):]
    body = body[:body.index("\n}\n")]
    vec = r"Vec\(([^()]*)\)"
    cur = {}
    cases = []
    for line in body.splitlines():
        m = re.search(r"ASSIGN_F3\((\w+),\s*\(?" + vec, line)
        if m:
            vals = [float(x) for x in m.group(2).split(",")]
            if ".normalized()" in line:
                n = float(np.linalg.norm(np.asarray(vals, np.float32)))
                vals = [float(np.float32(v) / np.float32(n)) for v in vals]
            cur[m.group(1)] = vals
            continue
        m = re.search(r"EXPECT_(TRUE|FALSE)\(_box_intersect", line)
        if m:
            cases.append(dict(box_start=cur["box_start"], box_end=cur["box_end"],
                              start_p=cur["start_p"], dir=cur["dir"],
                              expected=m.group(1) == "TRUE"))
    return cases


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def tree_hash(nodes, leaf):
    """Hash of the flattened tree without the cl_float3 padding lanes."""
    return sha(nodes["box_start"][:, :3], nodes["box_end"][:, :3], nodes["child"],
               nodes["parent"], nodes["sibling"], nodes["data"], leaf)


KD_SCENES = [("room", dict(config=0, seed=0)),
             ("spheres_small", dict(config=3, seed=5, family=1, target_triangles=4000,
                                    texture_size=16)),
             ("terrain_small", dict(config=3, seed=6, family=2, target_triangles=6000,
                                    texture_size=16)),
             ("room_tess", dict(config=3, seed=7, family=0, target_triangles=2000))]


# Camera of the Cornell fixture: the embree scene's usual viewpoint, with the
# reference CLI's conventions (forward = up x right, image-plane height =
# --angle at unit distance, src/hptracing.cpp:74-78).
CORNELL_CAM = dict(view_p=(278.0, 273.0, -800.0), top_dir=(0.0, 1.0, 0.0),
                   right_dir=(-1.0, 0.0, 0.0), width=0.68, height=0.68)
# Readme.md:53-55 renders it at 500 x 500, 50 samples, depth 5; the fixture
# keeps that camera and depth on a 100 x 100 raster, 256 samples per ray.
CORNELL_RES, CORNELL_SPP, CORNELL_DEPTH, CORNELL_SEED = 100, 256, 5, 77


def cornell_fixture():
    cb = os.path.join(REF, "scene", "simple-cornell-box", "cornell_box.obj")
    r = O.ref_load_scene(cb, os.path.dirname(cb) + "/")
    mesh = H.Mesh(r["points"], r["triangles"], r["materials"], r["normals"], r["texcoords"],
                  r["lights"])
    cs = O.CpuScene(mesh, r["nodes"], r["leaf_data"])
    w = CORNELL_RES
    acc, rgba, counts = cs.refcl_render(CORNELL_CAM, w, w, 1, 1, (0, 0, 0), CORNELL_SPP,
                                        CORNELL_DEPTH, 0, 1.0, seed=CORNELL_SEED, threads=1)
    acc_o, acc2, counts_o = cs.render(CORNELL_CAM, w, w, 1, 1, (0, 0, 0), CORNELL_SPP,
                                      CORNELL_DEPTH, 0, seed=CORNELL_SEED, rng_mode=0, threads=1)
    assert np.array_equal(acc, acc_o) and counts[0] == counts_o[0], "oracle != reference kernels"
    np.savez_compressed(os.path.join(HERE, "cornell_box.npz"),
                        points=r["points"], normals=r["normals"], texcoords=r["texcoords"],
                        triangles=r["triangles"], materials=r["materials"], lights=r["lights"],
                        nodes=r["nodes"], leaf_data=r["leaf_data"],
                        camera=np.array(list(CORNELL_CAM["view_p"]) + list(CORNELL_CAM["top_dir"])
                                        + list(CORNELL_CAM["right_dir"]) +
                                        [CORNELL_CAM["width"], CORNELL_CAM["height"]], np.float32),
                        res=w, spp=CORNELL_SPP, depth=CORNELL_DEPTH, seed=CORNELL_SEED,
                        ref_accum=acc, ref_accum_sq=acc2, ref_rgba=rgba, ref_queries=counts[0])


def main():
    from oracle import build as obuild
    obuild.build()
    if "--only" in sys.argv and sys.argv[sys.argv.index("--only") + 1] == "cornell":
        cornell_fixture()
        return
    assert O.refcl_lib() is not None and O.refscene_lib() is not None, "reference not built"
    out = {}
    cases = parse_box_cases()
    assert len(cases) == 7, cases
    json.dump(cases, open(os.path.join(HERE, "box_intersect.json"), "w"), indent=1)

    cb = os.path.join(REF, "scene", "simple-cornell-box", "cornell_box.obj")
    r = O.ref_load_scene(cb, os.path.dirname(cb) + "/")
    json.dump(dict(lights=r["lights"].tolist(),
                   count_s1_eq_14=int((r["lights"][:, 1] == 14).sum()),
                   points_xyz_sha=sha(r["points"][:, :3]),
                   tree_sha=tree_hash(r["nodes"], r["leaf_data"])),
              open(os.path.join(HERE, "cornell_lights.json"), "w"))

    hashes = {}
    import tempfile
    for name, kw in KD_SCENES:
        mesh = H.Mesh.generate(**kw)
        with tempfile.TemporaryDirectory() as d:
            path = objio.write_obj(mesh, d, name)
            text = open(path, "rb").read() + open(path[:-4] + ".mtl", "rb").read()
            ref = O.ref_load_scene(path, d + "/")
        hashes[name] = dict(kw=kw, obj_sha=hashlib.sha256(text).hexdigest(),
                            tree_sha=tree_hash(ref["nodes"], ref["leaf_data"]),
                            lights_sha=sha(ref["lights"]), nodes=int(len(ref["nodes"])))
    json.dump(hashes, open(os.path.join(HERE, "kdtree_hashes.json"), "w"), indent=1)

    # Stage fixtures on the box room.
    mesh, nodes, leaf = S.make_scene(0)
    cs = O.CpuScene(mesh, nodes, leaf)
    o, d = O.raygen(S.ROOM_CAM, 24, 16, 2, 2, impl="ref")
    po, pd = O.raygen(S.PANO_CAM, 24, 12, 1, 1, impl="ref")
    ro, rd = S.random_rays(3000, seed=2)
    allo = np.concatenate([o, ro]).astype(np.float32)
    alld = np.concatenate([d, rd]).astype(np.float32)
    import ctypes as C
    n = len(allo)
    geo = np.zeros((n, 4), np.int32)
    t = np.zeros(n, np.float32)
    hit = np.zeros(n, np.int32)
    O.refcl_lib().refcl_intersect(C.byref(cs.c), n, allo.ctypes.data, alld.ctypes.data,
                                  geo.ctypes.data, t.ctypes.data, hit.ctypes.data, 1)
    h = np.nonzero(hit)[0]
    tri_ids = np.array([int(np.nonzero((mesh.triangles == g).all(axis=1))[0][0])
                        for g in geo[h]], np.int32)
    rng = np.random.default_rng(4)
    st = rng.uniform(0, 1, (len(h), 3)).astype(np.float32)
    seeds = rng.integers(0, 2 ** 48, len(h), dtype=np.int64)
    sh = cs.shade(allo[h], alld[h], st, tri_ids, t[h], seeds, impl="ref")
    a = np.nonzero(sh["branch"] >= 0)[0]
    nx = cs.next_dir(sh["branch"][a], alld[h][a], sh["hit_p"][a], sh["normal"][a],
                     sh["strength"][a], sh["param"][a], sh["seeds"][a], impl="ref")
    acc = rng.gamma(1.0, 2.0, (24 * 2 * 16 * 2, 3)).astype(np.float32)
    img = O.resolve(acc, 24, 16, 2, 2, 5, 1.2, impl="ref")
    np.savez_compressed(os.path.join(HERE, "stages_room.npz"), cam_o=o, cam_d=d, pano_o=po,
                        pano_d=pd, ray_o=allo, ray_d=alld, hit=hit, geometry=geo, t=t,
                        shade_idx=h, shade_tri=tri_ids, shade_in_strength=st, shade_in_seeds=seeds,
                        **{"shade_" + k: v for k, v in sh.items()},
                        next_idx=a, **{"next_" + k: v for k, v in nx.items()},
                        resolve_accum=acc, resolve_rgba=img)
    acc, rgba, counts = cs.refcl_render(S.ROOM_CAM, 16, 12, 2, 2, (0.1, 0.2, 0.3), sample=3,
                                        depth=4, disable_diffuse=0, brightness=1.0, seed=11,
                                        threads=1)
    np.savez_compressed(os.path.join(HERE, "render_room.npz"), accum=acc, rgba=rgba,
                        counts=counts)
    cornell_fixture()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
