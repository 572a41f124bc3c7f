"""Seeded test scenes and cameras shared by the tests."""
import math

import numpy as np

import hptracing_b200 as H

# Box-room camera: eye (0.5, 0.5, -1.4), forward = up x right = +z, 40 deg.
ROOM_CAM = dict(view_p=(0.5, 0.5, -1.4), top_dir=(0.0, 1.0, 0.0), right_dir=(-1.0, 0.0, 0.0),
                width=2 * math.tan(math.radians(20)), height=2 * math.tan(math.radians(20)))
# Panorama from inside the room (height < 0 selects set_viewdirs_vr).
PANO_CAM = dict(view_p=(0.5, 0.5, 0.5), top_dir=(0.0, 1.0, 0.0), right_dir=(0.0, 0.0, 1.0),
                width=1.0, height=-1.0)


def terrain_cam(aspect=16 / 9):
    a = math.radians(25)
    h = 2 * math.tan(a)
    return dict(view_p=(0.0, 0.9, -1.6), top_dir=(0.0, math.cos(a), math.sin(a)),
                right_dir=(-1.0, 0.0, 0.0), width=aspect * h, height=h)


def hp_camera(c):
    return H.make_camera(c["view_p"], c["top_dir"], c["right_dir"], c["width"], c["height"])


def make_scene(config, seed=0, **kw):
    mesh = H.Mesh.generate(config, seed=seed, **kw)
    nodes, leaf = H.build_kdtree(mesh.points, mesh.triangles)
    return mesh, nodes, leaf


def random_rays(n, seed, lo=-0.1, hi=1.1):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o, d.astype(np.float32)


def edge_rays(mesh, nodes, n=600, seed=7):
    """mesh: anything with the reference's `points` and `triangles` arrays;
    nodes: the reference node array. Seeded ray sets aimed at the traversal's edge cases, by name:
    axis-parallel directions, directions with one zero component, origins on
    the reference tree's node faces (split planes), such origins with
    directions inside that plane, rays aimed exactly at mesh vertices and at
    edge midpoints (shared-edge ties), and a few degenerate rays (zero,
    NaN and infinite components, origins outside the scene)."""
    rng = np.random.default_rng(seed)
    lo, hi = mesh.points[:, :3].min(0), mesh.points[:, :3].max(0)
    out = {}

    def unit(v):
        return v / np.linalg.norm(v, axis=1, keepdims=True)

    o = rng.uniform(lo, hi, (n, 3))
    axes = np.concatenate([np.eye(3), -np.eye(3)])
    out["axis"] = (o, axes[rng.integers(0, 6, n)])
    d = rng.normal(size=(n, 3))
    d[np.arange(n), rng.integers(0, 3, n)] = 0
    out["one_zero"] = (o, unit(d))
    faces = np.concatenate([np.asarray(nodes["box_start"]).reshape(len(nodes), -1)[:, :3],
                            np.asarray(nodes["box_end"]).reshape(len(nodes), -1)[:, :3]])
    o2 = rng.uniform(lo, hi, (n, 3))
    ax = rng.integers(0, 3, n)
    o2[np.arange(n), ax] = faces[rng.integers(0, len(faces), n)][np.arange(n), ax]
    d2 = unit(rng.normal(size=(n, 3)))
    out["on_split"] = (o2, d2)
    d3 = d2.copy()
    d3[np.arange(n), ax] = 0
    out["in_split"] = (o2, unit(d3))
    P = mesh.points[:, :3].astype(np.float64)
    T = mesh.triangles[:, :3]
    o4 = rng.uniform(lo - 0.3, hi + 0.3, (n, 3))
    v = P[T[rng.integers(0, len(T), n), rng.integers(0, 3, n)]]
    out["vertex"] = (o4, unit(v - o4))
    t = T[rng.integers(0, len(T), n)]
    out["edge"] = (o4, unit(0.5 * (P[t[:, 0]] + P[t[:, 1]]) - o4))
    c = 0.5 * (lo + hi)
    out["degenerate"] = (
        np.array([c, c, c, c, [np.nan, c[1], c[2]], [c[0], np.inf, c[2]], hi + 4, lo - 3]),
        np.array([[0, 0, 0], [np.nan, 0, 1], [np.inf, 0, 0], [1e-30, 0, 0], [0, 0, 1], [0, 0, 1],
                  [1, 1, 1], [0, 0, 1]]))
    return {k: (np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32))
            for k, (a, b) in out.items()}


def check_edge_hits(name, o, d, ref, tri, t, u, v):
    """The contract for edge_rays(): bit-exact closest hits, except
    (a) a ray aimed exactly at a vertex or an edge may report another of the
        triangles meeting there, at the bit-identical t (it passes through a
        leaf's edge or corner, and the tie rank goes to a triangle of a leaf
        the walk only touches there), in under 1 % of such rays;
    (b) a ray lying exactly in a split plane is walked on both sides of it,
        yet where it also runs along a mesh edge in that plane it may still
        report the edge's other triangle (about 1 in 5000 such rays on the
        spheres scene, t within 1 ulp): under 0.5 % of such rays;
    (c) a zero direction vector is a miss (the reference reports t = +inf);
    and rays past the reference's 512-leaf gather cap are not compared."""
    ok = ref["overflow"] == 0
    bad = ok & ((ref["tri"] != tri) | (ref["t"].view(np.int32) != t.view(np.int32)) |
                (ref["u"].view(np.int32) != u.view(np.int32)) |
                (ref["v"].view(np.int32) != v.view(np.int32)))
    if name in ("vertex", "edge"):
        same_t = ref["t"].view(np.int32) == t.view(np.int32)
        assert (bad & ~same_t).sum() == 0, (name, np.flatnonzero(bad & ~same_t)[:5])
        assert bad.mean() < 0.01, (name, bad.sum())
    elif name == "in_split":
        assert bad.mean() < 0.005, (name, bad.sum())
    elif name == "degenerate":
        zero = ~(np.abs(d) > 0).any(axis=1)
        assert (bad & ~zero).sum() == 0, (name, np.flatnonzero(bad & ~zero))
        assert (tri[zero] < 0).all()
    else:
        assert bad.sum() == 0, (name, np.flatnonzero(bad)[:5])
