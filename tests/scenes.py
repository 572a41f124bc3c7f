"""Seeded test ray sets shared by the tests (the scenes and cameras live in
hptracing_b200.scenes)."""

import numpy as np

from hptracing_b200.scenes import PANO_CAM, ROOM_CAM, hp_camera, make_scene, terrain_cam  # noqa: F401


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


def aabb_random_rays(mesh, n, seed, pad=0.1):
    """Origins uniform in the scene's bounding box grown by `pad` of its
    extent on every side, directions uniform on the sphere."""
    lo, hi = mesh.points[:, :3].min(0), mesh.points[:, :3].max(0)
    g = pad * (hi - lo)
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo - g, hi + g, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o, d.astype(np.float32)


def oracle_bounce_rays(cpu, o, d, bounces, seed, threads=None):
    """The rays the oracle sends to its intersect stage after `bounces`
    shading passes (s1_run + s2_*_run) that start from rays (o, d) with
    strength 1 and seeded 48-bit LCG states; every stage is the oracle's."""
    rng = np.random.default_rng(seed)
    st = np.ones((len(o), 3), np.float32)
    sd = rng.integers(0, 2 ** 48, len(o), dtype=np.int64)
    kw = {} if threads is None else dict(threads=threads)
    for _ in range(bounces):
        r = cpu.intersect(o, d, **kw)
        h = r["tri"] >= 0
        sh = cpu.shade(o[h], d[h], st[h], r["tri"][h], r["t"][h], sd[h])
        a = sh["branch"] >= 0
        nd = cpu.next_dir(sh["branch"][a], d[h][a], sh["hit_p"][a], sh["normal"][a],
                          sh["strength"][a], sh["param"][a], sh["seeds"][a])
        k = nd["alive"] == 1
        o, d, st, sd = nd["origins"][k], nd["directions"][k], nd["strength"][k], nd["seeds"][k]
    return np.ascontiguousarray(o), np.ascontiguousarray(d)


def hit_parity(ref, tri, t, u, v):
    """Closest hits of the device against the oracle. Returns counts:
    rays, hits, `cap` (rays past the reference's 512-leaf gather cap, not
    compared), `ties` (another triangle at the bit-identical t: a ray
    through a shared edge or vertex) and `other` (any other difference)."""
    ok = ref["overflow"] == 0
    diff = ok & ((ref["tri"] != tri) | (ref["t"].view(np.int32) != t.view(np.int32)) |
                 (ref["u"].view(np.int32) != u.view(np.int32)) |
                 (ref["v"].view(np.int32) != v.view(np.int32)))
    tie = diff & (ref["t"].view(np.int32) == t.view(np.int32)) & (ref["tri"] >= 0) & (tri >= 0)
    return dict(rays=int(len(tri)), hits=int((ref["tri"] >= 0).sum()), cap=int((~ok).sum()),
                ties=int(tie.sum()), other=int((diff & ~tie).sum()),
                first_other=np.flatnonzero(diff & ~tie)[:5].tolist())
