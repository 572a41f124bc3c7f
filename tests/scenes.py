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
