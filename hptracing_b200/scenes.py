"""Seeded synthetic workloads: scenes and cameras of the benchmark configs.

The synthetic scene families are generated in C++ (hpt_mesh_generate,
csrc/scene_gen.cpp) and their KD-trees are built by the SAH builder
(hpt_kdtree_build); this module only names the cameras and wraps the two
calls. The reference renders scenes from OBJ files; these seeded families
stand in for its benchmark scenes:

    0  box room, ~36 triangles            (camera ROOM_CAM)
    1  room + 64 UV spheres, ~61k         (camera ROOM_CAM)
    2  heightfield + 16 columns, ~2.4M    (camera terrain_cam())
"""
import math

from . import Mesh, build_kdtree, make_camera

# Box-room camera: eye (0.5, 0.5, -1.4), forward = up x right = +z, 40 deg.
ROOM_CAM = dict(view_p=(0.5, 0.5, -1.4), top_dir=(0.0, 1.0, 0.0), right_dir=(-1.0, 0.0, 0.0),
                width=2 * math.tan(math.radians(20)), height=2 * math.tan(math.radians(20)))
# Panorama from inside the room (height < 0 selects set_viewdirs_vr).
PANO_CAM = dict(view_p=(0.5, 0.5, 0.5), top_dir=(0.0, 1.0, 0.0), right_dir=(0.0, 0.0, 1.0),
                width=1.0, height=-1.0)


def terrain_cam(aspect=16 / 9):
    """Camera over the heightfield family, 50 degrees vertical field."""
    a = math.radians(25)
    h = 2 * math.tan(a)
    return dict(view_p=(0.0, 0.9, -1.6), top_dir=(0.0, math.cos(a), math.sin(a)),
                right_dir=(-1.0, 0.0, 0.0), width=aspect * h, height=h)


def hp_camera(c):
    """A camera dict of this module -> the C ABI's hpt_camera."""
    return make_camera(c["view_p"], c["top_dir"], c["right_dir"], c["width"], c["height"])


def make_scene(config, seed=0, **kw):
    """Generates scene family `config` and builds its KD-tree.
    Returns (mesh, reference node array, leaf list)."""
    mesh = Mesh.generate(config, seed=seed, **kw)
    nodes, leaf = build_kdtree(mesh.points, mesh.triangles)
    return mesh, nodes, leaf
