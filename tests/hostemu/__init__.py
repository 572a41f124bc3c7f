"""ctypes wrapper of libhpt_emu.so: the GPU per-ray code built for the host
(test infrastructure only)."""
import ctypes as C
import os

import numpy as np

from hptracing_b200._lib import SceneDesc

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        from . import build
        build.build()
        L = C.CDLL(build.LIB)
        vp = C.c_void_p
        L.emu_scene_create.restype = vp
        L.emu_scene_create.argtypes = [C.POINTER(SceneDesc), C.POINTER(C.c_int)]
        L.emu_scene_destroy.argtypes = [vp]
        L.emu_scene_counts.argtypes = [vp, vp]
        L.emu_intersect.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp, vp, vp]
        L.emu_intersect_step.argtypes = L.emu_intersect.argtypes
        L.emu_shade.argtypes = [vp, C.c_int] + [vp] * 6 + [C.c_int] + [vp] * 6
        L.emu_next_dir.argtypes = [vp, C.c_int] + [vp] * 11
        L.emu_tree.argtypes = [vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None and a.size else None


class EmuScene:
    def __init__(self, mesh, nodes, leaf):
        self._keep = [mesh.points, mesh.normals, mesh.texcoords, mesh.triangles, nodes, leaf,
                      mesh.materials, mesh.lights, mesh.texture_data, mesh.texture_dims]
        d = SceneDesc()
        d.points, d.num_points = _p(mesh.points), len(mesh.points)
        d.normals, d.num_normals = _p(mesh.normals), len(mesh.normals)
        d.texcoords, d.num_texcoords = _p(mesh.texcoords), len(mesh.texcoords)
        d.triangles, d.num_triangles = _p(mesh.triangles), len(mesh.triangles)
        d.nodes, d.num_nodes = _p(nodes), len(nodes)
        d.leaf_data, d.num_leaf_data = _p(leaf), len(leaf)
        d.materials, d.num_materials = _p(mesh.materials), len(mesh.materials)
        d.lights, d.num_lights = _p(mesh.lights), len(mesh.lights)
        d.texture_data = _p(mesh.texture_data)
        d.num_textures = len(mesh.texture_dims)
        d.texture_dims = _p(mesh.texture_dims)
        self._desc = d
        st = C.c_int()
        self.h = lib().emu_scene_create(C.byref(d), C.byref(st))
        if not self.h:
            raise RuntimeError("pack failed: status %d" % st.value)

    def __del__(self):
        if getattr(self, "h", None):
            lib().emu_scene_destroy(self.h)

    def counts(self):
        c = np.zeros(4, np.int32)
        lib().emu_scene_counts(self.h, _p(c))
        return dict(nodes=int(c[0]), leaves=int(c[1]), refs=int(c[2]), max_depth=int(c[3]))

    def intersect(self, o, d, hints=None, smem_nodes=0, step=False):
        o = np.ascontiguousarray(o, np.float32)
        d = np.ascontiguousarray(d, np.float32)
        n = len(o)
        tri = np.zeros(n, np.int32)
        t, u, v = (np.zeros(n, np.float32) for _ in range(3))
        node = np.zeros(n, np.int32)
        cnt = np.zeros(4, np.int64)
        err = np.zeros(3, np.int64)
        h = None if hints is None else np.ascontiguousarray(hints, np.int32)
        fn = lib().emu_intersect_step if step else lib().emu_intersect
        fn(self.h, n, _p(o), _p(d), _p(h), smem_nodes, _p(tri), _p(t), _p(u), _p(v), _p(node),
           _p(cnt), _p(err))
        return dict(tri=tri, t=t, u=u, v=v, node=node, counts=cnt, err=err)

    def shade(self, o, d, strength, tri, t, seeds, disable_diffuse=0):
        o, d, s = (np.ascontiguousarray(x, np.float32) for x in (o, d, strength))
        tri = np.ascontiguousarray(tri, np.int32)
        t = np.ascontiguousarray(t, np.float32)
        sd = np.ascontiguousarray(seeds, np.uint64).copy()
        n = len(o)
        contrib, hit_p, normal, s_out = (np.zeros((n, 3), np.float32) for _ in range(4))
        branch = np.zeros(n, np.int32)
        param = np.zeros(n, np.float32)
        lib().emu_shade(self.h, n, _p(o), _p(d), _p(s), _p(tri), _p(t), _p(sd), disable_diffuse,
                        _p(contrib), _p(branch), _p(hit_p), _p(normal), _p(s_out), _p(param))
        return dict(contrib=contrib, branch=branch, hit_p=hit_p, normal=normal, strength=s_out,
                    param=param, seeds=sd)

    def next_dir(self, branch, d, hit_p, normal, strength, param, seeds):
        br = np.ascontiguousarray(branch, np.int32)
        d, hp_, nm, s = (np.ascontiguousarray(x, np.float32) for x in (d, hit_p, normal, strength))
        pa = np.ascontiguousarray(param, np.float32)
        sd = np.ascontiguousarray(seeds, np.uint64).copy()
        n = len(br)
        o_out, d_out, s_out = (np.zeros((n, 3), np.float32) for _ in range(3))
        alive = np.zeros(n, np.int32)
        lib().emu_next_dir(self.h, n, _p(br), _p(d), _p(hp_), _p(nm), _p(s), _p(pa), _p(sd),
                           _p(o_out), _p(d_out), _p(s_out), _p(alive))
        return dict(origins=o_out, directions=d_out, strength=s_out, alive=alive, seeds=sd)

    def tree(self):
        c = self.counts()
        meta = np.zeros(c["nodes"], np.uint32)
        split = np.zeros(c["nodes"], np.float32)
        leaves = np.zeros((c["leaves"], 16), np.int32)
        lib().emu_tree(self.h, _p(meta), _p(split), _p(leaves))
        return meta, split, leaves
