"""The oracle: CPU checker of the GPU path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
package, and only to check or time the reference behaviour; the product
(hptracing_b200) never touches it.

  - liboracle.so  : hpt_oracle.cpp, a restatement of the reference kernels
                    (src/hp/cl_src/kernel.cl) and host loop
                    (src/hp/trace_runner.cpp:116-356).
  - _ref/librefcl.so    : the reference's own kernel.cl compiled as C++
  - _ref/librefscene.so : the reference's own scene loader + SAH KD-tree
    (both built from the reference sources by oracle/build.py where they
    exist; they travel to GPU hosts as built files).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
i32, i64, u64, f32 = C.c_int32, C.c_int64, C.c_uint64, C.c_float
vp = C.c_void_p


class OracleScene(C.Structure):
    _fields_ = [("points", vp), ("normals", vp), ("num_normals", i32), ("texcoords", vp),
                ("num_texcoords", i32), ("triangles", vp), ("num_triangles", i32),
                ("nodes", vp), ("num_nodes", i32), ("leaf_data", vp), ("materials", vp),
                ("lights", vp), ("num_lights", i32), ("texture_data", vp),
                ("num_textures", i32), ("texture_dims", vp)]


class OracleCamera(C.Structure):
    _fields_ = [("view_p", f32 * 3), ("top_dir", f32 * 3), ("right_dir", f32 * 3),
                ("width", f32), ("height", f32)]


class RefSceneView(C.Structure):
    _fields_ = [("points", vp), ("num_points", C.c_int), ("normals", vp),
                ("num_normals", C.c_int), ("texcoords", vp), ("num_texcoords", C.c_int),
                ("triangles", vp), ("num_triangles", C.c_int), ("materials", vp),
                ("num_materials", C.c_int), ("lights", vp), ("num_lights", C.c_int),
                ("nodes", vp), ("num_nodes", C.c_int), ("leaf_data", vp),
                ("num_leaf_data", C.c_int)]


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data if a.size else None


_libs = {}


def _load(name, path, sigs):
    if name not in _libs:
        if not os.path.exists(path):
            if name == "oracle":
                from . import build
                build.build_oracle()
            else:
                return None
        L = C.CDLL(path)
        for fn, (res, args) in sigs.items():
            f = getattr(L, fn)
            f.restype = res
            f.argtypes = args
        _libs[name] = L
    return _libs[name]


_ORACLE_SIGS = {
    "oracle_box_intersect": (C.c_int, [vp, vp, vp, vp]),
    "oracle_intersect": (None, [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int]),
    "oracle_brute_f64": (None, [vp, C.c_int, vp, vp, vp, vp, C.c_int]),
    "oracle_shade": (None, [vp, C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp,
                            vp]),
    "oracle_next_dir": (None, [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "oracle_raygen": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp]),
    "oracle_resolve": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, f32, vp]),
    "oracle_render": (None, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int,
                             C.c_int, u64, C.c_int, C.c_int, vp, vp, vp]),
}
_REFCL_SIGS = {
    "refcl_sizeof_unit_data": (C.c_int, []),
    "refcl_intersect": (None, [vp, C.c_int, vp, vp, vp, vp, vp, C.c_int]),
    "refcl_shade": (None, [vp, C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp,
                           vp]),
    "refcl_next": (None, [vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "refcl_raygen": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp]),
    "refcl_get_image": (None, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, f32, vp]),
    "refcl_render": (None, [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int,
                            C.c_int, f32, u64, C.c_int, vp, vp, vp]),
}
_REFSCENE_SIGS = {
    "refscene_load": (vp, [C.c_char_p, C.c_char_p]),
    "refscene_view": (None, [vp, C.POINTER(RefSceneView)]),
    "refscene_free": (None, [vp]),
    "refscene_sizeof_node": (C.c_int, []),
    "refscene_sizeof_material": (C.c_int, []),
    "refscene_log": (None, [C.c_int]),
}


def oracle_lib():
    return _load("oracle", os.path.join(HERE, "liboracle.so"), _ORACLE_SIGS)


def refcl_lib():
    """The reference's kernel.cl compiled as C++, or None if not built."""
    return _load("refcl", os.path.join(HERE, "_ref", "librefcl.so"), _REFCL_SIGS)


def refscene_lib():
    """The reference's scene loader + KD-tree, or None if not built."""
    return _load("refscene", os.path.join(HERE, "_ref", "librefscene.so"), _REFSCENE_SIGS)


def _f32(a, cols=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a.reshape(-1, cols) if cols else a


class CpuScene:
    """Host arrays of a scene in the reference layouts, as both the oracle
    and the reference kernels consume them."""

    def __init__(self, mesh, nodes, leaf_data):
        self.points = np.ascontiguousarray(mesh.points, np.float32)
        self.normals = np.ascontiguousarray(mesh.normals, np.float32)
        self.texcoords = np.ascontiguousarray(mesh.texcoords, np.float32)
        self.triangles = np.ascontiguousarray(mesh.triangles, np.int32)
        self.materials = np.ascontiguousarray(mesh.materials)
        self.lights = np.ascontiguousarray(mesh.lights, np.int32)
        self.texture_data = np.ascontiguousarray(mesh.texture_data, np.uint8)
        self.texture_dims = np.ascontiguousarray(mesh.texture_dims, np.int32)
        self.nodes = np.ascontiguousarray(nodes)
        self.leaf_data = np.ascontiguousarray(leaf_data, np.int32)
        s = OracleScene()
        s.points = _p(self.points)
        s.normals = _p(self.normals)
        s.num_normals = len(self.normals)
        s.texcoords = _p(self.texcoords)
        s.num_texcoords = len(self.texcoords)
        s.triangles = _p(self.triangles)
        s.num_triangles = len(self.triangles)
        s.nodes = _p(self.nodes)
        s.num_nodes = len(self.nodes)
        s.leaf_data = _p(self.leaf_data)
        s.materials = _p(self.materials)
        s.lights = _p(self.lights)
        s.num_lights = len(self.lights)
        s.texture_data = _p(self.texture_data)
        s.num_textures = len(self.texture_dims)
        s.texture_dims = _p(self.texture_dims)
        self.c = s  # the refcl driver's struct has the same layout

    # ---- oracle restatement -------------------------------------------
    def intersect(self, o, d, threads=8):
        o, d = _f32(o, 3), _f32(d, 3)
        n = len(o)
        tri = np.zeros(n, np.int32)
        t, u, v = (np.zeros(n, np.float32) for _ in range(3))
        leaves = np.zeros(n, np.int32)
        ovf = np.zeros(n, np.int32)
        oracle_lib().oracle_intersect(C.byref(self.c), n, _p(o), _p(d), _p(tri), _p(t), _p(u),
                                      _p(v), _p(leaves), _p(ovf), threads)
        return dict(tri=tri, t=t, u=u, v=v, leaves=leaves, overflow=ovf)

    def brute_f64(self, o, d, threads=8):
        o, d = _f32(o, 3), _f32(d, 3)
        n = len(o)
        tri = np.zeros(n, np.int32)
        t = np.zeros(n, np.float64)
        oracle_lib().oracle_brute_f64(C.byref(self.c), n, _p(o), _p(d), _p(tri), _p(t), threads)
        return tri, t

    def shade(self, o, d, strength, tri, t, seeds, disable_diffuse=0, impl="oracle"):
        o, d, s = _f32(o, 3), _f32(d, 3), _f32(strength, 3)
        tri = np.ascontiguousarray(tri, np.int32)
        t = _f32(t)
        sd = np.ascontiguousarray(seeds, dtype=np.int64).copy()
        n = len(o)
        contrib, hit_p, normal, s_out = (np.zeros((n, 3), np.float32) for _ in range(4))
        branch = np.zeros(n, np.int32)
        param = np.zeros(n, np.float32)
        L = oracle_lib() if impl == "oracle" else refcl_lib()
        fn = L.oracle_shade if impl == "oracle" else L.refcl_shade
        fn(C.byref(self.c), n, _p(o), _p(d), _p(s), _p(tri), _p(t), _p(sd), disable_diffuse,
           _p(contrib), _p(branch), _p(hit_p), _p(normal), _p(s_out), _p(param))
        return dict(contrib=contrib, branch=branch, hit_p=hit_p, normal=normal, strength=s_out,
                    param=param, seeds=sd)

    def next_dir(self, branch, d, hit_p, normal, strength, param, seeds, impl="oracle"):
        br = np.ascontiguousarray(branch, np.int32)
        d, hp_, nm, s = (_f32(x, 3) for x in (d, hit_p, normal, strength))
        pa = _f32(param)
        sd = np.ascontiguousarray(seeds, dtype=np.int64).copy()
        n = len(br)
        o_out, d_out, s_out = (np.zeros((n, 3), np.float32) for _ in range(3))
        alive = np.zeros(n, np.int32)
        if impl == "oracle":
            oracle_lib().oracle_next_dir(C.byref(self.c), n, _p(br), _p(d), _p(hp_), _p(nm),
                                         _p(s), _p(pa), _p(sd), _p(o_out), _p(d_out), _p(s_out),
                                         _p(alive))
        else:
            # the reference runs one kernel per branch over its own list
            for b in range(4):
                idx = np.nonzero(br == b)[0]
                if not len(idx):
                    continue
                sub = [np.ascontiguousarray(x[idx]) for x in (d, hp_, nm, s)]
                spa = np.ascontiguousarray(pa[idx])
                ssd = np.ascontiguousarray(sd[idx])
                oo, dd, ss = (np.zeros((len(idx), 3), np.float32) for _ in range(3))
                al = np.zeros(len(idx), np.int32)
                refcl_lib().refcl_next(C.byref(self.c), b, len(idx), _p(sub[0]), _p(sub[1]),
                                       _p(sub[2]), _p(sub[3]), _p(spa), _p(ssd), _p(oo), _p(dd),
                                       _p(ss), _p(al))
                o_out[idx], d_out[idx], s_out[idx], alive[idx], sd[idx] = oo, dd, ss, al, ssd
        return dict(origins=o_out, directions=d_out, strength=s_out, alive=alive, seeds=sd)

    def render(self, camera, sample_x, sample_y, ssx=1, ssy=1, background=(0, 0, 0), sample=1,
               depth=5, disable_diffuse=0, seed=0, rng_mode=0, threads=8):
        cam = make_camera(camera)
        n = sample_x * ssx * sample_y * ssy
        acc = np.zeros((n, 3), np.float32)
        acc2 = np.zeros((n, 3), np.float32)
        counts = np.zeros(3, np.int64)
        bg = np.asarray(background, np.float32)
        oracle_lib().oracle_render(C.byref(self.c), C.byref(cam), sample_x, sample_y, ssx, ssy,
                                   _p(bg), sample, depth, disable_diffuse, seed, rng_mode,
                                   threads, _p(acc), _p(acc2), _p(counts))
        return acc, acc2, counts

    def refcl_render(self, camera, sample_x, sample_y, ssx=1, ssy=1, background=(0, 0, 0),
                     sample=1, depth=5, disable_diffuse=0, brightness=1.0, seed=0, threads=8):
        cam = make_camera(camera)
        n = sample_x * ssx * sample_y * ssy
        acc = np.zeros((n, 3), np.float32)
        rgba = np.zeros((sample_y, sample_x, 4), np.uint8)
        counts = np.zeros(2, np.int64)
        bg = np.asarray(background, np.float32)
        refcl_lib().refcl_render(C.byref(self.c), C.byref(cam), sample_x, sample_y, ssx, ssy,
                                 _p(bg), sample, depth, disable_diffuse, brightness, seed,
                                 threads, _p(rgba), _p(acc), _p(counts))
        return acc, rgba, counts


def make_camera(camera):
    """camera: dict(view_p, top_dir, right_dir, width, height) or an object
    with those attributes."""
    c = OracleCamera()
    get = (lambda k: camera[k]) if isinstance(camera, dict) else (lambda k: getattr(camera, k))
    c.view_p[:] = [float(x) for x in get("view_p")]
    c.top_dir[:] = [float(x) for x in get("top_dir")]
    c.right_dir[:] = [float(x) for x in get("right_dir")]
    c.width = float(get("width"))
    c.height = float(get("height"))
    return c


def raygen(camera, sample_x, sample_y, ssx=1, ssy=1, impl="oracle"):
    cam = make_camera(camera)
    n = sample_x * ssx * sample_y * ssy
    o = np.zeros((n, 3), np.float32)
    d = np.zeros((n, 3), np.float32)
    if impl == "oracle":
        oracle_lib().oracle_raygen(C.byref(cam), sample_x, sample_y, ssx, ssy, _p(o), _p(d))
    else:
        refcl_lib().refcl_raygen(C.byref(cam), sample_x, sample_y, ssx, ssy, _p(o), _p(d))
    return o, d


def resolve(accum, sample_x, sample_y, ssx, ssy, sample, brightness=1.0, impl="oracle"):
    a = _f32(accum, 3)
    rgba = np.zeros((sample_y, sample_x, 4), np.uint8)
    if impl == "oracle":
        oracle_lib().oracle_resolve(_p(a), sample_x, sample_y, ssx, ssy, sample,
                                    float(brightness), _p(rgba))
    else:
        refcl_lib().refcl_get_image(_p(a), sample_x, sample_y, ssx, ssy, sample,
                                    float(brightness), _p(rgba))
    return rgba


def box_intersect(box_start, box_end, p, d):
    a = [np.ascontiguousarray(x, np.float32) for x in (box_start, box_end, p, d)]
    return bool(oracle_lib().oracle_box_intersect(*[_p(x) for x in a]))


def ref_load_scene(filename, mtl_basepath=""):
    """Loads an OBJ with the reference's own hp::KDTree; returns numpy
    copies of its arrays, or None when the reference library is absent."""
    L = refscene_lib()
    if L is None:
        return None
    L.refscene_log(0)
    h = L.refscene_load(filename.encode(), mtl_basepath.encode())
    if not h:
        raise RuntimeError("reference loader failed on %s" % filename)
    v = RefSceneView()
    L.refscene_view(h, C.byref(v))

    def arr(p, n, width, dtype):
        nbytes = n * width * np.dtype(dtype).itemsize
        if not n:
            return np.zeros((0, width), dtype)
        return np.frombuffer(C.string_at(p, nbytes), dtype=dtype).reshape(n, width).copy()

    from hptracing_b200._lib import MATERIAL_DTYPE, NODE_DTYPE
    out = dict(points=arr(v.points, v.num_points, 4, np.float32),
               normals=arr(v.normals, v.num_normals, 4, np.float32),
               texcoords=arr(v.texcoords, v.num_texcoords, 2, np.float32),
               triangles=arr(v.triangles, v.num_triangles, 4, np.int32),
               lights=arr(v.lights, v.num_lights, 4, np.int32),
               materials=np.frombuffer(C.string_at(v.materials, v.num_materials * 96),
                                       dtype=MATERIAL_DTYPE).copy(),
               nodes=np.frombuffer(C.string_at(v.nodes, v.num_nodes * 48),
                                   dtype=NODE_DTYPE).copy(),
               leaf_data=np.frombuffer(C.string_at(v.leaf_data, v.num_leaf_data * 4),
                                       dtype=np.int32).copy())
    L.refscene_free(h)
    return out
