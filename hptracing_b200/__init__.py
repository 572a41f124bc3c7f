"""hptracing_b200 - B200 wavefront path tracer behind hpTracing's host surface.

Python mirror of the reference's host interface (src/hp/trace_runner.h,
src/hp/scene/kdtree.h) over the C ABI of libhpt.so (include/hpt.h):

    scene = KDTree("cornell_box.obj")          # hp::KDTree(filename, mtl)
    runner = TraceRunner(scene)                # hp::TraceRunner(scene)
    runner.run(pixels, view_p, top_dir, right_dir, width, height,
               sample_x, sample_y, ssx, ssy, background,
               sample=10, depth=6, disable_diffuse=0, brightness=1.0)

plus per-stage entry points (raygen / intersect / shade / next_dir /
compact / resolve), many-job batches and a continuous-batching server.
Every call runs on the GPU; there is no CPU path.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import (MATERIAL_DTYPE, NODE_DTYPE, Camera, GenParams, HptError, MeshArrays,
                   RenderParams, RenderStats, RequestInfo, SceneDesc, SceneInfo, ServerConfig,
                   Tuning, check, lib, ptr)

__all__ = ["Mesh", "KDTree", "Scene", "TraceRunner", "Batch", "Server", "build_kdtree",
           "light_table", "material_probabilities", "raygen", "compact", "resolve",
           "make_camera", "make_params", "HptError", "device_count", "NODE_DTYPE",
           "MATERIAL_DTYPE"]



def _copy_out(address, nbytes, dtype):
    """Copies nbytes at a C address into a new numpy array (sizes above
    2 GiB included, which ctypes.string_at cannot take)."""
    if not isinstance(address, int):
        address = C.cast(address, C.c_void_p).value
    buf = (C.c_uint8 * nbytes).from_address(address)
    return np.frombuffer(buf, dtype=np.uint8).view(dtype).copy()

def device_count():
    return lib().hpt_device_count()


def _f32(a, cols=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if cols is not None:
        a = a.reshape(-1, cols)
    return a


def _i32(a, cols=None):
    a = np.ascontiguousarray(a, dtype=np.int32)
    if cols is not None:
        a = a.reshape(-1, cols)
    return a


def _pad4(a):
    """(n,3) or (n,4) float -> (n,4) float32 with a zero pad (cl_float3)."""
    a = np.asarray(a, dtype=np.float32)
    if a.ndim == 1:
        a = a.reshape(-1, 4 if a.size % 4 == 0 and a.size % 3 != 0 else 3)
    if a.shape[1] == 4:
        return np.ascontiguousarray(a)
    out = np.zeros((a.shape[0], 4), np.float32)
    out[:, :3] = a
    return out


class Mesh:
    """hp::Scene arrays (src/hp/scene/base.h:30-40) as numpy copies."""

    def __init__(self, points, triangles, materials, normals=None, texcoords=None, lights=None,
                 texture_data=None, texture_dims=None, texture_names=None):
        self.points = _pad4(points)
        self.triangles = _i32(triangles, 4)
        self.materials = np.ascontiguousarray(materials, dtype=MATERIAL_DTYPE)
        self.normals = (_pad4(normals) if normals is not None and len(normals)
                        else np.zeros((0, 4), np.float32))
        self.texcoords = (_f32(texcoords, 2) if texcoords is not None and len(texcoords)
                          else np.zeros((0, 2), np.float32))
        self.lights = (_i32(lights, 4) if lights is not None and len(lights)
                       else np.zeros((0, 4), np.int32))
        self.texture_data = (np.ascontiguousarray(texture_data, dtype=np.uint8).ravel()
                             if texture_data is not None else np.zeros(0, np.uint8))
        self.texture_dims = (_i32(texture_dims, 2) if texture_dims is not None
                             else np.zeros((0, 2), np.int32))
        self.texture_names = list(texture_names or [])

    @staticmethod
    def _from_handle(h):
        v = MeshArrays()
        check(lib().hpt_mesh_view(h, C.byref(v)))

        def arr(p, n, cols, dtype):
            if n == 0 or not p:
                return np.zeros((0, cols), dtype)
            return np.ctypeslib.as_array(p, shape=(n * cols,)).astype(dtype).reshape(n, cols)

        m = Mesh.__new__(Mesh)
        m.points = arr(v.points, v.num_points, 4, np.float32)
        m.normals = arr(v.normals, v.num_normals, 4, np.float32)
        m.texcoords = arr(v.texcoords, v.num_texcoords, 2, np.float32)
        m.triangles = arr(v.triangles, v.num_triangles, 4, np.int32)
        m.lights = arr(v.lights, v.num_lights, 4, np.int32)
        nb = v.num_materials * MATERIAL_DTYPE.itemsize
        m.materials = (_copy_out(v.materials, nb, MATERIAL_DTYPE)
                       if nb else np.zeros(0, MATERIAL_DTYPE))
        m.texture_dims = arr(v.texture_dims, v.num_textures, 2, np.int32)
        m.texture_data = (_copy_out(v.texture_data, v.texture_bytes, np.uint8)
                          if v.texture_bytes else np.zeros(0, np.uint8))
        m.texture_names = ["tex%d" % i for i in range(v.num_textures)]
        lib().hpt_mesh_destroy(h)
        return m

    @classmethod
    def load_obj(cls, filename, mtl_basepath="", texture_size=512, ignore_textures=False):
        """hp::Scene::Scene (src/hp/scene/base.cpp:37-158). texture_size > 0
        resamples every texture to that square size (512: the reference's
        behaviour); 0 keeps each texture at its own size (texture_dims)."""
        h = C.c_void_p()
        check(lib().hpt_mesh_load_obj(filename.encode(), mtl_basepath.encode(),
                                      texture_size, int(ignore_textures), C.byref(h)))
        return cls._from_handle(h)

    @classmethod
    def generate(cls, config, seed=0, family=0, target_triangles=0, texture_size=0,
                 heightfield_n=0):
        """Seeded synthetic scene (0 box room, 1 spheres, 2 terrain, 3 scaled)."""
        p = GenParams(family, target_triangles, texture_size, heightfield_n)
        h = C.c_void_p()
        check(lib().hpt_mesh_generate(config, seed, C.byref(p), C.byref(h)))
        return cls._from_handle(h)

    def rebuild_lights(self):
        out = np.zeros((256, 4), np.int32)
        n = C.c_int32()
        check(lib().hpt_light_table(ptr(self.points), len(self.points), ptr(self.triangles),
                                    len(self.triangles), ptr(self.materials),
                                    len(self.materials), ptr(out), C.byref(n)))
        self.lights = out[:n.value].copy()
        return self.lights


def build_kdtree(points, triangles, threads=0):
    """KDTree::KDTree + getData (src/hp/scene/kdtree.cpp:235-292)."""
    pts = _pad4(points)
    tris = _i32(triangles, 4)
    h = C.c_void_p()
    check(lib().hpt_kdtree_build(ptr(pts), len(pts), ptr(tris), len(tris), threads, C.byref(h)))
    try:
        np_ = C.c_void_p()
        nn = C.c_int32()
        lp = C.c_void_p()
        nl = C.c_int32()
        check(lib().hpt_kdtree_view(h, C.byref(np_), C.byref(nn), C.byref(lp), C.byref(nl)))
        nodes = _copy_out(np_, nn.value * 48, NODE_DTYPE)
        leaf = _copy_out(lp, nl.value * 4, np.int32)
    finally:
        lib().hpt_kdtree_destroy(h)
    return nodes, leaf


def light_table(points, triangles, materials):
    m = Mesh(points, triangles, materials)
    return m.rebuild_lights()


def material_probabilities(material):
    """Fills the branch probabilities of one MATERIAL_DTYPE record in place."""
    rec = np.ascontiguousarray(material, dtype=MATERIAL_DTYPE).reshape(1)
    check(lib().hpt_material_probabilities(ptr(rec)))
    return rec[0]


class KDTree:
    """Mirror of hp::KDTree (src/hp/scene/kdtree.h:56-58): a loaded scene
    with its SAH tree. Attributes as hp::Scene; getData() as the reference."""

    def __init__(self, filename=None, mtl_basepath="", mesh=None, texture_size=512,
                 ignore_textures=False):
        if mesh is None:
            mesh = Mesh.load_obj(filename, mtl_basepath, texture_size, ignore_textures)
        self.mesh = mesh
        self.points = mesh.points
        self.normals = mesh.normals
        self.texcoords = mesh.texcoords
        self.geometries = mesh.triangles
        self.lights = mesh.lights
        self.materials = mesh.materials
        self.texture_data = mesh.texture_data
        self.texture_dims = mesh.texture_dims
        self.texture_names = mesh.texture_names
        self._data = build_kdtree(mesh.points, mesh.triangles)

    def getData(self):  # noqa: N802 - reference name
        return self._data


def make_camera(view_p, top_dir, right_dir, width, height):
    c = Camera()
    c.view_p[:] = [float(x) for x in view_p]
    c.top_dir[:] = [float(x) for x in top_dir]
    c.right_dir[:] = [float(x) for x in right_dir]
    c.width = float(width)
    c.height = float(height)
    return c


def make_params(sample_x, sample_y, supersample_x=1, supersample_y=1, background=(0, 0, 0),
                sample=10, depth=6, disable_diffuse=0, brightness=1.0, seed=0, first_sample=0):
    """hpt_render_params. first_sample: the frame's index of this render's
    first sample (a frame's spp split over several renders)."""
    p = RenderParams()
    p.sample_x, p.sample_y = int(sample_x), int(sample_y)
    p.supersample_x, p.supersample_y = int(supersample_x), int(supersample_y)
    p.background[:] = [float(x) for x in background]
    p.sample, p.depth = int(sample), int(depth)
    p.disable_diffuse = int(disable_diffuse)
    p.brightness = float(brightness)
    p.seed = int(seed)
    p.first_sample = int(first_sample)
    return p


class Scene:
    """A device-resident scene (hpt_scene). Owns its HBM buffers."""

    def __init__(self, mesh, nodes=None, leaf_data=None, device=0):
        if nodes is None:
            nodes, leaf_data = build_kdtree(mesh.points, mesh.triangles)
        self.mesh = mesh
        self.nodes = np.ascontiguousarray(nodes, dtype=NODE_DTYPE)
        self.leaf_data = _i32(leaf_data)
        d = SceneDesc()
        keep = []

        def put(arr):
            keep.append(arr)
            return ptr(arr)

        d.points, d.num_points = put(mesh.points), len(mesh.points)
        d.normals, d.num_normals = put(mesh.normals), len(mesh.normals)
        d.texcoords, d.num_texcoords = put(mesh.texcoords), len(mesh.texcoords)
        d.triangles, d.num_triangles = put(mesh.triangles), len(mesh.triangles)
        d.nodes, d.num_nodes = put(self.nodes), len(self.nodes)
        d.leaf_data, d.num_leaf_data = put(self.leaf_data), len(self.leaf_data)
        d.materials, d.num_materials = put(mesh.materials), len(mesh.materials)
        d.lights, d.num_lights = put(mesh.lights), len(mesh.lights)
        d.texture_data = put(mesh.texture_data)
        d.num_textures = len(mesh.texture_dims)
        d.texture_dims = put(mesh.texture_dims) if len(mesh.texture_dims) else None
        d.device = device
        h = C.c_void_p()
        check(lib().hpt_scene_create(C.byref(d), C.byref(h)))
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib().hpt_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self):
        i = SceneInfo()
        check(lib().hpt_scene_info_get(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in SceneInfo._fields_}

    def tuning(self):
        t = Tuning()
        check(lib().hpt_tuning_get(self._h, C.byref(t)))
        return t

    def set_tuning(self, t):
        check(lib().hpt_tuning_set(self._h, C.byref(t)))

    def autotune(self, camera, params, cache_path=None):
        """Searches the tuning on a short render of (camera, params), keeps
        the best in this scene and returns it (hpt_autotune)."""
        t = Tuning()
        path = cache_path.encode() if cache_path else None
        check(lib().hpt_autotune(self._h, C.byref(camera), C.byref(params), path, C.byref(t)))
        return t

    def render(self, camera, params, want_accum=False):
        rgba = np.zeros((params.sample_y, params.sample_x, 4), np.uint8)
        acc = None
        if want_accum:
            n = (params.sample_x * params.supersample_x * params.sample_y * params.supersample_y)
            acc = np.zeros((n, 3), np.float32)
        check(lib().hpt_render(self._h, C.byref(camera), C.byref(params), ptr(rgba), ptr(acc)))
        return (rgba, acc) if want_accum else rgba

    def stats(self):
        s = RenderStats()
        check(lib().hpt_render_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in RenderStats._fields_}

    # --- stage entry points ---------------------------------------------
    def intersect(self, origins, directions):
        o, d = _f32(origins, 3), _f32(directions, 3)
        n = len(o)
        tri = np.zeros(n, np.int32)
        t, u, v = (np.zeros(n, np.float32) for _ in range(3))
        check(lib().hpt_intersect(self._h, n, ptr(o), ptr(d), ptr(tri), ptr(t), ptr(u), ptr(v)))
        return tri, t, u, v

    def shade(self, origins, directions, strengths, tris, ts, seeds, disable_diffuse=0):
        o, d, s = _f32(origins, 3), _f32(directions, 3), _f32(strengths, 3)
        tri = _i32(tris)
        t = _f32(ts)
        sd = np.ascontiguousarray(seeds, dtype=np.uint64).copy()
        n = len(o)
        contrib, hit_p, normal, s_out = (np.zeros((n, 3), np.float32) for _ in range(4))
        branch = np.zeros(n, np.int32)
        param = np.zeros(n, np.float32)
        check(lib().hpt_shade(self._h, n, ptr(o), ptr(d), ptr(s), ptr(tri), ptr(t), ptr(sd),
                              int(disable_diffuse), ptr(contrib), ptr(branch), ptr(hit_p),
                              ptr(normal), ptr(s_out), ptr(param)))
        return dict(contrib=contrib, branch=branch, hit_p=hit_p, normal=normal, strength=s_out,
                    param=param, seeds=sd)

    def next_dir(self, branch, directions, hit_p, normal, strengths, param, seeds):
        br = _i32(branch)
        d, hp_, nm, s = (_f32(x, 3) for x in (directions, hit_p, normal, strengths))
        pa = _f32(param)
        sd = np.ascontiguousarray(seeds, dtype=np.uint64).copy()
        n = len(br)
        o_out, d_out, s_out = (np.zeros((n, 3), np.float32) for _ in range(3))
        alive = np.zeros(n, np.int32)
        check(lib().hpt_next_dir(self._h, n, ptr(br), ptr(d), ptr(hp_), ptr(nm), ptr(s),
                                 ptr(pa), ptr(sd), ptr(o_out), ptr(d_out), ptr(s_out),
                                 ptr(alive)))
        return dict(origins=o_out, directions=d_out, strength=s_out, alive=alive, seeds=sd)


def raygen(camera, sample_x, sample_y, supersample_x=1, supersample_y=1):
    n = sample_x * supersample_x * sample_y * supersample_y
    o = np.zeros((n, 3), np.float32)
    d = np.zeros((n, 3), np.float32)
    check(lib().hpt_raygen(C.byref(camera), sample_x, sample_y, supersample_x, supersample_y,
                           ptr(o), ptr(d)))
    return o, d


def compact(flags):
    f = np.ascontiguousarray(flags, dtype=np.uint32)
    out = np.zeros(max(1, len(f)), np.int32)
    cnt = C.c_int32()
    check(lib().hpt_compact(ptr(f), len(f), ptr(out), C.byref(cnt)))
    return out[:cnt.value].copy()


def resolve(accum, sample_x, sample_y, supersample_x, supersample_y, sample, brightness=1.0):
    a = _f32(accum, 3)
    rgba = np.zeros((sample_y, sample_x, 4), np.uint8)
    check(lib().hpt_resolve(ptr(a), sample_x, sample_y, supersample_x, supersample_y, sample,
                            float(brightness), ptr(rgba)))
    return rgba


class TraceRunner:
    """Mirror of hp::TraceRunner (src/hp/trace_runner.h:51-65)."""

    def __init__(self, scene, device=0):
        mesh = scene.mesh if hasattr(scene, "mesh") else Mesh(
            scene.points, scene.geometries, scene.materials, scene.normals, scene.texcoords,
            scene.lights, scene.texture_data, getattr(scene, "texture_dims", None))
        nodes, leaf = scene.getData()
        self.scene = Scene(mesh, nodes, leaf, device=device)

    def run(self, result_data, view_p, top_dir, right_dir, width, height, sample_x, sample_y,
            supersample_x, supersample_y, background_color, sample=10, depth=6,
            disable_diffuse=0, brightness=1.0, seed=0):
        cam = make_camera(view_p, top_dir, right_dir, width, height)
        par = make_params(sample_x, sample_y, supersample_x, supersample_y, background_color,
                          sample, depth, disable_diffuse, brightness, seed)
        out = np.zeros((sample_y, sample_x, 4), np.uint8)
        check(lib().hpt_render(self.scene.handle, C.byref(cam), C.byref(par), ptr(out), None))
        if result_data is not None:
            np.copyto(np.asarray(result_data).reshape(out.shape), out)
        return out


class Batch:
    """Many jobs in one persistent wavefront (hpt_batch)."""

    def __init__(self, device=0):
        h = C.c_void_p()
        check(lib().hpt_batch_create(device, C.byref(h)))
        self._h = h
        self._outputs = []

    def add(self, scene, camera, params, want_accum=False):
        rgba = np.zeros((params.sample_y, params.sample_x, 4), np.uint8)
        acc = None
        if want_accum:
            n = params.sample_x * params.supersample_x * params.sample_y * params.supersample_y
            acc = np.zeros((n, 3), np.float32)
        jid = C.c_int32()
        check(lib().hpt_batch_add(self._h, scene.handle, C.byref(camera), C.byref(params),
                                  ptr(rgba), ptr(acc), C.byref(jid)))
        self._outputs.append((rgba, acc))
        return jid.value

    def set_tuning(self, t):
        check(lib().hpt_batch_tuning_set(self._h, C.byref(t)))

    def run(self):
        check(lib().hpt_batch_run(self._h))
        out, self._outputs = self._outputs, []
        return out

    def stats(self):
        s = RenderStats()
        check(lib().hpt_batch_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in RenderStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().hpt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching render server (hpt_server)."""

    def __init__(self, device=0, max_jobs=64, memory_budget=8 << 30, capacity=1 << 22,
                 progressive=0, large_inflight_pct=0, pipeline_depth=0, keep_accum=1,
                 deadline_ms=0):
        cfg = ServerConfig(device, max_jobs, memory_budget, capacity, progressive,
                           large_inflight_pct, pipeline_depth, keep_accum, deadline_ms)
        h = C.c_void_p()
        check(lib().hpt_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._scenes = []

    def add_scene(self, scene):
        slot = C.c_int32()
        check(lib().hpt_server_add_scene(self._h, scene.handle, C.byref(slot)))
        self._scenes.append(scene)
        return slot.value

    def submit(self, slot, camera, params):
        rid = C.c_uint64()
        check(lib().hpt_server_submit(self._h, slot, C.byref(camera), C.byref(params),
                                      C.byref(rid)))
        return rid.value

    def shed(self):
        """Requests shed by the overload policy so far."""
        return lib().hpt_server_shed(self._h)

    def pump(self, max_iterations=1):
        check(lib().hpt_server_pump(self._h, max_iterations))

    def poll(self, rid, rgba=None, accum=None):
        info = RequestInfo()
        st = lib().hpt_server_poll(self._h, rid, C.byref(info), ptr(rgba), ptr(accum))
        if st not in (0, 9):
            check(st)
        return st, {k: getattr(info, k) for k, _ in RequestInfo._fields_}

    def cancel(self, rid):
        check(lib().hpt_server_cancel(self._h, rid))

    def pending(self):
        return lib().hpt_server_pending(self._h)

    def completed(self, max_ids=4096):
        """Ids of the requests that finished since the previous call."""
        ids = np.zeros(max_ids, np.uint64)
        n = C.c_int32()
        check(lib().hpt_server_drain_completed(self._h, ptr(ids), max_ids, C.byref(n)))
        return [int(x) for x in ids[:n.value]]

    def stats(self):
        s = RenderStats()
        check(lib().hpt_server_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in RenderStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().hpt_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
