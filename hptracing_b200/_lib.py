"""ctypes bindings of libhpt.so (declarations mirror include/hpt.h).

The shared library is built in-tree by hptracing_b200.build; importing this
module fails loudly if it is missing - there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# HPT_LIBRARY selects another build of the same ABI (e.g. a diagnostic one).
LIB_PATH = os.environ.get("HPT_LIBRARY") or os.path.join(HERE, "libhpt.so")

i32, i64, u64, f32, f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_float, C.c_double
P = C.POINTER
vp = C.c_void_p


class RefNode(C.Structure):
    _fields_ = [("box_start", f32 * 4), ("box_end", f32 * 4), ("child", i32),
                ("parent", i32), ("sibling", i32), ("data", i32)]


class RefMaterial(C.Structure):
    _fields_ = [("emission", f32 * 4), ("ambient", f32 * 4), ("diffuse", f32 * 4),
                ("specular", f32 * 4), ("optical_density", f32), ("dissolve", f32),
                ("shininess", f32), ("diffuse_texture_id", i32), ("ambient_texture_id", i32),
                ("specular_possibility", f32), ("refract_possibility", f32),
                ("diffuse_possibility", f32)]


NODE_DTYPE = np.dtype([("box_start", "<f4", 4), ("box_end", "<f4", 4), ("child", "<i4"),
                       ("parent", "<i4"), ("sibling", "<i4"), ("data", "<i4")])
MATERIAL_DTYPE = np.dtype([("emission", "<f4", 4), ("ambient", "<f4", 4),
                           ("diffuse", "<f4", 4), ("specular", "<f4", 4),
                           ("optical_density", "<f4"), ("dissolve", "<f4"),
                           ("shininess", "<f4"), ("diffuse_texture_id", "<i4"),
                           ("ambient_texture_id", "<i4"), ("specular_possibility", "<f4"),
                           ("refract_possibility", "<f4"), ("diffuse_possibility", "<f4")])
assert NODE_DTYPE.itemsize == 48 and MATERIAL_DTYPE.itemsize == 96


class MeshArrays(C.Structure):
    _fields_ = [("points", P(f32)), ("num_points", i32), ("normals", P(f32)),
                ("num_normals", i32), ("texcoords", P(f32)), ("num_texcoords", i32),
                ("triangles", P(i32)), ("num_triangles", i32), ("materials", vp),
                ("num_materials", i32), ("lights", P(i32)), ("num_lights", i32),
                ("texture_data", P(C.c_uint8)), ("num_textures", i32),
                ("texture_dims", P(i32)), ("texture_bytes", i64)]


class GenParams(C.Structure):
    _fields_ = [("family", i32), ("target_triangles", i32), ("texture_size", i32),
                ("heightfield_n", i32), ("reserved", i32 * 4)]


class SceneDesc(C.Structure):
    _fields_ = [("points", vp), ("num_points", i32), ("normals", vp), ("num_normals", i32),
                ("texcoords", vp), ("num_texcoords", i32), ("triangles", vp),
                ("num_triangles", i32), ("nodes", vp), ("num_nodes", i32),
                ("leaf_data", vp), ("num_leaf_data", i32), ("materials", vp),
                ("num_materials", i32), ("lights", vp), ("num_lights", i32),
                ("texture_data", vp), ("num_textures", i32), ("texture_dims", vp),
                ("device", i32)]


class SceneInfo(C.Structure):
    _fields_ = [("num_triangles", i32), ("num_ref_nodes", i32), ("num_device_nodes", i32),
                ("num_leaves", i32), ("num_leaf_triangles", i32), ("max_depth", i32),
                ("device_bytes", i64)]


class Camera(C.Structure):
    _fields_ = [("view_p", f32 * 3), ("top_dir", f32 * 3), ("right_dir", f32 * 3),
                ("width", f32), ("height", f32)]


class RenderParams(C.Structure):
    _fields_ = [("sample_x", i32), ("sample_y", i32), ("supersample_x", i32),
                ("supersample_y", i32), ("background", f32 * 3), ("sample", i32),
                ("depth", i32), ("disable_diffuse", i32), ("brightness", f32), ("seed", u64),
                ("first_sample", i32)]


class RenderStats(C.Structure):
    _fields_ = [("primary_rays", i64), ("intersect_queries", i64), ("shade_calls", i64),
                ("paths", i64), ("iterations", i32), ("error_flags", i32), ("ms_total", f32),
                ("ms_primary", f32), ("ms_shade", f32), ("ms_intersect", f32),
                ("ms_resolve", f32), ("ms_loop", f32), ("nodes_visited", i64),
                ("leaves_visited", i64), ("triangle_tests", i64), ("triangle_repeats", i64)]


class Tuning(C.Structure):
    _fields_ = [("capacity", i32), ("isect_block", i32), ("shade_block", i32),
                ("refill_chunk", i32), ("smem_nodes", i32), ("use_graph", i32),
                ("profile", i32), ("isect_min_blocks", i32), ("trav_steps", i32),
                ("max_steps", i32), ("shade_min_blocks", i32)]


class ServerConfig(C.Structure):
    _fields_ = [("device", i32), ("max_jobs", i32), ("memory_budget", i64), ("capacity", i32),
                ("progressive", i32), ("large_inflight_pct", i32), ("pipeline_depth", i32),
                ("keep_accum", i32), ("deadline_ms", i32)]


class RequestInfo(C.Structure):
    _fields_ = [("state", i32), ("samples_done", i32), ("submit_ms", f64), ("admit_ms", f64),
                ("done_ms", f64), ("intersect_queries", i64), ("due_ms", f64)]


# name -> (restype, argtypes); every function declared in include/hpt.h.
SIGNATURES = {
    "hpt_status_string": (C.c_char_p, [i32]),
    "hpt_last_error": (C.c_char_p, []),
    "hpt_version": (C.c_int, []),
    "hpt_device_count": (C.c_int, []),
    "hpt_mesh_load_obj": (i32, [C.c_char_p, C.c_char_p, i32, i32, P(vp)]),
    "hpt_mesh_generate": (i32, [i32, u64, P(GenParams), P(vp)]),
    "hpt_mesh_create": (i32, [P(MeshArrays), i32, P(vp)]),
    "hpt_mesh_view": (i32, [vp, P(MeshArrays)]),
    "hpt_mesh_destroy": (None, [vp]),
    "hpt_material_probabilities": (i32, [vp]),
    "hpt_light_table": (i32, [vp, i32, vp, i32, vp, i32, vp, P(i32)]),
    "hpt_kdtree_build": (i32, [vp, i32, vp, i32, i32, P(vp)]),
    "hpt_kdtree_view": (i32, [vp, P(vp), P(i32), P(vp), P(i32)]),
    "hpt_kdtree_destroy": (None, [vp]),
    "hpt_scene_create": (i32, [P(SceneDesc), P(vp)]),
    "hpt_scene_info_get": (i32, [vp, P(SceneInfo)]),
    "hpt_scene_destroy": (None, [vp]),
    "hpt_render": (i32, [vp, P(Camera), P(RenderParams), vp, vp]),
    "hpt_render_stats_get": (i32, [vp, P(RenderStats)]),
    "hpt_tuning_get": (i32, [vp, P(Tuning)]),
    "hpt_tuning_set": (i32, [vp, P(Tuning)]),
    "hpt_raygen": (i32, [P(Camera), i32, i32, i32, i32, vp, vp]),
    "hpt_intersect": (i32, [vp, i32, vp, vp, vp, vp, vp, vp]),
    "hpt_shade": (i32, [vp, i32, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp]),
    "hpt_next_dir": (i32, [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "hpt_compact": (i32, [vp, i32, vp, P(i32)]),
    "hpt_compact_noalloc": (i32, [vp, i32, vp, vp, vp]),
    "hpt_resolve": (i32, [vp, i32, i32, i32, i32, i32, f32, vp]),
    "hpt_batch_create": (i32, [i32, P(vp)]),
    "hpt_batch_add": (i32, [vp, vp, P(Camera), P(RenderParams), vp, vp, P(i32)]),
    "hpt_batch_run": (i32, [vp]),
    "hpt_batch_stats_get": (i32, [vp, P(RenderStats)]),
    "hpt_batch_tuning_set": (i32, [vp, P(Tuning)]),
    "hpt_batch_destroy": (None, [vp]),
    "hpt_server_create": (i32, [P(ServerConfig), P(vp)]),
    "hpt_server_add_scene": (i32, [vp, vp, P(i32)]),
    "hpt_server_submit": (i32, [vp, i32, P(Camera), P(RenderParams), P(u64)]),
    "hpt_server_pump": (i32, [vp, i32]),
    "hpt_server_poll": (i32, [vp, u64, P(RequestInfo), vp, vp]),
    "hpt_server_cancel": (i32, [vp, u64]),
    "hpt_server_pending": (i32, [vp]),
    "hpt_server_shed": (i64, [vp]),
    "hpt_server_stats_get": (i32, [vp, P(RenderStats)]),
    "hpt_server_drain_completed": (i32, [vp, vp, i32, P(i32)]),
    "hpt_server_destroy": (None, [vp]),
    "hpt_autotune": (i32, [vp, P(Camera), P(RenderParams), C.c_char_p, P(Tuning)]),
}

_lib = None


def lib():
    """Loads libhpt.so once; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libhpt.so is missing (%s); run `python -m hptracing_b200.build`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class HptError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s (%d): %s" % (lib().hpt_status_string(status).decode(), status, msg))
        self.status = status


def check(status):
    if status != 0:
        raise HptError(status, lib().hpt_last_error().decode())
    return status


def ptr(a):
    """Address of a contiguous numpy array (None for None / empty)."""
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data if a.size else None
