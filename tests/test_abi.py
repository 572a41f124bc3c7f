"""CPU tests of the C ABI boundary: the library loads, exports every symbol
include/*.h declares, validates its inputs before touching a device, and
fails loudly (HPT_ERR_CUDA) instead of falling back to the CPU."""
import ctypes as C
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import hptracing_b200 as H
from hptracing_b200 import _lib
from tests import scenes as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for hdr in ("hpt.h",):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(hpt_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_exports_every_declared_symbol(built):
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares a signature for each of them
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_status_strings(built):
    L = H.lib()
    assert L.hpt_status_string(0) == b"ok"
    assert L.hpt_status_string(2) == b"invalid scene"
    assert L.hpt_version() == 1000


def _desc_arrays():
    mesh, nodes, leaf = S.make_scene(0)
    return mesh, nodes, leaf


def _expect_status(fn, status):
    with pytest.raises(H.HptError) as e:
        fn()
    assert e.value.status == status, str(e.value)


def test_scene_validation_rejects_bad_inputs(built):
    mesh, nodes, leaf = _desc_arrays()
    bad = H.Mesh(mesh.points, mesh.triangles.copy(), mesh.materials, mesh.normals,
                 mesh.texcoords, mesh.lights)
    bad.triangles[3, 1] = len(mesh.points) + 5
    _expect_status(lambda: H.Scene(bad, nodes, leaf), 2)
    bad = H.Mesh(mesh.points, mesh.triangles.copy(), mesh.materials, mesh.normals,
                 mesh.texcoords, mesh.lights)
    bad.triangles[0, 3] = 99  # material out of range
    _expect_status(lambda: H.Scene(bad, nodes, leaf), 2)
    pts = mesh.points.copy()
    pts[4, 1] = np.nan
    bad = H.Mesh(pts, mesh.triangles, mesh.materials, mesh.normals, mesh.texcoords, mesh.lights)
    _expect_status(lambda: H.Scene(bad, nodes, leaf), 2)
    bad = H.Mesh(mesh.points, mesh.triangles, mesh.materials, mesh.normals[:-1],
                 mesh.texcoords, mesh.lights)
    _expect_status(lambda: H.Scene(bad, nodes, leaf), 2)
    # malformed trees: a cycle, a child that is not the next node, leaf ids out of range
    n2 = nodes.copy()
    n2[1]["sibling"] = 1
    _expect_status(lambda: H.Scene(mesh, n2, leaf), 2)
    n2 = nodes.copy()
    n2[0]["child"] = 2
    _expect_status(lambda: H.Scene(mesh, n2, leaf), 2)
    l2 = leaf.copy()
    l2[1] = 10 ** 6
    _expect_status(lambda: H.Scene(mesh, nodes, l2), 2)
    n2 = nodes.copy()
    n2[2]["box_end"][0] = n2[0]["box_end"][0] + 1.0  # child box outside the parent
    if H.device_count() == 0:
        _expect_status(lambda: H.Scene(mesh, n2, leaf), 2)


@pytest.mark.skipif(H.device_count() != 0, reason="checks the no-device error path")
def test_no_device_fails_loudly(built):
    mesh, nodes, leaf = _desc_arrays()
    _expect_status(lambda: H.Scene(mesh, nodes, leaf), 3)
    _expect_status(lambda: H.compact(np.ones(10, np.uint32)), 3)
    _expect_status(lambda: H.resolve(np.ones((4, 3), np.float32), 2, 2, 1, 1, 1), 3)
    _expect_status(lambda: H.Batch(), 3)
    cli = os.path.join(ROOT, "hptracing_b200", "hptracing")
    r = subprocess.run([cli, "-i", "generated:0", "-o", "/tmp/hpt_cpu.ppm", "-s", "1"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "CUDA" in r.stderr


def test_bad_render_arguments(built):
    """Argument checks that run before any device work."""
    L = H.lib()
    cam = S.hp_camera(S.ROOM_CAM)
    p = H.make_params(16, 16, 1, 1, sample=0)
    assert L.hpt_render(None, C.byref(cam), C.byref(p), None, None) == 1
    o = np.zeros((4, 3), np.float32)
    pano = S.hp_camera(S.PANO_CAM)
    assert L.hpt_raygen(C.byref(pano), 2, 2, 2, 1, o.ctypes.data, o.ctypes.data) == 1


def test_kdtree_rejects_bad_triangles(built):
    _expect_status(lambda: H.build_kdtree(np.zeros((3, 4), np.float32),
                                          np.array([[0, 1, 7, 0]], np.int32)), 2)
    _expect_status(lambda: H.build_kdtree(np.zeros((0, 4), np.float32),
                                          np.zeros((0, 4), np.int32)), 2)


def test_cli_builds_and_parses_flags(built):
    cli = os.path.join(ROOT, "hptracing_b200", "hptracing")
    assert os.access(cli, os.X_OK)
    r = subprocess.run([cli, "--bogus"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


def _write_textured_obj(d):
    """Two triangles, each with a PPM texture of its own size."""
    def ppm(name, w, h, seed):
        rng = np.random.default_rng(seed)
        px = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
        with open(os.path.join(d, name), "wb") as f:
            f.write(b"P6\n%d %d\n255\n" % (w, h) + px.tobytes())
        return px
    a = ppm("a.ppm", 3, 5, 1)
    b = ppm("b.ppm", 8, 2, 2)
    with open(os.path.join(d, "t.mtl"), "w") as f:
        f.write("newmtl ma\nKd 1 1 1\nmap_Kd a.ppm\n\nnewmtl mb\nKd 1 1 1\nmap_Kd b.ppm\n")
    with open(os.path.join(d, "t.obj"), "w") as f:
        f.write("mtllib t.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nvt 0 0\nvt 1 0\nvt 0 1\n"
                "vt 1 1\nusemtl ma\nf 1/1 2/2 3/3\nusemtl mb\nf 2/2 4/4 3/3\n")
    return os.path.join(d, "t.obj"), a, b


def _normalized(px):
    """CImg normalize(0, 255) of one texture, as the loader applies it."""
    lo, hi = px.min(), px.max()
    return ((px.astype(np.float32) - lo) * np.float32(255.0 / (hi - lo))).astype(np.uint8)


def test_loader_keeps_per_texture_sizes(built, tmp_path):
    """texture_size 0 keeps each texture at its own size; a positive size
    resamples all of them to it (512: the reference's behaviour)."""
    path, a, b = _write_textured_obj(str(tmp_path))
    m = H.Mesh.load_obj(path, str(tmp_path) + "/", texture_size=0)
    assert m.texture_dims.tolist() == [[3, 5], [8, 2]]
    data = np.asarray(m.texture_data, np.uint8)
    la = data[:3 * 5 * 4].reshape(5, 3, 4)
    lb = data[3 * 5 * 4:].reshape(2, 8, 4)
    assert np.array_equal(la[:, :, :3], _normalized(a)) and (la[:, :, 3] == 0).all()
    assert np.array_equal(lb[:, :, :3], _normalized(b)) and (lb[:, :, 3] == 0).all()
    m4 = H.Mesh.load_obj(path, str(tmp_path) + "/", texture_size=4)
    assert m4.texture_dims.tolist() == [[4, 4], [4, 4]]
    assert len(m4.texture_data) == 2 * 4 * 4 * 4
    with pytest.raises(H.HptError):
        H.Mesh.load_obj(path, str(tmp_path) + "/", texture_size=-1)


# Every struct the ctypes binding mirrors, against the C compiler's layout of
# include/hpt.h: size and the offset of each field.
_MIRRORS = {
    "hpt_ref_node": _lib.RefNode, "hpt_ref_material": _lib.RefMaterial,
    "hpt_mesh_arrays": _lib.MeshArrays, "hpt_gen_params": _lib.GenParams,
    "hpt_scene_desc": _lib.SceneDesc, "hpt_scene_info": _lib.SceneInfo,
    "hpt_camera": _lib.Camera, "hpt_render_params": _lib.RenderParams,
    "hpt_render_stats": _lib.RenderStats, "hpt_tuning": _lib.Tuning,
    "hpt_server_config": _lib.ServerConfig, "hpt_request_info": _lib.RequestInfo,
}


def test_ctypes_mirrors_match_the_c_layout(tmp_path):
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "hpt.h"', 'int main(void) {']
    for cname, cls in _MIRRORS.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in cls._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));'
                         % (cname, fname, cname, fname))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run([gcc, "-I", inc, str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True,
                               text=True).stdout.splitlines():
        cname, field, value = line.split()
        got[(cname, field)] = int(value)
    for cname, cls in _MIRRORS.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
