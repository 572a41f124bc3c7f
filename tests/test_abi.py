"""CPU tests of the C ABI boundary: the library loads, exports every symbol
include/*.h declares, validates its inputs before touching a device, and
fails loudly (HPT_ERR_CUDA) instead of falling back to the CPU."""
import ctypes as C
import os
import re
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
