"""The C++ drop-in against the reference's own types.

oracle/_ref/dropin_runner (built by oracle/build.py from
oracle/dropin_main.cpp) includes include/hpt_trace_runner.hpp together with
the reference's src/hp/scene/kdtree.h and base.h, loads a scene with the
reference's hp::KDTree (its OBJ loader and SAH builder), and calls
hp::TraceRunner(scene) and run(...) exactly as the reference's CLI does
(src/hptracing.cpp:74-78, 249). The image must match the oracle's render of
the same scene (loaded by the same reference loader) driven by the same
random streams: the first run() of a runner uses seed 0. The Cornell
box's paths are chaotic (its 556-unit scale rounds away the reference's 1e-5
offset of the next ray's origin; see test_gpu_cornell.py), so the pixel
agreement is held to the oracle's own agreement with its render from a
camera moved by one ulp, and the image means to 0.5 %."""
import os
import subprocess

import numpy as np
import pytest

import hptracing_b200 as H
import oracle as O
from oracle import build as obuild
from oracle import objio

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cornell_box.npz")
THREADS = max(1, os.cpu_count() or 1)


class _Arrays:
    def __init__(self, f):
        for k in ("points", "normals", "texcoords", "triangles", "materials"):
            setattr(self, k, f[k])


def test_dropin_header_with_reference_types(built, tmp_path):
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    if not os.path.exists(obuild.DROPIN_BIN) or O.refscene_lib() is None:
        pytest.skip("the drop-in checker was not built (needs the reference sources)")
    f = dict(np.load(GOLD))
    obj = objio.write_obj(_Arrays(f), str(tmp_path), "cornell")
    out = os.path.join(str(tmp_path), "out.rgba")
    w = h = 200
    spp, depth, angle = 16, 5, 0.68
    r = subprocess.run([obuild.DROPIN_BIN, obj, out, "278,273,-800", "0,1,0", "-1,0,0", str(w),
                        str(h), str(angle), str(spp), str(depth), "1.0", "0"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    img = np.fromfile(out, np.uint8).reshape(h, w, 4).astype(np.int32)
    ref_scene = O.ref_load_scene(obj, str(tmp_path) + "/")

    class Mesh:
        pass
    m = Mesh()
    for k in ("points", "normals", "texcoords", "triangles", "materials", "lights"):
        setattr(m, k, ref_scene[k])
    m.texture_data = np.zeros(0, np.uint8)
    m.texture_dims = np.zeros((0, 2), np.int32)
    cpu = O.CpuScene(m, ref_scene["nodes"], ref_scene["leaf_data"])
    cam = dict(view_p=(278.0, 273.0, -800.0), top_dir=(0.0, 1.0, 0.0),
               right_dir=(-1.0, 0.0, 0.0), width=float(np.float32(w) / np.float32(h)) * angle,
               height=angle)
    acc, _, counts = cpu.render(cam, w, h, 1, 1, (0, 0, 0), spp, depth, 0, seed=0, rng_mode=1,
                                threads=THREADS)
    ref = O.resolve(acc, w, h, 1, 1, spp).astype(np.int32)
    cam2 = dict(cam)
    v = np.asarray(cam["view_p"], np.float32).copy()
    v[0] = np.nextafter(v[0], np.float32(np.inf))
    cam2["view_p"] = tuple(float(x) for x in v)
    moved, _, _ = cpu.render(cam2, w, h, 1, 1, (0, 0, 0), spp, depth, 0, seed=0, rng_mode=1,
                             threads=THREADS)
    mimg = O.resolve(moved, w, h, 1, 1, spp).astype(np.int32)
    close = (np.abs(img - ref).max(axis=2) <= 1).mean()
    self_close = (np.abs(mimg - ref).max(axis=2) <= 1).mean()
    print("drop-in with the reference's types: %s; pixels within 1/255 %.4f (oracle vs its "
          "one-ulp camera move %.4f), mean %.3f vs %.3f (oracle %d queries)"
          % (r.stdout.strip(), close, self_close, img[:, :, :3].mean(), ref[:, :, :3].mean(),
             counts[0]))
    assert (img[:, :, 3] == 0).all()
    assert close >= self_close
    assert abs(img[:, :, :3].mean() - ref[:, :, :3].mean()) / ref[:, :, :3].mean() < 0.005
