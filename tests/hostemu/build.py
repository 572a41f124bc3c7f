"""Builds tests/hostemu/libhpt_emu.so: the GPU per-ray code compiled for the
host (test infrastructure)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CSRC = os.path.join(ROOT, "hptracing_b200", "csrc")
LIB = os.path.join(HERE, "libhpt_emu.so")


def build():
    srcs = [os.path.join(HERE, "emu.cu"), os.path.join(CSRC, "scene_pack.cpp"),
            os.path.join(CSRC, "kdtree_build.cpp"), os.path.join(CSRC, "obj_loader.cpp")]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                   if f.endswith((".h", ".cuh"))]
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(x) for x in deps):
        return LIB
    cmd = ["nvcc", "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
           "-DHPT_DEVICE_CHECKS",
           "-I", os.path.join(ROOT, "include"), "-shared", "-o", LIB] + srcs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("emu build failed\n%s%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build())
