"""Build recipe for the checker (test infrastructure only).

    python -m oracle.build

1. oracle/liboracle.so from oracle/hpt_oracle.cpp: the CPU restatement of
   the reference path (always built; it is the oracle).
2. When the reference sources are present (the directory named by
   REFERENCE_ROOT, else the container's read-only mount /root/reference if
   it exists), oracle/_ref/ receives:
     - librefcl.so: the reference's src/hp/cl_src/kernel.cl compiled as C++
       through refshim/opencl_c.h, driven by refcl_driver.cpp. The only
       change made to the kernel source on the way is a mechanical rewrite of
       OpenCL vector literals "(float4)(" / "(float3)(" / "(int2)(" into
       constructor calls, written to oracle/_ref/kernel_cl.inc (git-ignored).
     - librefscene.so: the reference's scene loader and SAH KD-tree
       (src/hp/scene/*.cpp, src/hp/common.cpp, src/objloader/*.cpp) compiled
       with refshim/Eigen/Core and refshim/CL/cl.h, driven by
       refscene_driver.cpp.
     - dropin_runner: dropin_main.cpp, the C++ drop-in header
       include/hpt_trace_runner.hpp used with the reference's own hp::KDTree
       and cl_float3 (the same scene sources and stand-ins), linked against
       hptracing_b200/libhpt.so (when that is built).
   Nothing is compiled with the reference's own build system and no
   reference source is copied into the repository.
"""
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REFCL_LIB = os.path.join(REF_OUT, "librefcl.so")
REFSCENE_LIB = os.path.join(REF_OUT, "librefscene.so")
DROPIN_BIN = os.path.join(REF_OUT, "dropin_runner")
REPO = os.path.dirname(HERE)
FLAGS = ["-O2", "-std=c++14", "-fPIC", "-shared", "-pthread", "-ffp-contract=off"]


DEFAULT_REFERENCE_MOUNT = "/root/reference"


def reference_root():
    """Directory of the reference sources, or None where they are absent
    (GPU hosts run only the prebuilt oracle/_ref files)."""
    root = os.environ.get("REFERENCE_ROOT")
    if root:
        return root if os.path.isdir(root) else None
    return DEFAULT_REFERENCE_MOUNT if os.path.isdir(DEFAULT_REFERENCE_MOUNT) else None


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle():
    src = os.path.join(HERE, "hpt_oracle.cpp")
    if _stale(ORACLE_LIB, [src]):
        _run(["g++"] + FLAGS + [src, "-o", ORACLE_LIB])
    return ORACLE_LIB


def build_reference():
    root = reference_root()
    if root is None:
        return None
    kernel = os.path.join(root, "src", "hp", "cl_src", "kernel.cl")
    types = os.path.join(root, "src", "hp", "cl_src", "types.h.cl")
    if not (os.path.exists(kernel) and os.path.exists(types)):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    text = open(kernel).read()
    text = re.sub(r"\(float4\)\(", "make_float4(", text)
    text = re.sub(r"\(float3\)\(", "make_float3(", text)
    text = re.sub(r"\(int2\)\(", "make_int2(", text)
    inc = os.path.join(REF_OUT, "kernel_cl.inc")
    if not os.path.exists(inc) or open(inc).read() != text:
        open(inc, "w").write(text)
    shutil.copyfile(types, os.path.join(REF_OUT, "types_h_cl.inc"))
    drv = os.path.join(HERE, "refcl_driver.cpp")
    shim = os.path.join(HERE, "refshim", "opencl_c.h")
    if _stale(REFCL_LIB, [drv, shim, inc]):
        _run(["g++"] + FLAGS + ["-I", HERE, "-w", drv, "-o", REFCL_LIB])
    # Scene loader + KD-tree from the reference sources.
    srcs = [os.path.join(root, "src", "hp", "scene", "base.cpp"),
            os.path.join(root, "src", "hp", "scene", "kdtree.cpp"),
            os.path.join(root, "src", "hp", "common.cpp"),
            os.path.join(root, "src", "objloader", "tiny_obj_loader.cpp"),
            os.path.join(HERE, "refscene_driver.cpp")]
    shims = [os.path.join(HERE, "refshim", "Eigen", "Core"),
             os.path.join(HERE, "refshim", "CL", "cl.h")]
    if all(os.path.exists(s) for s in srcs) and _stale(REFSCENE_LIB, srcs + shims):
        _run(["g++"] + FLAGS + ["-w", "-I", os.path.join(HERE, "refshim"),
                                "-I", os.path.join(root, "src"),
                                "-include", "map", "-include", "algorithm",
                                "-include", "functional", "-include", "cstring"]
             + srcs + ["-o", REFSCENE_LIB])
    build_dropin(root, srcs[:-1], shims)
    return REFCL_LIB


def build_dropin(root, scene_srcs, shims):
    """The drop-in checker: the reference's scene sources + dropin_main.cpp,
    linked against libhpt.so (found at run time next to the repository,
    $ORIGIN/../../hptracing_b200)."""
    lib = os.path.join(REPO, "hptracing_b200", "libhpt.so")
    main = os.path.join(HERE, "dropin_main.cpp")
    hdrs = [os.path.join(REPO, "include", "hpt_trace_runner.hpp"),
            os.path.join(REPO, "include", "hpt.h")]
    if not (os.path.exists(lib) and all(os.path.exists(s) for s in scene_srcs)):
        return None
    if _stale(DROPIN_BIN, scene_srcs + shims + hdrs + [main, lib]):
        _run(["g++", "-O2", "-std=c++14", "-pthread", "-ffp-contract=off", "-w",
              "-I", os.path.join(HERE, "refshim"), "-I", os.path.join(root, "src"),
              "-I", os.path.join(REPO, "include"),
              "-include", "map", "-include", "algorithm", "-include", "functional",
              "-include", "cstring"] + scene_srcs + [main, "-o", DROPIN_BIN,
                                                      "-L", os.path.dirname(lib), "-lhpt",
                                                      "-Wl,-rpath,$ORIGIN/../../hptracing_b200"])
    return DROPIN_BIN


def build():
    build_oracle()
    build_reference()


if __name__ == "__main__":
    build()
    print(ORACLE_LIB)
    for p in (REFCL_LIB, REFSCENE_LIB, DROPIN_BIN):
        print(p, os.path.exists(p))
