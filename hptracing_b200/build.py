"""Builds libhpt.so in-tree with nvcc for sm_100a.

    python -m hptracing_b200.build          (or hptracing_b200.build.build())

Every CUDA and host C++ source under csrc/ is compiled in parallel into
_build/ and linked into hptracing_b200/libhpt.so. Float contraction is off
everywhere (-fmad=false for device code, -ffp-contract=off for host code):
the kernels reproduce the reference's FP32 operation order bit for bit.

The device index guards (HPT_DEVICE_CHECKS, csrc/checks.cuh) are part of
the library: every index a kernel dereferences is range-checked, and a
failing check is returned as an error status naming its site instead of
touching memory.
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhpt.so")
CLI = os.path.join(HERE, "hptracing")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-DHPT_DEVICE_CHECKS", "-I", os.path.join(HERE, "..", "include")]
CUDA_FLAGS = ARCH + ["-lineinfo", "-fmad=false", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith(".cu") or name.endswith(".cpp"):
            out.append(os.path.join(CSRC, name))
    return out


def _newest_header():
    t = 0.0
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for name in os.listdir(d):
            if name.endswith((".h", ".cuh", ".hpp")):
                t = max(t, os.path.getmtime(os.path.join(d, name)))
    return t


def _compile(src, verbose, build_dir=None, extra=()):
    build_dir = build_dir or BUILD
    obj = os.path.join(build_dir, os.path.basename(src) + ".o")
    hdr = _newest_header()
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
        return obj
    cmd = [nvcc()] + COMMON + list(extra) + (
        CUDA_FLAGS if src.endswith(".cu") else ["-x", "c++"]) + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s%s" % (src, r.stdout, r.stderr))
    return obj


def build_cli(verbose=False):
    """The headless hptracing command line tool (C++, on the drop-in header)."""
    src = os.path.join(HERE, "cli", "hptracing.cpp")
    hdr = os.path.join(HERE, "..", "include", "hpt_trace_runner.hpp")
    if (os.path.exists(CLI) and os.path.getmtime(CLI) >= max(os.path.getmtime(src),
                                                             os.path.getmtime(hdr),
                                                             os.path.getmtime(LIB))):
        return CLI
    cmd = ["g++", "-O2", "-std=c++14", "-I", os.path.join(HERE, "..", "include"), src, "-o", CLI,
           "-L", HERE, "-lhpt", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("cli build failed\n%s%s" % (r.stdout, r.stderr))
    return CLI


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    srcs = _sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        build_cli(verbose)
        return LIB
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed\n%s%s" % (r.stdout, r.stderr))
    build_cli(verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
