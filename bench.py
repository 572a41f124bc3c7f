"""Benchmark: Mrays/s of the plain path on the mid-size scene.

Workload (one step = one full frame): the procedural box room + 64 UV
spheres (61,476 triangles, four 1024^2 RGBA8 value-noise textures),
512 x 512 rays, 64 samples per ray, depth 8, seeded synthetic data. A ray
is one intersect query (primary rays counted once per frame, as the
reference executes them once).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value: intersect queries of all ranks / max over ranks of the CUDA-event
       time of the frames (scene resident in HBM, L2 flushed between frames).
e2e:   the same queries / host wall time of the hpt_render C-ABI calls,
       which include the job upload and the RGBA read-back.
With N > 1 each rank renders its own frames (independent jobs, no
collective): weak scaling.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_RES, H_RES, SPP, DEPTH = 512, 512, 64, 8
WORKLOAD = "spheres64_61k_tris_512x512_spp64_d8"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # Overrides for profiling runs only (the headline workload is the default).
    ap.add_argument("--res", type=int, default=0)
    ap.add_argument("--spp", type=int, default=0)
    return ap.parse_args()


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


class ClockSampler:
    """Samples nvidia-smi clocks / throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, name in enumerate(names):
                if len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes (read + write) of one k_isect launch of this workload, from
    the committed ncu summary (None when the summary is absent)."""
    path = os.path.join(ROOT, "profiles", "k_isect_spheres64_512x512_spp64_d8.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(line.split(":")[1])
    except (OSError, ValueError):
        pass
    return None


def make_scene():
    import hptracing_b200 as H
    from tests import scenes as S
    mesh, nodes, leaf = S.make_scene(1, seed=1)
    return mesh, nodes, leaf, S.ROOM_CAM


def isect_bytes(stats):
    """Algorithmic bytes of all intersect-kernel work in one frame:
    per query 64 B (origin+direction in, strength+radiance carried) and
    72 B written per hit (next shade record) -- approximated with the hit
    count = shade calls; per inner node visited 8 B; per leaf visited 36 B
    (box + exit rope); per triangle test 48 B (a, b-a, c-a)."""
    q = stats["intersect_queries"] - stats["primary_rays"]
    hits = max(0, stats["shade_calls"] - stats["paths"])  # hits found by k_isect
    return (64 * q + 72 * hits + 8 * stats["nodes_visited"] + 36 * stats["leaves_visited"] +
            48 * stats["triangle_tests"])


def cpu_baseline(mesh, nodes, leaf, cam, kind):
    """The reference's kernels (kind 'reference') or the oracle restatement
    ('port') on all host cores, bounded sample: 1 sample of the frame."""
    import oracle as O
    cs = O.CpuScene(mesh, nodes, leaf)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    if kind == "reference":
        _, _, counts = cs.refcl_render(cam, W_RES, H_RES, 1, 1, (0, 0, 0), 1, DEPTH, 0, 1.0,
                                       seed=1, threads=threads)
    else:
        _, _, counts = cs.render(cam, W_RES, H_RES, 1, 1, (0, 0, 0), 1, DEPTH, 0, seed=1,
                                 rng_mode=0, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": counts[0] / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": kind,
            "sample": "%dx%d rays x 1 sample x depth %d of the same frame (%d queries, %.1f s)"
                      % (W_RES, H_RES, DEPTH, int(counts[0]), dt)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle as O
    from oracle import build as obuild
    obuild.build()
    kind = "reference" if O.refcl_lib() is not None else "port"
    mesh, nodes, leaf, cam = make_scene()
    for _ in range(args.warmup):
        cpu_baseline(mesh, nodes, leaf, cam, kind)
    vals = [cpu_baseline(mesh, nodes, leaf, cam, kind) for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    base = dict(vals[-1])
    base["value"] = v
    line = {"metric": "Mrays/s", "value": v, "unit": "Mrays/s", "impl": "reference",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene)",
            "config": {"workload": WORKLOAD, "res": [W_RES, H_RES], "spp": SPP, "depth": DEPTH,
                       "note": "reference runs 1 sample per step (bounded CPU sample)"},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    global W_RES, H_RES, SPP, WORKLOAD
    args = parse()
    if args.res or args.spp:
        W_RES = H_RES = args.res or W_RES
        SPP = args.spp or SPP
        WORKLOAD = "profiling_case_%dx%d_spp%d_d%d" % (W_RES, H_RES, SPP, DEPTH)
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_setup(args.gpus)
    import torch

    import hptracing_b200 as H
    from hptracing_b200 import build as hbuild
    hbuild.build()
    torch.cuda.set_device(local)
    mesh, nodes, leaf, cam = make_scene()
    scene = H.Scene(mesh, nodes, leaf, device=local)
    from tests import scenes as S
    camera = S.hp_camera(cam)
    tune = scene.tuning()
    tune.profile = 1
    scene.set_tuning(tune)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def frame(i):
        p = H.make_params(W_RES, H_RES, 1, 1, (0, 0, 0), SPP, DEPTH, 0, 1.0, 1000 + i)
        flush.zero_()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        rgba = scene.render(camera, p)
        wall = time.perf_counter() - t0
        return rgba, scene.stats(), wall

    for i in range(args.warmup):
        frame(i)
    sampler = ClockSampler(local)
    sampler.start()
    stats, walls = [], []
    for i in range(args.steps):
        _, st, wall = frame(args.warmup + i)
        stats.append(st)
        walls.append(wall)
    clocks = sampler.stop()
    torch.cuda.synchronize()
    barrier(world)
    dev_ms = sum(s["ms_total"] for s in stats)
    queries = sum(s["intersect_queries"] for s in stats)
    isect_ms = sum(s["ms_intersect"] for s in stats)
    launches = sum(3 * s["iterations"] + 3 for s in stats)
    wall_s = sum(walls)
    tot_q = allreduce_sum(float(queries), world)
    max_ms = allreduce_max(dev_ms, world)
    max_wall = allreduce_max(wall_s, world)
    value = tot_q / (max_ms / 1e3) / 1e6
    e2e = tot_q / max_wall / 1e6
    peak, peak_kind = measured_peak()
    ib = sum(isect_bytes(s) for s in stats)
    isect_launches = sum(s["iterations"] for s in stats)
    achieved = ib / (isect_ms / 1e3) / 1e9 if isect_ms > 0 else None
    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle as O
        from oracle import build as obuild
        obuild.build()
        kind = "reference" if O.refcl_lib() is not None else "port"
        base = cpu_baseline(mesh, nodes, leaf, cam, kind)
    if rank == 0:
        line = {
            "metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene, random textures)",
            "config": {"workload": WORKLOAD, "res": [W_RES, H_RES], "supersample": 1,
                       "spp": SPP, "depth": DEPTH, "triangles": int(len(mesh.triangles)),
                       "l2": "flushed between frames (512 MiB write)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": 320,
                    "d2h_bytes_per_step": W_RES * H_RES * 4 + 256},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": "k_isect", "achieved": achieved,
                         "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "peak_kind": peak_kind,
                         "traffic": profiled_traffic() if WORKLOAD.startswith("spheres64") else None,
                         "traffic_source": "ncu --set full, one full-queue launch (profiles/)",
                         "algorithmic_bytes_per_launch": ib / max(1, isect_launches),
                         "launches": isect_launches,
                         "avg_launch_ms": isect_ms / max(1, isect_launches)},
            "stages_ms_per_step": {
                "primary": sum(s["ms_primary"] for s in stats) / args.steps,
                "shade": sum(s["ms_shade"] for s in stats) / args.steps,
                "intersect": isect_ms / args.steps,
                "resolve": sum(s["ms_resolve"] for s in stats) / args.steps},
            "per_frame": {"queries": queries / args.steps,
                          "iterations": stats[-1]["iterations"],
                          "nodes_per_query": stats[-1]["nodes_visited"] / stats[-1][
                              "intersect_queries"],
                          "leaves_per_query": stats[-1]["leaves_visited"] / stats[-1][
                              "intersect_queries"],
                          "tri_tests_per_query": stats[-1]["triangle_tests"] / stats[-1][
                              "intersect_queries"]},
            "clocks": clocks,
            "cpu_baseline": base,
        }
        print(json.dumps(line), flush=True)
    scene.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
