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

The default line also carries the metric's other two parts, measured after
the frames: "batch" (the 32 mixed jobs one by one through hpt_render vs in
one hpt_batch wavefront; accumulators bit-identical, so equal relMSE) and,
at N = 1, "serve" (the Poisson stream over four resident scenes at 50
requests/s: pose and panorama p50/p99). --frame-only leaves them out.
Other modes print their own line: --mode batch | serve | compact.

--impl reference: the reference's own kernels (kernel.cl compiled as C++)
on the host cores, on the same frame's scene as the reference's own loader
and SAH builder build it from the stored workload file, without the
product library.
"""
import argparse
import json
import math
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
BG = (0.0, 0.0, 0.0)  # the terrain frame adds a constant environment term of 0.2
WORKLOAD = "spheres64_61k_tris_512x512_spp64_d8"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--frame-only", action="store_true",
                    help="frame: leave out the batch and serving parts of the default line")
    ap.add_argument("--serve-seconds", type=float, default=4.0,
                    help="frame: seconds of arrivals of the serving part")
    # Overrides for profiling runs only (the headline workload is the default).
    ap.add_argument("--res", type=int, default=0)
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--tuning", default="",
                    help="frame: hpt_tuning fields to override, e.g. shade_min_blocks=3")
    # Extra workloads (one JSON line each): the 32-job mixed batch, batched
    # vs one job at a time; the Poisson serving stream.
    ap.add_argument("--mode", default="frame", choices=["frame", "batch", "serve", "compact"])
    ap.add_argument("--compact-n", type=int, default=1 << 25,
                    help="compact: number of flags")
    ap.add_argument("--scene", default="spheres", choices=["spheres", "terrain", "room"],
                    help="frame: the 61k-triangle spheres frame (headline), the "
                         "2.4M-triangle terrain at 1920x1080, 256 spp, or the 38-triangle "
                         "box room at 256x256, 16 spp, depth 5")
    ap.add_argument("--rate", default="50", help="serve: requests per second (comma list)")
    ap.add_argument("--duration", type=float, default=4.0, help="serve: seconds of arrivals")
    ap.add_argument("--serve-capacity", default=str(1 << 20),
                    help="serve: wavefront capacity (paths in flight; comma list)")
    ap.add_argument("--large-pct", default="5",
                    help="serve: in-flight cap of the requests larger than the wavefront, "
                         "%% (comma list)")
    ap.add_argument("--depth-ahead", default="1",
                    help="serve: iterations queued ahead of the host (comma list)")
    ap.add_argument("--deadline-ms", default="0",
                    help="serve: overload policy deadline (0 = off; comma list)")
    ap.add_argument("--terrain-n", type=int, default=1024,
                    help="serve: heightfield vertices per side of the large scenes")
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
    from hptracing_b200 import shard
    return shard.allreduce_max(x, world, device="cuda")


def allreduce_sum(x, world):
    from hptracing_b200 import shard
    return shard.allreduce_sum(x, world, device="cuda")


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


SCENE = "spheres"


# The headline frame's scene as a file: written at build time by the
# product's generator (write_reference_workload), read by the reference arm,
# which never loads the product library: it rebuilds the scene's KD-tree
# with the reference's own loader and SAH builder from this file.
WORKLOAD_FILE = os.path.join(ROOT, "oracle", "_ref", "workload_spheres64_61k.npz")
_MESH_KEYS = ("points", "normals", "texcoords", "triangles", "materials", "lights",
              "texture_data", "texture_dims")


def write_reference_workload(path=None, force=False):
    """Stores the spheres frame's scene (hpt_mesh_generate config 1, seed 1:
    geometry, materials, light table and the four 1024^2 RGBA8 texture
    layers) for the reference arm. Called by __graft_entry__.build()."""
    import hptracing_b200 as H
    from hptracing_b200 import build as hbuild
    path = path or WORKLOAD_FILE
    if (not force and os.path.exists(path) and
            os.path.getmtime(path) >= os.path.getmtime(hbuild.LIB)):
        return path
    os.makedirs(os.path.dirname(path), exist_ok=True)
    mesh = H.Mesh.generate(1, seed=1)
    tmp = path + ".tmp.npz"
    np.savez(tmp, **{k: getattr(mesh, k) for k in _MESH_KEYS})
    os.replace(tmp, path)
    return path


class _StoredMesh:
    """hp::Scene arrays read from the stored workload file."""

    def __init__(self, data, **override):
        for k in _MESH_KEYS:
            setattr(self, k, override.get(k, data[k]))


def make_scene():
    import hptracing_b200 as H
    from hptracing_b200 import scenes as S
    if SCENE == "terrain":
        mesh = H.Mesh.generate(2, seed=2)
        nodes, leaf = H.build_kdtree(mesh.points, mesh.triangles)
        return mesh, nodes, leaf, S.terrain_cam(W_RES / H_RES)
    if SCENE == "room":
        mesh, nodes, leaf = S.make_scene(0)
        return mesh, nodes, leaf, S.ROOM_CAM
    mesh, nodes, leaf = S.make_scene(1, seed=1)
    return mesh, nodes, leaf, S.ROOM_CAM


def reference_scene():
    """The spheres frame's scene for the reference arm, without the product
    library: the stored workload's geometry and materials are written as
    OBJ + MTL and loaded by the reference's own hp::KDTree (its OBJ loader,
    material probabilities, light table and SAH builder, compiled from the
    reference sources into oracle/_ref/librefscene.so). The reference decodes
    texture maps through ImageMagick, which is absent here, so the texture
    ids and RGBA8 layers are attached from the stored workload, as
    TraceRunner uploads them (trace_runner.cpp:67-86)."""
    import tempfile

    import oracle as O
    from oracle import objio
    data = np.load(WORKLOAD_FILE)
    stored = _StoredMesh(data)
    with tempfile.TemporaryDirectory() as d:
        path = objio.write_obj(stored, d, "spheres64")
        r = O.ref_load_scene(path, d + "/")
    if r is None:
        raise RuntimeError("the reference's scene library is not built")
    mats = r["materials"].copy()
    mats["diffuse_texture_id"] = data["materials"]["diffuse_texture_id"]
    mats["ambient_texture_id"] = data["materials"]["ambient_texture_id"]
    mesh = _StoredMesh(data, points=r["points"], normals=r["normals"], texcoords=r["texcoords"],
                       triangles=r["triangles"], materials=mats, lights=r["lights"])
    return mesh, r["nodes"], r["leaf_data"]


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


def cpu_baseline(mesh, nodes, leaf, cam, kind, samples=1):
    """The reference's kernels (kind 'reference') or the oracle restatement
    ('port') on all host cores, bounded sample: `samples` samples per ray of
    the frame."""
    import oracle as O
    cs = O.CpuScene(mesh, nodes, leaf)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    if kind == "reference":
        _, _, counts = cs.refcl_render(cam, W_RES, H_RES, 1, 1, BG, samples, DEPTH, 0, 1.0,
                                       seed=1, threads=threads)
    else:
        _, _, counts = cs.render(cam, W_RES, H_RES, 1, 1, BG, samples, DEPTH, 0, seed=1,
                                 rng_mode=0, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": counts[0] / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": kind,
            "seconds": dt,
            "sample": "%dx%d rays x %d sample%s x depth %d of the same frame (%d queries, %.1f s)"
                      % (W_RES, H_RES, samples, "" if samples == 1 else "s", DEPTH,
                         int(counts[0]), dt)}


def run_reference(args):
    """The reference arm: the reference's own kernels (kernel.cl compiled as
    C++, driven like TraceRunner::run) on all host cores, on the spheres
    frame's scene as the reference's own loader and SAH builder build it.
    Each step is a bounded sample of the frame (1 of its 64 samples per ray);
    the metric (intersect queries per second) is the same as the GPU arm's."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle as O
    from oracle import build as obuild
    obuild.build()
    if O.refcl_lib() is None or O.refscene_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference kernels were not built (oracle/_ref missing)"}))
        return
    if not os.path.exists(WORKLOAD_FILE):
        print(json.dumps({"impl": "reference", "unavailable":
                          "workload file missing (written by __graft_entry__.build())"}))
        return
    from hptracing_b200 import scenes as S
    t0 = time.perf_counter()
    mesh, nodes, leaf = reference_scene()
    build_s = time.perf_counter() - t0
    cam = S.ROOM_CAM
    world = int(os.environ.get("WORLD_SIZE", "1"))
    for _ in range(args.warmup):
        cpu_baseline(mesh, nodes, leaf, cam, "reference")
    vals = [cpu_baseline(mesh, nodes, leaf, cam, "reference") for _ in range(args.steps)]
    v = statistics.median(x["value"] for x in vals)
    base = dict(vals[-1])
    base["value"] = v
    line = {"metric": "Mrays/s", "value": v, "unit": "Mrays/s", "impl": "reference",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.median(x["seconds"] for x in vals) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": DATA, "config": frame_config(len(mesh.triangles), world),
            "reference_sample": "each step renders 1 of the frame's %d samples per ray "
                                "(bounded CPU sample; the metric counts queries, so it is "
                                "comparable across spp)" % SPP,
            "reference_scene": {"source": "stored workload -> OBJ -> the reference's hp::KDTree "
                                          "(loader + SAH builder)",
                                "build_s": build_s, "triangles": int(len(mesh.triangles)),
                                "nodes": int(len(nodes))},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


DATA = "synthetic (seeded procedural scene, value-noise textures)"


def frame_config(triangles, world):
    """The frame workload's config dict, printed identically by both arms."""
    return {"workload": WORKLOAD, "res": [W_RES, H_RES], "supersample": 1, "spp": SPP,
            "depth": DEPTH, "triangles": int(triangles),
            "l2": "flushed between frames (512 MiB write)",
            "parallelism": "replicas" if world > 1 else "single"}


def serve_summary(line, cpu):
    """The serving keys of the default line: pose / panorama latency, the
    stream's Mrays/s and its roofline fraction, next to a CPU baseline."""
    keys = ("rate_per_s", "duration_s", "requests", "completed", "unfinished",
            "pose_512x512_4spp", "pano_2048x1024_64spp", "Mrays_per_s", "Msamples_per_s",
            "roofline", "scene_triangles", "scene_build_s", "server", "policy")
    out = {k: line[k] for k in keys if k in line}
    out["cpu_baseline"] = cpu
    return out


def serve_cpu_baseline(scene_arrays, cam):
    """The reference kernels on the host cores rendering one pose request of
    the spheres scene (512 x 512, depth 6) at 1 of its 4 samples: the pose
    latency a CPU host would give, scaled to 4 samples."""
    import oracle as O
    mesh, nodes, leaf = scene_arrays
    cs = O.CpuScene(mesh, nodes, leaf)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    _, _, counts = cs.refcl_render(cam, 512, 512, 1, 1, (0.05, 0.05, 0.05), 1, 6, 0, 1.0,
                                   seed=3, threads=threads)
    dt = time.perf_counter() - t0
    return {"pose_latency_ms": dt * 4 * 1e3, "value": counts[0] / dt / 1e6, "unit": "Mrays/s",
            "cores": threads, "kind": "reference",
            "sample": "one 512x512 pose request of the spheres scene at 1 of 4 spp "
                      "(%d queries, %.2f s), latency scaled x4" % (int(counts[0]), dt)}


def rotate(v, axis, ang):
    """Rodrigues rotation of v about the unit axis by ang radians."""
    v = np.asarray(v, np.float64)
    k = np.asarray(axis, np.float64)
    k = k / np.linalg.norm(k)
    return (v * math.cos(ang) + np.cross(k, v) * math.sin(ang) +
            k * np.dot(k, v) * (1 - math.cos(ang)))


def jitter_camera(cam, rng):
    """A pose request: yaw and pitch within +-30 degrees, translation within
    +-0.1 of the scene's base camera."""
    top, right = np.asarray(cam["top_dir"]), np.asarray(cam["right_dir"])
    yaw, pitch = np.radians(rng.uniform(-30, 30, 2))
    right2 = rotate(right, top, yaw)
    top2 = rotate(top, right2, pitch)
    eye = np.asarray(cam["view_p"]) + rng.uniform(-0.1, 0.1, 3)
    return dict(view_p=tuple(eye), top_dir=tuple(top2), right_dir=tuple(right2),
                width=cam["width"], height=cam["height"])


def c3_jobs(seed=0x48505403):
    """The 32 mixed jobs: scene family 0-2, triangles log-uniform in
    [1k, 500k], resolution in {128, 256, 512, 1024} squared, spp in
    {1, 4, 16, 64}, depth uniform in [3, 10]."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(32):
        jobs.append(dict(family=int(rng.integers(0, 3)),
                         tris=int(round(math.exp(rng.uniform(math.log(1e3), math.log(5e5))))),
                         res=int(rng.choice([128, 256, 512, 1024])),
                         spp=int(rng.choice([1, 4, 16, 64])),
                         depth=int(rng.integers(3, 11)), seed=7000 + j))
    return jobs


def batch_c3(world, rank):
    """C3: 32 jobs one by one through hpt_render (the plain per-job path)
    against the same jobs in one hpt_batch wavefront with the autotuned
    tuning. Accumulators are compared bit for bit (counter RNG + fixed-point
    sums), so the relMSE of both against the reference estimate is identical
    by construction. Returns the result line on rank 0 (None elsewhere)."""
    import hptracing_b200 as H
    from hptracing_b200 import shard
    from hptracing_b200 import scenes as S
    import torch
    dev = torch.cuda.current_device()  # this rank's GPU (set from LOCAL_RANK)
    all_jobs = c3_jobs()
    # With N ranks each runs its share (longest job first onto the least
    # loaded rank); the 32 jobs are the fixed total work (strong scaling).
    table = shard.assign_jobs([shard.job_cost(j["res"] ** 2, j["spp"], j["depth"])
                               for j in all_jobs], world)
    jobs = [all_jobs[i] for i in table[rank]]
    t0 = time.perf_counter()
    built = []
    for j in jobs:
        mesh = H.Mesh.generate(3, seed=j["seed"], family=j["family"], target_triangles=j["tris"])
        nodes, leaf = H.build_kdtree(mesh.points, mesh.triangles)
        cam = S.terrain_cam(1.0) if j["family"] == 2 else S.ROOM_CAM
        built.append((H.Scene(mesh, nodes, leaf, device=dev), S.hp_camera(cam),
                      H.make_params(j["res"], j["res"], 1, 1, (0.05, 0.05, 0.05), j["spp"],
                                    j["depth"], 0, 1.0, j["seed"]), len(mesh.triangles)))
    build_s = time.perf_counter() - t0
    # Autotune on the job with the most rays x spp, at reduced spp.
    big = max(range(len(jobs)), key=lambda k: jobs[k]["res"] ** 2 * jobs[k]["spp"])
    sc, cam, p, _ = built[big]
    probe = H.make_params(p.sample_x, p.sample_y, 1, 1, (0, 0, 0), min(4, p.sample), p.depth, 0,
                          1.0, 1)
    tune = sc.autotune(cam, probe)
    for sc, _, _, _ in built:
        sc.set_tuning(tune)

    per_job = []

    def plain():
        q = ms = 0.0
        accs = []
        per_job.clear()
        t = time.perf_counter()
        for sc, cam, p, _ in built:
            _, acc = sc.render(cam, p, want_accum=True)
            st = sc.stats()
            q += st["intersect_queries"]
            ms += st["ms_total"]
            per_job.append((st["ms_total"], st["intersect_queries"]))
            accs.append(acc)
        return q, ms, time.perf_counter() - t, accs

    def batched():
        b = H.Batch(device=dev)
        b.set_tuning(tune)
        for sc, cam, p, _ in built:
            b.add(sc, cam, p, want_accum=True)
        t = time.perf_counter()
        out = b.run()
        wall = time.perf_counter() - t
        st = b.stats()
        b.close()
        return st["intersect_queries"], st["ms_total"], wall, [o[1] for o in out]

    plain()
    batched()
    barrier(world)
    q_p, ms_p, wall_p, acc_p = plain()
    barrier(world)
    q_b, ms_b, wall_b, acc_b = batched()
    same = all(np.array_equal(a, b) for a, b in zip(acc_p, acc_b))
    q_p, q_b = allreduce_sum(q_p, world), allreduce_sum(q_b, world)
    ms_p, ms_b = allreduce_max(ms_p, world), allreduce_max(ms_b, world)
    wall_p, wall_b = allreduce_max(wall_p, world), allreduce_max(wall_b, world)
    same = allreduce_sum(0.0 if same else 1.0, world) == 0.0
    build_s = allreduce_max(build_s, world)
    for sc, _, _, _ in built:
        sc.close()
    if rank != 0:
        return None
    work = [j["res"] ** 2 * j["spp"] * j["depth"] for j in all_jobs]
    # Bound on the batch's gain for this job mix (one rank): the batch
    # cannot finish before its largest job does when that job runs at its
    # plain speed (it fills the wavefront alone), nor process the total
    # queries faster than the best plain rate any job reached.
    t_max = max(m for m, _ in per_job)
    best_rate = max(q / m for m, q in per_job if m > 0)
    bound = sum(m for m, _ in per_job) / max(t_max, sum(q for _, q in per_job) / best_rate)
    # A tighter bound: a query costs what it costs in its scene family, so
    # the batch needs at least sum over jobs of queries / (that family's
    # rate with the device full), the rate taken from the family's job with
    # the most queries (the one that fills the wavefront best).
    fam_rate = {}
    for j, (m, q) in zip(jobs, per_job):
        f = j["family"]
        if m > 0 and (f not in fam_rate or q > fam_rate[f][1]):
            fam_rate[f] = (q / m, q)
    fam_bound = sum(m for m, _ in per_job) / max(
        t_max, sum(q / fam_rate[j["family"]][0] for j, (_, q) in zip(jobs, per_job)))
    line = {
        "metric": "Mrays/s batched vs plain (C3, 32 mixed jobs)", "mode": "batch",
        "value": q_b / ms_b / 1e3, "unit": "Mrays/s", "plain": q_p / ms_p / 1e3,
        "speedup": (q_b / ms_b) / (q_p / ms_p), "higher_is_better": True, "n_gpus": world,
        "scaling": "strong", "jobs_per_rank": [len(t) for t in table],
        "ms_batched": ms_b, "ms_plain": ms_p, "queries": q_b,
        "e2e": {"batched": q_b / wall_b / 1e6, "plain": q_p / wall_p / 1e6, "unit": "Mrays/s"},
        "accumulators_bit_identical": same,
        "largest_job_share_of_work": max(work) / sum(work),
        "amdahl_bound": bound if world == 1 else None,
        "family_rate_bound": fam_bound if world == 1 else None,
        "family_rate_Mrays_per_s": {str(f): r[0] / 1e3 for f, r in fam_rate.items()},
        "plain_per_job": [{"family": j["family"], "tris": j["tris"], "res": j["res"],
                           "spp": j["spp"], "depth": j["depth"], "ms": m, "queries": q}
                          for j, (m, q) in zip(jobs, per_job)],
        "largest_job_share_of_plain_ms": t_max / sum(m for m, _ in per_job),
        "tuning": {"capacity": tune.capacity, "isect_block": tune.isect_block,
                   "isect_min_blocks": tune.isect_min_blocks, "refill": tune.refill_chunk,
                   "smem_nodes": tune.smem_nodes, "use_graph": tune.use_graph,
                   "trav_steps": tune.trav_steps},
        "jobs": all_jobs,
        "scene_build_s": build_s, "dtype": "f32", "data": "synthetic (seeded scene families)"}
    return line


def run_batch(args):
    import torch
    from hptracing_b200 import build as hbuild
    rank, world, local = dist_setup(args.gpus)
    hbuild.build()
    torch.cuda.set_device(local)
    line = batch_c3(world, rank)
    if line is not None:
        print(json.dumps(line), flush=True)


def serve_scenes(terrain_n=1024):
    """The four resident scenes of the serving stream: box room, spheres,
    terrain and a larger terrain (heightfield terrain_n and 1.33 x terrain_n
    vertices per side). Returns (scenes, cameras, triangle counts, build s)."""
    import hptracing_b200 as H
    from hptracing_b200 import scenes as S
    t0 = time.perf_counter()
    specs = [(0, {}), (1, dict(seed=1)),
             (2, dict(seed=2, heightfield_n=terrain_n)),
             (2, dict(seed=3, heightfield_n=int(terrain_n * 1.33)))]
    scenes, cams, tris = [], [], []
    for cfg, kw in specs:
        mesh = H.Mesh.generate(cfg, **kw)
        nodes, leaf = H.build_kdtree(mesh.points, mesh.triangles)
        scenes.append(H.Scene(mesh, nodes, leaf))
        cams.append(S.terrain_cam(1.0) if cfg == 2 else S.ROOM_CAM)
        tris.append(len(mesh.triangles))
        del mesh, nodes, leaf
    return scenes, cams, tris, time.perf_counter() - t0


def run_serve(args):
    """C4: Poisson arrivals over four resident scenes (box room, spheres,
    terrain, a larger terrain). 80 % pose requests (512x512, 4 spp), 20 %
    panoramas (2048x1024, 64 spp), depth 6. Latency = completion -
    submission on the server's clock. The scenes are built once and every
    rate of --rate runs against a fresh server."""
    import torch
    import hptracing_b200 as H
    from hptracing_b200 import build as hbuild
    from hptracing_b200 import scenes as S
    hbuild.build()
    torch.cuda.set_device(0)
    scenes, cams, tris, build_s = serve_scenes(args.terrain_n)
    for rate in [float(x) for x in str(args.rate).split(",")]:
        for cap in [int(x) for x in str(args.serve_capacity).split(",")]:
            for pct in [int(x) for x in str(args.large_pct).split(",")]:
                for ahead in [int(x) for x in str(args.depth_ahead).split(",")]:
                    for dl in [int(x) for x in str(args.deadline_ms).split(",")]:
                        line = serve_stream(H, S, scenes, cams, tris, build_s, rate,
                                            args.duration, cap, pct, ahead, dl)
                        print(json.dumps(line), flush=True)
    for sc in scenes:
        sc.close()


def serve_stream(H, S, scenes, cams, tris, build_s, rate, duration, capacity, large_pct, ahead,
                 deadline_ms=0):
    """One Poisson stream at `rate` requests/s for `duration` seconds
    against a fresh server; returns the result line."""
    server = H.Server(max_jobs=64, memory_budget=16 << 30, capacity=capacity,
                      large_inflight_pct=large_pct, pipeline_depth=ahead, keep_accum=0,
                      deadline_ms=deadline_ms)
    slots = [server.add_scene(s) for s in scenes]
    rng = np.random.default_rng(0x48505404 + int(rate))
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        k = int(rng.integers(0, 4))
        if rng.random() < 0.8:
            cam = jitter_camera(cams[k], rng)
            p = H.make_params(512, 512, 1, 1, (0.05, 0.05, 0.05), 4, 6, 0, 1.0,
                              int(rng.integers(1, 2 ** 31)))
            arrivals.append((t, "pose", k, cam, p))
        else:
            pano = dict(view_p=cams[k]["view_p"], top_dir=(0.0, 1.0, 0.0),
                        right_dir=(0.0, 0.0, 1.0), width=1.0, height=-1.0)
            p = H.make_params(2048, 1024, 1, 1, (0.2, 0.2, 0.2), 64, 6, 0, 1.0,
                              int(rng.integers(1, 2 ** 31)))
            arrivals.append((t, "pano", k, pano, p))
    # Warm-up: one small request per scene.
    for k in range(4):
        rid = server.submit(slots[k], S.hp_camera(cams[k]),
                            H.make_params(128, 128, 1, 1, (0, 0, 0), 1, 6, 0, 1.0, 1))
        while server.poll(rid)[0] != 0:
            server.pump(1)
    server.completed()
    st0 = server.stats()
    sampler = ClockSampler(0)
    sampler.start()
    start = time.perf_counter()
    outstanding = {}
    lat = {"pose": [], "pano": []}
    shed = {"pose": 0, "pano": 0}
    per_scene = {}
    sub_at, served_poses = {}, []
    pumps, gaps, last_pump_end = [], [], None
    samples = 0
    nxt = 0
    drain_cap = duration + 20.0
    while True:
        now = time.perf_counter() - start
        while nxt < len(arrivals) and arrivals[nxt][0] <= now:
            _, kind, k, cam, p = arrivals[nxt]
            rid = server.submit(slots[k], S.hp_camera(cam), p)
            outstanding[rid] = (kind, p, k)
            sub_at[rid] = now * 1e3
            nxt += 1
        if not outstanding and nxt >= len(arrivals):
            break
        if now > drain_cap:
            break
        if outstanding:
            tp = time.perf_counter()
            if last_pump_end is not None:
                gaps.append(((tp - start) * 1e3, (tp - last_pump_end) * 1e3))
            server.pump(1)
            last_pump_end = time.perf_counter()
            pumps.append(((tp - start) * 1e3, (last_pump_end - tp) * 1e3))
            for rid in server.completed():
                try:
                    st, info = server.poll(rid)
                except H.HptError as e:
                    if e.status == 8 and rid in outstanding:  # shed by the overload policy
                        shed[outstanding.pop(rid)[0]] += 1
                        continue
                    raise
                if st == 0 and rid in outstanding:
                    kind, p, k = outstanding.pop(rid)
                    lat[kind].append(info["done_ms"] - info["submit_ms"])
                    per_scene.setdefault((kind, k), []).append(
                        (info["done_ms"] - info["submit_ms"], info["admit_ms"] - info["submit_ms"],
                         info["submit_ms"]))
                    samples += p.sample_x * p.sample_y * p.sample
                    if kind == "pose":
                        served_poses.append({
                            "scene": k, "submitted_at_ms": sub_at.get(rid),
                            "admit_wait_ms": info["admit_ms"] - info["submit_ms"],
                            "latency_ms": info["done_ms"] - info["submit_ms"],
                            "done_minus_predicted_ms": (info["done_ms"] - info["due_ms"]
                                                        if info["due_ms"] >= 0 else None)})
        else:
            time.sleep(0.0005)
    elapsed = time.perf_counter() - start
    clocks = sampler.stop()
    st1 = server.stats()
    q = st1["intersect_queries"] - st0["intersect_queries"]

    def pct(v, x):
        return float(np.percentile(v, x)) if v else None

    d = {k: st1[k] - st0[k] for k in ("intersect_queries", "shade_calls", "nodes_visited",
                                        "leaves_visited", "triangle_tests")}
    alg = (64 * d["intersect_queries"] + 72 * d["shade_calls"] + 8 * d["nodes_visited"] +
           36 * d["leaves_visited"] + 48 * d["triangle_tests"])
    peak, peak_kind = measured_peak()
    line = {
        "metric": "serving p50/p99 latency (C4)", "mode": "serve", "rate_per_s": rate,
        "duration_s": duration, "elapsed_s": elapsed,
        "roofline": {"bound": "hbm", "kernel": "wavefront (traversal + queues), whole stream",
                     "achieved": alg / elapsed / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / elapsed / 1e9 / peak, "peak_kind": peak_kind,
                     "basis": "algorithmic bytes of every intersect query / the stream's wall "
                              "time"},
        "requests": len(arrivals), "completed": len(lat["pose"]) + len(lat["pano"]),
        "shed": shed,
        "policy": {"deadline_ms": deadline_ms,
                   "rule": ("requests of <= capacity paths granted first-come first-served "
                            "ahead of larger ones; each admitted when predicted to finish "
                            "within the deadline behind those admitted, shed once it could "
                            "not finish in time on an idle wavefront")
                   if deadline_ms > 0 else "smallest remaining work first, no shedding"},
        "unfinished": len(outstanding) + (len(arrivals) - nxt),
        "pose_512x512_4spp": {"n": len(lat["pose"]), "p50_ms": pct(lat["pose"], 50),
                              "p99_ms": pct(lat["pose"], 99)},
        "pano_2048x1024_64spp": {"n": len(lat["pano"]), "p50_ms": pct(lat["pano"], 50),
                                 "p99_ms": pct(lat["pano"], 99)},
        "per_scene": {"%s/scene%d" % key: {
            "n": len(v), "p50_ms": pct([x[0] for x in v], 50), "p99_ms": pct([x[0] for x in v], 99),
            "max_ms": max(x[0] for x in v), "admit_wait_max_ms": max(x[1] for x in v),
            "slowest_submitted_at_ms": max(v)[2]} for key, v in sorted(per_scene.items())},
        "slowest_poses": sorted(served_poses, key=lambda x: -x["latency_ms"])[:6],
        "host_loop": {"pumps": len(pumps),
                      "pump_ms_p50": pct([x[1] for x in pumps], 50),
                      "slowest_pumps_at_ms": sorted(pumps, key=lambda x: -x[1])[:5],
                      "slowest_gaps_at_ms": sorted(gaps, key=lambda x: -x[1])[:3]},
        "Mrays_per_s": q / elapsed / 1e6, "Msamples_per_s": samples / elapsed / 1e6,
        "server": {"capacity": capacity, "large_inflight_pct": large_pct,
                   "pipeline_depth": ahead, "max_jobs": 64, "memory_budget": 16 << 30},
        "scene_triangles": tris, "scene_build_s": build_s, "clocks": clocks,
        "dtype": "f32", "data": "synthetic (seeded scenes, seeded Poisson stream)"}
    server.close()
    return line


def run_compact(args):
    """Standalone stream compaction (the stage ABI's stable compaction
    kernels: per-tile counts, one-block scan, scatter). Device-resident
    flags of n = 2^25 u32 (128 MiB, survivors with probability 1/2), timed
    with CUDA events on the launching stream, L2 flushed between calls.
    Algorithmic bytes: 4 per flag read + 4 per survivor index written."""
    import ctypes as C

    import torch
    import hptracing_b200 as H
    from hptracing_b200 import _lib
    from hptracing_b200 import build as hbuild
    hbuild.build()
    torch.cuda.set_device(0)
    n = args.compact_n
    g = torch.Generator(device="cuda")
    g.manual_seed(0x48505400)
    flags = (torch.rand(n, device="cuda", generator=g) < 0.5).to(torch.int32)
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    L = _lib.lib()
    stream = torch.cuda.current_stream()

    def call():
        _lib.check(L.hpt_compact_noalloc(C.c_void_p(flags.data_ptr()), n,
                                         C.c_void_p(out.data_ptr()), C.c_void_p(cnt.data_ptr()),
                                         C.c_void_p(stream.cuda_stream)))

    for _ in range(args.warmup):
        call()
    torch.cuda.synchronize()
    times = []
    sampler = ClockSampler(0)
    sampler.start()
    for _ in range(args.steps):
        flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        call()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    clocks = sampler.stop()
    total = int(cnt.item())
    ref = torch.nonzero(flags).flatten().to(torch.int32)
    exact = total == ref.numel() and bool(torch.equal(out[:total], ref))
    ms = statistics.median(times)
    alg = 4.0 * n + 4.0 * total
    peak, peak_kind = measured_peak()
    # End to end through the host-array entry point (copies in and out).
    hflags = flags.cpu().numpy().astype(np.uint32)
    walls = []
    for _ in range(3):
        t0 = time.perf_counter()
        H.compact(hflags)
        walls.append(time.perf_counter() - t0)
    line = {"metric": "compaction GB/s", "mode": "compact", "value": alg / (ms / 1e3) / 1e9,
            "unit": "GB/s", "n": n, "survivors": total, "exact": exact,
            "ms_per_call": ms, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True,
            "roofline": {"bound": "hbm", "kernel": "k_compact_count+k_compact_scatter",
                         "achieved": alg / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_call": alg},
            "e2e": {"value": n / statistics.median(walls) / 1e9, "unit": "Gflags/s",
                    "h2d_bytes_per_step": 4 * n, "d2h_bytes_per_step": 4 * total + 4},
            "l2": "flushed between calls (512 MiB write)", "clocks": clocks,
            "dtype": "u32", "data": "synthetic (seeded flags, p = 0.5)"}
    print(json.dumps(line), flush=True)


def main():
    global W_RES, H_RES, SPP, DEPTH, WORKLOAD, SCENE, BG
    args = parse()
    if args.mode == "compact":
        run_compact(args)
        return
    if args.mode == "batch":
        run_batch(args)
        if int(os.environ.get("WORLD_SIZE", "1")) > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.mode == "serve":
        run_serve(args)
        return
    if args.scene == "terrain":
        SCENE = "terrain"
        W_RES, H_RES, SPP = 1920, 1080, 256
        BG = (0.2, 0.2, 0.2)
        WORKLOAD = "terrain_2.4M_tris_1920x1080_spp256_d8"
    if args.scene == "room":
        SCENE = "room"
        W_RES, H_RES, SPP, DEPTH = 256, 256, 16, 5
        WORKLOAD = "room_38_tris_256x256_spp16_d5"
    if args.impl == "reference" and SCENE != "spheres":
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm runs the "
                          "headline spheres frame only"}))
        return
    if args.res or args.spp:
        if args.res:
            H_RES = args.res * H_RES // W_RES
            W_RES = args.res
        SPP = args.spp or SPP
        WORKLOAD = "profiling_case_%s_%dx%d_spp%d_d%d" % (SCENE, W_RES, H_RES, SPP, DEPTH)
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
    from hptracing_b200 import scenes as S
    camera = S.hp_camera(cam)
    tune = scene.tuning()
    tune.profile = 1
    for kv in filter(None, args.tuning.split(",")):
        k, v = kv.split("=")
        setattr(tune, k, int(v))
    scene.set_tuning(tune)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def frame(i):
        p = H.make_params(W_RES, H_RES, 1, 1, BG, SPP, DEPTH, 0, 1.0, 1000 + i)
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
        # About 10 s of CPU work: as many samples per ray (up to the frame's)
        # as one sample's time allows.
        samples = max(1, min(SPP, int(10.0 / max(base["seconds"], 1e-3))))
        if samples > 1:
            base = cpu_baseline(mesh, nodes, leaf, cam, kind, samples)
    line = None
    if rank == 0:
        line = {
            "metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": DATA, "config": frame_config(len(mesh.triangles), world),
            "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": 320,
                    "d2h_bytes_per_step": W_RES * H_RES * 4 + 256},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": "k_isect", "achieved": achieved,
                         "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "peak_kind": peak_kind,
                         "traffic": profiled_traffic() if WORKLOAD.startswith("spheres64") else None,
                         "traffic_source": "ncu dram__bytes_read/write.sum, mean of two full-queue launches "
                                           "of this frame (profiles/)",
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
            "tuning": {f: getattr(tune, f) for f, _ in type(tune)._fields_},
            "cpu_baseline": base,
        }
    scene.close()
    del flush
    torch.cuda.empty_cache()
    if not args.frame_only and WORKLOAD.startswith("spheres64"):
        # The metric's other two parts on the same box: the 32-job batch
        # (batched vs one by one, bit-identical accumulators, hence equal
        # relMSE) and the serving stream at 50 requests/s.
        b = batch_c3(world, rank)
        if rank == 0:
            line["batch"] = {k: b[k] for k in (
                "metric", "value", "plain", "speedup", "unit", "ms_batched", "ms_plain",
                "queries", "e2e", "accumulators_bit_identical", "largest_job_share_of_work",
                "largest_job_share_of_plain_ms", "amdahl_bound", "family_rate_bound",
                "family_rate_Mrays_per_s", "tuning", "scene_build_s",
                "jobs_per_rank") if k in b}
        if world == 1:
            import hptracing_b200 as H
            from hptracing_b200 import scenes as S
            scenes, cams, tris, sbuild = serve_scenes()
            sl = serve_stream(H, S, scenes, cams, tris, sbuild, 50.0, args.serve_seconds,
                              1 << 20, 5, 1)
            for sc in scenes:
                sc.close()
            cpu = None if args.no_cpu_baseline else serve_cpu_baseline((mesh, nodes, leaf), cam)
            line["serve"] = serve_summary(sl, cpu)
        elif rank == 0:
            line["serve"] = {"skipped": "the serving stream runs at N = 1 (one server per "
                                        "device; requests are routed, not split)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
