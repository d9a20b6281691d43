"""Benchmark of the path tracing hot path (the reference's PathTracing Render).

Headline workload (default, --workload batch): the uneven batch: 64 seeded
instances (Cornell boxes holding noise-displaced icospheres or tori of 10k-2M
triangles, diffuse or GGX, 128^2-1024^2 films, 1-64 spp, depth 16; 834M
camera paths per step). ``value`` is Mpaths/s of one batched render of all
instances (one CUDA graph launch, autotuned); ``per_scene`` renders every
instance with its own gyt_render_device call; both render the same paths, so
the images have equal RMSE (``equal_rmse`` reports the largest film
difference). ``single_scene`` is the procedural-mesh workload (a 1,310,720-
triangle displaced icosphere, 1024x1024, 64 spp, depth 16) and ``adjoint`` the
inverse-rendering workload (gradients per second against finite differences).
--workload mesh | env | cornell make one of the single-scene workloads the
headline instead.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on rank 0. Device times are CUDA events on the render stream,
max over ranks; ``e2e`` is the same metric through the public host-image call.
Multi-GPU runs are weak scaling: every rank renders the whole workload
(independent renders, no collective on the data path). Synthetic seeded
geometry stands in for the reference's mesh assets.
"""
import argparse
import dataclasses
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the metric of the headline (batch) workload, and of the single-scene workloads
METRIC = "batched vs per-scene Mpaths/s at equal RMSE; adjoint vs FD grads/s on 1 B200"
METRIC_SINGLE = "Mpaths/s (path-traced camera paths per second)"
SAMPLER_NAMES = {"sobol": "Sobol", "halton": "Halton (Faure permutations)"}
UNIT = "Mpaths/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gyunity", choices=["gyunity", "reference"])
    ap.add_argument("--workload", default="batch", choices=["batch", "mesh", "env", "cornell"],
                    help="batch: the uneven 64-instance batch (default); mesh: procedural mesh; env: "
                         "environment-lit rough-glass torus knot (4M triangles, 1920x1080, 256 spp, depth 32); "
                         "cornell: the Cornell box (256x256, 16 spp)")
    ap.add_argument("--level", type=int, default=8, help="icosphere subdivision level (8 = 1.31M triangles)")
    ap.add_argument("--res", type=int, default=1024)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--depth", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sampler", default="sobol", choices=["sobol", "halton"],
                    help="sobol: SobolSampler + SobolEnum (default); halton: HaltonSampler (Faure) + HaltonEnum")
    ap.add_argument("--bvh-width", type=int, default=8, choices=[2, 8],
                    help="single-scene workloads: 8 = compressed 8-wide BVH (default), 2 = binary BVH; the batch "
                         "uses the library default (binary, built on the GPU)")
    ap.add_argument("--bvh-builder", default="device", choices=["device", "host"])
    ap.add_argument("--batch-instances", type=int, default=64, help="instances of the uneven batch workload")
    ap.add_argument("--batch-width", type=int, default=0, choices=[0, 2, 8],
                    help="batch BVH width instead of the autotuner's choice between both (0)")
    ap.add_argument("--batch-paths-in-flight", type=int, default=0,
                    help="batch pool size instead of the autotuner's choice (small cases for ncu captures)")
    ap.add_argument("--paths-in-flight", type=int, default=1 << 24,
                    help="path pool of the single-scene, volume and adjoint contexts (the batch's is autotuned)")
    ap.add_argument("--no-single-scene", action="store_true",
                    help="batch workload: skip the single-scene (procedural mesh) measurement")
    ap.add_argument("--adjoint-iters", type=int, default=200,
                    help="Adam iterations of the inverse-rendering run after the adjoint timing (0 = skip the run)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-light-tracing", action="store_true",
                    help="skip the light-tracing measurement (Cornell box, 512x512, 16 photons per pixel)")
    ap.add_argument("--no-volume", action="store_true",
                    help="skip the volumetric path-tracing measurement (Cornell box in fog, 512x512, 16 spp)")
    return ap.parse_args()


def workload(a):
    """The single-scene workload (--workload mesh, env, cornell; the batch
    line's single_scene object uses mesh)."""
    from gyunity_b200 import scenes
    if a.workload == "env":
        sd = scenes.env_torus_knot()
    elif a.workload == "cornell":
        sd = scenes.cornell_box(res=256, spp=16, max_depth=8, rr_depth=3)
    else:
        sd = scenes.procedural_mesh_box(level=a.level, res=a.res, spp=a.spp, max_depth=a.depth)
    sd.params.sampler = a.sampler
    return sd


def config(a, sd, extra=None):
    cam, prm = sd.camera, sd.params
    if a.workload == "env":
        c = {"workload": "env_lit_rough_glass_torus_knot", "material": "GGX rough dielectric alpha 0.1 IOR 1.5",
             "env_map": "2048x1024 synthetic sky, RGBE-rounded", "l2": "inputs larger than L2; no flush"}
    elif a.workload == "cornell":
        c = {"workload": "cornell_box_spheres", "material": "diffuse walls, mirror and glass spheres",
             "l2": "scene fits in L2 (the configuration's own size)"}
    else:
        c = {"workload": "procedural_mesh_cornell", "material": "GGX conductor", "groups": 64,
             "l2": "inputs larger than L2 (BVH + triangles exceed 126 MB); no flush"}
    c.update({"triangles": int(sd.n_triangles), "resolution": "%dx%d" % (cam.res_x, cam.res_y), "spp": prm.spp,
              "max_depth": prm.max_depth, "rr_depth": prm.rr_depth, "sampler": SAMPLER_NAMES[prm.sampler],
              "paths_per_step": int(sd.n_paths())})
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------ dist setup ---
class Dist:
    """One process per GPU (torchrun environment). Every rank renders its own
    full frame, so the only collectives are the barrier around the timed
    region and the max-over-ranks reduction of the timings. NCCL on GPUs;
    gloo where CUDA is absent (the CPU tests of this plumbing)."""

    def __init__(self, n, backend=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            self.dist = dist
            self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=120))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch
            if self.backend == "nccl":
                self.dist.barrier(device_ids=[self.local])
                torch.cuda.synchronize()
            else:
                self.dist.barrier()

    def max(self, v):
        if not self.pg:
            return v
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


# --------------------------------------------------------------- clocks ---
class Clocks:
    """Samples nvidia-smi during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.out.name) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------- CPU baseline ---
# The reference CPU integrator on the batch's own path mix: every instance, on
# a regular grid of every 16th column and 32nd row of its film with all of its
# samples per pixel, i.e. 1/512 of each instance's paths (1.6M of the 834M),
# so that each instance weighs in the sample as it weighs in the batch.
BATCH_GRID = (16, 32)


def _cpu_render(sd, spp, rows=None, threads=None):
    """One render of sd at spp by the reference CPU integrator (compiled from
    its sources, oracle/_ref) or, where that binary is absent, by the
    oracle's CPU restatement. Returns (paths, render seconds, kind, threads);
    scene loading and the BVH build are outside the timed render."""
    import copy
    from oracle import scene_io as io
    threads = threads or os.cpu_count() or 1
    s2 = copy.deepcopy(sd)
    s2.params.spp = spp
    if io.have_harness():
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "w.gyts")
            io.write_scene(path, s2)
            _, info = io.ref_render(tmp, path, rows=rows, spp=spp, threads=threads, sampler=sd.params.sampler)
        return info["paths"], info["render_s"], "reference", info["threads"]
    from oracle.port import oracle as orc
    o = orc.OracleScene(s2)
    r = rows or sd.camera.res_y
    t = time.perf_counter()
    o.render(rows=(0, r), precision=32, threads=threads, params=s2.params)
    return sd.camera.res_x * r * spp, time.perf_counter() - t, "port", threads


def cpu_baseline(sd, spp, rows=None, threads=None):
    """Single-scene CPU baseline: the full film of the same workload at spp."""
    n, sec, kind, th = _cpu_render(sd, spp, rows, threads)
    what = "TiledIntegrator::Render" if kind == "reference" else "CPU restatement"
    return {"value": n / sec / 1e6, "unit": UNIT, "cores": th, "kind": kind,
            "sample": "%d rows x %d px x %d spp of the same workload (%s, BVH build excluded)"
                      % (n // (sd.camera.res_x * spp), sd.camera.res_x, spp, what)}


def batch_workload(n, sampler="sobol", stride=1):
    """Instances 0, stride, 2 stride, ... < n of the uneven batch (seeds 1000 + i)."""
    from gyunity_b200 import scenes
    out = []
    for i in range(0, n, stride):
        sd = scenes.batch_instance(1000 + i)
        sd.params.sampler = sampler
        out.append((i, sd))
    return out


def batch_grid_samples(sd, i):
    """Instance i's share of the CPU sample: pixels on a grid of every
    BATCH_GRID[0]th column and BATCH_GRID[1]th row (offset by the instance
    index), every sample of each: (n, 3) uint32 x, y, s."""
    gx, gy = BATCH_GRID
    W, H, S = sd.camera.res_x, sd.camera.res_y, sd.params.spp
    xs = np.arange(i % gx, W, gx)
    ys = np.arange((i // gx) % gy, H, gy)
    X, Y = np.meshgrid(xs, ys)
    px = np.stack([X.ravel(), Y.ravel()], 1)
    return np.concatenate([np.repeat(px, S, axis=0), np.tile(np.arange(S), len(px))[:, None]], 1).astype(np.uint32)


def cpu_reference_batch(descs, warmup, steps, threads=None):
    """The batch CPU baseline: the reference's PathTracing::Li over every
    instance's grid sample (batch_grid_samples), instance after instance,
    scene loading and the reference's BVH build untimed; warmup + steps
    passes. Returns (Mpaths/s of each step, description). Without the
    reference binary the oracle's CPU restatement traces the same samples."""
    from oracle import scene_io as io
    sample = [(sd, batch_grid_samples(sd, i)) for i, sd in enumerate(descs)]
    paths = int(sum(len(x) for _, x in sample))
    total = int(sum(sd.n_paths() for sd in descs))
    if io.have_harness():
        with tempfile.TemporaryDirectory() as tmp:
            items = []
            for i, (sd, xys) in enumerate(sample):
                path = os.path.join(tmp, "inst%d.gyts" % i)
                io.write_scene(path, sd)
                items.append((path, xys))
            rec = io.ref_sample(tmp, items, warmup, steps, sampler=descs[0].params.sampler, threads=threads)
        vals = [rec["paths_per_step"] / t / 1e6 for t in rec["step_s"]]
        kind, cores, what = "reference", rec["threads"], "PathTracing::Li of the reference"
    else:
        from oracle.port import oracle as orc
        cores = threads or os.cpu_count() or 1
        secs = [0.0] * steps
        for sd, xys in sample:
            o = orc.OracleScene(sd)
            for k in range(warmup + steps):
                t = time.perf_counter()
                o.paths(xys[:, 0], xys[:, 1], xys[:, 2], precision=32, threads=cores)
                if k >= warmup:
                    secs[k - warmup] += time.perf_counter() - t
        vals = [paths / t / 1e6 for t in secs]
        kind, what = "port", "the CPU restatement"
    desc = ("all %d instances, every %dth column and %dth row of each film with all its samples per pixel: %d of "
            "the batch's %d paths (1/%d of every instance, the batch's own mix), %s, scene loading and BVH build "
            "untimed" % (len(descs), BATCH_GRID[0], BATCH_GRID[1], paths, total, BATCH_GRID[0] * BATCH_GRID[1],
                         what))
    return vals, {"kind": kind, "cores": cores, "sample": desc, "paths": paths}


def run_reference(a):
    # the reference is a CPU integrator: rank 0 runs it, other ranks exit at once
    if int(os.environ.get("RANK", "0")) != 0:
        return
    if a.workload == "batch":
        descs = [sd for _, sd in batch_workload(a.batch_instances, a.sampler)]
        vals, info = cpu_reference_batch(descs, a.warmup, a.steps)
        cfg = batch_config(a, descs)
        metric = METRIC
    else:
        sd = workload(a)
        vals, info = [], None
        for k in range(a.warmup + a.steps):
            info = cpu_baseline(sd, 1)
            if k >= a.warmup:
                vals.append(info["value"])
        info["paths"] = sd.camera.res_x * sd.camera.res_y
        cfg = config(a, sd, {"reference_sample_spp": 1})
        metric = METRIC_SINGLE
    v = statistics.median(vals)
    paths = info["paths"]
    line = {"impl": "reference", "metric": metric, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": paths / v / 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                             "sample": info["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ our arm ----
def run_ours(a):
    import torch
    d = Dist(a.gpus)
    torch.cuda.set_device(d.local)
    import gyunity_b200 as g
    if a.workload == "batch":
        line = measure_batch(a, d, g, torch)
        if not a.no_single_scene:
            a1 = argparse.Namespace(**vars(a))
            a1.workload = "mesh"
            single = measure_single(a1, d, g, torch)
            if d.rank == 0:
                for k in ("n_gpus", "steps", "warmup", "higher_is_better", "scaling", "vs_baseline", "dtype", "data"):
                    single.pop(k, None)
                line["single_scene"] = single
    else:
        line = measure_single(a, d, g, torch)
    if not a.no_adjoint:
        adj = measure_adjoint(a, d, g, torch)
        if d.rank == 0:
            line["adjoint"] = adj
    if not a.no_light_tracing:
        lt = measure_light_tracing(a, d, g, torch)
        if d.rank == 0:
            line["light_tracing"] = lt
    if not a.no_volume:
        vol = measure_volume(a, d, g, torch)
        if d.rank == 0:
            line["volume"] = vol
    if d.rank == 0:
        print(json.dumps(line), flush=True)
    d.close()


def bvh_label(width, builder):
    return "%s, %s-built" % ("8-wide" if width == 8 else "binary", builder)


def measure_single(a, d, g, torch):
    """One scene per step through gyt_render_device (--workload mesh, env,
    cornell); returns the JSON line on rank 0."""
    sd = workload(a)
    ctx = g.Context(d.local, capacity=a.paths_in_flight, bvh_width=a.bvh_width, bvh_builder=a.bvh_builder)
    t0 = time.perf_counter()
    scene = g.Scene(sd, ctx)
    scene_s = time.perf_counter() - t0
    W, H = sd.camera.res_x, sd.camera.res_y
    film = torch.zeros(W * H * 4, dtype=torch.float64, device="cuda")
    cam, prm = sd.camera, sd.params

    for _ in range(a.warmup):
        film.zero_()
        ctx.render_device(scene, cam, prm, film.data_ptr())
    d.barrier()
    torch.cuda.synchronize()
    stats = []
    with Clocks(d.local) as clk:
        wall0 = time.perf_counter()
        for _ in range(a.steps):
            stats.append(ctx.render_device(scene, cam, prm, film.data_ptr()))
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
    d.barrier()
    dev_ms = sum(s["ms"] for s in stats)
    dev_ms = d.max(dev_ms)
    paths = sum(s["paths"] for s in stats)
    value = paths * d.world / (dev_ms / 1e3) / 1e6
    launches = sum(s["launches"] for s in stats)

    # end to end through the public Render call (image back to host memory)
    e2e_steps = max(1, min(a.steps, 3))
    film_h = g.Film(W, H)
    pc = g.PinHoleCamera(film_h, cam.pos, cam.look_at, cam.up, cam.fovy, cam.film_distance)
    integ = g.GpuPathTracing(prm.spp, prm.max_depth, prm.rr_depth)
    integ.Render(scene, pc)
    d.barrier()
    t = time.perf_counter()
    for _ in range(e2e_steps):
        integ.Render(scene, pc)
    e2e_s = d.max(time.perf_counter() - t)
    e2e = paths / a.steps * e2e_steps * d.world / e2e_s / 1e6
    # cold path: scene upload + acceleration structure build + render
    t = time.perf_counter()
    s2 = g.Scene(sd, ctx)
    integ.Render(s2, pc)
    cold_s = time.perf_counter() - t
    s2.close()

    # scene creation (upload + acceleration structure) with every builder
    own = bvh_label(a.bvh_width, a.bvh_builder)
    builds = {own: scene_s}
    for w, b in ((2, "device"), (2, "host"), (8, "host")):
        if bvh_label(w, b) in builds:
            continue
        ctx_o = g.Context(d.local, bvh_width=w, bvh_builder=b)
        t = time.perf_counter()
        g.Scene(sd, ctx_o).close()
        builds[bvh_label(w, b)] = time.perf_counter() - t
        ctx_o.close()

    line = None
    if d.rank == 0:
        # kernel-level profile of one render (event timing) and traversal counts
        ctx.set_profile(1)
        film.zero_()
        torch.cuda.nvtx.range_push("single_profile")  # the launch list's capture window
        ctx.render_device(scene, cam, prm, film.data_ptr())
        torch.cuda.nvtx.range_pop()
        prof = ctx.read_profile()
        ctx.set_profile(2)
        film.zero_()
        ctx.render_device(scene, cam, prm, film.data_ptr())
        cnt = ctx.read_profile()
        ctx.set_profile(0)
        out = roofline(prof, cnt, stats[-1]["path_slots"], paths // a.steps,
                       node_bytes=80 if a.bvh_width == 8 else 64)
        line = {"metric": METRIC_SINGLE, "value": value, "unit": UNIT, "n_gpus": d.world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": dev_ms / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural mesh, no dataset)",
                "config": config(a, sd, {"parallelism": "independent frames per GPU" if d.world > 1 else "1 GPU",
                                         "paths_in_flight": a.paths_in_flight,
                                         "bvh": own}),
                "wall_ms_per_step": wall * 1e3 / a.steps,
                "iterations_per_step": stats[-1]["iterations"],
                "scene_upload_and_bvh_s": builds,
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": ctypes.sizeof(_c().GytCamera) +
                        ctypes.sizeof(_c().GytRenderParams), "d2h_bytes_per_step": W * H * 3 * 4,
                        "note": "public Render call with the scene resident, image copied to host each step"},
                "e2e_cold": {"value": paths / a.steps / cold_s / 1e6, "unit": UNIT,
                             "note": "scene upload from host arrays + BVH build + render + image readback"},
                "gpu_launches": launches, "roofline": out, "rays_per_s": rays_per_s(prof, dev_ms / a.steps),
                "clocks": clk.summary(), "profile": prof, "traversal_counts": cnt}
        if not a.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(sd, spp=2)
            except Exception as e:  # reported, never fatal for the GPU numbers
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    scene.close()
    ctx.close()
    return line


def _c():
    from gyunity_b200 import _capi
    return _capi


def batch_config(a, descs, extra=None):
    c = {"workload": "uneven_batch_%d_instances" % a.batch_instances,
         "instances": a.batch_instances, "instance_seeds": "1000..%d" % (1000 + a.batch_instances - 1),
         "scenes": "Cornell boxes holding a noise-displaced icosphere or ring torus (10k-2M triangles, log-uniform), "
                   "diffuse or GGX conductor; films 128^2-1024^2; 1-64 spp; depth 16, Russian roulette from 5",
         "sampler": SAMPLER_NAMES[a.sampler], "l2": "inputs larger than L2 (26M triangles resident); no flush"}
    if descs is not None:
        c.update({"triangles": int(sum(sd.n_triangles for sd in descs)),
                  "paths_per_step": int(sum(sd.n_paths() for sd in descs))})
    if extra:
        c.update(extra)
    return c


def measure_batch(a, d, g, torch):
    """The headline: the uneven batch (64 seeded instances) rendered by the
    per-scene integrator (gyt_render_device once per instance) and by the
    batched one (gyt_render_batch_device: one graph launch, autotuned). Both
    render the same paths, so the images have equal RMSE; the check reports
    the largest film difference. Returns the JSON line on rank 0."""
    t = time.perf_counter()
    descs = [sd for _, sd in batch_workload(a.batch_instances, a.sampler)]
    gen_s = time.perf_counter() - t
    ctx = g.Context(d.local)
    t = time.perf_counter()
    scs2 = [g.Scene(sd, ctx) for sd in descs]
    create_s = time.perf_counter() - t
    # the same scenes with the 8-wide BVH (built on the device too), so that
    # the autotuner can pick the width
    ctx8 = g.Context(d.local, bvh_width=8)
    t = time.perf_counter()
    scs8 = [g.Scene(sd, ctx8) for sd in descs]
    create8_s = time.perf_counter() - t
    cams = [sd.camera for sd in descs]
    prms = [sd.params for sd in descs]
    films = [torch.zeros(c.res_x * c.res_y * 4, dtype=torch.float64, device="cuda") for c in cams]
    ptrs = [f.data_ptr() for f in films]
    paths = sum(sd.n_paths() for sd in descs)

    t = time.perf_counter()
    if a.batch_width:
        cfg, tune_mp = ctx.batch_autotune(scs8 if a.batch_width == 8 else scs2, cams, prms, sample_spp=8)
    else:
        cfg, tune_mp = ctx.batch_autotune(scs2, cams, prms, scenes_alt=scs8, sample_spp=8)
    tune_s = time.perf_counter() - t
    if a.batch_paths_in_flight:
        cfg["paths_in_flight"] = a.batch_paths_in_flight
        ctx.set_batch_config(cfg["paths_in_flight"], cfg["stride_blocks_per_sm"], cfg["trace_blocks_per_sm"],
                             cfg["use_graph"])
    # both integrators render the scenes of the width the autotuner chose
    scs = scs8 if cfg["bvh_width"] == 8 else scs2

    def per_scene():
        ms = 0.0
        for sc, c, p, f in zip(scs, cams, prms, ptrs):
            ms += ctx.render_device(sc, c, p, f)["ms"]
        return ms

    for f in films:
        f.zero_()
    per_scene()  # warm-up pass (also the reference films)
    ref = [f.clone() for f in films]
    d.barrier()
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    per_ms = per_scene()
    torch.cuda.synchronize()
    per_wall = time.perf_counter() - w0
    per_ms = d.max(per_ms)

    for _ in range(a.warmup):
        ctx.render_batch_device(scs, cams, prms, ptrs)
    d.barrier()
    torch.cuda.synchronize()
    stats = []
    with Clocks(d.local) as clk:
        w0 = time.perf_counter()
        for _ in range(a.steps):
            stats.append(ctx.render_batch_device(scs, cams, prms, ptrs))
        torch.cuda.synchronize()
        b_wall = (time.perf_counter() - w0) / a.steps
    d.barrier()
    b_ms = d.max(sum(s["ms"] for s in stats)) / a.steps
    launches = sum(s["launches"] for s in stats)
    # equal RMSE: one more batched render from zeroed films against the per-scene films
    for f in films:
        f.zero_()
    ctx.render_batch_device(scs, cams, prms, ptrs)
    torch.cuda.synchronize()
    fdiff = max(float(((x - y).abs().max() / y.abs().max().clamp_min(1e-300)).item()) for x, y in zip(films, ref))
    del ref
    # end to end: the host-image batch call (cameras and parameters in, every image out)
    e2e_steps = max(1, min(a.steps, 2))
    imgs_bytes = sum(c.res_x * c.res_y * 3 * 4 for c in cams)
    h2d = len(descs) * (ctypes.sizeof(_c().GytCamera) + ctypes.sizeof(_c().GytRenderParams))
    # the images land in pinned host buffers that the steps reuse
    imgs = [torch.empty((c.res_y, c.res_x, 3), dtype=torch.float32, pin_memory=True).numpy() for c in cams]
    ctx.render_batch(scs, cams, prms, out=imgs)
    d.barrier()
    t = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.render_batch(scs, cams, prms, out=imgs)
    e2e_s = d.max(time.perf_counter() - t) / e2e_steps

    line = None
    if d.rank == 0:
        # per-kernel event timing of one batched render (host-driven loop),
        # and traversal counts from the per-scene counting pass: both trace
        # exactly the same rays
        ctx.set_profile(1)
        torch.cuda.nvtx.range_push("batch_profile")  # the launch list's capture window
        ctx.render_batch_device(scs, cams, prms, ptrs)
        torch.cuda.nvtx.range_pop()
        prof = ctx.read_profile()
        ctx.set_profile(2)
        per_scene()
        cnt = ctx.read_profile()
        ctx.set_profile(0)
        out = roofline(prof, cnt, prof["rays"]["extend"], paths, node_bytes=80 if cfg["bvh_width"] == 8 else 64)
        out["rays_match_counting_pass"] = prof["rays"] == cnt["rays"]
        value = paths * d.world / (b_ms / 1e3) / 1e6
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": b_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scenes, no dataset)",
                "config": batch_config(a, descs),
                "parallelism": "independent batches per GPU" if d.world > 1 else "1 GPU", "batch_config": cfg,
                "wall_ms_per_step": b_wall * 1e3,
                "per_scene": {"value": paths * d.world / (per_ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": per_ms,
                              "wall_ms_per_step": per_wall * 1e3,
                              "note": "gyt_render_device once per instance, events around each render"},
                "speedup_vs_per_scene": per_ms / b_ms,
                "equal_rmse": {"max_rel_film_diff": fdiff,
                               "note": "same paths in both runs; only the order of the FP64 film sums differs"},
                "autotune": {"config": cfg, "sample_mpaths": tune_mp, "seconds": tune_s,
                             "widths_tried": [a.batch_width] if a.batch_width else [2, 8],
                             "note": "coordinate search over BVH width (binary and 8-wide scenes, both built on "
                                     "the device), grid-stride and traversal blocks per SM on a sample of every "
                                     "instance at spp x 8 / 64 (the batch's mix), median of three renders per "
                                     "candidate; pool sizes 2M-32M on a sample at spp x 32 / 64; the per-scene "
                                     "renders use the chosen width and pool too"},
                "e2e": {"value": paths * d.world / e2e_s / 1e6, "unit": UNIT, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": imgs_bytes, "steps": e2e_steps,
                        "note": "gyt_render_batch with the scenes resident: cameras and parameters in, "
                                "films zeroed, every image resolved and copied to pinned host buffers "
                                "that the steps reuse"},
                "gpu_launches": launches, "graph_launches": a.steps,
                "iterations_per_step": stats[-1]["iterations"],
                "roofline": out, "rays_per_s": rays_per_s(prof, b_ms / d.world),
                "clocks": clk.summary(), "profile": prof, "traversal_counts": cnt,
                "scene_generation_s": gen_s, "scene_create_s": create_s, "scene_create_8wide_s": create8_s}
        if not a.no_cpu_baseline:
            try:
                vals, info = cpu_reference_batch(descs, 0, 1)
                line["cpu_baseline"] = {"value": vals[0], "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                                        "sample": info["sample"]}
            except Exception as e:  # reported, never fatal for the GPU numbers
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    del films
    for sc in scs2 + scs8:
        sc.close()
    ctx8.close()
    ctx.close()
    return line


def measure_light_tracing(a, d, g, torch):
    """LightTracing (integrator/LT.h) on the Cornell box with its spheres,
    512x512, 16 photons per pixel, depth 8: Mphotons/s on the GPU (device
    time, median of the steps) and the reference's LightTracing::Render on
    the host cores at 1 photon per pixel."""
    from gyunity_b200 import scenes
    sd = scenes.cornell_box(res=512, spp=16, max_depth=8)
    ctx = g.Context(d.local)
    sc = g.Scene(sd, ctx)
    buf = torch.zeros(512 * 512 * 3, dtype=torch.float64, device="cuda")
    ms = []
    for k in range(a.warmup + a.steps):
        st = ctx.render_light_tracing_device(sc, sd.camera, sd.params, buf.data_ptr())
        if k >= a.warmup:
            ms.append(st["ms"])
    t = d.max(statistics.median(ms))
    photons = 512 * 512 * 16
    out = {"workload": "Cornell box with mirror and glass spheres, 512x512, 16 photons per pixel, depth 8",
           "value": photons * d.world / (t / 1e3) / 1e6, "unit": "Mphotons/s", "ms_per_step": t,
           "note": "one kernel launch per render (a photon per thread, closest-hit and camera-join rays traced "
                   "inline); the splat buffer accumulates in FP64"}
    if d.rank == 0 and not a.no_cpu_baseline:
        try:
            import copy
            from oracle import scene_io as io
            if io.have_harness():
                s1 = copy.deepcopy(sd)
                s1.params.spp = 1
                with tempfile.TemporaryDirectory() as tmp:
                    path = os.path.join(tmp, "lt.gyts")
                    io.write_scene(path, s1)
                    _, info = io.ref_light_render(tmp, path)
                out["cpu_baseline"] = {"value": info["photons"] / info["render_s"] / 1e6, "unit": "Mphotons/s",
                                       "cores": os.cpu_count(), "kind": "reference",
                                       "sample": "LightTracing::Render of the same scene at 1 photon per pixel"}
        except Exception as e:  # reported, never fatal for the GPU numbers
            out["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    ctx.close()
    return out


def measure_volume(a, d, g, torch):
    """VolPathTracing (integrator/VPT.cpp) on the Cornell box filled with a
    homogeneous medium (sigma_a 0.05, sigma_s 0.5, HG g 0.3) behind a
    material-less front quad, with its mirror and glass spheres, 512x512,
    16 spp, depth 8: Mpaths/s on the GPU (device time, median of the steps)
    and the reference's TiledIntegrator::Render with VolPathTracing on the
    host cores over the first 128 rows."""
    from gyunity_b200 import scenes
    sd = scenes.cornell_fog(res=512, spp=16, max_depth=8)
    ctx = g.Context(d.local, capacity=a.paths_in_flight)
    sc = g.Scene(sd, ctx)
    film = torch.zeros(512 * 512 * 4, dtype=torch.float64, device="cuda")
    ms = []
    for k in range(a.warmup + a.steps):
        st = ctx.render_volume_device(sc, sd.camera, sd.params, film.data_ptr())
        if k >= a.warmup:
            ms.append(st["ms"])
    t = d.max(statistics.median(ms))
    torch.cuda.nvtx.range_push("volume_profile")  # one more render: the launch list's capture window
    ctx.render_volume_device(sc, sd.camera, sd.params, film.data_ptr())
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    paths = 512 * 512 * 16
    out = {"workload": "Cornell box in a homogeneous medium with mirror and glass spheres, 512x512, 16 spp, depth 8",
           "value": paths * d.world / (t / 1e3) / 1e6, "unit": "Mpaths/s", "ms_per_step": t,
           "note": "wavefront over a pool of paths in flight: closest hits, a volume shade kernel that queues "
                   "shadow segments and MIS rays, their transmittance walks, film and compaction; FP64 film"}
    # the same render with equi-angular sampling (VolPathTracing's default)
    sde = dataclasses.replace(sd, params=dataclasses.replace(sd.params, equi_angular=True))
    ms = []
    film.zero_()
    for k in range(a.warmup + a.steps):
        st = ctx.render_volume_device(sc, sde.camera, sde.params, film.data_ptr())
        if k >= a.warmup:
            ms.append(st["ms"])
    te = d.max(statistics.median(ms))
    out["equi_angular"] = {"value": paths * d.world / (te / 1e3) / 1e6, "unit": "Mpaths/s", "ms_per_step": te,
                           "note": "VolPathTracing with equalAngular = true: one light point per bounce, "
                                   "equi-angular distances in the medium, the connection to that point"}
    if d.rank == 0 and not a.no_cpu_baseline:
        for integ, key, dst in (("vpt", "cpu_baseline", out), ("vpt_eq", "cpu_baseline", out["equi_angular"])):
            try:
                from oracle import scene_io as io
                if io.have_harness():
                    with tempfile.TemporaryDirectory() as tmp:
                        path = os.path.join(tmp, "vpt.gyts")
                        io.write_scene(path, sd)
                        _, info = io.ref_render(tmp, path, rows=128, integrator=integ)
                    dst[key] = {"value": info["mpaths_per_s"], "unit": "Mpaths/s", "cores": info["threads"],
                                "kind": "reference",
                                "sample": "TiledIntegrator::Render with VolPathTracing (%s), first 128 rows" %
                                          ("equalAngular = true" if integ == "vpt_eq" else "equalAngular = false")}
            except Exception as e:  # reported, never fatal for the GPU numbers
                dst[key] = {"value": None, "error": str(e)[:200]}
    ctx.close()
    return out


def measure_adjoint(a, d, g, torch):
    """Differentiable inverse rendering: a level-5 icosphere (20,480
    triangles) in 256 GGX material groups and 4 emitter quads, 512x512, 32
    spp, depth 8; P = 256 * (3 albedo + 1 alpha) + 4 * 3 radiance = 1036
    parameters. Gradients per second by path replay (one primal + one adjoint
    pass gives all P) against central finite differences (2P primal renders),
    the FD check on 16 parameters (step 1e-3) and the Adam run from the
    perturbed parameters."""
    from gyunity_b200 import diff, scenes
    ctx = g.Context(d.local, capacity=a.paths_in_flight)
    hidden = scenes.inverse_params(groups=256, emitters=4, seed=7)
    sd = scenes.inverse_box(hidden, level=5, res=512, spp=32, max_depth=8, rr_depth=8)
    r = diff.DiffRenderer(ctx, sd)
    target = r.forward(hidden).clone()
    init = scenes.perturb_params(hidden, seed=8)
    P = init.count
    fwd, adj = [], []
    for k in range(a.warmup + a.steps):
        loss, grad = diff.loss_and_grad(r, init, target)
        if k >= a.warmup:
            fwd.append(r.last["forward_ms"])
            adj.append(r.last["backward_ms"])
    t_f = d.max(statistics.median(fwd))
    t_a = d.max(statistics.median(adj))
    # FD check: 8 albedo, 4 emitter (light sampling kept: exactly linear) and 4 alpha parameters
    picks = [("albedo", i, c) for i, c in ((0, 0), (31, 1), (77, 2), (101, 0), (150, 1), (199, 2), (230, 0),
                                           (255, 1))]
    picks += [("radiance", i, c) for i, c in ((0, 0), (1, 1), (2, 2), (3, 0))]
    picks += [("alpha", i, 0) for i in (5, 64, 128, 200)]

    def get(p, kind, i, c):
        return p.albedo[i, c] if kind == "albedo" else (p.alpha[i] if kind == "alpha" else p.radiance[i, c])

    def put(p, kind, i, c, v):
        q = scenes.InverseParams(p.albedo.copy(), p.alpha.copy(), p.radiance.copy())
        if kind == "albedo":
            q.albedo[i, c] = v
        elif kind == "alpha":
            q.alpha[i] = v
        else:
            q.radiance[i, c] = v
        return q

    checks, free = [], []
    for kind, i, c in picks:
        cur = get(init, kind, i, c)
        keep = kind == "radiance"
        up, dn = np.float32(cur + 1e-3), np.float32(cur - 1e-3)
        # alpha: BSDF sampling and pdfs frozen at the unstepped parameters, so
        # that the difference quotient is the detached-sampling derivative
        frozen = init if kind == "alpha" else None
        fd = (diff.loss_at(r, put(init, kind, i, c, up), target, keep, frozen) -
              diff.loss_at(r, put(init, kind, i, c, dn), target, keep, frozen)) / (float(up) - float(dn))
        ad = float(get(grad, kind, i, c))
        name = "%s[%d%s]" % (kind, i, "" if kind == "alpha" else ",%d" % c)
        checks.append({"param": name, "fd": fd, "adjoint": ad, "rel_err": abs(fd - ad) / max(abs(fd), 1e-30)})
        if kind == "alpha":
            fd_free = (diff.loss_at(r, put(init, kind, i, c, up), target) -
                       diff.loss_at(r, put(init, kind, i, c, dn), target)) / (float(up) - float(dn))
            free.append({"param": name, "fd": fd_free, "adjoint": ad})
    out = {"workload": "inverse rendering: 20,480-triangle icosphere, 256 GGX groups, 4 emitters, 512x512, 32 spp, "
                       "depth 8, %d parameters" % P,
           "forward_ms": t_f, "adjoint_ms": t_a,
           "grads_per_s": P / ((t_f + t_a) / 1e3), "fd_grads_per_s": P / (2 * P * t_f / 1e3),
           "speedup_vs_fd": 2 * P * t_f / (t_f + t_a),
           "paths_per_pass": int(sd.n_paths()),
           "adjoint_mpaths_per_s": sd.n_paths() / t_a / 1e3,
           "fd_check": checks,
           "fd_check_max_rel_err": {k: max(x["rel_err"] for x in checks if x["param"].startswith(k))
                                    for k in ("albedo", "radiance", "alpha")},
           "fd_check_note": "central differences of the full loss, step 1e-3; emitter steps keep the "
                            "light-selection distribution; alpha steps hold BSDF sampling and pdfs at the "
                            "unstepped parameters (gyt_scene_freeze_sampling), whose difference quotient is the "
                            "detached-sampling derivative",
           "fd_free_alpha": free,
           "fd_free_alpha_note": "the same alpha steps with sampling free: the sampled directions move with "
                                 "alpha, a far noisier estimator of the same derivative (one sample set; "
                                 "tests/test_gpu_adjoint.py checks its mean over 32 disjoint sample sets "
                                 "against the adjoint)"}
    if a.adjoint_iters > 0:
        t = time.perf_counter()
        p, hist = diff.optimize(r, target, init, iterations=a.adjoint_iters, lr=0.02)
        el = time.perf_counter() - t
        err0 = float(np.abs(init.flat() - hidden.flat()).mean())
        err1 = float(np.abs(p.flat() - hidden.flat()).mean())
        out["optimization"] = {"iterations": a.adjoint_iters, "optimizer": "Adam lr 0.02", "loss_first": hist[0],
                               "loss_last": hist[-1], "param_mae_first": err0, "param_mae_last": err1,
                               "seconds": el,
                               "e2e_grads_per_s": P * a.adjoint_iters / el,
                               "note": "wall clock of the whole loop: parameter upload, primal, loss, adjoint, "
                                       "gradient download and the Adam step through PathReplayRender"}
    ctx.close()
    return out


# Algorithmic bytes per path slot and per ray:
# path state read by a stage = origin 16 + direction 16 + throughput 16 +
# radiance 16 + Sobol' index 8 + meta 4 = 76 B; written back by shade = 68 B;
# closest hit 16 B; a queued segment ray (origin+tmax, direction) 32 B and its
# contribution 16 B; a BVH node 64 B (binary) or 80 B (8-wide); a triangle 48 B.
STATE_READ, STATE_WRITE, HIT, RAY, CONTRIB = 76, 68, 16, 32, 16


def kernel_bytes(kernel, prof, cnt, slots, node_bytes, gen_paths):
    """Algorithmic bytes of all launches of one kernel in a profiled render:
    traversal bytes per ray = BVH nodes x node size + triangle tests x 48 B
    (counts from the counting pass) on top of the ray and hit records; the
    shade and finish kernels by the path-state records of the slots they
    visit, the generate kernel by those of the gen_paths paths it writes."""
    rays = cnt["rays"]

    def trav(k):
        r = max(1, rays[k])
        return cnt["node_visits"][k] / r * node_bytes + cnt["tri_tests"][k] / r * 48

    if kernel == "extend":
        return rays["extend"] * (RAY + HIT + trav("extend"))
    if kernel == "connect":
        return sum(rays[k] * (RAY + CONTRIB + 16 + trav(k)) for k in ("shadow", "mis"))
    if kernel == "shade":
        return slots * (STATE_READ + HIT + STATE_WRITE) + (rays["shadow"] + rays["mis"]) * (RAY + CONTRIB)
    if kernel == "finish":
        return slots * (STATE_READ + 4) + slots * (STATE_READ + 8)
    return gen_paths * STATE_WRITE


def roofline(prof, cnt, slots, gen_paths, node_bytes=64):
    """Bandwidth roofline of the dominant kernel. achieved = algorithmic bytes
    of its launches / their CUDA-event time (kernel_bytes); the same figures
    for every kernel under "kernels", and the ncu issue utilisation and SIMD
    efficiency of the captured kernels (profiles/traffic.json) under "ncu"."""
    peak, src = peaks()
    ms = {k: v for k, v in prof["ms"].items() if k != "unused"}
    dom = max(ms, key=ms.get)
    launches = max(1, prof["launches"][dom])
    rays = cnt["rays"]
    byts = kernel_bytes(dom, prof, cnt, slots, node_bytes, gen_paths)
    achieved = byts / (ms[dom] / 1e3) / 1e9
    traffic, ncu = None, {}
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            recs = json.load(open(tf))
            rec = recs.get("k_" + dom)
            if rec and "bytes_per_slot" in rec:
                traffic = rec["bytes_per_slot"] * slots / launches
            ncu = {k: {f: v[f] for f in ("issue_active", "threads_per_inst", "source") if f in v}
                   for k, v in recs.items() if "issue_active" in v}
        except Exception:
            traffic = None
    kernels = {}
    for k, t in ms.items():
        n = max(1, prof["launches"][k])
        b = kernel_bytes(k, prof, cnt, slots, node_bytes, gen_paths)
        kernels["k_" + k] = {"share": t / sum(ms.values()), "launches": n, "avg_launch_ms": t / n,
                             "algorithmic_bytes_per_launch": b / n,
                             "achieved_gbs": b / (t / 1e3) / 1e9 if t > 0 else None,
                             "frac": b / (t / 1e3) / 1e9 / peak if t > 0 else None}
    per_ray = {k: {"nodes": cnt["node_visits"][k] / max(1, rays[k]), "tris": cnt["tri_tests"][k] / max(1, rays[k]),
                   "rays": rays[k]} for k in rays}
    return {"bound": "hbm", "kernel": "k_" + dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": src, "traffic": traffic,
            "algorithmic_bytes_per_launch": byts / launches, "launches": launches,
            "avg_launch_ms": ms[dom] / launches, "traversal": per_ray,
            "share": {k: v / sum(ms.values()) for k, v in ms.items()}, "kernels": kernels, "ncu": ncu}


def rays_per_s(prof, step_ms):
    """Extend, shadow and MIS rays traced per second of the timed step (the
    profiled render traces the same rays as each timed step)."""
    r = prof["rays"]
    out = {k: r[k] / (step_ms / 1e3) for k in ("extend", "shadow", "mis")}
    out["total"] = sum(out.values())
    out["unit"] = "rays/s"
    return out


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
