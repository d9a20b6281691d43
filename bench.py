"""Benchmark of the path tracing hot path (the reference's PathTracing Render).

Workload (default): a seeded noise-displaced icosphere of 1,310,720 triangles
with 64 GGX-conductor material groups in the Cornell box, 1024x1024 film,
64 spp Sobol', max depth 16 -> 67,108,864 camera paths per step. Synthetic
seeded geometry stands in for the reference's mesh assets.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on rank 0. ``value`` is Mpaths/s of whole renders with the
scene resident on the device (CUDA-event time on the render stream, max over
ranks); ``e2e`` is the same metric through the public Render call with the
image read back to host memory. Multi-GPU runs are weak scaling: every rank
renders its own full frame (independent frames, no collective on the data path).
"""
import argparse
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

METRIC = "Mpaths/s (path-traced camera paths per second)"
UNIT = "Mpaths/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gyunity", choices=["gyunity", "reference"])
    ap.add_argument("--level", type=int, default=8, help="icosphere subdivision level (8 = 1.31M triangles)")
    ap.add_argument("--res", type=int, default=1024)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--depth", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--bvh-width", type=int, default=None, choices=[2, 8])
    ap.add_argument("--bvh-builder", default="device", choices=["device", "host"])
    return ap.parse_args()


def workload(a):
    from gyunity_b200 import scenes
    return scenes.procedural_mesh_box(level=a.level, res=a.res, spp=a.spp, max_depth=a.depth)


def config(a, sd, extra=None):
    c = {"workload": "procedural_mesh_cornell", "triangles": int(sd.n_triangles), "material": "GGX conductor",
         "groups": 64, "resolution": "%dx%d" % (a.res, a.res), "spp": a.spp, "max_depth": a.depth,
         "rr_depth": sd.params.rr_depth, "sampler": "Sobol", "paths_per_step": int(sd.n_paths()),
         "l2": "inputs larger than L2 (BVH + triangles exceed 126 MB); no flush"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------ dist setup ---
class Dist:
    def __init__(self, n):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            self.dist = dist
            backend = "nccl"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch
            self.dist.barrier(device_ids=[self.local])
            torch.cuda.synchronize()

    def max(self, v):
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
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
def cpu_baseline(sd, spp, rows=None, threads=None):
    """The reference CPU integrator (compiled from its sources, oracle/_ref)
    or, when that binary is absent, the oracle's CPU restatement, on a bounded
    sample of the same workload (full film at reduced spp). Returns a dict."""
    from oracle import scene_io as io
    threads = threads or os.cpu_count() or 1
    import copy
    s2 = copy.deepcopy(sd)
    s2.params.spp = spp
    if io.have_harness():
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "w.gyts")
            io.write_scene(path, s2)
            _, info = io.ref_render(tmp, path, rows=rows, spp=spp, threads=threads)
        return {"value": info["mpaths_per_s"], "unit": UNIT, "cores": info["threads"], "kind": "reference",
                "sample": "%d rows x %d px x %d spp of the same workload (TiledIntegrator::Render, BVH build excluded)"
                          % (info["rows"], sd.camera.res_x, spp)}
    from oracle.port import oracle as orc
    o = orc.OracleScene(s2)
    t = time.perf_counter()
    r = rows or sd.camera.res_y
    o.render(rows=(0, r), precision=32, threads=threads, params=s2.params)
    dt = time.perf_counter() - t
    return {"value": sd.camera.res_x * r * spp / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d rows x %d px x %d spp of the same workload (CPU restatement)" % (r, sd.camera.res_x, spp)}


def run_reference(a):
    # the reference is a CPU integrator: rank 0 runs it, other ranks exit at once
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sd = workload(a)
    spp = 1
    vals = []
    info = None
    for k in range(a.warmup + a.steps):
        info = cpu_baseline(sd, spp)
        if k >= a.warmup:
            vals.append(info["value"])
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": sd.camera.res_x * sd.camera.res_y * spp / v / 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(a, sd, {"reference_sample_spp": spp}),
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
    sd = workload(a)
    ctx = g.Context(d.local, bvh_width=a.bvh_width, bvh_builder=a.bvh_builder)
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

    # scene creation with the other binary-BVH builder, for comparison
    other = "host" if a.bvh_builder == "device" else "device"
    ctx_o = g.Context(d.local, bvh_width=a.bvh_width, bvh_builder=other)
    t = time.perf_counter()
    g.Scene(sd, ctx_o).close()
    other_s = time.perf_counter() - t
    ctx_o.close()

    out = None
    if d.rank == 0:
        # kernel-level profile of one render (event timing) and traversal counts
        ctx.set_profile(1)
        film.zero_()
        ctx.render_device(scene, cam, prm, film.data_ptr())
        prof = ctx.read_profile()
        ctx.set_profile(2)
        film.zero_()
        ctx.render_device(scene, cam, prm, film.data_ptr())
        cnt = ctx.read_profile()
        ctx.set_profile(0)
        out = roofline(prof, cnt, stats, node_bytes=80 if a.bvh_width == 8 else 64)
        clocks = clk.summary()
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": dev_ms / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural mesh, no dataset)",
                "config": config(a, sd, {"parallelism": "independent frames per GPU" if d.world > 1 else "1 GPU",
                                         "paths_in_flight": 1 << 21,
                                         "bvh": "8-wide, host-built" if a.bvh_width == 8
                                         else "binary, %s-built" % a.bvh_builder}),
                "wall_ms_per_step": wall * 1e3 / a.steps,
                "iterations_per_step": stats[-1]["iterations"],
                "scene_upload_and_bvh_s": {a.bvh_builder: scene_s, other: other_s},
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 32 + 64 + 16,
                        "d2h_bytes_per_step": W * H * 3 * 4,
                        "note": "public Render call with the scene resident, image copied to host each step"},
                "e2e_cold": {"value": paths / a.steps / cold_s / 1e6, "unit": UNIT,
                             "note": "scene upload from host arrays + BVH build + render + image readback"},
                "gpu_launches": launches, "roofline": out, "clocks": clocks, "profile": prof,
                "traversal_counts": cnt}
        if not a.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(sd, spp=2)
            except Exception as e:  # reported, never fatal for the GPU numbers
                line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
        print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()
    d.close()


# Algorithmic bytes per path slot and per ray:
# path state read by a stage = origin 16 + direction 16 + throughput 16 +
# radiance 16 + Sobol' index 8 + meta 4 = 76 B; written back by shade = 68 B;
# closest hit 16 B; a queued segment ray (origin+tmax, direction) 32 B and its
# contribution 16 B; a BVH node 64 B (binary) or 80 B (8-wide); a triangle 48 B.
STATE_READ, STATE_WRITE, HIT, RAY, CONTRIB = 76, 68, 16, 32, 16


def roofline(prof, cnt, stats, node_bytes=64):
    """Bandwidth roofline of the dominant kernel. achieved = algorithmic bytes
    of its launches / their CUDA-event time; traversal bytes per ray = BVH
    nodes x node size + triangle tests x 48 B (counts from the counting pass)."""
    peak, src = peaks()
    ms = prof["ms"]
    dom = max(ms, key=ms.get)
    launches = max(1, prof["launches"][dom])
    slots = stats[-1]["path_slots"]
    rays = cnt["rays"]

    def trav(k):
        r = max(1, rays[k])
        return cnt["node_visits"][k] / r * node_bytes + cnt["tri_tests"][k] / r * 48

    if dom == "extend":
        byts = rays["extend"] * (RAY + HIT + trav("extend"))
    elif dom in ("shadow", "mis"):
        byts = rays[dom] * (RAY + CONTRIB + 16 + trav(dom))
    elif dom == "shade":
        byts = slots * (STATE_READ + HIT + STATE_WRITE) + (rays["shadow"] + rays["mis"]) * (RAY + CONTRIB)
    elif dom == "finish":
        byts = slots * (STATE_READ + 4) + slots * (STATE_READ + 8)
    else:
        byts = slots * STATE_WRITE
    achieved = byts / (ms[dom] / 1e3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            rec = json.load(open(tf)).get("k_" + dom)
            if rec:
                traffic = rec["bytes_per_slot"] * slots / launches
        except Exception:
            traffic = None
    per_ray = {k: {"nodes": cnt["node_visits"][k] / max(1, rays[k]), "tris": cnt["tri_tests"][k] / max(1, rays[k]),
                   "rays": rays[k]} for k in rays}
    return {"bound": "hbm", "kernel": "k_" + dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": src, "traffic": traffic,
            "algorithmic_bytes_per_launch": byts / launches, "launches": launches,
            "avg_launch_ms": ms[dom] / launches, "traversal": per_ray,
            "share": {k: v / sum(ms.values()) for k, v in ms.items()}}


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
