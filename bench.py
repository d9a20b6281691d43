"""Benchmark of the path tracing hot path (the reference's PathTracing Render).

Workload (default): a seeded noise-displaced icosphere of 1,310,720 triangles
with 64 GGX-conductor material groups in the Cornell box, 1024x1024 film,
64 spp Sobol', max depth 16 -> 67,108,864 camera paths per step. Synthetic
seeded geometry stands in for the reference's mesh assets. After it, the
uneven batch workload (64 seeded instances of 10k-2M triangles, 128^2-1024^2,
1-64 spp) is timed per scene and as one batched render ("batched" object).

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
    ap.add_argument("--workload", default="mesh", choices=["mesh", "env", "cornell"],
                    help="mesh: procedural mesh (default); env: environment-lit rough-glass torus knot "
                         "(4M triangles, 1920x1080, 256 spp, depth 32); cornell: the Cornell box (256x256, 16 spp)")
    ap.add_argument("--level", type=int, default=8, help="icosphere subdivision level (8 = 1.31M triangles)")
    ap.add_argument("--res", type=int, default=1024)
    ap.add_argument("--spp", type=int, default=64)
    ap.add_argument("--depth", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--bvh-width", type=int, default=None, choices=[2, 8])
    ap.add_argument("--bvh-builder", default="device", choices=["device", "host"])
    ap.add_argument("--batch-instances", type=int, default=64,
                    help="instances of the uneven batch workload measured after the main render (0 = skip)")
    ap.add_argument("--batch-steps", type=int, default=2)
    ap.add_argument("--adjoint-iters", type=int, default=200,
                    help="Adam iterations of the inverse-rendering run after the adjoint timing (0 = skip the run)")
    ap.add_argument("--no-adjoint", action="store_true")
    return ap.parse_args()


def workload(a):
    from gyunity_b200 import scenes
    if a.workload == "env":
        return scenes.env_torus_knot()
    if a.workload == "cornell":
        return scenes.cornell_box(res=256, spp=16, max_depth=8, rr_depth=3)
    return scenes.procedural_mesh_box(level=a.level, res=a.res, spp=a.spp, max_depth=a.depth)


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
              "max_depth": prm.max_depth, "rr_depth": prm.rr_depth, "sampler": "Sobol",
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
    scene.close()
    ctx.close()
    if a.batch_instances > 0:
        b = measure_batch(a, d, g, torch)
        if d.rank == 0:
            line["batched"] = b
    if not a.no_adjoint:
        adj = measure_adjoint(a, d, g, torch)
        if d.rank == 0:
            line["adjoint"] = adj
    if d.rank == 0:
        print(json.dumps(line), flush=True)
    d.close()


def measure_batch(a, d, g, torch):
    """The uneven batch workload (64 seeded instances: Cornell boxes holding
    displaced icospheres or tori of 10k-2M triangles, 128^2-1024^2 films,
    1-64 spp, depth 16): every instance rendered on its own with
    gyt_render_device (the per-scene integrator) against all of them in one
    batched render (one graph launch, autotuned). Both render the same paths,
    so their images have equal RMSE; the check reports the largest film
    difference."""
    from gyunity_b200 import scenes
    t = time.perf_counter()
    descs = scenes.batch_workload(a.batch_instances, seed=1000)
    gen_s = time.perf_counter() - t
    ctx = g.Context(d.local)
    t = time.perf_counter()
    scs = [g.Scene(sd, ctx) for sd in descs]
    create_s = time.perf_counter() - t
    cams = [sd.camera for sd in descs]
    prms = [sd.params for sd in descs]
    films = [torch.zeros(c.res_x * c.res_y * 4, dtype=torch.float64, device="cuda") for c in cams]
    ptrs = [f.data_ptr() for f in films]
    paths = sum(sd.n_paths() for sd in descs)

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

    t = time.perf_counter()
    cfg, tune_mp = ctx.batch_autotune(scs, cams, prms, sample_spp=1)
    tune_s = time.perf_counter() - t
    st = None
    for _ in range(a.warmup):
        st = ctx.render_batch_device(scs, cams, prms, ptrs)
    d.barrier()
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    b_ms = 0.0
    launches = 0
    for _ in range(a.batch_steps):
        st = ctx.render_batch_device(scs, cams, prms, ptrs)
        b_ms += st["ms"]
        launches += st["launches"]
    torch.cuda.synchronize()
    b_wall = (time.perf_counter() - w0) / a.batch_steps
    b_ms = d.max(b_ms / a.batch_steps)
    # equal RMSE: one more batched render from zeroed films against the per-scene films
    for f in films:
        f.zero_()
    ctx.render_batch_device(scs, cams, prms, ptrs)
    torch.cuda.synchronize()
    diff = max(float(((x - y).abs().max() / y.abs().max().clamp_min(1e-300)).item()) for x, y in zip(films, ref))
    # end to end: the host-image batch call (images copied back every step)
    imgs_bytes = sum(c.res_x * c.res_y * 3 * 4 for c in cams)
    ctx.render_batch(scs, cams, prms)
    t = time.perf_counter()
    ctx.render_batch(scs, cams, prms)
    e2e_s = d.max(time.perf_counter() - t)
    out = {"workload": "uneven batch: %d instances, %d triangles, %d paths per step" % (
               len(descs), sum(sd.n_triangles for sd in descs), paths),
           "value": paths * d.world / (b_ms / 1e3) / 1e6, "unit": UNIT,
           "ms_per_step": b_ms, "wall_ms_per_step": b_wall * 1e3, "steps": a.batch_steps,
           "gpu_launches_per_step": launches // max(1, a.batch_steps), "graph_launches_per_step": 1,
           "per_scene": {"value": paths * d.world / (per_ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": per_ms,
                         "wall_ms_per_step": per_wall * 1e3,
                         "note": "gyt_render_device once per instance, events around each render"},
           "speedup_vs_per_scene": per_ms / b_ms,
           "equal_rmse": {"max_rel_film_diff": diff,
                          "note": "same paths in both runs; only the order of the FP64 film sums differs"},
           "autotune": {"config": cfg, "sample_mpaths": tune_mp, "seconds": tune_s},
           "e2e": {"value": paths * d.world / e2e_s / 1e6, "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": imgs_bytes,
                   "note": "gyt_render_batch with the scenes resident, every image copied to host"},
           "scene_generation_s": gen_s, "scene_create_s": create_s}
    del films, ref
    for sc in scs:
        sc.close()
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
    ctx = g.Context(d.local)
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

    checks = []
    for kind, i, c in picks:
        cur = get(init, kind, i, c)
        keep = kind == "radiance"
        up, dn = np.float32(cur + 1e-3), np.float32(cur - 1e-3)
        fd = (diff.loss_at(r, put(init, kind, i, c, up), target, keep) -
              diff.loss_at(r, put(init, kind, i, c, dn), target, keep)) / (float(up) - float(dn))
        ad = float(get(grad, kind, i, c))
        checks.append({"param": "%s[%d%s]" % (kind, i, "" if kind == "alpha" else ",%d" % c), "fd": fd,
                       "adjoint": ad, "rel_err": abs(fd - ad) / max(abs(fd), 1e-30)})
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
           "fd_check_note": "central differences, step 1e-3; emitter steps keep the light-selection "
                            "distribution; alpha moves the sampled directions, which fixed-sample differences "
                            "follow and the detached adjoint does not"}
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


def roofline(prof, cnt, stats, node_bytes=64):
    """Bandwidth roofline of the dominant kernel. achieved = algorithmic bytes
    of its launches / their CUDA-event time; traversal bytes per ray = BVH
    nodes x node size + triangle tests x 48 B (counts from the counting pass)."""
    peak, src = peaks()
    ms = {k: v for k, v in prof["ms"].items() if k != "unused"}
    dom = max(ms, key=ms.get)
    launches = max(1, prof["launches"][dom])
    slots = stats[-1]["path_slots"]
    rays = cnt["rays"]

    def trav(k):
        r = max(1, rays[k])
        return cnt["node_visits"][k] / r * node_bytes + cnt["tri_tests"][k] / r * 48

    if dom == "extend":
        byts = rays["extend"] * (RAY + HIT + trav("extend"))
    elif dom == "connect":
        byts = sum(rays[k] * (RAY + CONTRIB + 16 + trav(k)) for k in ("shadow", "mis"))
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
