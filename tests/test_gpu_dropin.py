"""The drop-in, run: a program built from the reference's own sources
(oracle/ref/dropin.cpp) renders its Scene through Renderer::Render ->
GpuPathTracing::Render (include/gyt_integrator.h, on the GPU) ->
Film::SetImage -> Film::SaveImage, and through the reference's PathTracing
on the same objects. The GPU film must agree with the reference's and equal
what this package's own API renders for the same scene. Needs a B200 and the
oracle build (oracle/_ref, made by __graft_entry__.build())."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
import gyunity_b200 as g
from gyunity_b200 import scenes
from oracle import scene_io as io

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "oracle", "_ref", "gyref_dropin")


def _run(tmp_path, sd, kind):
    assert os.path.exists(EXE), "oracle/_ref/gyref_dropin is not built (run __graft_entry__.build())"
    path = str(tmp_path / "scene.gyts")
    io.write_scene(path, sd)
    outs = [str(tmp_path / n) for n in ("gpu.bin", "cpu.bin", "gpu.hdr", "cpu.hdr")]
    r = subprocess.run([EXE, path, kind] + outs, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]
    info = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    H, W = sd.camera.res_y, sd.camera.res_x
    gpu = np.fromfile(outs[0], np.float32).reshape(H, W, 3).astype(np.float64)
    cpu = np.fromfile(outs[1], np.float32).reshape(H, W, 3).astype(np.float64)
    for hdr in outs[2:]:  # Film::SaveImage wrote both images
        assert os.path.getsize(hdr) > W * H
    return gpu, cpu, info


def _compare(name, gpu, cpu, mean_tol, rmse_tol):
    rel_mean = abs(gpu.mean() - cpu.mean()) / cpu.mean()
    rmse = np.sqrt(np.mean((gpu - cpu) ** 2)) / np.sqrt(np.mean(cpu ** 2))
    print("%s: GPU drop-in vs the reference's integrator in the same program: relative mean %.2e, relative RMSE "
          "%.4f" % (name, rel_mean, rmse))
    assert np.isfinite(gpu).all()
    assert rel_mean < mean_tol and rmse < rmse_tol


def test_dropin_path_tracing_through_the_reference_renderer(tmp_path, ctx):
    sd = scenes.cornell_box(res=64, spp=16)
    gpu, cpu, info = _run(tmp_path, sd, "pt")
    print("render s:", info)
    _compare("PathTracing", gpu, cpu, 5e-3, 0.02)
    # the binding renders exactly what this package's API renders
    film = g.Film(64, 64)
    cam = g.PinHoleCamera(film, sd.camera.pos, sd.camera.look_at, sd.camera.up, sd.camera.fovy, 1.0)
    g.GpuPathTracing(sd.params.spp, sd.params.max_depth, sd.params.rr_depth).Render(g.Scene(sd, ctx), cam)
    np.testing.assert_allclose(gpu, film.image.astype(np.float64), rtol=1e-6, atol=1e-7)


def test_dropin_volumetric_path_tracing_through_the_reference_renderer(tmp_path):
    # VolPathTracing's default estimator (equi-angular sampling) on the fogged box
    sd = scenes.cornell_fog(res=48, spp=8, max_depth=6)
    gpu, cpu, _ = _run(tmp_path, sd, "vpt_eq")
    _compare("VolPathTracing (equi-angular)", gpu, cpu, 5e-3, 0.02)
