"""bench.py's reference arm on the CPU: rank 0 times the reference integrator
(or the restatement where the reference binary is absent) and prints one
JSON line carrying the contract's keys."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def _run(*args):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args], env=env,
                       stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_reference_arm_single_scene_line():
    line = _run("--workload", "cornell", "--steps", "1", "--warmup", "0")
    assert KEYS <= set(line)
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]


def test_reference_arm_with_halton_sampler():
    line = _run("--workload", "cornell", "--sampler", "halton", "--steps", "1", "--warmup", "0")
    assert line["value"] > 0 and line["config"]["sampler"].startswith("Halton")


def test_batch_cpu_sample_is_the_batch_mix():
    """The CPU sample covers every instance with 1/512 of its paths (every
    16th column and 32nd row, all samples per pixel), so its path mix is the
    batch's."""
    sys.path.insert(0, ROOT)
    import numpy as np
    import bench
    from gyunity_b200 import scenes
    for i in (0, 5, 37):
        sd = scenes.batch_instance(1000 + i)
        xys = bench.batch_grid_samples(sd, i)
        W, H, S = sd.camera.res_x, sd.camera.res_y, sd.params.spp
        assert len(xys) * 512 == W * H * S
        assert np.all(xys[:, 0] % 16 == i % 16) and np.all(xys[:, 1] % 32 == (i // 16) % 32)
        assert np.array_equal(np.bincount(xys[:, 2], minlength=S), np.full(S, W * H // 512))
    cfg = bench.batch_config(type("A", (), {"batch_instances": 64, "sampler": "sobol"})(), None)
    assert cfg["instances"] == 64 and cfg["workload"] == "uneven_batch_64_instances"


def test_reference_arm_batch_line_small():
    """The batch reference arm end to end on a 2-instance batch."""
    line = _run("--batch-instances", "2", "--steps", "2", "--warmup", "1")
    assert KEYS <= set(line)
    assert line["value"] > 0 and "every 16th column" in line["cpu_baseline"]["sample"]
    assert line["config"]["instances"] == 2
