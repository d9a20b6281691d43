"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (one process
each, as torchrun starts them) agree on the max-over-ranks timing and meet at
the barriers; the reference arm's non-zero ranks exit without work."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys, json
sys.path.insert(0, %(root)r)
import bench
d = bench.Dist(2)
assert d.world == 2 and d.backend == "gloo"
d.barrier()
v = d.max(float(10 + 5 * d.rank))
d.barrier()
print(json.dumps({"rank": d.rank, "max": v}))
d.close()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _launch(code, world=2):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        outs.append((p.returncode, out))
    return outs


def test_gloo_max_over_ranks():
    outs = _launch(CHILD % {"root": ROOT})
    import json
    vals = []
    for rc, out in outs:
        assert rc == 0, out
        vals.append(json.loads(out.strip().splitlines()[-1]))
    assert sorted(v["rank"] for v in vals) == [0, 1]
    assert all(v["max"] == 15.0 for v in vals)


def test_reference_arm_other_ranks_exit_without_work():
    # rank 1 of `bench.py --impl reference` under torchrun returns at once
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
    assert r.stdout.strip() == ""
