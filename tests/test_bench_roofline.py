"""The bench line's roofline arithmetic on a synthetic profile (CPU only).

bench.py turns the per-kernel event times of a profiled render and the
traversal counts of a counting pass into algorithmic bytes per launch,
achieved bandwidth and the fraction of the measured HBM peak. These checks
recompute those figures by hand, so a change to the byte model or to the
bookkeeping (launch counts, the dominant kernel, the traffic per slot from
profiles/traffic.json) shows up here rather than as a wrong number in a
bench line.
"""
import json
import os

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _profile():
    prof = {"ms": {"generate": 2.0, "extend": 30.0, "shade": 40.0, "connect": 20.0, "unused": 0.0,
                   "finish": 6.0},
            "launches": {"generate": 10, "extend": 10, "shade": 10, "connect": 10, "unused": 0, "finish": 10},
            "rays": {"extend": 4_000_000, "shadow": 2_500_000, "mis": 20_000}}
    cnt = {"rays": dict(prof["rays"]),
           "node_visits": {"extend": 12_000_000, "shadow": 5_000_000, "mis": 50_000},
           "tri_tests": {"extend": 16_000_000, "shadow": 11_000_000, "mis": 120_000}}
    return prof, cnt


def test_kernel_bytes_by_hand():
    prof, cnt = _profile()
    slots, gen, nb = 4_000_000, 1_000_000, 80
    R, H, C = bench.RAY, bench.HIT, bench.CONTRIB
    trav_ext = 12_000_000 / 4_000_000 * nb + 16_000_000 / 4_000_000 * 48
    assert bench.kernel_bytes("extend", prof, cnt, slots, nb, gen) == pytest.approx(4_000_000 * (R + H + trav_ext))
    trav_sh = 5_000_000 / 2_500_000 * nb + 11_000_000 / 2_500_000 * 48
    trav_mis = 50_000 / 20_000 * nb + 120_000 / 20_000 * 48
    assert bench.kernel_bytes("connect", prof, cnt, slots, nb, gen) == pytest.approx(
        2_500_000 * (R + C + 16 + trav_sh) + 20_000 * (R + C + 16 + trav_mis))
    assert bench.kernel_bytes("shade", prof, cnt, slots, nb, gen) == pytest.approx(
        slots * (bench.STATE_READ + H + bench.STATE_WRITE) + 2_520_000 * (R + C))
    assert bench.kernel_bytes("generate", prof, cnt, slots, nb, gen) == gen * bench.STATE_WRITE


def test_roofline_dominant_kernel_and_fractions():
    prof, cnt = _profile()
    slots, gen = 4_000_000, 1_000_000
    out = bench.roofline(prof, cnt, slots, gen, node_bytes=80)
    peak, src = bench.peaks()
    assert out["kernel"] == "k_shade" and out["peak"] == peak and out["peak_source"] == src
    byts = bench.kernel_bytes("shade", prof, cnt, slots, 80, gen)
    assert out["launches"] == 10
    assert out["avg_launch_ms"] == pytest.approx(4.0)
    assert out["algorithmic_bytes_per_launch"] == pytest.approx(byts / 10)
    assert out["achieved"] == pytest.approx(byts / 0.040 / 1e9)
    assert out["frac"] == pytest.approx(out["achieved"] / peak)
    # shares over the kernels that ran, summing to one; the unused slot is left out
    assert "unused" not in out["share"]
    assert sum(out["share"].values()) == pytest.approx(1.0)
    assert out["share"]["shade"] == pytest.approx(40.0 / 98.0)
    # every kernel's figures follow the same arithmetic
    for k in ("generate", "extend", "shade", "connect", "finish"):
        rec = out["kernels"]["k_" + k]
        b = bench.kernel_bytes(k, prof, cnt, slots, 80, gen)
        assert rec["avg_launch_ms"] == pytest.approx(prof["ms"][k] / 10)
        assert rec["frac"] == pytest.approx(b / (prof["ms"][k] / 1e3) / 1e9 / peak)
    # per-ray traversal counts
    assert out["traversal"]["extend"]["nodes"] == pytest.approx(3.0)
    assert out["traversal"]["shadow"]["tris"] == pytest.approx(4.4)


def test_roofline_traffic_from_profiles():
    """The traffic figure is the captured DRAM bytes per slot of the dominant
    kernel (profiles/traffic.json) scaled to one launch of this render."""
    prof, cnt = _profile()
    recs = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    out = bench.roofline(prof, cnt, 4_000_000, 1_000_000)
    per_slot = recs["k_shade"]["bytes_per_slot"]
    assert out["traffic"] == pytest.approx(per_slot * 4_000_000 / 10)
    # every captured kernel reports its issue utilisation and SIMD efficiency
    for k, v in recs.items():
        assert 0.0 < out["ncu"][k]["issue_active"] <= 1.0
        assert 1.0 <= out["ncu"][k]["threads_per_inst"] <= 32.0


def test_rays_per_s():
    prof, _ = _profile()
    r = bench.rays_per_s(prof, 2000.0)
    assert r["extend"] == pytest.approx(2_000_000.0)
    assert r["total"] == pytest.approx((4_000_000 + 2_500_000 + 20_000) / 2.0)
    assert r["unit"] == "rays/s"
