"""The GPU's BxDF lobes (diffuse, mirror, glass, GGX conductor, GGX rough
dielectric) directly against the reference's BxDFs compiled from its sources
(tests/golden/bsdf.npz: BxDF::Sample, Evaluate and Pdf on random directions,
sample numbers and the alpha grid), through gyt_bsdf_table. The per-path
tests reach the lobes only through whole paths; this pins each lobe on its
own. Needs a B200."""
import numpy as np
import pytest

from conftest import golden
from oracle import scene_io as io

pytestmark = pytest.mark.gpu


def test_gpu_lobes_match_reference_tables(ctx):
    g = golden("bsdf.npz")
    cases = g["cases"].view(io.BSDF_CASE_DTYPE)
    ref = g["out"].astype(np.float64)
    got = ctx.bsdf_table(cases["type"], cases["params"], cases["wo"], cases["u"], cases["we"]).astype(np.float64)
    assert np.isfinite(got).all()
    # FP32 on both sides; relative to max(|value|, 1e-3) per case (sampled f,
    # wi, pdf, evaluated f and pdf)
    rel = (np.abs(got - ref) / np.maximum(np.abs(ref), 1e-3)).max(1)
    for k, name in enumerate(["diffuse", "mirror", "glass", "GGX conductor", "GGX dielectric"]):
        m = cases["type"] == k
        print("%-15s cases %4d: within 1e-4 %.4f, worst %.2e" % (name, m.sum(), (rel[m] < 1e-4).mean(), rel[m].max()))
        assert (rel[m] < 1e-4).mean() > 0.99, name
        assert (rel[m] < 2e-3).all(), name
