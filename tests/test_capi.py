"""The C ABI library loads, exports every entry point include/gyt.h declares,
and its host-only pieces agree with the oracle (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
import gyunity_b200 as g
from gyunity_b200 import _capi, scenes


def header_functions():
    text = open(os.path.join(ROOT, "include", "gyt.h")).read()
    return sorted(set(re.findall(r"\b(gyt_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    declared = header_functions()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(_capi.EXPORTS) == declared


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_capi, "_lib", None)
    monkeypatch.setattr(_capi, "LIB_PATH", str(tmp_path / "absent.so"))
    with pytest.raises(_capi.GytError):
        _capi.load()


@pytest.mark.parametrize("res", ["256x256", "1920x1080"])
def test_raster_to_world_matches_reference(res):
    rx, ry = map(int, res.split("x"))
    film = g.Film(rx, ry)
    cam = g.PinHoleCamera(film, (0, 0, 3), (0, 0, 0), (0, 1, 0), scenes.CORNELL_FOVY, 1.0)
    got = cam.raster_to_world()
    ref = golden("camera.npz")[res].astype(np.float64)
    assert np.allclose(got, ref, rtol=1e-5, atol=1e-6)


def test_invalid_arguments_return_status():
    lib = _capi.load()
    assert lib.gyt_context_create(0, None) == 1
    assert lib.gyt_camera_raster_to_world(None, None) == 1
    assert lib.gyt_last_error(None) == b"null context"
