"""The C++ binding (include/gyt_integrator.h) compiles against the
reference's own headers (when the reference build folder is present) and the
C ABI; the C ABI header compiles as C."""
import os
import subprocess

import pytest

from conftest import ROOT

REF_SRC = os.path.join(ROOT, "oracle", "_ref", "src")
SHIMS = os.path.join(ROOT, "oracle", "ref", "shims")


def test_header_compiles_as_c():
    r = subprocess.run(["gcc", "-std=c99", "-fsyntax-only", "-x", "c", "-I", os.path.join(ROOT, "include"), "-"],
                       input='#include "gyt.h"\nint main(void){return GYT_OK;}\n', text=True,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    assert r.returncode == 0, r.stdout


@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference build folder absent")
def test_binding_compiles_against_reference_headers(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text('#include "gyt_integrator.h"\nint main() { return 0; }\n')
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-msse4.1", "-mavx", "-fpermissive", "-w",
           "-include", os.path.join(SHIMS, "compat.h"), "-I", REF_SRC, "-I", SHIMS,
           "-I", os.path.join(ROOT, "include"), "-I", str(tmp_path), str(src)]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout[-3000:]
