"""Build recipe of the native library ``gyunity_b200/libgyunity_b200.so``.

nvcc compiles the CUDA translation units for sm_100a only and links the CUDA
runtime statically, so the library loads through a plain ``dlopen`` (ctypes
or a C/C++ host) without any Python or torch dependency.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgyunity_b200.so")
SOURCES = ["gyt_render.cu", "gyt_bvh_gpu.cu", "gyt_bvh_host.cpp", "gyt_image.cpp", "gyt_obj.cpp"]
HEADERS = ["gyt_device.cuh", "gyt_bvh_host.h", "gyt_bvh_gpu.h", "gyt_image.h", "gyt_obj.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-shared", "-cudart", "static"]


def _inputs():
    from . import gen_tables  # noqa: F401  (import-time check that the module exists)
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(HERE, "..", "include", "gyt.h"))
    files.append(os.path.join(HERE, "_gen", "sobol_tables.h"))
    return files


def build(force=False, verbose=False):
    from . import gen_tables
    gen_tables.generate()
    if not force and os.path.exists(LIB):
        newest = max(os.path.getmtime(f) for f in _inputs())
        if os.path.getmtime(LIB) >= newest:
            return LIB
    cmd = [NVCC] + FLAGS + [os.path.join(CSRC, s) for s in SOURCES] + ["-o", LIB]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, cwd=CSRC)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout[-6000:])
    return LIB


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(HERE))
    from gyunity_b200 import build as b
    print(b.build(force="--force" in sys.argv, verbose=True))
