"""Build the reference path tracer (xiaoyxue/Gyunity) from its own sources as a
CPU oracle and CPU baseline.

TEST INFRASTRUCTURE ONLY: the product never links or calls anything built here.

Recipe (no reference build system is run):
  1. copy ``<reference>/Gyunity/src`` to ``oracle/_ref/src`` (a git-ignored
     build folder; the reference checkout itself is never written);
  2. apply the patch set below to that copy (each patch must match exactly
     once, so a changed reference fails loudly instead of building something
     else);
  3. compile the translation units on the PathTracing route with g++ and the
     shim headers in ``oracle/ref/shims`` (fmt, spdlog, tbb are absent
     submodules), plus ``oracle/ref/harness.cpp``;
  4. link ``oracle/_ref/gyref_harness``;
  5. when the product library is built, link ``oracle/_ref/gyref_dropin``
     (oracle/ref/dropin.cpp: the binding of include/gyt_integrator.h run
     inside the reference's own Renderer).

Patches (numbered P1-P9; each is an exact text replacement):
  P1 common/Core.h:42-43     int64/uint64 as long long so the Sampler override
                             at sampler/Sobol.h:70 matches sampler/Sampler.h:12
  P2 math/Linagl.h:155       dependent base-class name for GCC
  P3 math/Linagl.h:564       template parameter T shadows the class's T
  P4 math/MathUtils.h:16,28  'typename TensorType TType' is not valid C++
  P5 image/ImageIO.cpp:138   functional cast with a two-word type name
  P6 shape/Sphere.h:117      the world-space hit record is never written back
                             (any sphere hit dereferences a null phase function
                             in integrator/Integrator.cpp:125 without it)
  P7 shape/Sphere.h:134      the any-hit test uses a default-constructed ray
  P8 integrator/PT.cpp:53    Russian roulette start depth (hard-coded 5) made
                             a global so configurations that ask for another
                             start depth can be reproduced; default stays 5.
  P9 visual/Intersection.h:23 the BSDF pointer starts null: VolPathTracing
                             tests it to pass through surfaces of no material
                             (integrator/VPT.cpp:70-75) but the constructor
                             leaves it uninitialised.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref")
# the reference checkout: $GYUNITY_REFERENCE, else where this build's
# container mounts it
DEFAULT_REFERENCE = os.environ.get("GYUNITY_REFERENCE") or "/root/reference"

PATCHES = [
    ("common/Core.h", "using int64 = int64_t;", "using int64 = long long;"),
    ("common/Core.h", "using uint64 = uint64_t;", "using uint64 = unsigned long long;"),
    ("math/Linagl.h", "explicit GYT_FORCE_INLINE Vector() : VectorBase(_mm_set_ps1(0.f)) { }",
     "explicit GYT_FORCE_INLINE Vector() : VectorBase<dim__, T_, ISE_>(_mm_set_ps1(0.f)) { }"),
    ("math/Linagl.h",
     "template<int dim__ = dim, typename T, typename std::enable_if_t<dim__ == 3, int> = 0>\n"
     "\tGYT_FORCE_INLINE Vector Cross(const Vector<dim__, T> &a) const {\n"
     "\t\treturn Vector<dim__, T>(",
     "template<int dim__ = dim, typename T__, typename std::enable_if_t<dim__ == 3, int> = 0>\n"
     "\tGYT_FORCE_INLINE Vector Cross(const Vector<dim__, T__> &a) const {\n"
     "\t\treturn Vector<dim__, T__>("),
    ("math/MathUtils.h", "template<typename T, typename TensorType TType = T::tensorType,\n"
     "std::enable_if_t<TType == TensorType::VECTOR, int> = 0>",
     "template<typename T, TensorType TType = T::tensorType,\n"
     "std::enable_if_t<TType == TensorType::VECTOR, int> = 0>"),
    ("math/MathUtils.h", "template<typename T, typename TensorType TType = T::tensorType,\n"
     "\tstd::enable_if_t<TType == TensorType::MATRIX, int> = 0>",
     "template<typename T, TensorType TType = T::tensorType,\n"
     "\tstd::enable_if_t<TType == TensorType::MATRIX, int> = 0>"),
    ("image/ImageIO.cpp", "unsigned char(toInt(image[idx][k]))", "(unsigned char)(toInt(image[idx][k]))"),
    ("shape/Sphere.h", "\t\tObjectToWorld(it);\n", "\t\t*isect = ObjectToWorld(it);\n"),
    ("shape/Sphere.h", "\t\tWorldToObject(ray);\n\n\t\tVec3 op", "\t\tr = WorldToObject(ray);\n\n\t\tVec3 op"),
    ("integrator/PT.cpp", "if (p < 1 && i > 5) {", "if (p < 1 && i > gyref_rr_start_depth) {"),
    ("integrator/PT.cpp", "GYT_NAMESPACE_BEGIN\n", "int gyref_rr_start_depth = 5;\nGYT_NAMESPACE_BEGIN\n"),
    ("visual/Intersection.h", "\tBSDF* mpBSDF;\n", "\tBSDF* mpBSDF = nullptr;\n"),
]

SOURCES = [
    "math/AABB.cpp", "bsdf/BSDF.cpp", "accelerator/BVHAccel.cpp", "camera/Camera.cpp",
    "common/DebugUtils.cpp", "numeric/EFloat.cpp", "light/EnvLight.cpp", "system/Threading.cpp",
    "image/ImageIO.cpp", "integrator/Integrator.cpp", "visual/Intersection.cpp", "math/Linagl.cpp",
    "math/LowDiscrepency.cpp", "visual/Medium.cpp", "system/Memory.cpp", "visual/Microfacet.cpp",
    "integrator/PT.cpp", "camera/PinholeCamera.cpp", "visual/Primitive.cpp", "math/Ray.cpp",
    "sampler/Sampler.cpp", "visual/Sampling.cpp", "visual/Scene.cpp", "shape/Shape.cpp",
    "sampler/Sobol.cpp", "sampler/SobolEnum.cpp", "integrator/TiledIntegrator.cpp", "mesh/Mesh.cpp",
    "integrator/VPT.cpp", "volume/Homogeneous.cpp",
    "math/Transform.cpp", "shape/Triangle.cpp", "visual/Film.cpp", "visual/Visibility.cpp",
]

CXXFLAGS = ["-std=c++17", "-O2", "-msse4.1", "-mavx", "-ffp-contract=off", "-fpermissive",
            "-DNDEBUG", "-w", "-pthread"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout[-4000:]))


def build(reference=DEFAULT_REFERENCE, verbose=True):
    src_ref = os.path.join(reference, "Gyunity", "src")
    if not os.path.isdir(src_ref):
        raise FileNotFoundError("reference sources not found at %s" % src_ref)
    src = os.path.join(OUT, "src")
    obj = os.path.join(OUT, "obj")
    if os.path.isdir(src):
        shutil.rmtree(src)
    os.makedirs(obj, exist_ok=True)
    shutil.copytree(src_ref, src, ignore=shutil.ignore_patterns("*.exe"))
    for rel, old, new in PATCHES:
        path = os.path.join(src, rel)
        with open(path, "r", encoding="utf-8", errors="surrogateescape") as f:
            text = f.read()
        n = text.count(old)
        if n != 1:
            raise RuntimeError("patch for %s matched %d times (expected 1): %r" % (rel, n, old[:60]))
        with open(path, "w", encoding="utf-8", errors="surrogateescape") as f:
            f.write(text.replace(old, new))
    shims = os.path.join(HERE, "shims")
    inc = ["-I", src, "-I", shims, "-I", os.path.join(reference, "external"),
           "-include", os.path.join(shims, "compat.h")]
    units = [(os.path.join(src, s), os.path.join(obj, s.replace("/", "_") + ".o")) for s in SOURCES]
    units.append((os.path.join(shims, "logger_stub.cpp"), os.path.join(obj, "logger_stub.o")))
    units.append((os.path.join(HERE, "harness.cpp"), os.path.join(obj, "harness.o")))

    def compile_one(u):
        _run(["g++"] + CXXFLAGS + inc + ["-c", u[0], "-o", u[1]])

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(compile_one, units))
    exe = os.path.join(OUT, "gyref_harness")
    _run(["g++"] + CXXFLAGS + [o for _, o in units] + ["-o", exe])
    if verbose:
        print("built", exe)
    build_dropin(reference, verbose)
    return exe


def build_dropin(reference=DEFAULT_REFERENCE, verbose=True):
    """``oracle/_ref/gyref_dropin``: oracle/ref/dropin.cpp (the reference's
    Renderer with the GPU integrators of include/gyt_integrator.h) on the
    reference objects of build(), linked against the product library
    (gyunity_b200/libgyunity_b200.so, found at run time next to the
    repository through an $ORIGIN-relative rpath). Skipped when that library
    has not been built."""
    lib_dir = os.path.join(os.path.dirname(ORACLE), "gyunity_b200")
    if not os.path.exists(os.path.join(lib_dir, "libgyunity_b200.so")):
        return None
    src = os.path.join(OUT, "src")
    obj = os.path.join(OUT, "obj")
    shims = os.path.join(HERE, "shims")
    inc = ["-I", src, "-I", shims, "-I", os.path.join(reference, "external"),
           "-I", os.path.join(os.path.dirname(ORACLE), "include"), "-include", os.path.join(shims, "compat.h")]
    dobj = os.path.join(obj, "dropin.o")
    _run(["g++"] + CXXFLAGS + inc + ["-c", os.path.join(HERE, "dropin.cpp"), "-o", dobj])
    objs = [os.path.join(obj, s.replace("/", "_") + ".o") for s in SOURCES] + [os.path.join(obj, "logger_stub.o")]
    exe = os.path.join(OUT, "gyref_dropin")
    _run(["g++"] + CXXFLAGS + objs + [dobj, "-L", lib_dir, "-lgyunity_b200",
                                      "-Wl,-rpath,$ORIGIN/../../gyunity_b200", "-o", exe])
    if verbose:
        print("built", exe)
    return exe


if __name__ == "__main__":
    build(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_REFERENCE)
