// Scene files of oracle/scene_io.py (write_scene documents every field)
// turned into the reference's own objects: Scene with its primitives, lights
// and BVHAccel, Film, PinHoleCamera. Shared by the reference harness and the
// drop-in program. TEST INFRASTRUCTURE ONLY.
//
// Include after the reference headers it uses (the includer decides whether
// private members are opened up) and after <stb/stb_image_write.h>.
#pragma once
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

extern int gyref_rr_start_depth;

namespace gyref {
using namespace Gyunity;

inline std::vector<char> read_file(const char* path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error(std::string("cannot open ") + path);
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

inline void write_file(const char* path, const void* data, size_t n) {
  FILE* f = std::fopen(path, "wb");
  if (!f) throw std::runtime_error(std::string("cannot write ") + path);
  std::fwrite(data, 1, n, f);
  std::fclose(f);
}

struct Reader {
  const char* p;
  const char* end;
  template <typename T> T get() {
    if (p + sizeof(T) > end) throw std::runtime_error("truncated input");
    T v;
    std::memcpy(&v, p, sizeof(T));
    p += sizeof(T);
    return v;
  }
  template <typename T> std::vector<T> arr(size_t n) {
    if (p + n * sizeof(T) > end) throw std::runtime_error("truncated array");
    std::vector<T> v(n);
    if (n) std::memcpy(v.data(), p, n * sizeof(T));
    p += n * sizeof(T);
    return v;
  }
};

// GGX conductor with alpha given directly: the reference RoughnessMaterial
// (material/Roughness.h:36-46) with its RoughnessToAlpha step left out.
class AlphaConductorMaterial : public Material {
 public:
  AlphaConductorMaterial(Vec3 r, real ax, real ay, Vec3 eta, Vec3 k) : r(r), ax(ax), ay(ay), eta(eta), k(k) {}
  void ComputeScatteringFunction(Intersection* isect, MemoryPool& arena, TransportMode) const override {
    MicrofacetDistribution* d = MEMORY_POOL_ALLOC(arena, GGXDistribution)(ax, ay, true);
    isect->mpBSDF = MEMORY_POOL_ALLOC(arena, BSDF)(*isect);
    Fresnel* fr = MEMORY_POOL_ALLOC(arena, FresnelConductor)(Vec3(1.0, 1.0, 1.0), eta, k);
    isect->mpBSDF->Add(MEMORY_POOL_ALLOC(arena, MicrofacetReflectionBSDF)(d, fr, r));
  }
  Vec3 r; real ax, ay; Vec3 eta, k;
};

// GGX rough dielectric with alpha given directly: RoughDielectricMaterial
// (material/RoughDielectric.h:21-41) without RoughnessToAlpha.
class AlphaDielectricMaterial : public Material {
 public:
  AlphaDielectricMaterial(Vec3 kr, Vec3 kt, real ax, real ay, real eta) : kr(kr), kt(kt), ax(ax), ay(ay), eta(eta) {}
  void ComputeScatteringFunction(Intersection* isect, MemoryPool& arena, TransportMode mode) const override {
    isect->mpBSDF = MEMORY_POOL_ALLOC(arena, BSDF)(*isect);
    MicrofacetDistribution* d = MEMORY_POOL_ALLOC(arena, GGXDistribution)(ax, ay, true);
    isect->mpBSDF->Add(MEMORY_POOL_ALLOC(arena, RoughDielectricBSDF)(d, kr, kt, 1.f, eta, mode));
  }
  Vec3 kr, kt; real ax, ay, eta;
};

inline std::shared_ptr<Texture<Vec3>> ctex(float r, float g, float b) {
  return std::make_shared<ConstantTexture<Vec3>>(Vec3(r, g, b));
}

struct LoadedScene {
  std::shared_ptr<Scene> scene;
  std::shared_ptr<Film> film;
  std::shared_ptr<PinHoleCamera> camera;
  int spp = 1, maxDepth = 1, rrDepth = 5;
  int resX = 0, resY = 0;
};

// Scene file layout: oracle/scene_io.py (write_scene) documents every field.
inline LoadedScene load_scene(const char* path) {
  std::vector<char> buf = read_file(path);
  Reader r{buf.data(), buf.data() + buf.size()};
  if (r.get<uint32_t>() != 0x53545947u) throw std::runtime_error("bad scene magic");
  uint32_t version = r.get<uint32_t>();
  if (version != 1 && version != 2) throw std::runtime_error("bad scene version");
  uint32_t nv = r.get<uint32_t>(), nt = r.get<uint32_t>(), ns = r.get<uint32_t>();
  uint32_t nm = r.get<uint32_t>(), ne = r.get<uint32_t>(), has_normals = r.get<uint32_t>();
  uint32_t env_w = r.get<uint32_t>(), env_h = r.get<uint32_t>();
  LoadedScene out;
  out.resX = (int)r.get<uint32_t>();
  out.resY = (int)r.get<uint32_t>();
  out.spp = (int)r.get<uint32_t>();
  out.maxDepth = (int)r.get<uint32_t>();
  out.rrDepth = (int)r.get<uint32_t>();
  std::vector<float> cam = r.arr<float>(11);  // pos3 look3 up3 fovy filmdist
  float env_scale = r.get<float>();
  std::vector<float> V = r.arr<float>((size_t)nv * 3);
  std::vector<float> N = has_normals ? r.arr<float>((size_t)nv * 3) : std::vector<float>();
  std::vector<uint32_t> I = r.arr<uint32_t>((size_t)nt * 3);
  std::vector<uint32_t> TM = r.arr<uint32_t>(nt);
  std::vector<int32_t> TE = r.arr<int32_t>(nt);
  std::vector<float> SP = r.arr<float>((size_t)ns * 4);
  std::vector<uint32_t> SM = r.arr<uint32_t>(ns);
  std::vector<uint32_t> MT = r.arr<uint32_t>(nm);
  std::vector<float> MP = r.arr<float>((size_t)nm * 16);
  std::vector<float> EM = r.arr<float>((size_t)ne * 3);
  std::vector<float> ENV = r.arr<float>((size_t)env_w * env_h * 3);
  // version 2: homogeneous media (sigma_a, sigma_s, g) and the triangles'
  // MediumInterface (inside, outside; -1 none)
  std::vector<const Medium*> media;
  std::vector<int32_t> TMED;
  if (version == 2) {
    const uint32_t n_media = r.get<uint32_t>(), has_tmed = r.get<uint32_t>();
    std::vector<float> MD = r.arr<float>((size_t)n_media * 7);
    for (uint32_t k = 0; k < n_media; ++k) {
      const float* q = &MD[7 * k];
      media.push_back(new HomogeneousMedium(Vec3(q[0], q[1], q[2]), Vec3(q[3], q[4], q[5]), q[6]));
    }
    if (has_tmed) TMED = r.arr<int32_t>((size_t)nt * 2);
  }
  auto medium_of = [&](int32_t k) -> const Medium* { return k < 0 ? nullptr : media.at((size_t)k); };

  std::vector<std::shared_ptr<Material>> mats;
  for (uint32_t m = 0; m < nm; ++m) {
    const float* p = &MP[m * 16];
    switch (MT[m]) {
      case 0: mats.push_back(std::make_shared<DiffuseMaterial>(ctex(p[0], p[1], p[2]))); break;
      case 1: mats.push_back(std::make_shared<MirrorMaterial>(ctex(p[0], p[1], p[2]))); break;
      case 2: mats.push_back(std::make_shared<GlassMaterial>(ctex(p[0], p[1], p[2]), ctex(p[3], p[4], p[5]), p[15], p[8])); break;
      case 3: mats.push_back(std::make_shared<AlphaConductorMaterial>(Vec3(p[0], p[1], p[2]), p[6], p[7],
                                                                      Vec3(p[9], p[10], p[11]), Vec3(p[12], p[13], p[14]))); break;
      case 4: mats.push_back(std::make_shared<AlphaDielectricMaterial>(Vec3(p[0], p[1], p[2]), Vec3(p[3], p[4], p[5]),
                                                                       p[6], p[7], p[8])); break;
      case 5: mats.push_back(nullptr); break;  // no material: a medium boundary
      default: throw std::runtime_error("unknown material type");
    }
  }
  out.scene = std::make_shared<Scene>();
  out.scene->mShapeNum = 0;
  out.scene->mPrimitiveNum = 0;
  for (uint32_t t = 0; t < nt; ++t) {
    uint32_t a = I[3 * t], b = I[3 * t + 1], c = I[3 * t + 2];
    Vec3 p0(V[3 * a], V[3 * a + 1], V[3 * a + 2]);
    Vec3 p1(V[3 * b], V[3 * b + 1], V[3 * b + 2]);
    Vec3 p2(V[3 * c], V[3 * c + 1], V[3 * c + 2]);
    Vec3 n0, n1, n2;
    if (has_normals) {
      n0 = Vec3(N[3 * a], N[3 * a + 1], N[3 * a + 2]);
      n1 = Vec3(N[3 * b], N[3 * b + 1], N[3 * b + 2]);
      n2 = Vec3(N[3 * c], N[3 * c + 1], N[3 * c + 2]);
    } else {
      n0 = n1 = n2 = Cross(p1 - p0, p2 - p0).Norm();
    }
    auto shape = std::make_shared<Triangle>(Transform(), Transform(), p0, p1, p2, n0, n1, n2);
    std::shared_ptr<Light> light;
    if (TE[t] >= 0) {
      const float* e = &EM[3 * TE[t]];
      light = std::make_shared<AreaLight>(shape, Vec3(e[0], e[1], e[2]));
      out.scene->AddLight(light);
    }
    MediumInterface mi;
    if (!TMED.empty()) mi = MediumInterface(medium_of(TMED[2 * t]), medium_of(TMED[2 * t + 1]));
    out.scene->AddPrimitive(std::make_shared<Primitive>(shape, mats[TM[t]], light, mi));
  }
  for (uint32_t s = 0; s < ns; ++s) {
    auto shape = std::make_shared<Sphere>(Transform(), Transform(), SP[4 * s + 3],
                                          Vec3(SP[4 * s], SP[4 * s + 1], SP[4 * s + 2]));
    out.scene->AddPrimitive(std::make_shared<Primitive>(shape, mats[SM[s]]));
  }
  if (env_w * env_h > 0) {
    // The reference loads environment maps from files only (light/EnvMap.h:291);
    // the texels in the scene file are already RGBE-exact, so the round trip
    // through an .hdr file is lossless.
    // Rows are stored in file order (row 0 = top of the lat-long map).
    std::string tmp = std::string(path) + ".env.hdr";
    stbi_write_hdr(tmp.c_str(), (int)env_w, (int)env_h, 3, ENV.data());
    out.scene->AddLight(std::make_shared<EnvironmentLight>(tmp, 0.f, env_scale));
  }
  out.scene->SetAccelerator(std::make_shared<BVHAccel>(out.scene->GetPrimitives()));
  out.scene->Initialize();
  out.film = std::make_shared<Film>(out.resX, out.resY, new BoxFilter());
  out.camera = std::make_shared<PinHoleCamera>(out.film, Vec3(cam[0], cam[1], cam[2]), Vec3(cam[3], cam[4], cam[5]),
                                               Vec3(cam[6], cam[7], cam[8]), cam[9], cam[10]);
  gyref_rr_start_depth = out.rrDepth;
  return out;
}

}  // namespace gyref
