// Driver for the reference path tracer compiled from its own sources
// (oracle/ref/build_ref.py). TEST INFRASTRUCTURE ONLY: it produces golden
// vectors and the CPU baseline timing; nothing in the product links it.
//
// Commands (all binary I/O is little-endian, see oracle/scene_io.py):
//   sobol   <pairs.bin> <out.bin>             (u32 dim, u64 index) -> f32 sobol::sample
//   enum    <resx> <resy> <trip.bin> <out.bin> (u32 s,x,y) -> u64 SobolEnum::GetIndex
//   halton  <pairs.bin> <out.bin>             (u32 dim, u64 index) -> f32 HaltonSampler (Faure) Sample
//   henum   <resx> <resy> <trip.bin> <out.bin> (u32 s,x,y) -> u64 HaltonEnum::GetIndex
//   hits    <scene> <rays.bin> <out.bin>       closest-hit through BVHAccel::Intersect
//   anyhit  <scene> <rays.bin> <out.bin>       occlusion through BVHAccel::Intersect(ray)
//   paths   <scene> <trip.bin> <out.bin>       PathTracing::Li for (x,y,s) triplets
//   sample  <list.txt> <warmup> <steps>        timed PathTracing::Li over many scenes: each line of the
//           list is "<scene> <trip.bin>"; scene after scene (loading and BVH build untimed), its
//           samples are traced warmup + steps times on all host threads; prints one JSON line with
//           the paths of one step and each step's seconds summed over the scenes
//   render  <scene> <out.bin> [rows]           TiledIntegrator::Render, timed
//   camera  <scene> <out.bin>                  RasterToWorld matrix (row-major f32)
//   bsdf    <cases.bin> <out.bin>              BxDF Sample/Evaluate/Pdf tables
//   toint   <in.bin> <gamma> <out.bin>         f32 -> i32 ImageIO::toInt
//   image   <rgb.bin> <w> <h> <path>           f32 RGB -> ImageIO::WriteImage (.png .bmp .hdr)
//   lt      <scene> <photons.bin> <out.bin>    LightTracing: per photon (u64 index) max_depth records of
//           (on film 1/0 or -1, X, Y, splatted RGB)
//   ltrender <scene> <out.bin>                 LightTracing::Render, the film's splat buffer (W*H*3 f32)
//   obj     <file.obj> <reverse> <spec> <out.bin>  Mesh::LoadFromFile, then Triangle::SetTransform
//           by the transform of spec ("-": none; else "T x y z;S x y z;RX a;RY a;RZ a" composed
//           left to right); 18 f32 per triangle: p0 p1 p2 n0 n1 n2
// paths and render use SobolSampler + SobolEnum, or HaltonSampler (Faure
// permutations) + HaltonEnum when GYREF_SAMPLER=halton; PathTracing, or
// VolPathTracing (without equi-angular sampling) when GYREF_INTEGRATOR=vpt,
// with it (the constructor's default) when GYREF_INTEGRATOR=vpt_eq.
// Standard and shim headers first, so the access override below only reaches
// the reference's own classes (Film's pixel buffer, Scene's counters).
#include <algorithm>
#include <atomic>
#include <functional>
#include <iostream>
#include <map>
#include <list>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <vector>
#include "fmt/fmt.h"
#include "tbb/parallel_for.h"
#define private public
#define protected public
#include "visual/Scene.h"
#include "visual/Film.h"
#include "camera/PinholeCamera.h"
#include "integrator/PT.h"
#include "accelerator/BVHAccel.h"
#include "sampler/Sobol.h"
#include "sampler/SobolEnum.h"
#include "sampler/Halton.h"
#include "sampler/HaltonEnum.h"
#include "material/Diffuse.h"
#include "material/Mirror.h"
#include "material/Glass.h"
#include "material/RoughDielectric.h"
#include "texture/ConstantTexture.h"
#include "light/AreaLight.h"
#include "light/EnvLight.h"
#include "shape/Sphere.h"
#include "system/Memory.h"
#include "image/ImageIO.h"
#include "mesh/Mesh.h"
#include "integrator/LT.h"
#include "integrator/VPT.h"
#include "volume/Homogeneous.h"
#undef private
#undef protected

#undef STB_IMAGE_WRITE_IMPLEMENTATION
#include <stb/stb_image_write.h>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "scene_loader.h"

using namespace Gyunity;
using namespace gyref;

namespace {

struct RayIn { float o[3], d[3], tmax; };
struct HitOut { int32_t prim; float t, b1, b2; };

Ray make_ray(const RayIn& in) {
  Ray r;  // default ctor: no RayEps shift, so the origin is exactly the given one
  r.mOrig = Vec3(in.o[0], in.o[1], in.o[2]);
  r.mDir = Vec3(in.d[0], in.d[1], in.d[2]);
  r.m_tMax = in.tmax;
  r.m_tMin = 0.f;
  return r;
}

int cmd_sobol(int argc, char** argv) {
  std::vector<char> in = read_file(argv[2]);
  size_t n = in.size() / 12;
  std::vector<float> out(n);
  for (size_t i = 0; i < n; ++i) {
    uint32_t dim; uint64_t idx;
    std::memcpy(&dim, &in[12 * i], 4);
    std::memcpy(&idx, &in[12 * i + 4], 8);
    out[i] = sobol::sample(idx, dim);
  }
  write_file(argv[3], out.data(), out.size() * 4);
  return 0;
}

int cmd_enum(int argc, char** argv) {
  SobolEnum e((uint32)std::atoi(argv[2]), (uint32)std::atoi(argv[3]));
  std::vector<char> in = read_file(argv[4]);
  size_t n = in.size() / 12;
  std::vector<uint64_t> out(n);
  for (size_t i = 0; i < n; ++i) {
    uint32_t v[3];
    std::memcpy(v, &in[12 * i], 12);
    out[i] = e.GetIndex(v[0], v[1], v[2]);
  }
  write_file(argv[5], out.data(), out.size() * 8);
  return 0;
}

// HaltonSampler(w, h) as the demo driver builds it (Gyunity_exe/main.cpp:134):
// a non-zero first argument selects the Faure permutations.
const HaltonSampler& faure_halton() {
  static HaltonSampler h(true);
  return h;
}

int cmd_halton(int argc, char** argv) {
  std::vector<char> in = read_file(argv[2]);
  size_t n = in.size() / 12;
  std::vector<float> out(n);
  const HaltonSampler& h = faure_halton();
  for (size_t i = 0; i < n; ++i) {
    uint32_t dim; uint64_t idx;
    std::memcpy(&dim, &in[12 * i], 4);
    std::memcpy(&idx, &in[12 * i + 4], 8);
    out[i] = h.sample(dim, idx);
  }
  write_file(argv[3], out.data(), out.size() * 4);
  return 0;
}

int cmd_henum(int argc, char** argv) {
  HaltonEnum e((uint32)std::atoi(argv[2]), (uint32)std::atoi(argv[3]));
  std::vector<char> in = read_file(argv[4]);
  size_t n = in.size() / 12;
  std::vector<uint64_t> out(n);
  for (size_t i = 0; i < n; ++i) {
    uint32_t v[3];
    std::memcpy(v, &in[12 * i], 12);
    out[i] = e.GetIndex(v[0], v[1], v[2]);
  }
  write_file(argv[5], out.data(), out.size() * 8);
  return 0;
}

int cmd_hits(int argc, char** argv, bool any) {
  LoadedScene ls = load_scene(argv[2]);
  std::vector<char> in = read_file(argv[3]);
  size_t n = in.size() / sizeof(RayIn);
  std::vector<HitOut> out(n);
  for (size_t i = 0; i < n; ++i) {
    RayIn ri;
    std::memcpy(&ri, &in[i * sizeof(RayIn)], sizeof(RayIn));
    Ray r = make_ray(ri);
    HitOut h{-1, 0.f, 0.f, 0.f};
    if (any) {
      h.prim = ls.scene->Intersect(r) ? 1 : 0;
    } else {
      Intersection isect;
      if (ls.scene->Intersect(r, &isect)) {
        h.prim = (int32_t)isect.mPrimId;
        h.t = r.m_tMax;
        h.b1 = isect.mB1;
        h.b2 = isect.mB2;
      }
    }
    out[i] = h;
  }
  write_file(argv[4], out.data(), out.size() * sizeof(HitOut));
  return 0;
}

std::shared_ptr<TiledIntegrator> make_integrator(const LoadedScene& ls, std::shared_ptr<Sampler>* sampler,
                                                 std::shared_ptr<SamplerEnum>* senum) {
  const char* kind = std::getenv("GYREF_SAMPLER");
  if (kind && std::string(kind) == "halton") {
    *sampler = std::make_shared<HaltonSampler>(faure_halton());
    *senum = std::make_shared<HaltonEnum>(ls.resX, ls.resY);
  } else {
    *sampler = std::make_shared<SobolSampler>();
    *senum = std::make_shared<SobolEnum>(ls.resX, ls.resY);
  }
  const char* integ = std::getenv("GYREF_INTEGRATOR");
  if (integ && std::string(integ) == "vpt")  // the estimator without equi-angular sampling
    return std::make_shared<VolPathTracing>(ls.spp, ls.maxDepth, *sampler, *senum, false);
  if (integ && std::string(integ) == "vpt_eq")  // equi-angular sampling, the constructor's default
    return std::make_shared<VolPathTracing>(ls.spp, ls.maxDepth, *sampler, *senum);
  return std::make_shared<PathTracing>(ls.spp, ls.maxDepth, *sampler, *senum);
}

// One sample of TiledIntegrator::Render's inner loop
// (integrator/TiledIntegrator.cpp:40-47) for pixel (x, y), sample s.
Vec3 one_path(const LoadedScene& ls, const TiledIntegrator& pt, const std::shared_ptr<Sampler>& sampler,
              const SamplerEnum& senum, uint32_t x, uint32_t y, uint32_t s, MemoryPool& arena, int* cursor) {
  uint64 instance = senum.GetIndex(s, x, y);
  RandomStateSequence rand(sampler, instance);
  real u = senum.SampleX(x, rand());
  real v = senum.SampleY(y, rand());
  Ray ray = static_cast<const Camera&>(*ls.camera).GenerateRay(x, y, Vec2(u, v));
  Vec3 L = pt.Li(ray, *ls.scene, rand, arena);
  arena.Reset();
  if (cursor) *cursor = rand.GetCursor();
  return L;
}

void trace_listed(const LoadedScene& ls, const TiledIntegrator& pt, const std::shared_ptr<Sampler>& sampler,
                  const SamplerEnum& senum, const std::vector<char>& in, float* L, unsigned nth);
unsigned host_threads();

int cmd_paths(int argc, char** argv) {
  LoadedScene ls = load_scene(argv[2]);
  std::shared_ptr<Sampler> sampler;
  std::shared_ptr<SamplerEnum> senum;
  auto pt = make_integrator(ls, &sampler, &senum);
  std::vector<char> in = read_file(argv[3]);
  std::vector<float> out(in.size() / 12 * 4);
  // contiguous chunks on the host threads (the reference's Li is const and
  // each thread has its own memory pool, as TiledIntegrator::Render's workers)
  trace_listed(ls, *pt, sampler, *senum, in, out.data(), host_threads());
  write_file(argv[4], out.data(), out.size() * 4);
  return 0;
}

// Li over listed (x, y, s) samples on nth threads (contiguous chunks, one
// memory pool per thread); L (4 floats per sample: radiance, dimensions
// used) may be null.
void trace_listed(const LoadedScene& ls, const TiledIntegrator& pt, const std::shared_ptr<Sampler>& sampler,
                  const SamplerEnum& senum, const std::vector<char>& in, float* L, unsigned nth) {
  const size_t n = in.size() / 12;
  nth = (unsigned)std::min<size_t>(nth, std::max<size_t>(1, n / 256));
  auto work = [&](size_t a, size_t b) {
    MemoryPool arena;
    for (size_t i = a; i < b; ++i) {
      uint32_t v[3];
      std::memcpy(v, &in[12 * i], 12);
      int cursor = 0;
      Vec3 r = one_path(ls, pt, sampler, senum, v[0], v[1], v[2], arena, &cursor);
      if (L) {
        L[4 * i] = r.x; L[4 * i + 1] = r.y; L[4 * i + 2] = r.z;
        L[4 * i + 3] = (float)cursor;
      }
    }
  };
  std::vector<std::thread> th;
  for (unsigned k = 0; k < nth; ++k) th.emplace_back(work, n * k / nth, n * (k + 1) / nth);
  for (auto& t : th) t.join();
}

unsigned host_threads() {
  unsigned nth = std::max(1u, std::thread::hardware_concurrency());
  if (const char* e = std::getenv("GYREF_THREADS")) nth = std::max(1, std::atoi(e));
  return nth;
}

int cmd_sample(int argc, char** argv) {
  if (argc < 5) throw std::runtime_error("sample <list.txt> <warmup> <steps>");
  const int warmup = std::atoi(argv[3]), steps = std::atoi(argv[4]);
  std::ifstream list(argv[2]);
  if (!list) throw std::runtime_error(std::string("cannot open ") + argv[2]);
  const unsigned nth = host_threads();
  std::vector<double> step_s((size_t)std::max(steps, 0), 0.0);
  double load_s = 0.0;
  size_t paths = 0, scenes = 0;
  std::string scene_path, trip_path;
  while (list >> scene_path >> trip_path) {
    auto t0 = std::chrono::steady_clock::now();
    LoadedScene ls = load_scene(scene_path.c_str());
    std::shared_ptr<Sampler> sampler;
    std::shared_ptr<SamplerEnum> senum;
    auto pt = make_integrator(ls, &sampler, &senum);
    const std::vector<char> in = read_file(trip_path.c_str());
    load_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int k = 0; k < warmup + steps; ++k) {
      const auto a = std::chrono::steady_clock::now();
      trace_listed(ls, *pt, sampler, *senum, in, nullptr, nth);
      const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
      if (k >= warmup) step_s[k - warmup] += sec;
    }
    paths += in.size() / 12;
    ++scenes;
  }
  std::printf("{\"scenes\": %zu, \"paths_per_step\": %zu, \"threads\": %u, \"load_s\": %.3f, \"step_s\": [", scenes,
              paths, nth, load_s);
  for (size_t k = 0; k < step_s.size(); ++k) std::printf("%s%.6f", k ? ", " : "", step_s[k]);
  std::printf("]}\n");
  return 0;
}

// Full TiledIntegrator::Render on all host threads. With [rows] < resY only the
// first `rows` image rows are rendered (a bounded CPU-baseline sample); the
// film keeps the reference Render's per-pixel accumulation either way.
int cmd_render(int argc, char** argv) {
  LoadedScene ls = load_scene(argv[2]);
  int rows = argc > 4 ? std::atoi(argv[4]) : ls.resY;
  if (rows <= 0 || rows > ls.resY) rows = ls.resY;
  if (argc > 5) ls.spp = std::atoi(argv[5]);
  std::shared_ptr<Sampler> sampler;
  std::shared_ptr<SamplerEnum> senum;
  auto pt = make_integrator(ls, &sampler, &senum);
  int fullY = ls.film->mResY;
  if (rows < fullY) ls.film->mResY = rows;  // TiledIntegrator::Render tiles [0, mResY)
  auto t0 = std::chrono::steady_clock::now();
  pt->Render(*ls.scene, *ls.camera);
  auto t1 = std::chrono::steady_clock::now();
  ls.film->mResY = fullY;
  double sec = std::chrono::duration<double>(t1 - t0).count();
  size_t npx = (size_t)ls.resX * ls.resY;
  std::vector<float> img(npx * 4);
  for (size_t i = 0; i < npx; ++i) {
    const Pixel& p = ls.film->mPixelBuffer[i];
    img[4 * i] = p.color.x; img[4 * i + 1] = p.color.y; img[4 * i + 2] = p.color.z; img[4 * i + 3] = p.weight;
  }
  write_file(argv[3], img.data(), img.size() * 4);
  double paths = (double)ls.resX * rows * ls.spp;
  std::printf("{\"render_s\": %.6f, \"paths\": %.0f, \"mpaths_per_s\": %.6f, \"threads\": %d, \"rows\": %d, \"spp\": %d}\n",
              sec, paths, paths / sec / 1e6, tbb::detail_shim::thread_count(), rows, ls.spp);
  return 0;
}

int cmd_camera(int argc, char** argv) {
  LoadedScene ls = load_scene(argv[2]);
  float m[16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) m[4 * i + j] = ls.camera->RasterToWorld.mat(i, j);
  write_file(argv[3], m, sizeof(m));
  return 0;
}

// BxDF tables in the local shading frame. Case record: u32 type, f32 params[16],
// f32 wo[3], f32 u[3], f32 wi_eval[3]. Output: f32 sample_f[3], wi[3], pdf,
// eval_f[3], eval_pdf (11 floats).
int cmd_bsdf(int argc, char** argv) {
  std::vector<char> in = read_file(argv[2]);
  const size_t rec = 4 + 4 * (16 + 9);
  size_t n = in.size() / rec;
  std::vector<float> out(n * 11);
  for (size_t i = 0; i < n; ++i) {
    uint32_t type;
    float p[25];
    std::memcpy(&type, &in[i * rec], 4);
    std::memcpy(p, &in[i * rec + 4], sizeof(p));
    Vec3 wo(p[16], p[17], p[18]), u(p[19], p[20], p[21]), we(p[22], p[23], p[24]);
    std::unique_ptr<BxDF> b;
    switch (type) {
      case 0: b.reset(new DiffuseBSDF(Vec3(p[0], p[1], p[2]))); break;
      case 1: b.reset(new SpecularBSDF(Vec3(p[0], p[1], p[2]))); break;
      case 2: b.reset(new TransmissionBSDF(Vec3(p[3], p[4], p[5]), Vec3(p[0], p[1], p[2]), TransportMode::Radiance, p[15], p[8])); break;
      case 3: b.reset(new MicrofacetReflectionBSDF(new GGXDistribution(p[6], p[7], true),
                                                   new FresnelConductor(Vec3(1, 1, 1), Vec3(p[9], p[10], p[11]), Vec3(p[12], p[13], p[14])),
                                                   Vec3(p[0], p[1], p[2]))); break;
      case 4: b.reset(new RoughDielectricBSDF(new GGXDistribution(p[6], p[7], true), Vec3(p[0], p[1], p[2]),
                                              Vec3(p[3], p[4], p[5]), 1.f, p[8], TransportMode::Radiance)); break;
      default: throw std::runtime_error("bad bsdf type");
    }
    Vec3 wi;
    real pdf = 0;
    Vec3 f = b->Sample(wo, &wi, &pdf, u);
    Vec3 fe = b->Evaluate(wo, we);
    real pe = b->Pdf(wo, we);
    float* o = &out[i * 11];
    o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = wi.x; o[4] = wi.y; o[5] = wi.z; o[6] = pdf;
    o[7] = fe.x; o[8] = fe.y; o[9] = fe.z; o[10] = pe;
  }
  write_file(argv[3], out.data(), out.size() * 4);
  return 0;
}

int cmd_toint(int argc, char** argv) {
  std::vector<char> in = read_file(argv[2]);
  const float gamma = (float)std::atof(argv[3]);
  size_t n = in.size() / 4;
  std::vector<int32_t> out(n);
  for (size_t i = 0; i < n; ++i) {
    float x;
    std::memcpy(&x, &in[4 * i], 4);
    out[i] = ImageIO::toInt(x, gamma);
  }
  write_file(argv[4], out.data(), out.size() * 4);
  return 0;
}

std::shared_ptr<Sampler> lt_sampler() {
  const char* kind = std::getenv("GYREF_SAMPLER");
  if (kind && std::string(kind) == "halton") return std::make_shared<HaltonSampler>(faure_halton());
  return std::make_shared<SobolSampler>();
}

// LightTracing::Render's inner loop (integrator/LT.h:30-44) for listed photons.
int cmd_lt(int argc, char** argv) {
  LoadedScene ls = load_scene(argv[2]);
  std::vector<char> in = read_file(argv[3]);
  const size_t n = in.size() / 8;
  std::shared_ptr<Sampler> sampler = lt_sampler();
  LightTracing lt(sampler, ls.maxDepth, ls.spp);
  const Camera& camera = *ls.camera;
  const int64 resX = ls.resX, resY = ls.resY;
  const int64 total = (int64)ls.spp * resX * resY;
  std::vector<float> out(n * (size_t)ls.maxDepth * 6, 0.f);
  MemoryPool arena;
  for (size_t i = 0; i < n; ++i) {
    uint64_t g;
    std::memcpy(&g, &in[8 * i], 8);
    float* rec = &out[i * (size_t)ls.maxDepth * 6];
    for (int k = 0; k < ls.maxDepth; ++k) rec[6 * k] = -1.f;
    RandomStateSequence rand(sampler, g);
    std::vector<PathVertex> lightPath(ls.maxDepth + 1);
    int nv = lt.GenerateLightPath(*ls.scene, camera, rand, arena, lightPath);
    for (int s = 0; s < nv && s < ls.maxDepth; ++s) {
      Vec3 pRaster;
      bool inScreen = false;
      Vec3 L = lt.ConnectToCamera(*ls.scene, camera, rand, lightPath[s], s, &pRaster, &inScreen);
      L = L * ls.film->mResX * ls.film->mResY / total;
      rec[6 * s] = inScreen ? 1.f : 0.f;
      rec[6 * s + 1] = pRaster.x;
      rec[6 * s + 2] = pRaster.y;
      rec[6 * s + 3] = L.x; rec[6 * s + 4] = L.y; rec[6 * s + 5] = L.z;
    }
    arena.Reset();
  }
  write_file(argv[4], out.data(), out.size() * 4);
  return 0;
}

int cmd_ltrender(int argc, char** argv) {
  LoadedScene ls = load_scene(argv[2]);
  LightTracing lt(lt_sampler(), ls.maxDepth, ls.spp);
  auto t0 = std::chrono::steady_clock::now();
  lt.Render(*ls.scene, *ls.camera);
  auto t1 = std::chrono::steady_clock::now();
  const size_t npx = (size_t)ls.resX * ls.resY;
  std::vector<float> img(npx * 3);
  for (size_t i = 0; i < npx; ++i) {
    const Pixel& p = ls.film->mPixelBuffer[i];
    img[3 * i] = p.splat.x; img[3 * i + 1] = p.splat.y; img[3 * i + 2] = p.splat.z;
  }
  write_file(argv[3], img.data(), img.size() * 4);
  const double sec = std::chrono::duration<double>(t1 - t0).count();
  std::printf("{\"render_s\": %.6f, \"photons\": %.0f}\n", sec, (double)ls.spp * npx);
  return 0;
}

int cmd_obj(int argc, char** argv) {
  Mesh mesh;
  mesh.LoadFromFile(argv[2], std::atoi(argv[3]) != 0);
  const std::string spec = argv[4];
  const bool apply = spec != "-";
  Transform t;
  if (apply) {
    std::stringstream ss(spec);
    std::string item;
    while (std::getline(ss, item, ';')) {
      std::stringstream is(item);
      std::string op;
      is >> op;
      float a = 0, b = 0, c = 0;
      is >> a >> b >> c;
      Transform u;
      if (op == "T") u = Transform::Translate(Vec3(a, b, c));
      else if (op == "S") u = Transform::Scale(a, b, c);
      else if (op == "RX") u = Transform::RotateX(a);
      else if (op == "RY") u = Transform::RotateY(a);
      else if (op == "RZ") u = Transform::RotateZ(a);
      else throw std::runtime_error("bad transform " + op);
      t = t * u;
    }
  }
  std::vector<float> out;
  for (const Triangle& src : mesh.untransformedTriangles) {
    Triangle tri = src;
    if (apply) tri.SetTransform(t);
    const Vec3* v[6] = {&tri.p0, &tri.p1, &tri.p2, &tri.n0, &tri.n1, &tri.n2};
    for (const Vec3* q : v) out.insert(out.end(), {q->x, q->y, q->z});
  }
  write_file(argv[5], out.data(), out.size() * 4);
  return 0;
}

int cmd_image(int argc, char** argv) {
  std::vector<char> in = read_file(argv[2]);
  const uint32_t w = (uint32_t)std::atoi(argv[3]), h = (uint32_t)std::atoi(argv[4]);
  std::vector<Vec3> img((size_t)w * h);
  for (size_t i = 0; i < img.size(); ++i) {
    float c[3];
    std::memcpy(c, &in[12 * i], 12);
    img[i] = Vec3(c[0], c[1], c[2]);
  }
  ImageIO::WriteImage(argv[5], img, w, h);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: gyref_harness <sobol|enum|halton|henum|toint|image|obj|lt|ltrender|hits|anyhit|paths|sample|render|camera|bsdf> ...\n");
    return 2;
  }
  try {
    std::string c = argv[1];
    if (c == "sobol") return cmd_sobol(argc, argv);
    if (c == "enum") return cmd_enum(argc, argv);
    if (c == "halton") return cmd_halton(argc, argv);
    if (c == "henum") return cmd_henum(argc, argv);
    if (c == "hits") return cmd_hits(argc, argv, false);
    if (c == "anyhit") return cmd_hits(argc, argv, true);
    if (c == "paths") return cmd_paths(argc, argv);
    if (c == "sample") return cmd_sample(argc, argv);
    if (c == "render") return cmd_render(argc, argv);
    if (c == "camera") return cmd_camera(argc, argv);
    if (c == "bsdf") return cmd_bsdf(argc, argv);
    if (c == "toint") return cmd_toint(argc, argv);
    if (c == "image") return cmd_image(argc, argv);
    if (c == "obj") return cmd_obj(argc, argv);
    if (c == "lt") return cmd_lt(argc, argv);
    if (c == "ltrender") return cmd_ltrender(argc, argv);
    std::fprintf(stderr, "unknown command %s\n", c.c_str());
    return 2;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
