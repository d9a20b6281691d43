// The drop-in, run: the reference's own Scene, PinHoleCamera, Film and
// Renderer (visual/Renderer.h:22-26) with the GPU integrators of
// include/gyt_integrator.h as the Integrator, against the same program's
// reference integrator on the same objects. TEST INFRASTRUCTURE: built by
// oracle/ref/build_ref.py from the reference's sources and linked against
// libgyunity_b200 (the product), whose use through the binding it checks.
//
//   gyref_dropin <scene.gyts> <pt|vpt|vpt_eq> <gpu.bin> <cpu.bin> <gpu.hdr> <cpu.hdr>
//
// The scene file is read twice, as an application would build its scene:
// once into the reference's objects (Scene::AddPrimitive / AddLight, BVHAccel)
// and once into the GytSceneExport record the binding uploads, one record per
// AddPrimitive in the same order. Renderer::Render runs the integrator and
// Film::SaveImage (the .hdr files); the films' pixel buffers (colour / weight)
// go to the .bin files as float32 W*H*3. Prints one JSON line with both
// render times.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <functional>
#include <iostream>
#include <list>
#include <map>
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
#include "visual/Renderer.h"
#include "camera/PinholeCamera.h"
#include "integrator/PT.h"
#include "integrator/VPT.h"
#include "accelerator/BVHAccel.h"
#include "sampler/Sobol.h"
#include "sampler/SobolEnum.h"
#include "material/Diffuse.h"
#include "material/Mirror.h"
#include "material/Glass.h"
#include "material/RoughDielectric.h"
#include "texture/ConstantTexture.h"
#include "light/AreaLight.h"
#include "light/EnvLight.h"
#include "shape/Sphere.h"
#include "system/Memory.h"
#include "volume/Homogeneous.h"
#undef private
#undef protected

#undef STB_IMAGE_WRITE_IMPLEMENTATION
#include <stb/stb_image_write.h>

#include "scene_loader.h"
#include "gyt_integrator.h"

using namespace Gyunity;

namespace {

// The scene file's arrays as the binding's export record (the field order of
// oracle/scene_io.py's write_scene, as gyref::load_scene reads it).
std::shared_ptr<GytSceneExport> export_scene(const char* path) {
  std::vector<char> buf = gyref::read_file(path);
  gyref::Reader r{buf.data(), buf.data() + buf.size()};
  if (r.get<uint32_t>() != 0x53545947u) throw std::runtime_error("bad scene magic");
  const uint32_t version = r.get<uint32_t>();
  const uint32_t nv = r.get<uint32_t>(), nt = r.get<uint32_t>(), ns = r.get<uint32_t>();
  const uint32_t nm = r.get<uint32_t>(), ne = r.get<uint32_t>(), has_normals = r.get<uint32_t>();
  const uint32_t env_w = r.get<uint32_t>(), env_h = r.get<uint32_t>();
  if (env_w * env_h) throw std::runtime_error("the export record holds no environment map");
  r.arr<uint32_t>(5);  // resolution, spp, depth, roulette depth
  r.arr<float>(12);    // camera, environment scale
  const std::vector<float> V = r.arr<float>((size_t)nv * 3);
  const std::vector<float> N = has_normals ? r.arr<float>((size_t)nv * 3) : std::vector<float>();
  const std::vector<uint32_t> I = r.arr<uint32_t>((size_t)nt * 3);
  const std::vector<uint32_t> TM = r.arr<uint32_t>(nt);
  const std::vector<int32_t> TE = r.arr<int32_t>(nt);
  const std::vector<float> SP = r.arr<float>((size_t)ns * 4);
  const std::vector<uint32_t> SM = r.arr<uint32_t>(ns);
  const std::vector<uint32_t> MT = r.arr<uint32_t>(nm);
  const std::vector<float> MP = r.arr<float>((size_t)nm * 16);
  const std::vector<float> EM = r.arr<float>((size_t)ne * 3);
  auto ex = std::make_shared<GytSceneExport>();
  std::vector<int32_t> TMED;
  if (version == 2) {
    const uint32_t n_media = r.get<uint32_t>(), has_tmed = r.get<uint32_t>();
    const std::vector<float> MD = r.arr<float>((size_t)n_media * 7);
    for (uint32_t k = 0; k < n_media; ++k) {
      const float* q = &MD[7 * k];
      ex->AddMedium(Vec3(q[0], q[1], q[2]), Vec3(q[3], q[4], q[5]), q[6]);
    }
    if (has_tmed) TMED = r.arr<int32_t>((size_t)nt * 2);
  }
  for (uint32_t m = 0; m < nm; ++m) ex->AddMaterial(MT[m], &MP[16 * m]);
  for (uint32_t t = 0; t < nt; ++t) {
    Vec3 p[3], n[3];
    for (int k = 0; k < 3; ++k) {
      const uint32_t v = I[3 * t + k];
      p[k] = Vec3(V[3 * v], V[3 * v + 1], V[3 * v + 2]);
    }
    for (int k = 0; k < 3; ++k) {
      const uint32_t v = I[3 * t + k];
      n[k] = has_normals ? Vec3(N[3 * v], N[3 * v + 1], N[3 * v + 2]) : Cross(p[1] - p[0], p[2] - p[0]).Norm();
    }
    Vec3 le;
    const Vec3* radiance = nullptr;
    if (TE[t] >= 0) {
      const float* e = &EM[3 * TE[t]];
      le = Vec3(e[0], e[1], e[2]);
      radiance = &le;
    }
    ex->AddTriangle(p, n, TM[t], radiance, TMED.empty() ? -1 : TMED[2 * t], TMED.empty() ? -1 : TMED[2 * t + 1]);
  }
  for (uint32_t s = 0; s < ns; ++s) ex->AddSphere(Vec3(SP[4 * s], SP[4 * s + 1], SP[4 * s + 2]), SP[4 * s + 3], SM[s]);
  return ex;
}

void write_film(const Film& film, const char* path) {
  std::vector<float> out((size_t)film.mResX * film.mResY * 3);
  for (size_t i = 0; i < (size_t)film.mResX * film.mResY; ++i) {
    const auto& px = film.mPixelBuffer[i];
    for (int c = 0; c < 3; ++c) out[3 * i + c] = px.color[c] / px.weight;
  }
  gyref::write_file(path, out.data(), out.size() * 4);
}

double render(const gyref::LoadedScene& ls, const std::shared_ptr<Integrator>& integrator,
              const std::shared_ptr<Film>& film, const std::shared_ptr<Camera>& camera, const char* image) {
  film->SetFileName(image);
  Renderer renderer(ls.scene, camera, integrator, film);
  const auto t0 = std::chrono::steady_clock::now();
  renderer.Render();  // Integrator::Render, then Film::SaveImage
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s <scene.gyts> <pt|vpt|vpt_eq> <gpu.bin> <cpu.bin> <gpu.hdr> <cpu.hdr>\n", argv[0]);
    return 2;
  }
  try {
    gyref::LoadedScene ls = gyref::load_scene(argv[1]);
    const std::string kind = argv[2];
    auto ex = export_scene(argv[1]);
    std::shared_ptr<Integrator> gpu, cpu;
    auto sampler = std::make_shared<SobolSampler>();
    auto senum = std::make_shared<SobolEnum>(ls.resX, ls.resY);
    if (kind == "pt") {
      gpu = std::make_shared<GpuPathTracing>(ls.spp, ls.maxDepth, ex, 0, ls.rrDepth);
      cpu = std::make_shared<PathTracing>(ls.spp, ls.maxDepth, sampler, senum);
    } else if (kind == "vpt" || kind == "vpt_eq") {
      const bool eq = kind == "vpt_eq";
      gpu = std::make_shared<GpuVolPathTracing>(ls.spp, ls.maxDepth, ex, eq);
      cpu = std::make_shared<VolPathTracing>(ls.spp, ls.maxDepth, sampler, senum, eq);
    } else {
      throw std::runtime_error("unknown integrator " + kind);
    }
    // the GPU integrator on the loaded scene's own film and camera
    const double tg = render(ls, gpu, ls.film, ls.camera, argv[5]);
    write_film(*ls.film, argv[3]);
    // the reference integrator on a fresh film seen by the same camera set-up
    auto film = std::make_shared<Film>(ls.resX, ls.resY, new BoxFilter());
    auto cam = std::make_shared<PinHoleCamera>(film, ls.camera->mPos, ls.camera->mLookAt, ls.camera->mUp,
                                               ls.camera->mFovy, ls.camera->mFilmDistance);
    const double tc = render(ls, cpu, film, cam, argv[6]);
    write_film(*film, argv[4]);
    std::printf("{\"gpu_s\": %.6f, \"cpu_s\": %.6f, \"res\": [%d, %d], \"spp\": %d}\n", tg, tc, ls.resX, ls.resY,
                ls.spp);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "gyref_dropin: %s\n", e.what());
    return 1;
  }
  return 0;
}
