/*
 * gyt_integrator.h - the C++ binding a Gyunity code base adds to use the B200
 * path tracer: GytSceneExport records the flat scene arrays of GytSceneDesc
 * next to Scene::AddPrimitive / AddLight (visual/Scene.h:39-65), and
 * GpuPathTracing is an Integrator (integrator/Integrator.h:17-27) whose
 * Render calls the C ABI of gyt.h and hands the image to Film::SetImage
 * (visual/Film.h:106-117), so Renderer::Render (visual/Renderer.h:22-26)
 * and Film::SaveImage work unchanged.
 *
 * Header-only; include it from the reference's source tree (it uses the
 * reference's Integrator, Camera, Film and Vec3) and link libgyunity_b200.
 */
#pragma once
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "integrator/Integrator.h"
#include "camera/Camera.h"
#include "visual/Film.h"
#include "gyt.h"  // from this repository's include/

GYT_NAMESPACE_BEGIN

// Flat scene arrays recorded next to Scene::AddPrimitive / AddLight.
struct GytSceneExport {
  std::vector<float> vertices, normals, spheres, mat_params, emission;
  std::vector<uint32_t> indices, tri_material, sphere_material, mat_type;
  std::vector<int32_t> tri_emission;
  std::vector<float> media;         // 7 floats per HomogeneousMedium: sigma_a rgb, sigma_s rgb, g
  std::vector<int32_t> tri_medium;  // per triangle: inside, outside medium (-1: none)

  // one material record; kind = GYT_MAT_*, 16 parameters as in include/gyt.h
  uint32_t AddMaterial(uint32_t kind, const float params[16]) {
    mat_type.push_back(kind);
    mat_params.insert(mat_params.end(), params, params + 16);
    return (uint32_t)mat_type.size() - 1;
  }
  // a HomogeneousMedium(sigma_a, sigma_s, g) (volume/Homogeneous.h); returns its index
  int32_t AddMedium(const Vec3& sa, const Vec3& ss, float g) {
    media.insert(media.end(), {sa.x, sa.y, sa.z, ss.x, ss.y, ss.z, g});
    return (int32_t)(media.size() / 7) - 1;
  }
  // a Triangle(p0, p1, p2, n0, n1, n2) primitive; emitting triangles are AreaLights;
  // inside/outside: the primitive's MediumInterface as AddMedium indices
  void AddTriangle(const Vec3 p[3], const Vec3 n[3], uint32_t material, const Vec3* radiance = nullptr,
                   int32_t inside = -1, int32_t outside = -1) {
    uint32_t base = (uint32_t)(vertices.size() / 3);
    for (int k = 0; k < 3; ++k) {
      vertices.insert(vertices.end(), {p[k].x, p[k].y, p[k].z});
      normals.insert(normals.end(), {n[k].x, n[k].y, n[k].z});
      indices.push_back(base + k);
    }
    tri_material.push_back(material);
    tri_medium.insert(tri_medium.end(), {inside, outside});
    if (radiance) {
      tri_emission.push_back((int32_t)(emission.size() / 3));
      emission.insert(emission.end(), {radiance->x, radiance->y, radiance->z});
    } else {
      tri_emission.push_back(-1);
    }
  }
  // a Sphere(radius, centre) primitive (added after all triangles)
  void AddSphere(const Vec3& c, float r, uint32_t material) {
    spheres.insert(spheres.end(), {c.x, c.y, c.z, r});
    sphere_material.push_back(material);
  }
  GytSceneDesc Desc() const {
    GytSceneDesc d = {};
    d.n_vertices = (uint32_t)(vertices.size() / 3);
    d.n_triangles = (uint32_t)tri_material.size();
    d.n_spheres = (uint32_t)sphere_material.size();
    d.n_materials = (uint32_t)mat_type.size();
    d.n_emission = (uint32_t)(emission.size() / 3);
    d.vertices = vertices.data();
    d.normals = normals.data();
    d.indices = indices.data();
    d.tri_material = tri_material.data();
    d.tri_emission = tri_emission.data();
    d.spheres = spheres.data();
    d.sphere_material = sphere_material.data();
    d.mat_type = mat_type.data();
    d.mat_params = mat_params.data();
    d.emission = emission.data();
    if (!media.empty()) {
      d.n_media = (uint32_t)(media.size() / 7);
      d.media = media.data();
      d.tri_medium = tri_medium.data();
    }
    return d;
  }
};

// What the GPU integrators share: a context and the exported scene on the
// device, the camera and film conversions and the error check (a failing
// call throws, where the reference logs and exits, common/Core.h:160-166).
class GpuIntegratorBase : public Integrator {
 public:
  GpuIntegratorBase(std::shared_ptr<GytSceneExport> scene, int device) : mExport(std::move(scene)) {
    Check(gyt_context_create(device, &mCtx), "gyt_context_create");
    GytSceneDesc d = mExport->Desc();
    Check(gyt_scene_create(mCtx, &d, &mScene), "gyt_scene_create");
  }
  ~GpuIntegratorBase() override {
    gyt_scene_destroy(mScene);
    gyt_context_destroy(mCtx);
  }
  GpuIntegratorBase(const GpuIntegratorBase&) = delete;
  GpuIntegratorBase& operator=(const GpuIntegratorBase&) = delete;

 protected:
  static GytCamera ToGyt(const Camera& camera) {
    std::shared_ptr<Film> film = camera.GetFilm();
    return GytCamera{{camera.mPos.x, camera.mPos.y, camera.mPos.z},
                     {camera.mLookAt.x, camera.mLookAt.y, camera.mLookAt.z},
                     {camera.mUp.x, camera.mUp.y, camera.mUp.z},
                     camera.mFovy, camera.mFilmDistance, (uint32_t)film->mResX, (uint32_t)film->mResY};
  }
  static void SetFilm(Film& film, const std::vector<float>& rgb) {
    std::vector<Vec3> image((size_t)film.mResX * film.mResY);
    for (size_t i = 0; i < image.size(); ++i) image[i] = Vec3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
    film.SetImage(image);  // weight 1 per pixel (visual/Film.h:106-117)
  }
  void Check(int32_t rc, const char* what) {
    if (rc != GYT_OK) throw std::runtime_error(std::string(what) + ": " + gyt_last_error(mCtx));
  }
  std::shared_ptr<GytSceneExport> mExport;
  gyt_context* mCtx = nullptr;
  gyt_scene* mScene = nullptr;
};

// Drop-in for PathTracing(spp, maxDepth, SobolSampler, SobolEnum) (integrator/PT.h:12).
class GpuPathTracing : public GpuIntegratorBase {
 public:
  GpuPathTracing(int spp, int maxDepth, std::shared_ptr<GytSceneExport> scene, int device = 0, int rrDepth = 5)
      : GpuIntegratorBase(std::move(scene), device) {
    mParams = GytRenderParams{(uint32_t)spp, (uint32_t)maxDepth, (uint32_t)rrDepth, 0};
  }

  void Render(const Scene& scene, const Camera& camera) override {
    std::shared_ptr<Film> film = camera.GetFilm();
    GytCamera c = ToGyt(camera);
    std::vector<float> rgb((size_t)film->mResX * film->mResY * 3);
    Check(gyt_render(mCtx, mScene, &c, &mParams, rgb.data()), "gyt_render");
    SetFilm(*film, rgb);
  }

  // Several cameras of the scene (an animation's frames, probe views) in one
  // batched call: one pool of paths over all of them, one film each.
  void RenderBatch(const std::vector<std::shared_ptr<Camera>>& cameras, bool autotune = false) {
    const uint32_t n = (uint32_t)cameras.size();
    std::vector<const gyt_scene*> scenes(n, mScene);
    std::vector<GytCamera> cams;
    std::vector<GytRenderParams> prms(n, mParams);
    std::vector<std::vector<float>> rgb(n);
    std::vector<float*> outs;
    for (uint32_t i = 0; i < n; ++i) {
      cams.push_back(ToGyt(*cameras[i]));
      rgb[i].resize((size_t)cams[i].res_x * cams[i].res_y * 3);
      outs.push_back(rgb[i].data());
    }
    if (autotune) {
      GytBatchConfig best;
      Check(gyt_batch_autotune(mCtx, n, scenes.data(), nullptr, cams.data(), prms.data(), 1, &best, nullptr),
            "gyt_batch_autotune");
    }
    Check(gyt_render_batch(mCtx, n, scenes.data(), cams.data(), prms.data(), outs.data()), "gyt_render_batch");
    for (uint32_t i = 0; i < n; ++i) SetFilm(*cameras[i]->GetFilm(), rgb[i]);
  }

 private:
  GytRenderParams mParams;
};

// Drop-in for VolPathTracing(spp, maxDepth, SobolSampler, SobolEnum,
// equalAngular) (integrator/VPT.h:12-19; equalAngular defaults to true there
// too) over the media the export recorded.
class GpuVolPathTracing : public GpuIntegratorBase {
 public:
  GpuVolPathTracing(int spp, int maxDepth, std::shared_ptr<GytSceneExport> scene, bool equalAngular = true,
                    int device = 0)
      : GpuIntegratorBase(std::move(scene), device) {
    mParams = GytRenderParams{(uint32_t)spp, (uint32_t)maxDepth, 0, equalAngular ? GYT_VOLUME_EQUI_ANGULAR : 0u};
  }

  void Render(const Scene& scene, const Camera& camera) override {
    std::shared_ptr<Film> film = camera.GetFilm();
    GytCamera c = ToGyt(camera);
    std::vector<float> rgb((size_t)film->mResX * film->mResY * 3);
    Check(gyt_render_volume(mCtx, mScene, &c, &mParams, rgb.data()), "gyt_render_volume");
    SetFilm(*film, rgb);
  }

 private:
  GytRenderParams mParams;
};

GYT_NAMESPACE_END
