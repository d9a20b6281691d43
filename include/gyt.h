/*
 * gyt.h - C ABI of the B200 path tracer that stands in for the reference
 * renderer's PathTracing integrator (xiaoyxue/Gyunity).
 *
 * Plain C types only: handles, POD descriptors, pointers and sizes, int32
 * status codes. No C++ or CUDA types cross this boundary, so the reference's
 * C++ host (or ctypes, or any FFI) can bind it directly.
 *
 * Reference interfaces replaced (paths inside Gyunity/src):
 *   Integrator::Render(const Scene&, const Camera&)   integrator/Integrator.h:20
 *     -> gyt_render / gyt_render_device
 *   TiledIntegrator::Render + PathTracing::Li          integrator/TiledIntegrator.cpp:7-60,
 *                                                       integrator/PT.cpp:10-67
 *   Scene + BVHAccel construction                      visual/Scene.h:26-77, accelerator/BVHAccel.cpp:154-200
 *     -> gyt_scene_create / gyt_scene_destroy
 *   PinHoleCamera / ProjectiveCamera::Initialize        camera/PinholeCamera.h:22-29, camera/Camera.cpp:6-59
 *     -> GytCamera
 *   Film::SetImage / Film pixel buffer                  visual/Film.h:106-117
 *     -> rgb_out of gyt_render (colour / weight per pixel)
 *
 * Error behaviour: every call returns GYT_OK or a negative-free status code
 * and never aborts the process (the reference logs and exits, common/Core.h:160-166);
 * gyt_last_error() gives the message of the last failing call on a context.
 *
 * Threading: one host thread per context at a time. Calls are synchronous
 * unless stated otherwise.
 */
#ifndef GYT_H
#define GYT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gyt_context gyt_context;
typedef struct gyt_scene gyt_scene;

enum {
  GYT_OK = 0,
  GYT_ERR_INVALID = 1,      /* bad argument or scene description */
  GYT_ERR_CUDA = 2,         /* CUDA runtime error (message in gyt_last_error) */
  GYT_ERR_OUT_OF_MEMORY = 3,
  GYT_ERR_UNSUPPORTED = 4,  /* feature or size outside what this build handles */
  GYT_ERR_WATCHDOG = 5      /* a bounded loop hit its iteration cap (twice the iterations the work can
                               need); a film then holds the paths finished so far */
};

/* Material kinds. Parameters are 16 floats per material:
 *   0 diffuse          (material/Diffuse.h:27-31)        [0:3] kd
 *   1 mirror           (material/Mirror.h:26-32)         [0:3] kr
 *   2 glass            (material/Glass.h:30-34)          [0:3] kr [3:6] kt [15] eta1 [8] eta2
 *   3 GGX conductor    (material/Roughness.h:36-46)      [0:3] R [6] alpha_x [7] alpha_y [9:12] eta [12:15] k
 *   4 GGX dielectric   (material/RoughDielectric.h:21-41) [0:3] kr [3:6] kt [6] alpha_x [7] alpha_y [8] eta
 * Alpha is the GGX alpha (the reference maps roughness to alpha with
 * GGXDistribution::RoughnessToAlpha, visual/Microfacet.h:49-54, before this). */
enum { GYT_MAT_DIFFUSE = 0, GYT_MAT_MIRROR = 1, GYT_MAT_GLASS = 2, GYT_MAT_CONDUCTOR = 3, GYT_MAT_DIELECTRIC = 4,
       GYT_MAT_NONE = 5 /* no material: a GeometryPrimitive with a null material (a medium boundary) */ };

/* Scene description (all host pointers; copied by gyt_scene_create).
 * Primitive ids: triangle t has id t, sphere s has id n_triangles + s, the
 * order Scene::AddPrimitive assigns (visual/Scene.h:39-58). Every triangle
 * with tri_emission >= 0 is one AreaLight (light/AreaLight.h); the light list
 * is those triangles in order, then the environment light if env != NULL. */
typedef struct {
  uint32_t n_vertices, n_triangles, n_spheres, n_materials, n_emission;
  const float* vertices;          /* n_vertices * 3 */
  const float* normals;           /* n_vertices * 3, or NULL for face normals */
  const uint32_t* indices;        /* n_triangles * 3 */
  const uint32_t* tri_material;   /* n_triangles */
  const int32_t* tri_emission;    /* n_triangles, index into emission or -1 */
  const float* spheres;           /* n_spheres * 4: centre xyz, radius */
  const uint32_t* sphere_material;/* n_spheres */
  const uint32_t* mat_type;       /* n_materials */
  const float* mat_params;        /* n_materials * 16 */
  const float* emission;          /* n_emission * 3 radiance */
  uint32_t env_w, env_h;          /* lat-long environment map, 0 if none */
  const float* env;               /* env_h * env_w * 3, row 0 = top (theta = 0) */
  float env_scale;
  /* Participating media for volumetric path tracing (HomogeneousMedium,
   * volume/Homogeneous.h): n_media * 7 floats (sigma_a rgb, sigma_s rgb,
   * Henyey-Greenstein g); tri_medium: n_triangles * 2 (medium inside,
   * outside; -1 none), the triangle's MediumInterface (visual/Medium.h), or
   * NULL. A triangle whose inside and outside differ is a medium boundary;
   * one of material GYT_MAT_NONE has no BSDF (rays pass through it). */
  uint32_t n_media;
  const float* media;
  const int32_t* tri_medium;
} GytSceneDesc;

/* PinHoleCamera(film, position, lookAt, up, fovy, filmDistance) on a
 * res_x x res_y film (Gyunity_exe/main.cpp:708-714). */
typedef struct {
  float pos[3], look_at[3], up[3];
  float fovy, film_distance;
  uint32_t res_x, res_y;
} GytCamera;

/* PathTracing(spp, maxDepth, sampler, samplerEnum) (integrator/PT.h:12).
 * Russian roulette is applied at bounce i when i > rr_depth (the reference
 * hard-codes 5 at integrator/PT.cpp:53). The sampler is SobolSampler +
 * SobolEnum unless flags holds GYT_SAMPLER_HALTON. */
typedef struct {
  uint32_t spp, max_depth, rr_depth;
  uint32_t flags;                 /* GYT_SAMPLER_* bits; other bits must be 0 */
} GytRenderParams;

/* HaltonSampler with Faure permutations + HaltonEnum (sampler/Halton.h,
 * sampler/HaltonEnum.h), as the demo driver builds them
 * (Gyunity_exe/main.cpp:134-137): 256 dimensions, later dimensions give 0. */
#define GYT_SAMPLER_HALTON 1u

/* Per-render statistics filled by gyt_render_device. */
typedef struct {
  uint64_t paths;                 /* camera paths traced */
  uint64_t path_slots;            /* path-state slots processed (sum of live paths per iteration) */
  uint32_t iterations;            /* wavefront iterations */
  uint32_t launches;              /* kernels launched */
  float ms;                       /* device time of the render (CUDA events on the context stream) */
} GytRenderStats;

/* Kernel-level profile of the renders since the last gyt_profile_read.
 * Kernel slots: 0 generate, 1 extend (continuation rays), 2 shade,
 * 3 connect (next-event shadow rays, then the BSDF-sampled MIS rays, in one
 * launch), 4 unused (0), 5 finish (film and compaction). Traversal slots:
 * 0 extend, 1 shadow, 2 mis. */
typedef struct {
  float ms[6];                    /* summed device time per kernel (CUDA events) */
  uint32_t launches[6];
  uint64_t rays[3];               /* rays traced per traversal kernel */
  uint64_t node_visits[3];        /* BVH nodes fetched (counting mode only) */
  uint64_t tri_tests[3];          /* triangle tests (counting mode only) */
} GytProfile;

/* Context on one CUDA device; owns a stream and the path-state pools. */
int32_t gyt_context_create(int32_t device, gyt_context** out);
void gyt_context_destroy(gyt_context* ctx);
const char* gyt_last_error(const gyt_context* ctx);
/* Maximum number of paths in flight (default 2M); call before rendering. */
int32_t gyt_context_set_capacity(gyt_context* ctx, uint32_t paths_in_flight);
/* Profiling: 0 off (default), 1 per-kernel event timing, 2 timing plus
 * traversal counters (slower kernels; counts only, not for timing). */
int32_t gyt_context_set_profile(gyt_context* ctx, int32_t mode);
/* Branching factor of the BVH built by later gyt_scene_create calls: 2
 * (binary, two child boxes per 64-byte node; the default) or 8 (quantized
 * child boxes, 80-byte nodes). Both replace BVHAccel (accelerator/BVHAccel.cpp). */
int32_t gyt_context_set_bvh_width(gyt_context* ctx, int32_t width);
/* Where later gyt_scene_create calls build the BVH: GYT_BVH_BUILD_DEVICE
 * (the default) or GYT_BVH_BUILD_HOST. For a binary (width 2) BVH both make
 * the same tree: 16-bin SAH, at most 8 triangles per leaf, identical splits,
 * leaves and child boxes, each leaf's triangles in ascending id order (only
 * the node numbering differs). For the 8-wide BVH both collapse the binary
 * tree of at most 3 triangles per leaf into the same quantized nodes, word
 * for word (breadth-first numbering). Replaces the BVHAccel constructor's
 * build (accelerator/BVHAccel.cpp:154-200). */
#define GYT_BVH_BUILD_HOST 0
#define GYT_BVH_BUILD_DEVICE 1
int32_t gyt_context_set_bvh_builder(gyt_context* ctx, int32_t builder);
/* Copies the accumulated profile into *out and resets it. */
int32_t gyt_profile_read(gyt_context* ctx, GytProfile* out);

/* Uploads the scene and builds the acceleration structure on the device.
 * Replaces Scene::Initialize + new BVHAccel(primitives) (Gyunity_exe/main.cpp:735-738). */
int32_t gyt_scene_create(gyt_context* ctx, const GytSceneDesc* desc, gyt_scene** out);
void gyt_scene_destroy(gyt_scene* scene);
/* Triangle count, BVH node count and device bytes of a scene. */
int32_t gyt_scene_info(const gyt_scene* scene, uint64_t* n_triangles, uint64_t* n_nodes, uint64_t* device_bytes);
/* Copies a binary BVH to the host: node slots (16 floats each, the layout of
 * the traversal kernels; slots a tree does not reach are left as found) and,
 * per leaf-order position, the triangle's index in the scene description.
 * *n_slots receives the slot count; with nodes == NULL only that is set.
 * Capacities are in elements (floats, uint32s). GYT_ERR_UNSUPPORTED for an
 * 8-wide BVH. Inspection and tests; no counterpart in the reference. */
int32_t gyt_scene_read_bvh(const gyt_scene* scene, float* nodes, uint64_t node_capacity, uint32_t* tri_ids,
                           uint64_t tri_capacity, uint64_t* n_slots);
/* The same for an 8-wide BVH: n_nodes nodes of 20 words (5 x uint4, the
 * layout of the traversal kernels) and the leaf-order triangle ids;
 * GYT_ERR_UNSUPPORTED for a binary BVH. Inspection and tests; no counterpart
 * in the reference. */
int32_t gyt_scene_read_wide_bvh(const gyt_scene* scene, uint32_t* words, uint64_t word_capacity, uint32_t* tri_ids,
                                uint64_t tri_capacity, uint64_t* n_nodes);

/* Integrator::Render: renders the full image and writes rgb_out (host,
 * res_x*res_y*3 floats, row-major from the top-left pixel) = colour/weight
 * per pixel, as Film::WriteToPixelBuffer (visual/Film.h:128-136) computes. */
int32_t gyt_render(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                   const GytRenderParams* params, float* rgb_out);

/* Same render into a caller-owned DEVICE film of res_x*res_y*4 doubles
 * (colour sums and filter weights, accumulated, not cleared), on the
 * context's stream; returns when the render is complete. */
int32_t gyt_render_device(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                          const GytRenderParams* params, double* d_film, GytRenderStats* stats);

/* Traces an explicit list of camera paths (xys: n triplets x, y, s; host)
 * and returns per-path radiance (L_out: n*3 floats), the number of Sobol'
 * dimensions each path used (cursor_out) and its discrete decisions for a
 * replay, bit i = bounce i < 64: a Russian roulette number was drawn
 * (rr_mask_out), the next-event shadow ray was occluded (occ_mask_out), the
 * BSDF-sampled MIS ray reached the sampled light (mis_mask_out). Any output
 * may be NULL. This is PathTracing::Li for the samples
 * TiledIntegrator::Render would make (integrator/TiledIntegrator.cpp:40-47). */
int32_t gyt_trace_paths(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                        const GytRenderParams* params, uint64_t n, const uint32_t* xys,
                        float* L_out, uint32_t* cursor_out, uint64_t* rr_mask_out,
                        uint64_t* occ_mask_out, uint64_t* mis_mask_out);

/* Closest-hit (any_hit = 0) or occlusion (any_hit = 1) queries for n rays
 * (host rays: 7 floats each = origin, direction, tmax; tmin = 0). Outputs
 * (host, may be NULL): prim (-1 = miss; for any_hit 1/0), t, b1, b2 where b1
 * and b2 weight vertices 1 and 2 as Triangle::Intersect reports them
 * (shape/Triangle.cpp:71-103). BVHAccel::Intersect (accelerator/BVHAccel.cpp:401-487). */
int32_t gyt_intersect(gyt_context* ctx, const gyt_scene* scene, uint64_t n, const float* rays,
                      int32_t any_hit, int32_t* prim, float* t, float* b1, float* b2);

/* sobol::sample (sampler/Sobol.h:46-61) for n (dimension, index) pairs. */
int32_t gyt_sobol(gyt_context* ctx, uint64_t n, const uint32_t* dims, const uint64_t* indices, float* out);

/* The BxDF lobes of the shading kernels in their local frame, for n cases
 * (host arrays): material kind types[i] (GYT_MAT_DIFFUSE..GYT_MAT_DIELECTRIC)
 * with parameters params[16 i..] (the GytSceneDesc.mat_params layout); vec[9 i..]
 * = wo, u, we. out[11 i..] = the sample BxDF::Sample(wo, u) gives (f rgb, wi,
 * pdf), then BxDF::Evaluate(wo, we) (rgb) and BxDF::Pdf(wo, we): the BxDFs of
 * bsdf/BSDF.h:162-616 on the GPU, for parity tests. */
int32_t gyt_bsdf_table(gyt_context* ctx, uint64_t n, const uint32_t* types, const float* params, const float* vec,
                       float* out);

/* SobolEnum::GetIndex (sampler/SobolEnum.h:23-28) for n (s, x, y) triplets. */
int32_t gyt_sobol_enum_index(gyt_context* ctx, uint32_t res_x, uint32_t res_y, uint64_t n,
                             const uint32_t* sxy, uint64_t* out);

/* ---- Light tracing ---------------------------------------------------------
 * LightTracing(sampler, maxDepth, spp) (integrator/LT.h:11-230) on the GPU:
 * spp * res_x * res_y photons, photon g with sampler index g. Each light
 * path starts on a power-sampled area light (cosine-weighted direction about
 * the interpolated normal), follows BSDF samples in importance transport up
 * to max_depth vertices (no roulette), and each vertex is joined to the
 * pinhole camera; unoccluded joins are splatted (Film::AddSplat,
 * visual/Film.h:89-104) scaled by res_x * res_y / photons. params: spp,
 * max_depth and the sampler flag (rr_depth unused). Scenes with an
 * environment light are refused (the reference samples area lights only).
 * gyt_render_light_tracing: the splat image (res_x*res_y*3 floats, host);
 * _device: accumulated into d_splat (res_x*res_y*3 doubles). Differences: a
 * light direction or BSDF sample of pdf 0 ends the path (the reference
 * divides by the zero pdf, or continues with an undefined direction). */
int32_t gyt_render_light_tracing(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                 const GytRenderParams* params, float* rgb_out);
int32_t gyt_render_light_tracing_device(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                        const GytRenderParams* params, double* d_splat, GytRenderStats* stats);
/* Per-photon records for parity tests: for photons[i], max_depth records of
 * 6 floats (on film 1 / 0, or -1 where the path has no such vertex; pixel X,
 * Y; the splatted RGB), vertex 0 = the light vertex; a missing vertex's
 * record is (-1, 0, 0, 0, 0, 0). */
int32_t gyt_trace_light_paths(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                              const GytRenderParams* params, uint64_t n, const uint64_t* photons, float* records);

/* ---- Volumetric path tracing -----------------------------------------------
 * VolPathTracing(spp, maxDepth, sampler, samplerEnum, equalAngular)
 * (integrator/VPT.h:12-19, integrator/VPT.cpp:7-171) with the scene's
 * homogeneous media (GytSceneDesc::media, tri_medium). Without
 * GYT_VOLUME_EQUI_ANGULAR in params->flags, the estimator of
 * equalAngular = false:
 * camera rays start in no medium; a ray through a medium samples a
 * scattering distance (HomogeneousMedium::Sample, volume/Homogeneous.cpp);
 * at a medium point light is gathered with the Henyey-Greenstein phase
 * function (both halves of the MIS estimate, transmittance along shadow
 * rays) and the path continues in a phase-sampled direction; surfaces of
 * GYT_MAT_NONE are passed through without using a bounce. No Russian
 * roulette (the reference's test is always false). Environment lights are
 * refused. _device accumulates into a film as gyt_render_device; the
 * reference's VolPathTracing needs its BSDF pointer initialised to null to
 * pass through surfaces of no material (it reads it uninitialised). A hit
 * at the very end of a shadow segment (the light's own surface) is settled
 * in FP64, as in the path tracer's occlusion test.
 * With GYT_VOLUME_EQUI_ANGULAR, the estimator of equalAngular = true (the
 * reference constructor's default): every bounce draws one area light and
 * one point on it (AreaLight::SampleOnePoint); a ray in a medium samples its
 * scattering distance in [0, 3] along the ray with density proportional to
 * the inverse squared distance to that point
 * (HomogeneousMedium::EquiAngularSampling, volume/Homogeneous.cpp:38-64),
 * and a medium point gathers light only through the connection to that
 * point (ConnectToLight, VPT.cpp:108-146: phase function, transmittance of
 * the segment, cosine at the light over the squared distance and the area
 * pdf, no MIS weight); surface points gather as without the flag. Needs an
 * area light (GYT_ERR_UNSUPPORTED otherwise). The flag is accepted by the
 * three volumetric entry points only. */
#define GYT_VOLUME_EQUI_ANGULAR 2u
int32_t gyt_render_volume(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                          const GytRenderParams* params, float* rgb_out);
int32_t gyt_render_volume_device(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                 const GytRenderParams* params, double* d_film, GytRenderStats* stats);
/* VolPathTracing::Li for listed samples (xys: n triplets x, y, s): radiance
 * (n*3 floats) and the sampler dimensions each used (n). */
int32_t gyt_trace_volume_paths(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                               const GytRenderParams* params, uint64_t n, const uint32_t* xys, float* L_out,
                               uint32_t* cursor_out);

/* ---- Meshes from Wavefront OBJ files ---------------------------------------
 * Mesh::LoadFromFile (mesh/Mesh.cpp:7-90) with the reference's vendored
 * tinyobjloader (external/tinyobjloader, v2.0.0-rc) restated: its number
 * parsing, face-index rules (1-based, negative = relative) and polygon
 * triangulation (ear clipping). One record per triangle, three new vertices
 * each; normals from the file, else the face normal Cross(p1 - p0, p2 - p0)
 * normalised; reverse_vertices swaps the second and third vertex. Malformed
 * input (index 0, out-of-range indices, a face with normals on some of its
 * vertices only) fails with a message in err (err_len bytes, may be NULL).
 * Host only: no GPU needed. */
typedef struct gyt_mesh gyt_mesh;
int32_t gyt_mesh_load_obj(const char* path, int32_t reverse_vertices, gyt_mesh** out, char* err, uint32_t err_len);
int32_t gyt_mesh_size(const gyt_mesh* mesh, uint32_t* n_triangles);
/* positions and normals: n_triangles*9 floats (p0 p1 p2, n0 n1 n2), uvs:
 * n_triangles*6; any may be NULL. */
int32_t gyt_mesh_read(const gyt_mesh* mesh, float* positions, float* normals, float* uvs);
/* Scene::AddMesh's Triangle::SetTransform (visual/Scene.h:68-77,
 * shape/Triangle.h:78-88) on the GPU of ctx: positions by matrix (w-divide
 * unless w is 0 or 1), normals by the transpose of inverse, normalised; both
 * 4x4 row-major, as Transform holds them (math/Transform.h). The mesh keeps
 * the result. */
int32_t gyt_mesh_transform(gyt_context* ctx, gyt_mesh* mesh, const float* matrix, const float* inverse);
void gyt_mesh_destroy(gyt_mesh* mesh);

/* ---- Film output ----------------------------------------------------------
 * Film::SaveImage (visual/Film.cpp:6-9) on the GPU: colour / weight per pixel
 * (Film::WriteToPixelBuffer, visual/Film.h:128-136) and ImageIO::toInt
 * (image/ImageIO.cpp:66-68): int(pow(clamp(c, 0, 1), 1 / gamma) * 255 + 0.5)
 * per channel, in float as the reference. d_film: res_x*res_y*4 doubles on
 * the context's device (colour sums and weights, as gyt_render_device
 * accumulates them); rgb8_out: host, res_x*res_y*3 bytes, row 0 = the top
 * image row. Pixels of weight 0 give 0. */
int32_t gyt_film_quantize(gyt_context* ctx, const double* d_film, uint32_t res_x, uint32_t res_y, float gamma,
                          uint8_t* rgb8_out);

/* ImageIO::WriteImage (image/ImageIO.cpp:117-149) of a device film by the
 * file name's suffix: .png and .bmp with gyt_film_quantize's bytes at gamma
 * 2.2, .hdr as Radiance RGBE of colour / weight (the RGBE encoding on the
 * GPU). The containers are this library's own encoders (uncompressed PNG
 * deflate blocks, 24-bit BMP, run-length-layout HDR); decoded pixels equal
 * the reference's. */
int32_t gyt_film_save(gyt_context* ctx, const double* d_film, uint32_t res_x, uint32_t res_y, const char* path);

/* HaltonSampler::sample with Faure permutations (sampler/Halton.h:648-905)
 * for n (dimension, index) pairs; dimensions >= 256 give 0. */
int32_t gyt_halton(gyt_context* ctx, uint64_t n, const uint32_t* dims, const uint64_t* indices, float* out);

/* HaltonEnum::GetIndex (sampler/HaltonEnum.h) for n (s, x, y) triplets. */
int32_t gyt_halton_enum_index(gyt_context* ctx, uint32_t res_x, uint32_t res_y, uint64_t n,
                              const uint32_t* sxy, uint64_t* out);

/* ---- Differentiable rendering (path replay backpropagation) ---------------
 * Gradients of an image loss with respect to every material's albedo a
 * (mat_params[0..2]) and GGX roughness alpha (mat_params[6] = [7]) and every
 * emission row's radiance. The adjoint pass replays the primal's paths from
 * their Sobol' indices (nothing per vertex is stored; the primal keeps one
 * radiance value per path) with detached sampling: pdfs, MIS weights, light
 * selection and roulette are constants of the derivative. Albedo gradients
 * cover the diffuse and GGX-conductor lobes, alpha gradients the GGX lobe;
 * other lobes pass radiance through without parameter gradients. Gradient
 * sums are FP64. No counterpart in the reference (it has no derivatives). */

/* Replaces the scene's material parameters (n_materials x 16 floats, the
 * GytSceneDesc.mat_params layout; NULL keeps them) and emission rows
 * (n_emission x 3; NULL keeps them). The light-selection distribution is
 * rebuilt from the new powers unless flags holds GYT_KEEP_LIGHT_SAMPLING
 * (sampling then stays that of the previous emission: the estimator remains
 * unbiased and becomes linear in the emission, as a detached-sampling
 * derivative assumes). Material types and geometry are unchanged. */
#define GYT_KEEP_LIGHT_SAMPLING 1u
int32_t gyt_scene_set_materials(gyt_scene* scene, const float* mat_params, const float* emission, uint32_t flags);
/* Freezes BSDF sampling for difference checks: while set, gyt_render,
 * gyt_render_device, gyt_diff_forward and gyt_trace_paths sample BSDF
 * directions and evaluate every BSDF pdf (sample pdfs and MIS weights) with
 * mat_params (n_materials x 16 floats, the GytSceneDesc.mat_params layout),
 * while the BSDF values of the GGX lobes use the scene's current parameters.
 * Rendered with roulette off and the scene's parameters stepped about the
 * frozen ones, central differences of an image loss then equal the
 * detached-sampling derivative gyt_diff_backward computes (for the GGX alpha
 * as for the albedo). NULL ends it. The adjoint pass, batched renders, light
 * tracing, volumetric path tracing and gyt_render_device_noalloc refuse a
 * frozen scene (GYT_ERR_UNSUPPORTED). No counterpart in the reference. */
int32_t gyt_scene_freeze_sampling(gyt_scene* scene, const float* mat_params);
/* Primal render for differentiation: gyt_render_device into d_film plus the
 * radiance of every path (d_path_L: device, res_x*res_y*spp*3 floats,
 * indexed by path id = pixel * spp + sample). */
int32_t gyt_diff_forward(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                         const GytRenderParams* params, double* d_film, float* d_path_L, GytRenderStats* stats);
/* Adjoint of the image (colour / weight per pixel, as gyt_render returns it):
 * d_image_grad = dLoss/dImage (device, res_x*res_y*3 floats), d_film and
 * d_path_L from gyt_diff_forward with the same parameters. Adds dLoss/dparam
 * into d_grad_mat (device, n_materials*4 doubles: a.r, a.g, a.b, alpha) and
 * d_grad_em (device, n_emission*3 doubles). */
int32_t gyt_diff_backward(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                          const GytRenderParams* params, const float* d_image_grad, const double* d_film,
                          const float* d_path_L, double* d_grad_mat, double* d_grad_em, GytRenderStats* stats);
/* The adjoint of an explicit path list (host arrays): n (x, y, s) samples
 * with their adjoint weights delta (n*3: dLoss/d(path radiance)) and primal
 * radiance L_total (n*3, from gyt_trace_paths); grad_mat and grad_em (host)
 * receive the gradient sums. For parity tests against an FP64 adjoint. */
int32_t gyt_diff_backward_paths(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                const GytRenderParams* params, uint64_t n, const uint32_t* xys, const float* delta,
                                const float* L_total, double* grad_mat, double* grad_em);

/* ---- Batched renders ------------------------------------------------------
 * Many scenes and cameras of uneven sizes, resolutions and sample counts in
 * one wavefront: one path pool refilled across the instances (instance after
 * instance), each path carrying its instance, so the pool stays full until
 * the last instance's tail. Each instance's film receives exactly what
 * gyt_render_device would accumulate for it (the same paths; only the order
 * of the FP64 additions differs). All scenes of a batch must have the same
 * BVH width. No counterpart in the reference (its Integrator::Render takes
 * one scene and one camera, integrator/Integrator.h:17-27). */
typedef struct GytBatchConfig {
  uint32_t paths_in_flight;      /* path pool size; 0 keeps the context's */
  uint32_t stride_blocks_per_sm; /* blocks per SM of the refill, shade and finish kernels; 0 = 8 */
  uint32_t trace_blocks_per_sm;  /* blocks per SM of the extend and shadow traversals; 0 = occupancy limit */
  uint32_t use_graph;            /* 1: the render is one CUDA graph launch whose while-loop node runs
                                    the wavefront iterations on the device; 0: a host loop */
  uint32_t bvh_width;            /* set by gyt_batch_autotune: 2 or 8 */
} GytBatchConfig;
/* Configuration of later batched renders (NULL restores the defaults). */
int32_t gyt_context_set_batch_config(gyt_context* ctx, const GytBatchConfig* config);
int32_t gyt_context_get_batch_config(const gyt_context* ctx, GytBatchConfig* out);
/* Renders n instances: scenes[i] seen through cameras[i] with params[i],
 * accumulated into d_films[i] (device, res_x*res_y*4 doubles as in
 * gyt_render_device; not cleared). stats (may be NULL) covers the batch;
 * launches counts the kernels the batch ran, iterations the half-iterations
 * (pool swaps). GYT_ERR_WATCHDOG if the device loop hit its iteration bound. */
int32_t gyt_render_batch_device(gyt_context* ctx, uint32_t n, const gyt_scene* const* scenes,
                                const GytCamera* cameras, const GytRenderParams* params, double* const* d_films,
                                GytRenderStats* stats);
/* The same with host images: rgb_out[i] receives res_x*res_y*3 floats as
 * gyt_render writes them. Like gyt_render, the context keeps its FP64 film
 * and RGB staging buffers (grown to the largest call) until it is destroyed;
 * copies into page-locked rgb_out buffers run at full PCIe rate. */
int32_t gyt_render_batch(gyt_context* ctx, uint32_t n, const gyt_scene* const* scenes, const GytCamera* cameras,
                         const GytRenderParams* params, float* const* rgb_out);
/* Autotuner: times batched renders of the given instances with at most
 * sample_spp samples per pixel (0 = 1; each instance's spp scaled by
 * sample_spp / the batch's largest spp, at least 1, so that the sample keeps
 * the batch's mix of instances) over grid shapes and, when scenes_alt (the
 * same scenes built with the other BVH width) is given, the BVH width; the
 * pool sizes (2M to 32M paths in flight, those the sample can fill) on a
 * sample four times larger, since a short sample undervalues large pools.
 * Sets the fastest configuration on the context and returns it in *best
 * with its throughput on the base sample in *best_mpaths (Mpaths/s; may be
 * NULL). */
int32_t gyt_batch_autotune(gyt_context* ctx, uint32_t n, const gyt_scene* const* scenes,
                           const gyt_scene* const* scenes_alt, const GytCamera* cameras,
                           const GytRenderParams* params, uint32_t sample_spp, GytBatchConfig* best,
                           float* best_mpaths);

/* Render without allocating: the same render as gyt_render_device, for
 * callers that must not allocate GPU memory during the call (an engine that
 * owns all device memory through its own allocator or a fixed budget, or code
 * running where cudaMalloc is not allowed). The paths in flight, their queues
 * and the compaction counter live in a scratch array built into the library
 * (GYT_NOALLOC_MAX_PATHS path slots, about 10 MB, reserved on every device that
 * loads the library until the process exits) instead of the context's pools,
 * which are allocated on first use. paths_in_flight (1..GYT_NOALLOC_MAX_PATHS)
 * sets how many paths share it; larger values are rejected with
 * GYT_ERR_UNSUPPORTED, and so is a pool so small for the render that its
 * iteration bound passes 2^24 wavefront iterations (each waits for the GPU
 * once). The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls on a device share the array: calls whose GPU work
 * overlaps (other streams or threads) race on it. The scene, the Sobol' tables
 * of the context and the caller's device film (accumulated, not cleared) are
 * the inputs and output. No counterpart in the reference. */
#define GYT_NOALLOC_MAX_PATHS 32768u
int32_t gyt_render_device_noalloc(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                  const GytRenderParams* params, double* d_film, uint32_t paths_in_flight);

/* ProjectiveCamera::RasterToWorld (camera/Camera.cpp:38) as a row-major 4x4. */
int32_t gyt_camera_raster_to_world(const GytCamera* camera, double* out16);

#ifdef __cplusplus
}
#endif

#endif /* GYT_H */
