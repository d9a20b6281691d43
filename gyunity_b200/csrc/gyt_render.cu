// Wavefront path tracer for B200 (sm_100a) behind the C ABI of include/gyt.h.
//
// One render = a loop of wavefront iterations over a pool of paths in flight:
//   k_generate  new camera paths into free pool slots (Sobol' pixel sample,
//               pinhole ray)                       TiledIntegrator.cpp:40-45
//   k_extend    closest hit of every continuation ray (binary BVH, watertight
//               triangles, analytic spheres)       BVHAccel.cpp:401-445
//   k_shade     surface interaction, emission, light sample + BSDF sample of
//               the MIS next-event estimate (queued as shadow / MIS rays),
//               continuation BSDF sample, Russian roulette
//                                                  PT.cpp:16-65, Integrator.cpp:9-107
//   k_shadow    next-event shadow rays (any hit) from a compact queue
//                                                  Visibility.cpp:7-10
//   k_mis       BSDF-sampled MIS rays (closest hit) from a compact queue
//                                                  Integrator.cpp:86-101
//   k_finish    film accumulation of finished paths (FP64 atomics) and
//               compaction of live paths into the other pool (warp-aggregated
//               atomics)                           Film.h:61-87
// The three traversal kernels are persistent: lanes whose ray is done fetch
// the next queue entry before each traversal step (dynamic ray fetching), so
// warps stay full while rays of very different lengths are in flight.
// Path state is SoA in HBM; pools are ping-ponged each iteration so live
// paths stay dense and new paths fill the tail.
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gyt.h"
#include "../_gen/sobol_tables.h"
#include "gyt_bvh_gpu.h"
#include "gyt_bvh_host.h"
#include "gyt_device.cuh"
#include "gyt_image.h"
#include "gyt_obj.h"

namespace cg = cooperative_groups;
using namespace gyt;

// ----------------------------------------------------------- structures ---
namespace {

struct DevScene {
  const uint4* wnodes;        // 8-wide BVH, 5 uint4 per node (gyt_bvh_host.h), or null
  const float4* nodes;        // binary BVH, 4 float4 per node (gyt_bvh_host.h), or null
  const float4* tris;         // leaf order: (p0, original id), (p1, -), (p2, -)
  const float4* tnrm;         // leaf order: (n0, material), (n1, light index or -1), (n2, -)
  const float4* spheres;
  const uint32_t* sphere_mat;
  const float* mparams;
  const uint32_t* mtypes;
  const float4* ltab;         // kLightRec float4 per light (see light record below)
  const float* lcdf;          // n_lights + 1
  const float* lfunc;         // n_lights
  float lfunc_int;
  int n_lights, n_tris, n_spheres;
  int n_area;        // area lights come first; light n_area is the environment
  int has_env;
  EnvDev env;
  const float4* media;        // 2 float4 per medium: (sigma_a, g), (sigma_s, 0); or null
  int n_media;
  // BSDF sampling parameters (16 floats per material) while sampling is
  // frozen by gyt_scene_freeze_sampling; null otherwise
  const float* sparams;
};

// Light record (kLightRec float4): (p0, Le.r) (p1, Le.g) (p2, Le.b)
// (n0, area) (n1, leaf index) (n2, original id) (face normal, emission row).
constexpr int kLightRec = 7;

struct PathBuf {
  float4* o;      // origin
  float4* d;      // direction
  float4* tp;     // throughput
  float4* L;      // radiance so far
  unsigned long long* sidx;  // Sobol' index of the sample
  uint32_t* meta; // depth 0-7 | delta 8 | cursor 9-19 | alive 31
  uint32_t* pix;  // pixel index 0-27 | spill x 30 | spill y 31
  uint32_t* pid;  // path id within the render (debug outputs)
  uint32_t* inst; // instance of the path (batched renders)
};

// Compact ray queues filled by k_shade (positions from warp-aggregated
// atomics on counts[0] and counts[1]) and the closest hit of every path slot.
struct Queues {
  float4* so;  // shadow ray: origin, tmax
  float4* sd;  // shadow ray: direction, path slot bits
  float4* sc;  // shadow ray: contribution, bounce bits
  float4* mo;  // MIS ray: origin, bounce bits
  float4* md;  // MIS ray: direction, light index bits
  float4* mc;  // MIS ray: contribution, path slot bits
  float4* hit; // per path slot: t, b1, b2, prim bits
  uint32_t* counts;  // [0] shadow rays, [1] MIS rays, [2..4] fetch counters, [5] compaction
  float4* madd; // per path slot: its MIS ray's contribution (k_connect; added by k_finish)
  float4* sx;  // adjoint pass, shadow ray: material bits, d log f / d alpha, light bits, -
  float4* mx;  // adjoint pass, MIS ray: material bits, d log f / d alpha, -, -
};

// Adjoint (path replay) state per path slot, ping-ponged with the pool.
struct AdjBuf {
  float4* delta;  // dLoss / d(path radiance), RGB
  float4* Ltot;   // the path's radiance from the primal pass
  uint2* pend;    // the last continuation: material | kPendValid, d log f / d alpha bits
};

// Parameter gradients (FP64): per material (dL/da.r, dL/da.g, dL/da.b,
// dL/dalpha) and per emission row (dL/dLe.rgb).
struct GradOut {
  double* mat;
  double* em;
};
constexpr uint32_t kPendValid = 1u << 31;

struct Params {
  uint32_t spp, max_depth, rr_depth;
  uint32_t sampler;  // 0 Sobol', 1 Halton (GYT_SAMPLER_HALTON)
};

// Per-path replay record, indexed by path id (explicit path lists only).
// Bit i of a mask refers to bounce i (< 64): rr = a roulette number was
// drawn, occ = the shadow ray was occluded, mis = the MIS ray reached the
// sampled light.
struct DebugOut {
  float* L;
  uint32_t* cursor;
  unsigned long long* rr;
  unsigned long long* occ;
  unsigned long long* mis;
};

constexpr uint32_t kAlive = 1u << 31;
constexpr uint32_t kPixMask = 0x0fffffffu;
constexpr int kWStack = 48;  // node groups: one per level of the wide BVH
constexpr int kBStack = 64;  // binary BVH: one entry per level
constexpr int kBlock = 256;  // every kernel that traverses the BVH runs blocks of kBlock threads

// The primitive word of a closest-hit record (q.hit .w): -1 for a miss, the
// leaf-order triangle (< 2^28) or n_tris + sphere index; hits of the
// closest-hit kernels carry the triangle's shading class + 1 in bits 28-30
// (0: not recorded, as for spheres).
constexpr int kClsShift = 28;
GYT_D int hit_prim(int w) { return w < 0 ? w : (w & ((1 << kClsShift) - 1)); }
GYT_D uint32_t hit_cls(int w) { return w < 0 ? 0u : (uint32_t)w >> kClsShift; }

// Traversal stacks live in a per-warp slab of shared memory: each lane keeps
// its top kBStackSh binary entries (4 bytes) or kWStackSh wide node groups
// (8 bytes) there, deeper entries in a local-memory tail that only deep
// traversals reach. The slab is [warp][entry][lane]: entry k of lane l sits
// at word 32 k + l of the binary view (bank l) or at element 32 k + l of the
// 8-byte view, so a warp's pushes and pops never conflict in the binary view
// and take the two phases any 8-byte warp access takes in the wide one,
// whatever depth each lane is at. 32 bytes per lane: 8 KB per block of 256
// threads. Measured on 16 instances of the uneven batch against stacks in
// local memory: 8 entries +0.2% (both widths), 16 entries -0.5% (the larger
// slab takes L1 capacity from the node fetches); the 1.31M-triangle mesh +1%.
constexpr int kBStackSh = 8;
constexpr int kWStackSh = 4;
constexpr int kSlabWarps = kBlock / 32;
__shared__ uint2 g_trav_slab[kSlabWarps * kWStackSh * 32];

// Entry k of this lane's stack in the slab (binary and 8-byte views).
GYT_D uint32_t& slab_b(int k) {
  return reinterpret_cast<uint32_t*>(g_trav_slab)[(threadIdx.x >> 5) * (kBStackSh * 32) + k * 32 + (threadIdx.x & 31)];
}
GYT_D uint2& slab_w(int k) { return g_trav_slab[(threadIdx.x >> 5) * (kWStackSh * 32) + k * 32 + (threadIdx.x & 31)]; }
static_assert(kBStackSh * 4 == kWStackSh * 8, "both views cover the same slab");
// Traversal kernels are latency-bound (dependent node fetches): a register
// cap that fits four blocks per SM (a few spilled values) beats fewer blocks
// for the shadow/MIS kernels of both widths (measured on the procedural mesh
// and the uneven batch). The closest-hit kernels, whose lanes keep little
// state, run five (48 registers: 2% faster than four, a few spilled values).
template <int W>
constexpr int shadow_blocks_per_sm() { return 4; }
template <int W>
constexpr int extend_blocks_per_sm() { return 5; }
// The shade kernels, once their blocks are sorted by lobe type, are bound by
// latency at two blocks per SM (124 registers): a cap of 80 registers (three
// blocks, some spilled values) shades 11-13% faster on the procedural mesh
// and the uneven batch, and 64 registers (four blocks) another 3% (2% of the
// whole render on both). 128-thread blocks at the same occupancy were slower:
// the sort window is the block.
constexpr int kShadeBlocksPerSm = 4;

// meta bit 20: the bounce queued an MIS ray whose contribution k_finish adds
constexpr uint32_t kMisQueued = 1u << 20;

GYT_D uint32_t meta_pack(uint32_t depth, bool delta, uint32_t cursor, bool alive, bool mis_queued = false) {
  return (depth & 255u) | (delta ? 256u : 0u) | ((cursor & 2047u) << 9) | (alive ? kAlive : 0u) |
         (mis_queued ? kMisQueued : 0u);
}

// ------------------------------------------------------------ traversal ---
struct TraceCount {
  uint32_t nodes = 0, tris = 0;
};

// Per-ray constants shared by both traversals.
struct RayConst {
  WtRay wr;
  float ix, iy, iz;  // reciprocal direction (tiny components clamped to 2^-80)
};

struct Inst {
  DevScene s;
  Cam cam;
  Params prm;
  double* film;
  unsigned long long first;  // first global path index of the instance
};

// The instance table lives in constant memory: warps almost always hold paths
// of one instance (the pool is refilled instance after instance), so the
// per-path reads of scene fields are uniform constant-cache hits and the
// compiler can keep them out of the way of the kernels' global stores.
// Larger batches run as consecutive groups of kMaxBatch instances.
constexpr uint32_t kMaxBatch = 128;
__constant__ Inst c_insts[kMaxBatch];

// The geometry one ray of a batch is traced against: its instance, whose
// fields the traversal reads from the instance table when it needs them (a
// lane keeps one index instead of four pointers and two counts).
struct TraceGeo {
  uint32_t inst;
};
GYT_D const uint4* geo_wnodes(const DevScene& s) { return s.wnodes; }
GYT_D const float4* geo_nodes(const DevScene& s) { return s.nodes; }
GYT_D const float4* geo_tris(const DevScene& s) { return s.tris; }
GYT_D const float4* geo_spheres(const DevScene& s) { return s.spheres; }
GYT_D int geo_ntris(const DevScene& s) { return s.n_tris; }
GYT_D int geo_nspheres(const DevScene& s) { return s.n_spheres; }
GYT_D const uint4* geo_wnodes(const TraceGeo& g) { return c_insts[g.inst].s.wnodes; }
GYT_D const float4* geo_nodes(const TraceGeo& g) { return c_insts[g.inst].s.nodes; }
GYT_D const float4* geo_tris(const TraceGeo& g) { return c_insts[g.inst].s.tris; }
GYT_D const float4* geo_spheres(const TraceGeo& g) { return c_insts[g.inst].s.spheres; }
GYT_D int geo_ntris(const TraceGeo& g) { return c_insts[g.inst].s.n_tris; }
GYT_D int geo_nspheres(const TraceGeo& g) { return c_insts[g.inst].s.n_spheres; }

GYT_D RayConst ray_const(float3 o, float3 d) {
  RayConst c;
  c.wr = wt_setup(o, d);
  const float ooeps = 8.271806125530277e-25f;  // 2^-80
  c.ix = 1.f / (fabsf(d.x) > ooeps ? d.x : copysignf(ooeps, d.x));
  c.iy = 1.f / (fabsf(d.y) > ooeps ? d.y : copysignf(ooeps, d.y));
  c.iz = 1.f / (fabsf(d.z) > ooeps ? d.z : copysignf(ooeps, d.z));
  return c;
}

// Triangles [first, first + count) in leaf order against the ray. ANY stops
// at the first hit (returns true). CLS: the hit's shading class + 1 (the
// .w word of the triangle's second vertex) goes to bits 28-30 of prim.
template <bool ANY, bool COUNT, bool CLS = false, class S>
GYT_D bool test_tris(const S& s, const WtRay& wr, uint32_t first, uint32_t count, float& tmax, float& b1,
                     float& b2, int& prim, TraceCount* cnt) {
  if (COUNT) cnt->tris += count;
  for (uint32_t k = 0; k < count; ++k) {
    const float4* t = geo_tris(s) + 3 * (size_t)(first + k);
    float4 t0 = __ldg(t), t1 = __ldg(t + 1), t2 = __ldg(t + 2);
    float th, u, v;
    if (wt_intersect<ANY>(wr, f3(t0), f3(t1), f3(t2), tmax, &th, &u, &v)) {
      prim = CLS ? (int)((first + k) | (__float_as_uint(t1.w) << kClsShift)) : (int)(first + k);
      if (ANY) return true;
      tmax = th;
      b1 = u;
      b2 = v;
    }
  }
  return false;
}

// Binary BVH (two child boxes per 64-byte node, gyt_bvh_host.h). One step =
// the inner nodes down to the next leaf, then that leaf ("while-while"
// traversal): the lanes of a warp stay on inner nodes together and test
// their leaves together, instead of alternating between the two at every
// step. The stack holds one far child per level.
struct BinaryTraversal {
  int node, sp;
  int tail[kBStack - kBStackSh];  // entries past the lane's part of the shared slab

  GYT_D void init(const RayConst&) { node = 0; sp = 0; }
  GYT_D void push(int v) {
    if (sp < kBStackSh) slab_b(sp) = (uint32_t)v;
    else tail[sp - kBStackSh] = v;
    ++sp;
  }
  GYT_D int pop() {
    --sp;
    return sp < kBStackSh ? (int)slab_b(sp) : tail[sp - kBStackSh];
  }

  // Returns true when the traversal is finished (or, for ANY, on a hit).
  template <bool ANY, bool COUNT, bool CLS = false, class S>
  GYT_D bool step(const S& s, const RayConst& rc, float3 o, float& tmax, float& b1, float& b2, int& prim,
                  TraceCount* cnt) {
#pragma unroll 1
    while (node >= 0) {
      if (COUNT) cnt->nodes++;
      const float4* n = geo_nodes(s) + 4 * (size_t)node;
      float4 n0 = __ldg(n), n1 = __ldg(n + 1), n2 = __ldg(n + 2);
      int4 n3 = __ldg((const int4*)(n + 3));
      const float ox = o.x * rc.ix, oy = o.y * rc.iy, oz = o.z * rc.iz;
      float a0 = fmaf(n0.x, rc.ix, -ox), a1 = fmaf(n0.y, rc.ix, -ox);
      float a2 = fmaf(n0.z, rc.iy, -oy), a3 = fmaf(n0.w, rc.iy, -oy);
      float a4 = fmaf(n2.x, rc.iz, -oz), a5 = fmaf(n2.y, rc.iz, -oz);
      float c0 = fmaf(n1.x, rc.ix, -ox), c1 = fmaf(n1.y, rc.ix, -ox);
      float c2 = fmaf(n1.z, rc.iy, -oy), c3 = fmaf(n1.w, rc.iy, -oy);
      float c4 = fmaf(n2.z, rc.iz, -oz), c5 = fmaf(n2.w, rc.iz, -oz);
      float lo0 = fmaxf(fmaxf(fminf(a0, a1), fminf(a2, a3)), fmaxf(fminf(a4, a5), 0.f));
      float hi0 = fminf(fminf(fmaxf(a0, a1), fmaxf(a2, a3)), fminf(fmaxf(a4, a5), tmax));
      float lo1 = fmaxf(fmaxf(fminf(c0, c1), fminf(c2, c3)), fmaxf(fminf(c4, c5), 0.f));
      float hi1 = fminf(fminf(fmaxf(c0, c1), fmaxf(c2, c3)), fminf(fmaxf(c4, c5), tmax));
      bool h0 = lo0 <= hi0, h1 = lo1 <= hi1;
      if (!h0 && !h1) {
        if (sp == 0) return true;
        node = pop();
        continue;
      }
      if (h0 && h1) {
        int nearc = n3.x, farc = n3.y;
        if (lo1 < lo0) { nearc = n3.y; farc = n3.x; }
        push(farc);
        node = nearc;
      } else {
        node = h0 ? n3.x : n3.y;
      }
    }
    uint32_t code = ~(uint32_t)node;
    if (test_tris<ANY, COUNT, CLS>(s, rc.wr, code >> 3, (code & 7u) + 1u, tmax, b1, b2, prim, cnt)) return true;
    if (sp == 0) return true;
    node = pop();
    return false;
  }
};

// Byte k of w as a float: PRMT builds the bit pattern 2^23 + byte, the
// subtraction removes 2^23 (both exact).
GYT_D float qbyte(uint32_t w, int k) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440 + k)) - 8388608.f; }

// 8-wide BVH with quantized child boxes (gyt_bvh_host.h), traversed as in
// Ylitie, Karras and Laine, "Efficient Incoherent Ray Traversal on GPUs
// Through Compressed Wide BVHs" (HPG 2017). The builder puts the child whose
// centre lies towards octant s of the node in slot s (axis a positive when
// bit a of s is set); a ray whose direction has its negative axes in the bits
// of `oct` meets the children roughly in increasing order of slot ^ oct. One
// node group = the inner children of a node still to visit (bit slot ^ oct of
// the hit mask) and the node's first inner child index: 8 bytes on the stack,
// no per-node sort. A step tests the triangles of the last node's hit leaves,
// then fetches the nearest pending inner child and tests its eight boxes.
struct WideTraversal {
  uint2 grp;        // .x first inner child; .y hit mask (bits 0-7) | inner-slot mask (bits 8-15)
  uint32_t tri_base, tmask;  // the last node's hit leaf triangles (bit k = tri_base + k)
  uint32_t oct;
  int sp;
  uint2 tail[kWStack - kWStackSh];  // node groups past the lane's part of the shared slab

  GYT_D void push(uint2 v) {
    if (sp < kWStackSh) slab_w(sp) = v;
    else tail[sp - kWStackSh] = v;
    ++sp;
  }
  GYT_D uint2 pop() {
    --sp;
    return sp < kWStackSh ? slab_w(sp) : tail[sp - kWStackSh];
  }

  GYT_D void init(const RayConst& rc) {
    grp = make_uint2(0u, 1u);  // the root as the single pending child of a virtual group
    tri_base = tmask = 0u;
    oct = (rc.ix < 0.f ? 1u : 0u) | (rc.iy < 0.f ? 2u : 0u) | (rc.iz < 0.f ? 4u : 0u);
    sp = 0;
  }

  template <bool ANY, bool COUNT, bool CLS = false, class S>
  GYT_D bool step(const S& s, const RayConst& rc, float3 o, float& tmax, float& b1, float& b2, int& prim,
                  TraceCount* cnt) {
#pragma unroll 1
    while (tmask) {
      const uint32_t k = __ffs(tmask) - 1;
      tmask &= tmask - 1u;
      if (test_tris<ANY, COUNT, CLS>(s, rc.wr, tri_base + k, 1u, tmax, b1, b2, prim, cnt)) return true;
    }
    if ((grp.y & 0xffu) == 0u) {
      if (sp == 0) return true;
      grp = pop();
    }
    const uint32_t p = __ffs(grp.y & 0xffu) - 1;
    const uint32_t slot = p ^ oct;
    // the virtual root group holds node 0 with an empty inner-slot mask
    const uint32_t node = grp.x + __popc((grp.y >> 8) & ((1u << slot) - 1u));
    grp.y &= ~(1u << p);
    if (grp.y & 0xffu) push(grp);
    if (COUNT) cnt->nodes++;
    const uint4* n = geo_wnodes(s) + 5 * (size_t)node;
    const uint4 w0 = __ldg(n), w1 = __ldg(n + 1), w2 = __ldg(n + 2), w3 = __ldg(n + 3), w4 = __ldg(n + 4);
    const float sx = __int_as_float(((int)(int8_t)(w0.w & 0xffu) + 127) << 23);
    const float sy = __int_as_float(((int)(int8_t)((w0.w >> 8) & 0xffu) + 127) << 23);
    const float sz = __int_as_float(((int)(int8_t)((w0.w >> 16) & 0xffu) + 127) << 23);
    const uint32_t imask = w0.w >> 24;
    const float ax = sx * rc.ix, ay = sy * rc.iy, az = sz * rc.iz;
    const float bx = (__uint_as_float(w0.x) - o.x) * rc.ix, by = (__uint_as_float(w0.y) - o.y) * rc.iy,
                bz = (__uint_as_float(w0.z) - o.z) * rc.iz;
    // near and far planes per axis by the direction's sign (t is monotone in
    // the quantized coordinate, so this equals the min / max of the two)
    const bool fx = oct & 1u, fy = oct & 2u, fz = oct & 4u;
    const uint32_t nxa = fx ? w2.z : w2.x, nxb = fx ? w2.w : w2.y, fxa = fx ? w2.x : w2.z, fxb = fx ? w2.y : w2.w;
    const uint32_t nya = fy ? w3.z : w3.x, nyb = fy ? w3.w : w3.y, fya = fy ? w3.x : w3.z, fyb = fy ? w3.y : w3.w;
    const uint32_t nza = fz ? w4.z : w4.x, nzb = fz ? w4.w : w4.y, fza = fz ? w4.x : w4.z, fzb = fz ? w4.y : w4.w;
    uint32_t hits = 0u, tm = 0u;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int k = i & 3;
      const float tn = fmaxf(fmaxf(fmaf(qbyte(i < 4 ? nxa : nxb, k), ax, bx), fmaf(qbyte(i < 4 ? nya : nyb, k), ay, by)),
                             fmaxf(fmaf(qbyte(i < 4 ? nza : nzb, k), az, bz), 0.f));
      const float tf = fminf(fminf(fmaf(qbyte(i < 4 ? fxa : fxb, k), ax, bx), fmaf(qbyte(i < 4 ? fya : fyb, k), ay, by)),
                             fminf(fmaf(qbyte(i < 4 ? fza : fzb, k), az, bz), tmax));
      const uint32_t meta = ((i < 4 ? w1.z : w1.w) >> (8 * k)) & 0xffu;
      if (tn <= tf) {
        if ((imask >> i) & 1u) hits |= 1u << (i ^ oct);
        else if (meta) tm |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
      }
    }
    grp = make_uint2(w1.x, hits | (imask << 8));
    tri_base = w1.y;
    tmask = tm;
    return false;
  }
};

template <int W>
struct TraversalOf { using type = BinaryTraversal; };
template <>
struct TraversalOf<8> { using type = WideTraversal; };

// The analytic spheres after the BVH (linear; the configurations hold few).
template <bool ANY, class S>
GYT_D void trace_spheres(const S& s, float3 o, float3 d, float& tmax, int& prim) {
  const int ns = geo_nspheres(s);
  for (int k = 0; k < ns; ++k) {
    if (ANY && prim >= 0) return;
    float4 sp4 = __ldg(geo_spheres(s) + k);
    Ray r = sphere_object_ray(o, d, tmax, 0.f);
    float th;
    if (sphere_root(sp4, r, &th)) {
      prim = geo_ntris(s) + k;
      tmax = th;
    }
  }
}

// Closest hit (ANY = false) or occlusion (ANY = true) of one ray over the BVH
// (binary or 8-wide) and the spheres. Returns the triangle's leaf position
// (< n_tris; the original id is in tris[3k].w), n_tris + sphere index, or -1.
// tmax is updated to the hit distance; spheres report the distance along the
// re-made object ray of Sphere::Intersect (shape/Sphere.h:35).
template <int W, bool ANY, bool COUNT = false>
GYT_D int trace(const DevScene& s, float3 o, float3 d, float& tmax, float& b1, float& b2, TraceCount* cnt = nullptr) {
  int prim = -1;
  if (s.n_tris > 0) {
    RayConst rc = ray_const(o, d);
    typename TraversalOf<W>::type tv;
    tv.init(rc);
    while (!tv.template step<ANY, COUNT>(s, rc, o, tmax, b1, b2, prim, cnt)) {
    }
  }
  trace_spheres<ANY>(s, o, d, tmax, prim);
  return prim;
}

// Persistent traversal with dynamic ray fetching: every lane of a warp keeps
// a ray; lanes whose ray is finished take new ray indices before the next
// traversal step (one atomicAdd per warp), so warps stay full until the
// queue runs dry. (Reserving 64 indices per atomic and handing them out as
// lanes go idle was slower on the uneven batch: 365 against 373 Mpaths/s.)
// load(i, o, d, tmax) fetches ray i; done(i, prim, tmax, b1, b2) consumes
// its result.
//
// Traversal steps between two fetch checks of a persistent traversal kernel.
// 8-wide closest hit: 2 (4: 372.5, 1: 358 against 377.5 Mpaths/s on the
// uneven batch); 8-wide any hit: 4 (2 and 8 were slower).
template <int W, bool ANY>
__host__ __device__ constexpr int steps_per_fetch() { return W == 8 ? (ANY ? 4 : 2) : 2; }

// BATCH: every ray carries its own geometry (load fills the lane's TraceGeo);
// otherwise all rays use the scene s. CLS: triangle hits carry their shading
// class (test_tris).
template <int W, bool ANY, bool COUNT, bool BATCH = false, bool CLS = false, class Load, class Done>
GYT_D void persistent_trace(const DevScene& s, uint32_t* next, uint32_t n, Load load, Done done,
                            unsigned long long* counters) {
  const uint32_t lane = threadIdx.x & 31u;
  int ri = -1;  // -1 idle, -2 queue exhausted
  float3 o = mk(0.f, 0.f, 0.f), d = o;
  float tmax = 0.f, b1 = 0.f, b2 = 0.f;
  int prim = -1;
  RayConst rc;
  typename TraversalOf<W>::type tv;
  TraceCount cnt;
  TraceGeo lg{};  // the lane's geometry (BATCH)
  for (;;) {
    const uint32_t idle = __ballot_sync(0xffffffffu, ri == -1);
    if (idle) {
      const int leader = __ffs(idle) - 1;
      uint32_t base = 0;
      if ((int)lane == leader) base = atomicAdd(next, (uint32_t)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (ri == -1) {
        const uint32_t r = base + __popc(idle & ((1u << lane) - 1u));
        if (r < n) {
          ri = (int)r;
          load(r, o, d, tmax, lg);
          b1 = b2 = 0.f;
          prim = -1;
          rc = ray_const(o, d);
          tv.init(rc);
          if ((BATCH ? geo_ntris(lg) : s.n_tris) == 0) {
            if (BATCH) trace_spheres<ANY>(lg, o, d, tmax, prim);
            else trace_spheres<ANY>(s, o, d, tmax, prim);
            done((uint32_t)ri, prim, tmax, b1, b2);
            ri = -1;
          }
        } else {
          ri = -2;
        }
      }
    }
    if (__all_sync(0xffffffffu, ri == -2)) break;
    if (ri >= 0) {
      // a few steps per fetch check keep the ballot cost small (a binary step
      // already walks down to a leaf)
#pragma unroll 1
      for (int k = 0; k < steps_per_fetch<W, ANY>(); ++k) {
        const bool fin = BATCH ? tv.template step<ANY, COUNT, CLS>(lg, rc, o, tmax, b1, b2, prim, &cnt)
                               : tv.template step<ANY, COUNT, CLS>(s, rc, o, tmax, b1, b2, prim, &cnt);
        if (fin) {
          if ((BATCH ? geo_nspheres(lg) : s.n_spheres) > 0) {
            // the direction again from the ray's record (load only reads):
            // the traversal needs the origin and the ray constants, so the
            // lane does not keep the direction live through it
            float3 o2, d2;
            float t2;
            TraceGeo g2;
            load((uint32_t)ri, o2, d2, t2, g2);
            if (BATCH) trace_spheres<ANY>(lg, o, d2, tmax, prim);
            else trace_spheres<ANY>(s, o, d2, tmax, prim);
          }
          done((uint32_t)ri, prim, tmax, b1, b2);
          ri = -1;
          break;
        }
      }
    }
  }
  if (COUNT) {
    unsigned long long nodes = cnt.nodes, tris = cnt.tris;
    for (int off = 16; off > 0; off >>= 1) {
      nodes += __shfl_down_sync(0xffffffffu, nodes, off);
      tris += __shfl_down_sync(0xffffffffu, tris, off);
    }
    if (lane == 0) {
      atomicAdd(counters, nodes);
      atomicAdd(counters + 1, tris);
    }
  }
}

// Hit triangle k in leaf order: positions, shading normals, face normal
// (Triangle ctor, shape/Triangle.h:52), material and light index.
GYT_D void load_leaf_tri(const DevScene& s, int k, float3* p0, float3* p1, float3* p2, float3* n0, float3* n1,
                         float3* n2, float3* face, int* mat, int* light) {
  const float4* t = s.tris + 3 * k;
  const float4* n = s.tnrm + 3 * k;
  float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
  float4 na = __ldg(n), nb = __ldg(n + 1), nc = __ldg(n + 2);
  *p0 = f3(a); *p1 = f3(b); *p2 = f3(c);
  *n0 = f3(na); *n1 = f3(nb); *n2 = f3(nc);
  *face = norm(cross(*p1 - *p0, *p2 - *p0));
  *mat = __float_as_int(na.w);
  *light = __float_as_int(nb.w);
}

struct LightTri {
  float3 p0, p1, p2, n0, n1, n2, face, Le;
  float area;
};

GYT_D LightTri load_light(const DevScene& s, int li) {
  const float4* r = s.ltab + kLightRec * li;
  float4 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2), d = __ldg(r + 3), e = __ldg(r + 4), f = __ldg(r + 5),
         g = __ldg(r + 6);
  LightTri l;
  l.p0 = f3(a); l.p1 = f3(b); l.p2 = f3(c);
  l.Le = mk(a.w, b.w, c.w);
  l.n0 = f3(d); l.n1 = f3(e); l.n2 = f3(f);
  l.area = d.w;
  l.face = f3(g);
  return l;
}

// Distribution1D::SampleDiscrete over light powers (visual/Sampling.h:86-97,
// visual/Scene.h:97-109): upper_bound on the CDF.
GYT_D int sample_light(const DevScene& s, float u, float* pdf) {
  int lo = 0, hi = s.n_lights + 1;  // first index with cdf > u in [0, n+1)
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(s.lcdf + mid) > u) hi = mid; else lo = mid + 1;
  }
  int off = max(0, lo - 1);
  off = min(off, s.n_lights - 1);
  *pdf = __ldg(s.lfunc + off) / (s.lfunc_int * (float)s.n_lights);
  return off;
}

// Shape::Pdf for a triangle light (shape/Shape.h:34-47): re-intersect the
// light from the shading point along wi.
GYT_D float tri_light_pdf(const LightTri& l, const Hit& h, float3 o, float3 wi) {
  WtRay wr = wt_setup(o, wi);
  float th, b1, b2;
  if (!wt_intersect(wr, l.p0, l.p1, l.p2, __int_as_float(0x7f800000), &th, &b1, &b2)) return 0.f;
  Hit lp;
  tri_hit(l.p0, l.p1, l.p2, l.n0, l.n1, l.n2, l.face, b1, b2, o, wi, &lp);
  float3 dd = lp.pos - h.pos;
  float pdf = dot(dd, dd) / (fabsf(dot(lp.n, -wi)) * l.area);
  if (isinf(pdf)) return 0.f;
  return pdf;
}

// -------------------------------------------------------------- kernels ---
// Path p of a film (pixel after pixel, spp samples each): its pixel (x, y)
// and sample s. Integer divisions, 32-bit while p fits (every film of fewer
// than 2^32 samples), 64-bit beyond.
GYT_D void path_coords(unsigned long long p, uint32_t spp, uint32_t res_x, uint32_t* x, uint32_t* y, uint32_t* s) {
  if (p < (1ull << 32)) {
    const uint32_t q = (uint32_t)p;
    const uint32_t pixel = q / spp;
    *s = q - pixel * spp;
    *y = pixel / res_x;
    *x = pixel - *y * res_x;
  } else {
    const unsigned long long pixel = p / spp;
    *s = (uint32_t)(p - pixel * spp);
    *y = (uint32_t)(pixel / res_x);
    *x = (uint32_t)(pixel - (unsigned long long)*y * res_x);
  }
}

// Camera path of sample s in pixel (x, y) into slot k (TiledIntegrator::Render
// body, integrator/TiledIntegrator.cpp:37-48).
GYT_D void gen_path(PathBuf& dst, uint32_t k, uint32_t x, uint32_t y, uint32_t s, const Cam& cam, SamplerTables tab) {
  const bool halton = cam.sampler != 0;
  uint64_t idx = halton ? halton_enum_index(cam, s, x, y) : enum_index(tab, cam.log2_res, s, x, y);
  Rng rng{idx, 0};
  float su = rng.next(tab, cam.sampler), sv = rng.next(tab, cam.sampler);
  // SobolEnum::SampleX/Y (SobolEnum.h:30-36) or HaltonEnum::scale_x/y, kept
  // unfused as the reference
  float u = __fsub_rn(__fmul_rn(halton ? cam.h_sx : cam.res_pow2, su), (float)x);
  float v = __fsub_rn(__fmul_rn(halton ? cam.h_sy : cam.res_pow2, sv), (float)y);
  float3 o, d;
  camera_ray(cam, __fadd_rn((float)x, u), __fadd_rn((float)y, v), &o, &d);
  dst.o[k] = make_float4(o.x, o.y, o.z, 0.f);
  dst.d[k] = make_float4(d.x, d.y, d.z, 0.f);
  dst.tp[k] = make_float4(1.f, 1.f, 1.f, 0.f);
  dst.L[k] = make_float4(0.f, 0.f, 0.f, 0.f);
  dst.sidx[k] = idx;
  dst.meta[k] = meta_pack(0, false, rng.cursor, true);
  uint32_t pix = (y * cam.res_x + x) | ((u == 0.f && x > 0) ? (1u << 30) : 0u) | ((v == 0.f && y > 0) ? (1u << 31) : 0u);
  dst.pix[k] = pix;
}

__global__ void __launch_bounds__(kBlock) k_generate(PathBuf dst, uint32_t base, uint32_t n_new,
                                                     unsigned long long first, Cam cam, uint32_t spp,
                                                     const uint32_t* __restrict__ list, SamplerTables tab) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_new) return;
  unsigned long long p = first + j;
  uint32_t x, y, s;
  if (list) {
    x = __ldg(list + 3 * p);
    y = __ldg(list + 3 * p + 1);
    s = __ldg(list + 3 * p + 2);
  } else {
    path_coords(p, spp, cam.res_x, &x, &y, &s);
  }
  gen_path(dst, base + j, x, y, s, cam, tab);
  dst.pid[base + j] = (uint32_t)p;
}

template <int W, bool COUNT>
__global__ void __launch_bounds__(kBlock, extend_blocks_per_sm<W>())
    k_extend(PathBuf cur, uint32_t n, DevScene s, float4* __restrict__ hits, uint32_t* __restrict__ fetch,
             unsigned long long* counters) {
  persistent_trace<W, false, COUNT, false, true>(
      s, fetch, n,
      [&](uint32_t i, float3& o, float3& d, float& tmax, TraceGeo&) {
        o = f3(cur.o[i]);
        d = f3(cur.d[i]);
        tmax = __int_as_float(0x7f800000);
      },
      [&](uint32_t i, int prim, float tmax, float b1, float b2) {
        hits[i] = make_float4(tmax, b1, b2, __int_as_float(prim));
      },
      counters);
}

// Append to a compact queue: one atomicAdd per warp.
GYT_D uint32_t queue_slot(uint32_t* count) {
  cg::coalesced_group g = cg::coalesced_threads();
  uint32_t base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(count, g.size());
  return g.shfl(base, 0) + g.thread_rank();
}

// Gradient accumulation: lanes with the same key sum their values first
// (FP64), one atomic per key and warp.
GYT_D void grad_add(double* g, uint32_t key, int n, const double* v) {
  cg::coalesced_group act = cg::coalesced_threads();
  cg::coalesced_group grp = cg::labeled_partition(act, key);
  for (int k = 0; k < n; ++k) {
    const double r = cg::reduce(grp, v[k], cg::plus<double>());
    if (grp.thread_rank() == 0) atomicAdd(g + (size_t)key * n + k, r);
  }
}

// A contribution C (RGB) whose path carries the adjoint weight delta and
// whose BSDF factor belongs to material m (albedo a, d log f / d alpha = da):
// dL/da_c += delta_c C_c / a_c (f is linear in a for the diffuse and GGX
// lobes), dL/dalpha += sum_c delta_c C_c da.
GYT_D void grad_material(const GradOut& G, const DevScene& s, uint32_t m, float3 Cd, float da) {
  const uint32_t type = __ldg(s.mtypes + m);
  if (type != 0 && type != 3) return;
  const float* a = s.mparams + 16u * m;
  const float a0 = __ldg(a), a1 = __ldg(a + 1), a2 = __ldg(a + 2);
  double v[4];
  v[0] = a0 != 0.f ? (double)Cd.x / a0 : 0.0;
  v[1] = a1 != 0.f ? (double)Cd.y / a1 : 0.0;
  v[2] = a2 != 0.f ? (double)Cd.z / a2 : 0.0;
  v[3] = ((double)Cd.x + Cd.y + Cd.z) * da;
  grad_add(G.mat, m, 4, v);
}

// Contribution through area light li: dL/dLe_c += delta_c C_c / Le_c into its emission row.
GYT_D void grad_emitter(const GradOut& G, const DevScene& s, int li, float3 Cd) {
  const float4* r = s.ltab + kLightRec * li;
  const float l0 = __ldg(r).w, l1 = __ldg(r + 1).w, l2 = __ldg(r + 2).w;
  const uint32_t row = __float_as_uint(__ldg(r + 6).w);
  double v[3];
  v[0] = l0 != 0.f ? (double)Cd.x / l0 : 0.0;
  v[1] = l1 != 0.f ? (double)Cd.y / l1 : 0.0;
  v[2] = l2 != 0.f ? (double)Cd.z / l2 : 0.0;
  grad_add(G.em, row, 3, v);
}

// One bounce of path slot i (PathTracing::Li loop body, integrator/PT.cpp:14-63,
// with Integrator::DirectIllumination, integrator/Integrator.cpp:9-107): emission,
// light and BSDF samples queued as shadow and MIS rays, the continuation ray.
//
// ADJ (path replay backpropagation): the same bounce, replayed with the same
// samples, also moves gradient into G. Sampling decisions are detached: the
// BSDF and light sample pdfs, MIS weights, light selection and roulette
// probabilities are constants of the derivative, which is then an unbiased
// estimate of the gradient of the expected image. The radiance a BSDF factor
// f_k scales is known from the primal radiance: everything after vertex k's
// continuation is Ltot - (radiance gathered through vertex k), settled at the
// next bounce.
//
// DEFER: the MIS ray's contribution is added by k_finish (k_connect traces
// the shadow and MIS rays in one launch and leaves it in q.madd), not by the
// MIS kernel.
//
// FROZEN: BSDF sampling and the BSDF pdfs (sample pdfs and MIS weights) use
// the scene's frozen sampling parameters s.sparams, the BSDF values f of the
// GGX lobes the current parameters. With roulette off, the radiance is then a
// smooth function of the GGX alpha whose central differences equal the
// detached-sampling derivative of the adjoint pass.
//
// SAMPLER: 0 Sobol', 1 Halton, -1 prm.sampler at run time. A kernel compiled
// for one sampler keeps fewer registers live than one with both (-2.4% shade
// time on the uneven batch).
template <bool ADJ, bool DEFER = false, bool FROZEN = false, int SAMPLER = -1>
GYT_D void shade_path(const PathBuf& cur, uint32_t i, const DevScene& s, const Params& prm, const Queues& q,
                      SamplerTables tab, const DebugOut& dbg, const AdjBuf& A = AdjBuf{}, const GradOut& G = GradOut{}) {
  float4 h4 = q.hit[i];
  int prim = hit_prim(__float_as_int(h4.w));
  uint32_t meta = cur.meta[i];
  uint32_t depth = meta & 255u;
  bool delta = (meta >> 8) & 1u;
  Rng rng{cur.sidx[i], (meta >> 9) & 2047u};
  float3 ro = f3(cur.o[i]), rd = f3(cur.d[i]);
  float3 tp = f3(cur.tp[i]);
  // the path's radiance changes only on emission (a light or the environment
  // seen directly): added to the stored sum there, not carried through
  auto add_L = [&](float3 v) {
    const float3 L = f3(cur.L[i]) + v;
    cur.L[i] = make_float4(L.x, L.y, L.z, 0.f);
  };
  const uint32_t bounce = depth;
  bool alive = false;
  float3 adj = mk(0.f, 0.f, 0.f);
  uint2 pend_new = make_uint2(0u, 0u);
  bool mis_queued = false;
  if (ADJ) {
    adj = f3(A.delta[i]);
    const uint2 pend = A.pend[i];
    if (pend.x & kPendValid) {
      // the previous continuation's BSDF factor scales all radiance after it
      const float3 after = f3(A.Ltot[i]) - f3(cur.L[i]);
      grad_material(G, s, pend.x & ~kPendValid, adj * after, __uint_as_float(pend.y));
    }
  }
  if (prim < 0) {
    // PT.cpp:18-21: environment emission on the camera ray or after a delta bounce
    if ((depth == 0 || delta) && s.has_env) add_L(tp * env_lookup(s.env, rd));
  } else {
    Hit h;
    uint32_t mat;
    int light = -1;
    if (prim < s.n_tris) {
      float3 p0, p1, p2, n0, n1, n2, face;
      int m;
      load_leaf_tri(s, prim, &p0, &p1, &p2, &n0, &n1, &n2, &face, &m, &light);
      tri_hit(p0, p1, p2, n0, n1, n2, face, h4.y, h4.z, ro, rd, &h);
      mat = (uint32_t)m;
    } else {
      int k = prim - s.n_tris;
      Ray r = sphere_object_ray(ro, rd, __int_as_float(0x7f800000), 0.f);
      sphere_hit(__ldg(s.spheres + k), r, h4.x, &h);
      mat = __ldg(s.sphere_mat + k);
    }
    // the spawned rays' offset distance, once for the three rays of this bounce
    const float ofs_d = offset_dist(h.perr, h.abs_n);
    Bsdf bsdf;
    bsdf.lobe = load_lobe(s.mparams, s.mtypes, mat);
    bsdf.su = h.su; bsdf.sv = h.sv; bsdf.n = h.n; bsdf.gn = h.geo_n;
    // the BSDF that samples directions and gives their pdfs (bsdf itself
    // unless FROZEN)
    Bsdf fz;
    if (FROZEN) {
      fz = bsdf;
      fz.lobe = load_lobe(s.sparams, s.mtypes, mat);
    }
    const Bsdf& sbsdf = FROZEN ? fz : bsdf;
    // a sample's BSDF value at the current parameters (FROZEN, GGX lobes)
    auto refit = [&](float3 f, float3 wi_) {
      if (FROZEN && (bsdf.lobe.type == 3 || bsdf.lobe.type == 4) && !is_zero(f))
        return bsdf.lobe.eval(bsdf.local(h.wo), bsdf.local(wi_));
      return f;
    };
    // the ten dimensions this bounce can use: six for direct lighting (PT.cpp:38
    // arguments in GCC's right-to-left order: v.z v.y v.x u.y u.x uLight), three
    // for the BSDF sample (PT.cpp:47, again z y x) and one for roulette
    float u10[10];
    if (SAMPLER == 1 || (SAMPLER < 0 && prm.sampler)) halton10(tab, rng.index, rng.cursor, u10);
    else sobol10(tab.bits, rng.index, rng.cursor, u10);
    const bool emit = (depth == 0 || delta) && light >= 0;
    // the continuation's four dimensions (arguments again in right-to-left
    // order) wait in shared memory while direct lighting runs: four registers
    // fewer live across it in the 64-register build (blocks of kBlock threads)
    __shared__ float s_cont[4][kBlock];
    s_cont[0][threadIdx.x] = emit ? u10[0] : u10[6];
    s_cont[1][threadIdx.x] = emit ? u10[1] : u10[7];
    s_cont[2][threadIdx.x] = emit ? u10[2] : u10[8];
    s_cont[3][threadIdx.x] = emit ? u10[3] : u10[9];
    if (emit) {
      LightTri l = load_light(s, light);
      if (dot(h.n, h.wo) > 0.f) {
        add_L(tp * l.Le);  // AreaLight::Emission (AreaLight.h:40-43)
        if (ADJ) grad_emitter(G, s, light, adj * (tp * l.Le));
      }
    } else {
      float vz = u10[0], vy = u10[1], vx = u10[2];
      float uy = u10[3], ux = u10[4];
      float ul = u10[5];
      rng.cursor += 6;
      float lsel = 0.f;
      int li = s.n_lights > 0 ? sample_light(s, ul, &lsel) : 0;
      if (lsel > 0.f) {
        const bool env_light = li >= s.n_area;
        LightTri l;
        float3 wi, Li, lpos, lerr, labs;
        float pdf;
        if (!env_light) {
          // light sample: AreaLight::Sample_Li -> Shape::Sample -> Triangle::Sample
          l = load_light(s, li);
          float su0 = sqrtf(ux);
          float bb0 = 1.f - su0, bb1 = uy * su0, bb2 = 1.f - bb0 - bb1;
          lpos = l.p0 * bb0 + l.p1 * bb1 + l.p2 * bb2;
          float3 ln = l.n0 * bb0 + l.n1 * bb1 + l.n2 * bb2;
          lerr = (vabs(l.p0 * bb0) + vabs(l.p1 * bb1) + vabs(l.p2 * bb2)) * gammaf(6);
          labs = l.face;
          pdf = 1.f / l.area;
          float3 w = h.pos - lpos;
          if (length(w) == 0.f) {
            pdf = 0.f;
          } else {
            w = norm(w);
            pdf *= dot(h.pos - lpos, h.pos - lpos) / fabsf(dot(ln, -w));
            if (isinf(pdf)) pdf = 0.f;
          }
          wi = norm(lpos - h.pos);
          Li = dot(ln, -wi) > 0.f ? l.Le : mk(0.f, 0.f, 0.f);
        } else {
          // EnvironmentLight::Sample_Li (light/EnvLight.cpp:41-51): a point 2R away
          float3 sd;
          Li = env_sample(s.env, ux, uy, &sd, &pdf);
          wi = norm(sd);
          lpos = h.pos + wi * (2.f * s.env.radius);
          lerr = mk(0.f, 0.f, 0.f);
          labs = wi;
        }
        if (pdf > 0.f && !is_zero(Li)) {
          float spdf = sbsdf.pdf(h.wo, wi);
          float3 f = bsdf.eval(h.wo, wi);
          float cosT = fabsf(dot(h.n, wi));
          if (!is_zero(f)) {
            // Intersection::SpawnTo (Intersection.h:64-72)
            float3 org = offset_origin_d(h.pos, ofs_d, h.abs_n, lpos - h.pos);
            float3 tgt = offset_origin(lpos, lerr, labs, org - lpos);
            float3 dd = tgt - org;
            float dis = length(dd);
            dd = dd / dis;
            float3 so = org + dd * kRayEps;
            float w1 = power_heuristic(pdf, spdf);
            float3 c = tp * (Li * f * cosT / pdf) * w1 / lsel;
            const uint32_t j = queue_slot(q.counts);
            q.so[j] = make_float4(so.x, so.y, so.z, dis - kShadowEps);
            q.sd[j] = make_float4(dd.x, dd.y, dd.z, __uint_as_float(i));
            q.sc[j] = make_float4(c.x, c.y, c.z, __uint_as_float(bounce));
            if (ADJ)
              q.sx[j] = make_float4(__uint_as_float(mat), lobe_dlog_alpha(bsdf.lobe, bsdf.local(h.wo), bsdf.local(wi)),
                                    __int_as_float(li), 0.f);
          }
        }
        // BSDF-sampled half of the MIS estimate (Integrator.cpp:66-101)
        float3 wi2;
        float pdf2;
        float3 f2 = sbsdf.sample(h.wo, &wi2, &pdf2, vx, vy, vz);
        if (FROZEN) f2 = refit(f2, wi2);
        float cos2 = fabsf(dot(h.n, wi2));
        if (pdf2 != 0.f && !is_zero(f2)) {
          float3 o2 = offset_origin_d(h.pos, ofs_d, h.abs_n, wi2) + wi2 * kRayEps;  // SpawnRay
          // the light triangle again from the light table rather than kept live
          // across the BSDF evaluation and sampling
          float lpdf = env_light ? env_pdf_dir(s.env, wi2) : tri_light_pdf(load_light(s, li), h, o2, wi2);
          if (lpdf != 0.f) {
            float w2 = power_heuristic(pdf2, lpdf);
            float3 c = tp * (f2 * cos2 / pdf2) * w2 / lsel;
            const uint32_t j = queue_slot(q.counts + 1);
            q.mo[j] = make_float4(o2.x, o2.y, o2.z, __uint_as_float(bounce));
            q.md[j] = make_float4(wi2.x, wi2.y, wi2.z, __int_as_float(li));
            q.mc[j] = make_float4(c.x, c.y, c.z, __uint_as_float(i));
            mis_queued = true;
            if (ADJ)
              q.mx[j] = make_float4(__uint_as_float(mat), lobe_dlog_alpha(bsdf.lobe, bsdf.local(h.wo), bsdf.local(wi2)),
                                    0.f, 0.f);
          }
        }
      }
    }
    // continuation (PT.cpp:45-62)
    float rz = s_cont[0][threadIdx.x], ry = s_cont[1][threadIdx.x], rx = s_cont[2][threadIdx.x];
    const float urr = s_cont[3][threadIdx.x];
    rng.cursor += 3;
    float3 wi;
    float pdf;
    float3 f = sbsdf.sample(h.wo, &wi, &pdf, rx, ry, rz);
    if (FROZEN) f = refit(f, wi);
    if (!(is_zero(f) || pdf == 0.f)) {
      float3 est = f * fabsf(dot(h.n, wi)) / pdf;
      delta = bsdf.lobe.delta();
      float qv = lum(est * tp) / lum(tp);
      float p = qv < 1.f ? qv : 1.f;  // std::min(1, q): 1 when q is NaN
      bool survive = true;
      if (p < 1.f && depth > prm.rr_depth) {
        if (dbg.rr && depth < 64) dbg.rr[cur.pid[i]] |= 1ull << depth;
        rng.cursor += 1;
        if (urr < p) tp = tp / p;
        else survive = false;
      }
      if (survive) {
        tp = tp * est;
        float3 no = offset_origin_d(h.pos, ofs_d, h.abs_n, wi) + wi * kRayEps;
        cur.o[i] = make_float4(no.x, no.y, no.z, 0.f);
        cur.d[i] = make_float4(wi.x, wi.y, wi.z, 0.f);
        cur.tp[i] = make_float4(tp.x, tp.y, tp.z, 0.f);
        depth += 1;
        alive = depth < prm.max_depth;
        if (ADJ && alive)
          pend_new = make_uint2(mat | kPendValid,
                                __float_as_uint(lobe_dlog_alpha(bsdf.lobe, bsdf.local(h.wo), bsdf.local(wi))));
      }
    }
  }
  cur.meta[i] = meta_pack(depth, delta, rng.cursor, alive, DEFER && mis_queued);
  if (ADJ) A.pend[i] = pend_new;
}

// Shading classes: the lobe type of the surface hit (GYT_MAT_*), a miss, an
// idle thread past the live paths.
constexpr uint32_t kClassMiss = 5, kClassIdle = 6, kShadeClasses = 7;

GYT_D uint32_t shade_class(const DevScene& s, const Queues& q, uint32_t i) {
  const int prim = __float_as_int(q.hit[i].w);
  if (prim < 0) return kClassMiss;
  const uint32_t c = hit_cls(prim);
  if (c) return c - 1u;
  const uint32_t m = prim < s.n_tris ? (uint32_t)__float_as_int(__ldg(&s.tnrm[3 * prim].w))
                                     : __ldg(s.sphere_mat + (prim - s.n_tris));
  return min(__ldg(s.mtypes + m), 4u);
}

// Block-local counting sort of the block's path slots by shading class, so
// that a warp shades surfaces of one kind (one BSDF branch) instead of a mix.
// Returns the slot this thread shades, ~0u for none. Every thread of the
// block must call it.
GYT_D uint32_t coherent_slot(uint32_t i, uint32_t key) {
  __shared__ uint32_t cnt[kShadeClasses];
  __shared__ uint32_t order[kBlock];
  if (threadIdx.x < kShadeClasses) cnt[threadIdx.x] = 0u;
  __syncthreads();
  const uint32_t rank = atomicAdd(&cnt[key], 1u);
  __syncthreads();
  uint32_t base = 0;
  for (uint32_t c = 0; c < key; ++c) base += cnt[c];
  order[base + rank] = key == kClassIdle ? ~0u : i;
  __syncthreads();
  return order[threadIdx.x];
}

template <bool FROZEN, int SAMPLER>
__global__ void __launch_bounds__(kBlock, kShadeBlocksPerSm)
    k_shade(PathBuf cur, uint32_t n, DevScene s, Params prm, Queues q, SamplerTables tab, DebugOut dbg) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t j = coherent_slot(i, i < n ? shade_class(s, q, i) : kClassIdle);
  if (j != ~0u) shade_path<false, true, FROZEN, SAMPLER>(cur, j, s, prm, q, tab, dbg);
}

// MIS-ray result of one queue entry (every MIS kernel). DEFER: the
// contribution (zero when the light is missed) goes to the path's q.madd slot
// for k_finish instead of into its radiance.
template <bool ADJ = false, bool DEFER = false>
GYT_D void mis_done(const PathBuf& cur, const Queues& q, const DevScene& s, uint32_t j, int prim, float b1, float b2,
                    const DebugOut& dbg, const AdjBuf& A = AdjBuf{}, const GradOut& G = GradOut{}) {
  const float4 md = q.md[j], mc = q.mc[j];
  const int li = __float_as_int(md.w);
  const uint32_t slot = __float_as_uint(mc.w);
  const float3 wi = f3(md);
  bool reach = false;
  float3 add = mk(0.f, 0.f, 0.f);
  if (prim < 0 && li >= s.n_area) {
    add = f3(mc) * env_lookup(s.env, wi);  // Integrator.cpp:97-99
    reach = true;
  } else if (prim >= 0 && prim < s.n_tris && __float_as_int(__ldg(s.tnrm + 3 * prim + 1).w) == li) {
    float3 n0 = f3(__ldg(s.tnrm + 3 * prim)), n1 = f3(__ldg(s.tnrm + 3 * prim + 1));
    float3 n2 = f3(__ldg(s.tnrm + 3 * prim + 2));
    float b0 = 1.f - b1 - b2;
    float3 ns = norm(n0 * b0 + n1 * b1 + n2 * b2);
    if (dot(ns, -wi) > 0.f) {
      const float4* r = s.ltab + kLightRec * li;
      add = f3(mc) * mk(__ldg(r).w, __ldg(r + 1).w, __ldg(r + 2).w);
    }
    reach = true;
  }
  if (DEFER) q.madd[slot] = make_float4(add.x, add.y, add.z, 0.f);
  if (reach) {
    if (!DEFER) {
      float4 l = cur.L[slot];
      cur.L[slot] = make_float4(l.x + add.x, l.y + add.y, l.z + add.z, 0.f);
    }
    if (ADJ) {
      const float3 Cd = f3(A.delta[slot]) * add;
      const float4 x = q.mx[j];
      grad_material(G, s, __float_as_uint(x.x), Cd, x.y);
      if (li < s.n_area) grad_emitter(G, s, li, Cd);
    }
    if (dbg.mis) {
      const uint32_t b = __float_as_uint(q.mo[j].w);
      if (b < 64) dbg.mis[cur.pid[slot]] |= 1ull << b;
    }
  }
}

// The rays k_shade queued, in one persistent launch: first the next-event
// shadow rays (any hit; an unoccluded ray adds its contribution to its path's
// radiance, VisibilityTester::Unoccluded, Visibility.cpp:7-10), then the
// BSDF-sampled MIS rays (closest hit; the sampled light's emission where the
// ray reaches it, Integrator.cpp:86-101). The MIS rays are few: traced in the
// same launch they fill the shadow rays' tail instead of paying a launch of
// their own. Their contribution goes to q.madd (k_finish adds it), since the
// path's radiance may still be in use by a shadow ray of another warp.
// counters: node and triangle counts of the shadow rays, then of the MIS rays.
template <int W, bool COUNT>
__global__ void __launch_bounds__(kBlock, shadow_blocks_per_sm<W>()) k_connect(PathBuf cur, DevScene s, Queues q,
                                                                                DebugOut dbg,
                                                                                unsigned long long* counters) {
  const uint32_t ns = *(volatile uint32_t*)q.counts;
  persistent_trace<W, true, COUNT>(
      s, q.counts + 3, ns,
      [&](uint32_t j, float3& o, float3& d, float& tmax, TraceGeo&) {
        float4 a = q.so[j], b = q.sd[j];
        o = f3(a);
        d = f3(b);
        tmax = a.w;
      },
      [&](uint32_t j, int prim, float, float, float) {
        const uint32_t slot = __float_as_uint(q.sd[j].w);
        if (prim < 0) {
          float4 c = q.sc[j], l = cur.L[slot];
          cur.L[slot] = make_float4(l.x + c.x, l.y + c.y, l.z + c.z, 0.f);
        } else if (dbg.occ) {
          const uint32_t b = __float_as_uint(q.sc[j].w);
          if (b < 64) dbg.occ[cur.pid[slot]] |= 1ull << b;
        }
      },
      counters);
  const uint32_t nm = *(volatile uint32_t*)(q.counts + 1);
  persistent_trace<W, false, COUNT>(
      s, q.counts + 4, nm,
      [&](uint32_t j, float3& o, float3& d, float& tmax, TraceGeo&) {
        o = f3(q.mo[j]);
        d = f3(q.md[j]);
        tmax = __int_as_float(0x7f800000);
      },
      [&](uint32_t j, int prim, float, float b1, float b2) {
        mis_done<false, true>(cur, q, s, j, prim, b1, b2, dbg);
      },
      COUNT ? counters + 2 : nullptr);
}

// Stream compaction at block granularity: the position in the next pool of
// this thread's live path, in thread order within the block, with one atomic
// per block on the shared counter (a warp-granular atomic puts 16K+ requests
// per launch on that one address). Every thread of the block calls it.
GYT_D uint32_t block_compact(bool live, uint32_t* __restrict__ counter) {
  __shared__ uint32_t warp_base[kBlock / 32];
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t ball = __ballot_sync(0xffffffffu, live);
  if (lane == 0) warp_base[w] = __popc(ball);
  __syncthreads();
  if (w == 0) {
    const uint32_t c = lane < kBlock / 32 ? warp_base[lane] : 0u;
    uint32_t inc = c;
#pragma unroll
    for (int o = 1; o < kBlock / 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= (uint32_t)o) inc += t;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, inc, kBlock / 32 - 1);
    uint32_t base = 0;
    if (lane == 0 && total) base = atomicAdd(counter, total);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (lane < kBlock / 32) warp_base[lane] = base + inc - c;
  }
  __syncthreads();
  return warp_base[w] + __popc(ball & ((1u << lane) - 1u));
}

GYT_D void film_add(double* film, uint32_t w, uint32_t x, uint32_t y, float3 L) {
  double* p = film + 4ull * ((unsigned long long)y * w + x);
  atomicAdd(p, (double)L.x);
  atomicAdd(p + 1, (double)L.y);
  atomicAdd(p + 2, (double)L.z);
  atomicAdd(p + 3, 1.0);
}

// Finished paths go to the film (FP64 atomics, Film::AddSample with the box
// filter, visual/Film.h:61-87); live paths are compacted into the next pool.
__global__ void __launch_bounds__(kBlock) k_finish(PathBuf cur, PathBuf nxt, uint32_t n, double* __restrict__ film,
                                                   uint32_t res_x, uint32_t* __restrict__ counter,
                                                   const float4* __restrict__ madd, DebugOut dbg) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x * blockDim.x >= n) return;  // the whole block is idle
  uint32_t meta = i < n ? cur.meta[i] : 0u;
  float4 L4 = i < n ? cur.L[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  if (meta & kMisQueued) {  // the MIS contribution of this bounce (k_connect)
    const float4 m = madd[i];
    L4 = make_float4(L4.x + m.x, L4.y + m.y, L4.z + m.z, 0.f);
    meta &= ~kMisQueued;
  }
  const uint32_t j = block_compact(meta & kAlive, counter);
  if (i >= n) return;
  if (meta & kAlive) {
    nxt.o[j] = cur.o[i];
    nxt.d[j] = cur.d[i];
    nxt.tp[j] = cur.tp[i];
    nxt.L[j] = L4;
    nxt.sidx[j] = cur.sidx[i];
    nxt.meta[j] = meta;
    nxt.pix[j] = cur.pix[i];
    nxt.pid[j] = cur.pid[i];
  } else {
    const float3 L = f3(L4);
    uint32_t pix = cur.pix[i];
    if (film) {
      uint32_t p = pix & kPixMask;
      uint32_t y = p / res_x, x = p - y * res_x;
      film_add(film, res_x, x, y, L);
      if (pix & (1u << 30)) film_add(film, res_x, x - 1, y, L);
      if (pix & (1u << 31)) film_add(film, res_x, x, y - 1, L);
      if ((pix & (1u << 30)) && (pix & (1u << 31))) film_add(film, res_x, x - 1, y - 1, L);
    }
    uint32_t pid = cur.pid[i];
    if (dbg.L) {
      dbg.L[3ull * pid] = L.x;
      dbg.L[3ull * pid + 1] = L.y;
      dbg.L[3ull * pid + 2] = L.z;
    }
    if (dbg.cursor) dbg.cursor[pid] = (meta >> 9) & 2047u;
  }
}

// ------------------------------------------------------- adjoint pass ---
// Inputs of the path replay: the image gradient and the primal film (its
// per-pixel weights) for full renders, or per-path adjoint weights for an
// explicit path list; the primal radiance of every path.
struct AdjIn {
  const float* img_grad;    // dLoss/dImage, res_x * res_y * 3 (full renders)
  const double* film;       // the primal film, res_x * res_y * 4 (weights in .w)
  const float* path_delta;  // per path id, 3 floats (explicit lists)
  const float* path_L;      // per path id, 3 floats: the primal radiance
};

__global__ void __launch_bounds__(kBlock) k_generate_adj(PathBuf dst, AdjBuf A, uint32_t base, uint32_t n_new,
                                                         unsigned long long first, Cam cam, uint32_t spp,
                                                         const uint32_t* __restrict__ list, SamplerTables tab,
                                                         AdjIn in) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_new) return;
  const unsigned long long p = first + j;
  uint32_t x, y, s;
  if (list) {
    x = __ldg(list + 3 * p);
    y = __ldg(list + 3 * p + 1);
    s = __ldg(list + 3 * p + 2);
  } else {
    path_coords(p, spp, cam.res_x, &x, &y, &s);
  }
  const uint32_t k = base + j;
  gen_path(dst, k, x, y, s, cam, tab);
  dst.pid[k] = (uint32_t)p;
  float3 d = mk(0.f, 0.f, 0.f);
  if (in.path_delta) {
    d = mk(in.path_delta[3 * p], in.path_delta[3 * p + 1], in.path_delta[3 * p + 2]);
  } else {
    // the pixels the sample reaches (Film::AddSample's box filter, as
    // k_finish splats it), each image value = colour / weight
    const uint32_t pix = dst.pix[k];
    const uint32_t q = pix & kPixMask;
    const uint32_t py = q / cam.res_x, px = q - py * cam.res_x;
    auto add = [&](uint32_t xx, uint32_t yy) {
      const size_t o = (size_t)yy * cam.res_x + xx;
      const double w = in.film[4 * o + 3];
      if (w > 0.0) {
        const float iw = (float)(1.0 / w);
        d = d + mk(in.img_grad[3 * o], in.img_grad[3 * o + 1], in.img_grad[3 * o + 2]) * iw;
      }
    };
    add(px, py);
    if (pix & (1u << 30)) add(px - 1, py);
    if (pix & (1u << 31)) add(px, py - 1);
    if ((pix & (1u << 30)) && (pix & (1u << 31))) add(px - 1, py - 1);
  }
  A.delta[k] = make_float4(d.x, d.y, d.z, 0.f);
  A.Ltot[k] = make_float4(in.path_L[3 * p], in.path_L[3 * p + 1], in.path_L[3 * p + 2], 0.f);
  A.pend[k] = make_uint2(0u, 0u);
}

__global__ void __launch_bounds__(kBlock) k_shade_adj(PathBuf cur, AdjBuf A, uint32_t n, DevScene s, Params prm,
                                                      Queues q, SamplerTables tab, GradOut G) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  shade_path<true>(cur, i, s, prm, q, tab, DebugOut{}, A, G);
}

template <int W>
__global__ void __launch_bounds__(kBlock, shadow_blocks_per_sm<W>()) k_shadow_adj(PathBuf cur, AdjBuf A, DevScene s, Queues q, GradOut G) {
  const uint32_t n = *(volatile uint32_t*)q.counts;
  persistent_trace<W, true, false>(
      s, q.counts + 3, n,
      [&](uint32_t j, float3& o, float3& d, float& tmax, TraceGeo&) {
        const float4 a = q.so[j], b = q.sd[j];
        o = f3(a);
        d = f3(b);
        tmax = a.w;
      },
      [&](uint32_t j, int prim, float, float, float) {
        if (prim >= 0) return;
        const uint32_t slot = __float_as_uint(q.sd[j].w);
        const float4 c = q.sc[j], l = cur.L[slot];
        cur.L[slot] = make_float4(l.x + c.x, l.y + c.y, l.z + c.z, 0.f);
        const float3 Cd = f3(A.delta[slot]) * f3(c);
        const float4 x = q.sx[j];
        grad_material(G, s, __float_as_uint(x.x), Cd, x.y);
        const int li = __float_as_int(x.z);
        if (li < s.n_area) grad_emitter(G, s, li, Cd);
      },
      nullptr);
}

template <int W>
__global__ void __launch_bounds__(kBlock) k_mis_adj(PathBuf cur, AdjBuf A, DevScene s, Queues q, GradOut G) {
  const uint32_t n = *(volatile uint32_t*)(q.counts + 1);
  persistent_trace<W, false, false>(
      s, q.counts + 4, n,
      [&](uint32_t j, float3& o, float3& d, float& tmax, TraceGeo&) {
        o = f3(q.mo[j]);
        d = f3(q.md[j]);
        tmax = __int_as_float(0x7f800000);
      },
      [&](uint32_t j, int prim, float, float b1, float b2) {
        mis_done<true>(cur, q, s, j, prim, b1, b2, DebugOut{}, A, G);
      },
      nullptr);
}

// Live paths (and their adjoint state) compacted; finished paths are done
// (their gradient was moved at their last bounce).
__global__ void __launch_bounds__(kBlock) k_finish_adj(PathBuf cur, PathBuf nxt, AdjBuf A, AdjBuf AN, uint32_t n,
                                                       uint32_t* __restrict__ counter) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x * blockDim.x >= n) return;  // the whole block is idle
  const uint32_t meta = i < n ? cur.meta[i] : 0u;
  const uint32_t j = block_compact(meta & kAlive, counter);
  if (!(meta & kAlive)) return;
  nxt.o[j] = cur.o[i];
  nxt.d[j] = cur.d[i];
  nxt.tp[j] = cur.tp[i];
  nxt.L[j] = cur.L[i];
  nxt.sidx[j] = cur.sidx[i];
  nxt.meta[j] = meta;
  nxt.pix[j] = cur.pix[i];
  nxt.pid[j] = cur.pid[i];
  AN.delta[j] = A.delta[i];
  AN.Ltot[j] = A.Ltot[i];
  AN.pend[j] = A.pend[i];
}

// ------------------------------------------------------ batched renders ---
// Many scenes, cameras and sample counts in one wavefront: the path pool is
// refilled from the concatenation of all instances' paths (instance-major),
// every path slot carries its instance, and each kernel reads the scene,
// camera, parameters and film of the instance it works on.


// Device-side loop state of a batched render (one half-iteration moves the
// pool from one buffer to the other).
struct IterState {
  unsigned long long generated, total;
  uint32_t active;    // live paths at the start of a half-iteration
  uint32_t n_new;     // paths generated in it
  uint32_t n;         // active + n_new
  uint32_t iter;      // half-iterations run
  uint32_t max_iter;  // watchdog
  uint32_t watchdog;  // set when max_iter stopped the loop
  uint32_t n_inst, capacity;
};

__global__ void k_batch_begin(IterState* __restrict__ st, uint32_t* __restrict__ counts) {
  if (threadIdx.x == 0) {
    const unsigned long long rem = st->total - st->generated;
    const uint32_t room = st->capacity - st->active;
    const uint32_t n_new = (uint32_t)(rem < room ? rem : room);
    st->n_new = n_new;
    st->n = st->active + n_new;
  }
  if (threadIdx.x < 8) counts[threadIdx.x] = 0;
}

__global__ void __launch_bounds__(kBlock) k_generate_batch(PathBuf dst, const IterState* __restrict__ st,
                                                           SamplerTables tab) {
  const uint32_t n_new = st->n_new, base = st->active, ni = st->n_inst;
  const unsigned long long first = st->generated;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n_new; j += gridDim.x * blockDim.x) {
    const unsigned long long g = first + j;
    // last instance whose first path is <= g
    uint32_t lo = 0, hi = ni;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (c_insts[mid].first <= g) lo = mid; else hi = mid;
    }
    const Inst& I = c_insts[lo];
    uint32_t x, y, s;
    path_coords(g - I.first, I.prm.spp, I.cam.res_x, &x, &y, &s);
    const Cam cam = I.cam;
    gen_path(dst, base + j, x, y, s, cam, tab);
    dst.inst[base + j] = lo;
  }
}



template <int W>
__global__ void __launch_bounds__(kBlock, extend_blocks_per_sm<W>())
    k_extend_batch(PathBuf cur, const IterState* __restrict__ st, float4* __restrict__ hits,
                   uint32_t* __restrict__ fetch) {
  const uint32_t n = st->n;
  persistent_trace<W, false, false, true, true>(
      c_insts[0].s, fetch, n,
      [&](uint32_t i, float3& o, float3& d, float& tmax, TraceGeo& g) {
        o = f3(cur.o[i]);
        d = f3(cur.d[i]);
        tmax = __int_as_float(0x7f800000);
        g.inst = cur.inst[i];
      },
      [&](uint32_t i, int prim, float tmax, float b1, float b2) {
        hits[i] = make_float4(tmax, b1, b2, __int_as_float(prim));
      },
      nullptr);
}

// One path per thread over a grid sized for the whole pool (threads past
// the live count return at once): the work per path varies a lot, and the
// block scheduler balances it far better than a grid-stride loop does.
template <int SAMPLER>
__global__ void __launch_bounds__(kBlock, kShadeBlocksPerSm)
    k_shade_batch(PathBuf cur, const IterState* __restrict__ st, Queues q, SamplerTables tab) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = st->n;
  if (blockIdx.x * blockDim.x >= n) return;  // the whole block is idle
  const uint32_t j = coherent_slot(i, i < n ? shade_class(c_insts[cur.inst[i]].s, q, i) : kClassIdle);
  if (j == ~0u) return;
  const Inst& I = c_insts[cur.inst[j]];
  shade_path<false, true, false, SAMPLER>(cur, j, I.s, I.prm, q, tab, DebugOut{});
}

// Shadow then MIS rays of the batch in one launch (k_connect, every ray with
// its instance's geometry).
template <int W>
__global__ void __launch_bounds__(kBlock, shadow_blocks_per_sm<W>()) k_connect_batch(PathBuf cur, Queues q) {
  const uint32_t ns = *(volatile uint32_t*)q.counts;
  persistent_trace<W, true, false, true>(
      c_insts[0].s, q.counts + 3, ns,
      [&](uint32_t j, float3& o, float3& d, float& tmax, TraceGeo& g) {
        const float4 a = q.so[j], b = q.sd[j];
        o = f3(a);
        d = f3(b);
        tmax = a.w;
        g.inst = cur.inst[__float_as_uint(b.w)];
      },
      [&](uint32_t j, int prim, float, float, float) {
        if (prim < 0) {
          const uint32_t slot = __float_as_uint(q.sd[j].w);
          const float4 c = q.sc[j], l = cur.L[slot];
          cur.L[slot] = make_float4(l.x + c.x, l.y + c.y, l.z + c.z, 0.f);
        }
      },
      nullptr);
  const uint32_t nm = *(volatile uint32_t*)(q.counts + 1);
  persistent_trace<W, false, false, true>(
      c_insts[0].s, q.counts + 4, nm,
      [&](uint32_t j, float3& o, float3& d, float& tmax, TraceGeo& g) {
        o = f3(q.mo[j]);
        d = f3(q.md[j]);
        tmax = __int_as_float(0x7f800000);
        g.inst = cur.inst[__float_as_uint(q.mc[j].w)];
      },
      [&](uint32_t j, int prim, float, float b1, float b2) {
        const uint32_t slot = __float_as_uint(q.mc[j].w);
        mis_done<false, true>(cur, q, c_insts[cur.inst[slot]].s, j, prim, b1, b2, DebugOut{});
      },
      nullptr);
}

// Finished paths to their instance's film, live paths compacted.
__global__ void __launch_bounds__(kBlock) k_finish_batch(PathBuf cur, PathBuf nxt, const IterState* __restrict__ st,
                                                         uint32_t* __restrict__ counter,
                                                         const float4* __restrict__ madd) {
  // one path per thread over a grid sized for the pool, every field loaded
  // before the branch (more loads in flight than a grid-stride loop that
  // loads after testing the path: 14% faster on the uneven batch); batched
  // renders keep no path ids
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = st->n;
  if (blockIdx.x * blockDim.x >= n) return;  // the whole block is idle
  const bool in = i < n;
  uint32_t meta = in ? cur.meta[i] : 0u;
  float4 L4 = in ? cur.L[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  uint32_t pix = 0, inst = 0;
  float4 o = L4, d = L4, tp = L4;
  unsigned long long sidx = 0;
  if (in) {
    pix = cur.pix[i];
    inst = cur.inst[i];
    o = cur.o[i];
    d = cur.d[i];
    tp = cur.tp[i];
    sidx = cur.sidx[i];
  }
  if (meta & kMisQueued) {  // the MIS contribution of this bounce (k_connect_batch)
    const float4 m = madd[i];
    L4 = make_float4(L4.x + m.x, L4.y + m.y, L4.z + m.z, 0.f);
    meta &= ~kMisQueued;
  }
  const uint32_t j = block_compact(meta & kAlive, counter);
  if (!in) return;
  if (meta & kAlive) {
    nxt.o[j] = o;
    nxt.d[j] = d;
    nxt.tp[j] = tp;
    nxt.L[j] = L4;
    nxt.sidx[j] = sidx;
    nxt.meta[j] = meta;
    nxt.pix[j] = pix;
    nxt.inst[j] = inst;
  } else {
    const Inst& I = c_insts[inst];
    const float3 L = f3(L4);
    const uint32_t res_x = I.cam.res_x;
    double* film = I.film;
    const uint32_t p = pix & kPixMask;
    const uint32_t y = p / res_x, x = p - y * res_x;
    film_add(film, res_x, x, y, L);
    if (pix & (1u << 30)) film_add(film, res_x, x - 1, y, L);
    if (pix & (1u << 31)) film_add(film, res_x, x, y - 1, L);
    if ((pix & (1u << 30)) && (pix & (1u << 31))) film_add(film, res_x, x - 1, y - 1, L);
  }
}

// Closes a half-iteration: live count, refill progress, and the loop
// condition of the enclosing graph (while more paths remain, bounded by the
// watchdog).
__global__ void k_batch_end(IterState* __restrict__ st, const uint32_t* __restrict__ counts,
                            cudaGraphConditionalHandle cond, int in_graph) {
  if (threadIdx.x != 0) return;
  st->generated += st->n_new;
  st->active = counts[5];
  st->iter += 1;
  bool more = st->generated < st->total || st->active > 0;
  if (more && st->iter >= st->max_iter) {
    st->watchdog = 1;
    more = false;
  }
  if (in_graph) cudaGraphSetConditional(cond, more ? 1u : 0u);
}

__global__ void k_resolve(const double* __restrict__ film, float* __restrict__ rgb, uint32_t npix) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npix) return;
  const double* p = film + 4ull * i;
  double w = p[3];
  // Film::WriteToPixelBuffer: colour / weight (visual/Film.h:128-136)
  rgb[3ull * i] = (float)(p[0] / w);
  rgb[3ull * i + 1] = (float)(p[1] / w);
  rgb[3ull * i + 2] = (float)(p[2] / w);
}

// ImageIO::toInt (image/ImageIO.cpp:66-68) in float as the reference
// computes it: int(pow(Clamp(x, 0, 1), 1 / gamma) * 255 + 0.5). A pixel
// without samples (weight 0, colour NaN) gives 0.
GYT_D uint8_t to_int8(float x, float inv_gamma) {
  const float c = x < 0.f ? 0.f : (x > 1.f ? 1.f : x);
  const float v = __fadd_rn(__fmul_rn(powf(c, inv_gamma), 255.f), 0.5f);
  return (v >= 0.f && v < 256.f) ? (uint8_t)(int)v : (uint8_t)0;
}

// Film::SaveImage for 8-bit formats: colour / weight per pixel
// (Film::WriteToPixelBuffer, visual/Film.h:128-136), then toInt per channel.
__global__ void k_film_rgb8(const double* __restrict__ film, uint8_t* __restrict__ rgb, uint32_t npix,
                            float inv_gamma) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npix) return;
  const double* p = film + 4ull * i;
  const double w = p[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) rgb[3ull * i + k] = to_int8((float)(p[k] / w), inv_gamma);
}

// Film::SaveImage for .hdr: colour / weight in Ward's RGBE (shared exponent
// e of the largest component m: frexp(m) = f * 2^e, each channel stored as
// trunc(c * f * 256 / m), exponent byte e + 128; components below 1e-32 give
// zero), as stbi_write_hdr stores the float image (image/ImageIO.cpp:121-131).
__global__ void k_film_rgbe(const double* __restrict__ film, uint8_t* __restrict__ rgbe, uint32_t npix) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npix) return;
  const double* p = film + 4ull * i;
  const double w = p[3];
  float c[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float v = (float)(p[k] / w);
    c[k] = v > 0.f ? v : 0.f;  // negative or NaN: no light
  }
  const float m = fmaxf(fmaxf(c[0], c[1]), c[2]);
  uint8_t* o = rgbe + 4ull * i;
  if (!(m >= 1e-32f)) {
    o[0] = o[1] = o[2] = o[3] = 0;
    return;
  }
  int e;
  const float f = frexpf(m, &e);
  const float norm = __fdiv_rn(__fmul_rn(f, 256.f), m);
#pragma unroll
  for (int k = 0; k < 3; ++k) o[k] = (uint8_t)(int)__fmul_rn(c[k], norm);
  o[3] = (uint8_t)(e + 128);
}

// --------------------------------------------------------- light tracing ---
// LightTracing (integrator/LT.h:11-230): photon g (< spp * W * H) uses the
// sampler index g with the dimension cursor at 0. The light path starts on a
// power-sampled area light (Triangle::Sample + cosine hemisphere about the
// interpolated normal, AreaLight::SampleOnLight, light/AreaLight.h:60-78),
// follows BSDF samples in importance transport without roulette, and every
// vertex is joined to the pinhole camera (ConnectToCamera): the light vertex
// with its emission, the others with We * f * throughput * |cos| / pdfW.
// Unoccluded joins whose truncated raster position lies in [0, W] x [0, H]
// are splatted (Film::AddSplat, visual/Film.h:89-104) scaled by
// W * H / total photons.
struct LtCam {
  float w2r[16];             // world to raster (CameraToRaster * WorldToCamera), row-major
  float3 pos, cz;            // camera position and viewing direction (camera/Camera.cpp:8)
  float film_dist, film_area;
  uint32_t res_x, res_y;
  float fx, fy, ftotal;      // the splat scale factors in float: res_x, res_y, total photons
};

// ConnectToCamera for a vertex at pos: returns whether it lands on the film
// (pixel X, Y) and leaves the direction to the camera and its distance.
template <int W>
GYT_D bool lt_join(const DevScene& s, const LtCam& c, float3 pos, int* X, int* Y, float3* dir, float* dist) {
  const float3 h2c = c.pos - pos;
  const float len = length(h2c);
  const float3 d = h2c / len;
  *dir = d;
  *dist = len;
  if (dot(c.cz, -d) < 0.f) return false;
  float r[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) r[k] = ((c.w2r[4 * k + 3] + c.w2r[4 * k + 2] * pos.z) + c.w2r[4 * k + 1] * pos.y) +
                                     c.w2r[4 * k] * pos.x;
  if (!(r[3] == 1.f || r[3] == 0.f)) {
    r[0] = r[0] / r[3];
    r[1] = r[1] / r[3];
  }
  const int xi = __float2int_rz(r[0]), yi = __float2int_rz(r[1]);
  *X = xi;
  *Y = yi;
  if (!(xi >= 0 && xi <= (int)c.res_x && yi >= 0 && yi <= (int)c.res_y)) return false;
  float tmax = len, b1 = 0.f, b2 = 0.f;  // Ray(pos, dir, len): the constructor's RayEps shift
  return trace<W, true>(s, pos + d * kRayEps, d, tmax, b1, b2) < 0;
}

GYT_D void lt_splat(double* splat, const LtCam& c, int X, int Y, float3 L) {
  X = min(max(X, 0), (int)c.res_x - 1);
  Y = min(max(Y, 0), (int)c.res_y - 1);
  double* p = splat + 3ull * ((unsigned long long)Y * c.res_x + X);
  atomicAdd(p, (double)L.x);
  atomicAdd(p + 1, (double)L.y);
  atomicAdd(p + 2, (double)L.z);
}

// One thread per photon (grid-stride). rec (debug, may be null): per photon
// max_depth records of (on film 1/0 or -1 for no vertex, X, Y, scaled L).
// Capped at four blocks per SM (64 registers; spills, but more warps to hide
// the dependent node fetches): 446 -> 462 Mphotons/s on the Cornell box.
template <int W>
__global__ void __launch_bounds__(kBlock, 4) k_light_trace(DevScene s, LtCam c, Params prm, SamplerTables tab,
                                                        unsigned long long n, const unsigned long long* __restrict__ ids,
                                                        double* __restrict__ splat, float* __restrict__ rec) {
  for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long g = ids ? ids[t] : t;
    float* out = rec ? rec + 6ull * prm.max_depth * t : nullptr;
    if (out)  // no vertex: (-1, 0, 0, 0, 0, 0)
      for (uint32_t k = 0; k < prm.max_depth; ++k)
        for (int f = 0; f < 6; ++f) out[6 * k + f] = f == 0 ? -1.f : 0.f;
    auto emit = [&](uint32_t k, bool on, int X, int Y, float3 L) {
      L = ((L * c.fx) * c.fy) / c.ftotal;
      if (out) {
        out[6 * k] = on ? 1.f : 0.f;
        out[6 * k + 1] = (float)X;
        out[6 * k + 2] = (float)Y;
        out[6 * k + 3] = L.x;
        out[6 * k + 4] = L.y;
        out[6 * k + 5] = L.z;
      }
      if (on && splat) lt_splat(splat, c, X, Y, L);
    };
    if (s.n_area <= 0) continue;
    Rng rng{g, 0};
    // GCC evaluates the arguments right to left: light choice, then v (y, x), then u (y, x)
    const float ul = rng.next(tab, prm.sampler);
    const float vy = rng.next(tab, prm.sampler), vx = rng.next(tab, prm.sampler);
    const float uy = rng.next(tab, prm.sampler), ux = rng.next(tab, prm.sampler);
    float lsel = 0.f;
    const int li = sample_light(s, ul, &lsel);
    if (li >= s.n_area) continue;  // environment light (rejected on the host)
    const LightTri l = load_light(s, li);
    const float su0 = sqrtf(ux);
    const float b0 = 1.f - su0, b1 = uy * su0, b2 = 1.f - b0 - b1;
    const float3 lpos = l.p0 * b0 + l.p1 * b1 + l.p2 * b2;
    const float3 ln = l.n0 * b0 + l.n1 * b1 + l.n2 * b2;
    // CoordinateSystem (math/GeometryUtils.h:11-17) and CosineSampleHemisphere
    float3 ss;
    {
      const bool xz = fabsf(ln.x) > fabsf(ln.y);
      const float den = xz ? sqrtf(ln.x * ln.x + ln.z * ln.z) : sqrtf(ln.y * ln.y + ln.z * ln.z);
      ss = den == 0.f ? mk(0.f, 0.f, 0.f) : (xz ? mk(-ln.z, 0.f, ln.x) : mk(0.f, ln.z, -ln.y)) / den;  // Vector / 0 = 0
    }
    const float3 ts = cross(ln, ss);
    float dx = 0.f, dy = 0.f;
    {
      const float ox = 2.f * vx - 1.f, oy = 2.f * vy - 1.f;
      if (!(ox == 0.f && oy == 0.f)) {
        float th, r;
        if (fabsf(ox) > fabsf(oy)) { r = ox; th = kPiOver4 * (oy / ox); }
        else { r = oy; th = kPiOver2 - kPiOver4 * (ox / oy); }
        float sn, cs;
        sincosf(th, &sn, &cs);
        dx = r * cs;
        dy = r * sn;
      }
    }
    const float dz = sqrtf(fmaxf(0.f, 1.f - dx * dx - dy * dy));
    const float3 dir = norm(ss * dx + ts * dy + ln * dz);
    const float pdf_dir = dz * kInvPi, pdf_a = 1.f / l.area;
    const float cos_l = fabsf(dot(ln, dir));
    float3 tp = l.Le * cos_l / lsel / pdf_a / pdf_dir;
    {
      int X = 0, Y = 0;
      float3 wd;
      float dist;
      const bool on = lt_join<W>(s, c, lpos, &X, &Y, &wd, &dist);
      emit(0, on, X, Y, l.Le);
    }
    // a direction of pdf 0 (on the hemisphere's rim, where this GPU's cosine
    // and the host library's can round differently) carries no flux
    if (!(pdf_dir > 0.f)) continue;
    float3 o = (lpos + dir * kRayEps) + dir * kRayEps, d = dir;
    for (uint32_t bounce = 1; bounce < prm.max_depth;) {
      float tmax = __int_as_float(0x7f800000), hb1 = 0.f, hb2 = 0.f;
      const int prim = trace<W, false>(s, o, d, tmax, hb1, hb2);
      if (prim < 0) break;
      Hit h;
      uint32_t mat;
      if (prim < s.n_tris) {
        float3 p0, p1, p2, n0, n1, n2, face;
        int m, light;
        load_leaf_tri(s, prim, &p0, &p1, &p2, &n0, &n1, &n2, &face, &m, &light);
        tri_hit(p0, p1, p2, n0, n1, n2, face, hb1, hb2, o, d, &h);
        mat = (uint32_t)m;
      } else {
        const int k = prim - s.n_tris;
        Ray r = sphere_object_ray(o, d, __int_as_float(0x7f800000), 0.f);
        sphere_hit(__ldg(s.spheres + k), r, tmax, &h);
        mat = __ldg(s.sphere_mat + k);
      }
      Bsdf bsdf;
      bsdf.lobe = load_lobe(s.mparams, s.mtypes, mat);
      bsdf.lobe.importance = true;
      bsdf.su = h.su; bsdf.sv = h.sv; bsdf.n = h.n; bsdf.gn = h.geo_n;
      {
        int X = 0, Y = 0;
        float3 wi;
        float dist;
        const bool on = lt_join<W>(s, c, h.pos, &X, &Y, &wi, &dist);
        // PinHoleCamera::Sample_Wi and We (camera/PinholeCamera.h:31-49)
        const float cos_c = dot(c.cz, -wi);
        const float pdf_w = 1.f * (dist * dist) / cos_c;
        const float c2 = cos_c * cos_c;
        const float we = c.film_dist * c.film_dist * 1.f / (c.film_area * c2 * c2);
        const float3 f = bsdf.eval(h.wo, wi);
        const float3 L = mk(we, we, we) * f * tp * fabsf(dot(wi, h.n)) / pdf_w;
        emit(bounce, on, X, Y, L);
      }
      ++bounce;
      if (bounce >= prm.max_depth) break;
      const float rz = rng.next(tab, prm.sampler), ry = rng.next(tab, prm.sampler), rx = rng.next(tab, prm.sampler);
      float3 wi;
      float pdf;
      const float3 f = bsdf.sample(h.wo, &wi, &pdf, rx, ry, rz);
      if (pdf == 0.f) break;  // the reference continues with an undefined direction here
      o = (h.pos + wi * kRayEps) + wi * kRayEps;
      d = wi;
      tp = tp * f * fabsf(dot(wi, h.n)) / pdf;
    }
  }
}

// ------------------------------------------------ volumetric path tracing ---
// VolPathTracing::Li without equi-angular sampling (integrator/VPT.cpp:7-104)
// with HomogeneousMedium (volume/Homogeneous.cpp:7-35) and the
// Henyey-Greenstein phase function (visual/Medium.cpp). One camera sample
// per thread; the closest-hit, transmittance and shadow rays are traced
// inline. A ray carries its medium (-1 none); a surface hit takes the
// triangle's MediumInterface when it is a transition, else the ray's medium
// (Primitive::Intersect, visual/Primitive.cpp:5-18); a ray leaving a surface
// takes the outside medium when it leaves along the shading normal, else the
// inside (Intersection::GetMedium, visual/Intersection.h:80-82).
struct MediumDev {
  float3 sa, ss, st;
  float g;
};

GYT_D MediumDev load_medium(const DevScene& s, int m) {
  const float4 a = __ldg(s.media + 2 * m), b = __ldg(s.media + 2 * m + 1);
  MediumDev r;
  r.sa = f3(a);
  r.ss = f3(b);
  r.st = r.ss + r.sa;
  r.g = a.w;
  return r;
}

// HomogeneousMedium::Tr over a segment of parametric length t of direction d
GYT_D float3 medium_tr(const MediumDev& m, float t, float dlen) {
  const float tt = fminf(t * dlen, FLT_MAX);
  return mk(expf(-m.st.x * tt), expf(-m.st.y * tt), expf(-m.st.z * tt));
}

// PhaseHG (visual/Medium.h:20-23)
GYT_D float phase_hg(float cos_t, float g) {
  const float denom = 1.f + g * g + 2.f * g * cos_t;
  return 0.07957747154594766788f * (1.f - g * g) / (denom * sqrtf(denom));
}

// CoordinateSystem (math/GeometryUtils.h:11-17): a zero denominator gives a
// zero vector (Vector / 0 in math/Linagl.h:353-361)
GYT_D void coord_system(float3 v, float3* a, float3* b) {
  const bool xz = fabsf(v.x) > fabsf(v.y);
  const float den = xz ? sqrtf(v.x * v.x + v.z * v.z) : sqrtf(v.y * v.y + v.z * v.z);
  *a = den == 0.f ? mk(0.f, 0.f, 0.f) : (xz ? mk(-v.z, 0.f, v.x) : mk(0.f, v.z, -v.y)) / den;
  *b = cross(v, *a);
}

// HenyeyGreenstein::Sample_p: returns the phase value, sets wi
GYT_D float phase_sample(float g, float3 wo, float u0, float u1, float3* wi) {
  float cos_t;
  if (fabsf(g) < 1e-3f) {
    cos_t = 1.f - 2.f * u0;
  } else {
    const float sq = (1.f - g * g) / (1.f - g + 2.f * g * u0);
    cos_t = (1.f + g * g - sq * sq) / (2.f * g);
  }
  const float sin_t = sqrtf(fmaxf(0.f, 1.f - cos_t * cos_t));
  const float phi = 2.f * (float)3.14159265358979 * u1;
  float3 v1, v2;
  coord_system(wo, &v1, &v2);
  *wi = v1 * (sin_t * cosf(phi)) + v2 * (sin_t * sinf(phi)) + (-wo) * cos_t;
  return phase_hg(-cos_t, g);
}

// A scattering point: a surface hit (its shading data and MediumInterface)
// or a medium point (no normal, no position error, one medium both sides).
struct VPoint {
  float3 pos, perr, abs_n, n, wo;
  int m_in, m_out;
  bool surface;
  GYT_D int medium_along(float3 w) const { return dot(w, n) > 0.f ? m_out : m_in; }
};

// The triangle's MediumInterface when it is a transition, else the ray's medium
GYT_D void surface_media(const DevScene& s, int prim, int ray_medium, int* in, int* out) {
  *in = *out = ray_medium;
  if (!s.media || prim < 0 || prim >= s.n_tris) return;
  const uint32_t packed = __float_as_uint(__ldg(&s.tnrm[3 * prim + 2].w));
  const int a = (int)(packed & 0xffffu) - 1, b = (int)(packed >> 16) - 1;
  if (a != b) {
    *in = a;
    *out = b;
  }
}

GYT_D uint32_t material_type(const DevScene& s, int prim) {
  const uint32_t m = prim < s.n_tris ? (uint32_t)__float_as_int(__ldg(&s.tnrm[3 * prim].w))
                                     : __ldg(s.sphere_mat + (prim - s.n_tris));
  return __ldg(s.mtypes + m);
}

// Full hit record of prim along (o, d) (Scene::QueryIntersectionInfo)
GYT_D void vpt_hit(const DevScene& s, int prim, float t, float b1, float b2, float3 o, float3 d, Hit* h,
                   uint32_t* mat, int* light) {
  if (prim < s.n_tris) {
    float3 p0, p1, p2, n0, n1, n2, face;
    int m;
    load_leaf_tri(s, prim, &p0, &p1, &p2, &n0, &n1, &n2, &face, &m, light);
    tri_hit(p0, p1, p2, n0, n1, n2, face, b1, b2, o, d, h);
    *mat = (uint32_t)m;
  } else {
    const int k = prim - s.n_tris;
    Ray r = sphere_object_ray(o, d, __int_as_float(0x7f800000), 0.f);
    sphere_hit(__ldg(s.spheres + k), r, t, h);
    *mat = __ldg(s.sphere_mat + k);
    *light = -1;
  }
}

// A point on light l for the sample numbers u = (ux, uy): Triangle::Sample
// (shape/Triangle.cpp:141-158) as AreaLight::SampleOnePoint
// (light/AreaLight.h:54-58) and Shape::Sample(ref) (shape/Shape.cpp:6-19) take
// it: position, interpolated normal (not normalised), position error; the
// area pdf is 1 / area.
struct LightPoint {
  float3 pos, n, err;
};

GYT_D LightPoint light_point(const LightTri& l, float ux, float uy) {
  const float su0 = sqrtf(ux);
  const float bb0 = 1.f - su0, bb1 = uy * su0, bb2 = 1.f - bb0 - bb1;
  LightPoint q;
  q.pos = l.p0 * bb0 + l.p1 * bb1 + l.p2 * bb2;
  q.n = l.n0 * bb0 + l.n1 * bb1 + l.n2 * bb2;
  q.err = (vabs(l.p0 * bb0) + vabs(l.p1 * bb1) + vabs(l.p2 * bb2)) * gammaf(6);
  return q;
}

// ----------------------------------------------- volumetric wavefront ---
// VolPathTracing as a wavefront over the path pool: the path tracer's
// k_generate, k_extend and k_finish around three kernels of its own. Per
// bounce k_vshade samples the medium (distance or equi-angular sampling),
// gathers direct light by queueing a shadow segment (a transmittance walk to
// the light point) and an MIS ray (a walk to the first surface with a
// material), and samples the continuation; k_vshadow and k_vmis walk the
// queued rays and add what they carry to the path's radiance. Each kernel is
// small and its warps run one kind of work, where the single persistent
// kernel spent its time on instruction fetch and on a spilled 1.2 KB frame.
// Path slot fields beyond the path tracer's: o.w = medium + 1 and d.w = the
// material-less surfaces crossed, both as integer bits (0 for a new camera
// path: no medium, none crossed).
//
// Shadow segment entry (q.so, q.sd, q.sc, q.madd): (origin, segment length),
// (direction, medium bits), (contribution without the transmittance, path
// slot bits), (light bits, ux, uy, -): the light point, recomputed at every
// hop. MIS ray entry (q.mo, q.md, q.mc): (origin, medium bits), (direction,
// light bits), (contribution without emission and transmittance, slot bits).
GYT_D int vmedium(float w) { return (int)__float_as_uint(w) - 1; }
GYT_D float vmedium_bits(int m) { return __uint_as_float((uint32_t)(m + 1)); }

// The first segment of VisibilityTester::Tr (visual/Visibility.cpp:13-30)
// from p to the light point (Intersection::SpawnTo, visual/Intersection.h:64-72),
// queued with its contribution c.
GYT_D void queue_vshadow(const Queues& q, const VPoint& p, const LightTri& l, const LightPoint& lp, int li, float ux,
                         float uy, float3 c, uint32_t slot) {
  const float3 org = offset_origin(p.pos, p.perr, p.abs_n, lp.pos - p.pos);
  const float3 tgt = offset_origin(lp.pos, lp.err, l.face, org - lp.pos);
  float3 d = tgt - org;
  const float dis = length(d);
  d = d / dis;
  const int medium = dot(d, p.n) > 0.f ? p.m_out : p.m_in;
  const float3 o = org + d * kRayEps;
  const uint32_t j = queue_slot(q.counts);
  q.so[j] = make_float4(o.x, o.y, o.z, dis - kShadowEps);
  q.sd[j] = make_float4(d.x, d.y, d.z, vmedium_bits(medium));
  q.sc[j] = make_float4(c.x, c.y, c.z, __uint_as_float(slot));
  q.madd[j] = make_float4(__int_as_float(li), ux, uy, 0.f);
}

// Integrator::DirectIllumination with handleMedia (integrator/Integrator.cpp:9-107)
// at p, queued: the light half as a shadow segment, the BSDF/phase half as an
// MIS ray. u: uLight, u.y, u.x, v.z, v.y, v.x as the caller draws them.
GYT_D void vpt_direct_queue(const DevScene& s, const Queues& q, const VPoint& p, const Bsdf* bsdf, float g, float3 tp,
                            uint32_t slot, float ul, float ux, float uy, float vx, float vy, float vz) {
  if (s.n_lights <= 0) return;
  float lsel = 0.f;
  const int li = sample_light(s, ul, &lsel);
  if (!(lsel > 0.f) || li >= s.n_area) return;
  const LightTri l = load_light(s, li);
  {
    // AreaLight::Sample_Li -> Shape::Sample(ref) -> Triangle::Sample
    const LightPoint lp = light_point(l, ux, uy);
    float pdf = 1.f / l.area;
    float3 w = p.pos - lp.pos;
    if (length(w) == 0.f) {
      pdf = 0.f;
    } else {
      w = norm(w);
      pdf *= dot(p.pos - lp.pos, p.pos - lp.pos) / fabsf(dot(lp.n, -w));
      if (isinf(pdf)) pdf = 0.f;
    }
    const float3 wi = norm(lp.pos - p.pos);
    const float3 Li = dot(lp.n, -wi) > 0.f ? l.Le : mk(0.f, 0.f, 0.f);
    if (pdf > 0.f && !is_zero(Li)) {
      float spdf, cos_t = 1.f;
      float3 f;
      if (p.surface) {
        spdf = bsdf->pdf(p.wo, wi);
        f = bsdf->eval(p.wo, wi);
        cos_t = fabsf(dot(p.n, wi));
      } else {
        const float ph = phase_hg(dot(p.wo, wi), g);
        f = mk(ph, ph, ph);
        spdf = ph;
      }
      if (!is_zero(f)) {
        const float w1 = power_heuristic(pdf, spdf);
        queue_vshadow(q, p, l, lp, li, ux, uy, tp * (Li * f * cos_t / pdf * w1 / lsel), slot);
      }
    }
  }
  float3 wi, f;
  float pdf, cos_t = 1.f;
  if (p.surface) {
    f = bsdf->sample(p.wo, &wi, &pdf, vx, vy, vz);
    cos_t = fabsf(dot(p.n, wi));
  } else {
    const float ph = phase_sample(g, p.wo, vx, vy, &wi);
    f = mk(ph, ph, ph);
    pdf = ph;
  }
  if (pdf != 0.f && !is_zero(f)) {
    // Intersection::SpawnRay (visual/Intersection.h:74-78)
    const float3 o2 = offset_origin(p.pos, p.perr, p.abs_n, wi) + wi * kRayEps;
    Hit hh;
    hh.pos = p.pos;
    hh.perr = p.perr;
    hh.abs_n = p.abs_n;
    hh.n = p.n;
    const float lpdf = tri_light_pdf(l, hh, o2, wi);
    if (lpdf != 0.f) {
      const float w2 = power_heuristic(pdf, lpdf);
      const float3 c = tp * (f * cos_t / pdf * w2 / lsel);
      const uint32_t j = queue_slot(q.counts + 1);
      q.mo[j] = make_float4(o2.x, o2.y, o2.z, vmedium_bits(p.medium_along(wi)));
      q.md[j] = make_float4(wi.x, wi.y, wi.z, __int_as_float(li));
      q.mc[j] = make_float4(c.x, c.y, c.z, __uint_as_float(slot));
    }
  }
}

// One bounce of VolPathTracing::Li (integrator/VPT.cpp:13-101) for path slot
// i, whose closest hit k_extend left in q.hit.
//
// EQUI: VolPathTracing with equi-angular sampling (its constructor's default,
// integrator/VPT.h:13-15): every bounce draws one light and one point on it
// (VPT.cpp:22-27); a ray through a medium samples its scattering distance
// equi-angularly about that point (HomogeneousMedium::EquiAngularSampling,
// volume/Homogeneous.cpp:38-64), and a medium point gathers light only by the
// connection to that point (ConnectToLight, VPT.cpp:108-146), queued as a
// shadow segment. The light point is recomputed from its two numbers where it
// is used rather than kept.
template <int W, bool EQUI>
__global__ void __launch_bounds__(kBlock, EQUI ? 4 : 3) k_vshade(PathBuf cur, uint32_t n, DevScene s, Params prm,
                                                                 Queues q, SamplerTables tab) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 h4 = q.hit[i];
  const int prim = hit_prim(__float_as_int(h4.w));
  const float tmax = h4.x;
  const uint32_t meta = cur.meta[i];
  uint32_t depth = meta & 255u;
  bool delta = (meta >> 8) & 1u;
  Rng rng{cur.sidx[i], (meta >> 9) & 2047u};
  const float4 o4 = cur.o[i], d4 = cur.d[i];
  float3 o = f3(o4);
  const float3 d = f3(d4);
  int medium = vmedium(o4.w);
  uint32_t crossings = __float_as_uint(d4.w);
  float3 tp = f3(cur.tp[i]);
  float3 nd = d;
  const uint32_t dim_limit = prm.sampler ? kHaltonDims : 1024u;
  bool end = rng.cursor + 16u > dim_limit;  // the sampler's dimensions are spent
  if (!end) {
    bool scattered = false;
    float3 mpos = o;
    float g = 0.f;
    int eli = 0;  // EQUI: the bounce's light, its selection probability and point sample
    float elsel = 0.f, eux = 0.f, euy = 0.f;
    if (EQUI) {
      // VPT.cpp:23-24: Scene::SampleOneLight, then SampleOnePoint's
      // Vec2(rand(), rand()) in right-to-left order
      const float ul = rng.next(tab, prm.sampler);
      euy = rng.next(tab, prm.sampler);
      eux = rng.next(tab, prm.sampler);
      eli = sample_light(s, ul, &elsel);
      if (medium >= 0) {
        // HomogeneousMedium::EquiAngularSampling (volume/Homogeneous.cpp:38-64)
        const MediumDev md = load_medium(s, medium);
        g = md.g;
        const float u = rng.next(tab, prm.sampler);
        const float3 lpos = light_point(load_light(s, eli), eux, euy).pos;
        const float dl = dot(lpos - o, d);
        const float D = length(o + d * dl - lpos);
        const float ta = atan2f(0.f - dl, D), tb = atan2f(3.f - dl, D);
        const float tau = D * tanf((1.f - u) * ta + u * tb);
        const float tt = dl + tau;
        scattered = tt < tmax;
        if (scattered) {
          const float3 tr = mk(expf(-md.st.x * tt), expf(-md.st.y * tt), expf(-md.st.z * tt));
          const float pdf = D / ((tb - ta) * (D * D + tau * tau));
          tp = tp * (tr * md.ss / pdf);
          mpos = o + d * tt;
        } else {
          const float pdf = 1.f - (atan2f(fminf(3.f, tmax) - dl, D) - ta) / (tb - ta);
          tp = tp * (medium_tr(md, tmax, length(d)) / pdf);
        }
      }
    } else if (medium >= 0) {
      // HomogeneousMedium::Sample (volume/Homogeneous.cpp:12-30)
      const MediumDev md = load_medium(s, medium);
      g = md.g;
      const float uc = rng.next(tab, prm.sampler), ud = rng.next(tab, prm.sampler);
      const int ch = min((int)(uc * 3.f), 2);
      const float sc = ch == 0 ? md.st.x : (ch == 1 ? md.st.y : md.st.z);
      const float dist = -logf(1.f - ud) / sc;
      const float dlen = length(d);
      const float tt = fminf(dist / dlen, tmax);
      scattered = tt < tmax;
      const float tc = fminf(tt, FLT_MAX);  // Exp(-sigma_t * min(t, MaxReal) * |d|)
      const float3 tr = mk(expf((-md.st.x * tc) * dlen), expf((-md.st.y * tc) * dlen), expf((-md.st.z * tc) * dlen));
      const float3 dens = scattered ? md.st * tr : tr;
      float pdf = ((0.f + dens.x) + dens.y) + dens.z;
      pdf *= 1.f / 3.f;
      if (pdf == 0.f) pdf = 1.f;
      tp = tp * (scattered ? tr * md.ss / pdf : tr / pdf);
      if (scattered) mpos = o + d * tt;
    }
    VPoint p;
    Bsdf bsdf;
    bool gather = false, pass = false;
    if (is_zero(tp)) {
      end = true;
    } else if (scattered) {
      p.pos = mpos;
      p.perr = p.abs_n = p.n = mk(0.f, 0.f, 0.f);
      p.wo = -d;
      p.m_in = p.m_out = medium;
      p.surface = false;
      gather = true;
    } else if (prim < 0) {
      end = true;  // no environment light with media
    } else {
      Hit h;
      uint32_t mat;
      int light;
      vpt_hit(s, prim, tmax, h4.y, h4.z, o, d, &h, &mat, &light);
      surface_media(s, prim, medium, &p.m_in, &p.m_out);
      p.pos = h.pos;
      p.perr = h.perr;
      p.abs_n = h.abs_n;
      p.n = h.n;
      p.wo = h.wo;
      p.surface = true;
      if (__ldg(s.mtypes + mat) == 5u) {
        // no BSDF: pass through without using a bounce (VPT.cpp:70-75)
        pass = true;
        o = offset_origin(h.pos, h.perr, h.abs_n, d) + d * kRayEps;
        medium = dot(d, h.n) > 0.f ? p.m_out : p.m_in;
        if (++crossings > 64) end = true;
      } else {
        bsdf.lobe = load_lobe(s.mparams, s.mtypes, mat);
        bsdf.su = h.su; bsdf.sv = h.sv; bsdf.n = h.n; bsdf.gn = h.geo_n;
        if ((depth == 0 || delta) && light >= 0) {
          if (dot(h.n, h.wo) > 0.f) {
            const float3 L = f3(cur.L[i]) + tp * load_light(s, light).Le;
            cur.L[i] = make_float4(L.x, L.y, L.z, 0.f);
          }
        } else {
          gather = true;
        }
      }
    }
    if (EQUI && gather && scattered) {
      // VPT.cpp:36: the connection to the bounce's light point
      // (ConnectToLight, VPT.cpp:108-146) as a shadow segment
      if (elsel > 0.f) {
        const LightTri l = load_light(s, eli);
        const LightPoint lp = light_point(l, eux, euy);
        const float3 dir = p.pos - lp.pos;
        const float3 wi = -norm(dir);
        float cos_t = 1.f;
        if (!is_zero(lp.n)) cos_t = dot(norm(dir), lp.n);
        if (!(cos_t < 0.f)) {
          const float ph = phase_hg(dot(p.wo, wi), g);
          const float pdf = 1.f / l.area;
          queue_vshadow(q, p, l, lp, eli, eux, euy, tp * (l.Le * ph * cos_t / dot(dir, dir) / pdf) / elsel, i);
        }
      }
    } else if (gather) {
      // one call site for surface and medium points
      const float vz = rng.next(tab, prm.sampler), vy = rng.next(tab, prm.sampler), vx = rng.next(tab, prm.sampler);
      const float uy = rng.next(tab, prm.sampler), ux = rng.next(tab, prm.sampler);
      const float ul = rng.next(tab, prm.sampler);
      vpt_direct_queue(s, q, p, scattered ? nullptr : &bsdf, g, tp, i, ul, ux, uy, vx, vy, vz);
    }
    if (!end && !pass) {
      if (scattered) {
        const float py = rng.next(tab, prm.sampler), px = rng.next(tab, prm.sampler);
        float3 wi;
        phase_sample(g, -d, px, py, &wi);
        o = mpos + wi * kRayEps;  // MediumIntersection::SpawnRay: no offset
        nd = wi;
        delta = false;
      } else {
        const float rz = rng.next(tab, prm.sampler), ry = rng.next(tab, prm.sampler), rx = rng.next(tab, prm.sampler);
        float3 wi;
        float pdf;
        const float3 f = bsdf.sample(p.wo, &wi, &pdf, rx, ry, rz);
        if (is_zero(f) || pdf == 0.f) {
          end = true;
        } else {
          tp = tp * (f * fabsf(dot(p.n, wi)) / pdf);
          delta = bsdf.lobe.delta();
          o = offset_origin(p.pos, p.perr, p.abs_n, wi) + wi * kRayEps;
          nd = wi;
          medium = dot(wi, p.n) > 0.f ? p.m_out : p.m_in;
        }
      }
      if (!end && ++depth >= prm.max_depth) end = true;
    }
  }
  if (!end) {
    cur.o[i] = make_float4(o.x, o.y, o.z, vmedium_bits(medium));
    cur.d[i] = make_float4(nd.x, nd.y, nd.z, __uint_as_float(crossings));
    cur.tp[i] = make_float4(tp.x, tp.y, tp.z, 0.f);
  }
  cur.meta[i] = meta_pack(depth, delta, rng.cursor, !end);
}

// The queued shadow segments: VisibilityTester::Tr (visual/Visibility.cpp:13-30),
// segment after segment through surfaces of no material (a surface with a
// material blocks), each attenuated by its medium; an unblocked walk adds its
// contribution times the transmittance to the path. A hit at the very end of
// a segment (the light's own surface) is settled in FP64, as the path
// tracer's occlusion test settles it. Grid-stride over the queue.
template <int W>
__global__ void __launch_bounds__(kBlock) k_vshadow(PathBuf cur, DevScene s, Queues q) {
  const uint32_t nq = *(volatile uint32_t*)q.counts;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += gridDim.x * blockDim.x) {
    const float4 a = q.so[j], b = q.sd[j], c4 = q.sc[j], x = q.madd[j];
    float3 o = f3(a), d = f3(b);
    float seg = a.w;
    int medium = vmedium(b.w);
    const int li = __float_as_int(x.x);
    float3 tr = mk(1.f, 1.f, 1.f);
    bool lit = false;
#pragma unroll 1
    for (int hop = 0; hop < 64; ++hop) {
      float tmax = seg, b1 = 0.f, b2 = 0.f;
      int prim = trace<W, false>(s, o, d, tmax, b1, b2);
      if (prim >= 0 && prim < s.n_tris && tmax >= seg * 0.999998f) {
        const float4* tv = s.tris + 3 * (size_t)prim;
        if (!wt_intersect_fp64(wt_setup(o, d), f3(__ldg(tv)), f3(__ldg(tv + 1)), f3(__ldg(tv + 2)), seg)) {
          prim = -1;
          tmax = seg;
        }
      }
      if (prim >= 0 && material_type(s, prim) != 5u) break;  // blocked
      if (medium >= 0) tr = tr * medium_tr(load_medium(s, medium), tmax, length(d));
      if (prim < 0) {
        lit = true;
        break;
      }
      Hit h;
      uint32_t mat;
      int light;
      vpt_hit(s, prim, tmax, b1, b2, o, d, &h, &mat, &light);
      int m_in, m_out;
      surface_media(s, prim, medium, &m_in, &m_out);
      // the next segment: SpawnTo from the crossed surface to the light point
      const LightTri l = load_light(s, li);
      const LightPoint lp = light_point(l, x.y, x.z);
      const float3 org = offset_origin(h.pos, h.perr, h.abs_n, lp.pos - h.pos);
      const float3 tgt = offset_origin(lp.pos, lp.err, l.face, org - lp.pos);
      d = tgt - org;
      const float dis = length(d);
      d = d / dis;
      medium = dot(d, h.n) > 0.f ? m_out : m_in;
      o = org + d * kRayEps;
      seg = dis - kShadowEps;
    }
    if (lit) {
      const uint32_t slot = __float_as_uint(c4.w);
      const float3 L = f3(cur.L[slot]) + f3(c4) * tr;
      cur.L[slot] = make_float4(L.x, L.y, L.z, 0.f);
    }
  }
}

// The queued MIS rays: Scene::IntersectTr (visual/Scene.cpp:14-26), the first
// surface with a material along the ray and the transmittance up to it (a
// passed surface restarts at its barycentric point in its inside medium); a
// ray that reaches the sampled light's front adds its contribution times the
// emission and the transmittance (Integrator.cpp:86-101). Grid-stride.
template <int W>
__global__ void __launch_bounds__(kBlock) k_vmis(PathBuf cur, DevScene s, Queues q) {
  const uint32_t nq = *(volatile uint32_t*)(q.counts + 1);
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += gridDim.x * blockDim.x) {
    const float4 a = q.mo[j], b = q.md[j], c4 = q.mc[j];
    float3 o = f3(a);
    const float3 wi = f3(b);
    int medium = vmedium(a.w);
    const int li = __float_as_int(b.w);
    float3 tr = mk(1.f, 1.f, 1.f);
#pragma unroll 1
    for (int hop = 0; hop < 64; ++hop) {
      float tmax = __int_as_float(0x7f800000), b1 = 0.f, b2 = 0.f;
      const int prim = trace<W, false>(s, o, wi, tmax, b1, b2);
      if (medium >= 0) tr = tr * medium_tr(load_medium(s, medium), tmax, length(wi));
      if (prim < 0) break;
      if (material_type(s, prim) != 5u || prim >= s.n_tris) {
        if (prim < s.n_tris && __float_as_int(__ldg(&s.tnrm[3 * prim + 1].w)) == li) {
          Hit lh;
          uint32_t mat;
          int light;
          vpt_hit(s, prim, tmax, b1, b2, o, wi, &lh, &mat, &light);
          if (dot(lh.n, -wi) > 0.f) {  // AreaLight::Emission(isect, -wi)
            const uint32_t slot = __float_as_uint(c4.w);
            const float4* r = s.ltab + kLightRec * li;
            const float3 Le = mk(__ldg(r).w, __ldg(r + 1).w, __ldg(r + 2).w);
            const float3 L = f3(cur.L[slot]) + f3(c4) * Le * tr;
            cur.L[slot] = make_float4(L.x, L.y, L.z, 0.f);
          }
        }
        break;
      }
      float3 p0, p1, p2, n0, n1, n2, face;
      int m, light;
      load_leaf_tri(s, prim, &p0, &p1, &p2, &n0, &n1, &n2, &face, &m, &light);
      const float3 pos = p0 * (1.f - b1 - b2) + p1 * b1 + p2 * b2;
      int in, out;
      surface_media(s, prim, medium, &in, &out);
      medium = in;
      o = pos + wi * kRayEps;
    }
  }
}

// Scene::AddMesh's Triangle::SetTransform (shape/Triangle.h:78-88) per
// vertex, in the reference's float arithmetic: a point is M (x, y, z, 1) with
// the matrix applied column by column from the last (((M.3 + M.2 z) + M.1 y)
// + M.0 x per row, unfused), divided by w unless w is 0 or 1
// (math/Transform.h:106-115); a normal is M^-T (x, y, z, 0) the same way
// (Transform::TransformNormal, math/Transform.h:247-251), then divided by its
// length ((x x + y y) + z z).
struct Xform {
  float m[16], inv[16];  // row-major
};

__global__ void k_mesh_transform(float* __restrict__ pos, float* __restrict__ nrm, uint32_t nvert, Xform t) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nvert) return;
  float* p = pos + 3ull * i;
  const float x = p[0], y = p[1], z = p[2];
  float r[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float a = t.m[4 * k + 3];
    a = __fadd_rn(__fmul_rn(t.m[4 * k + 2], z), a);
    a = __fadd_rn(__fmul_rn(t.m[4 * k + 1], y), a);
    r[k] = __fadd_rn(__fmul_rn(t.m[4 * k + 0], x), a);
  }
  if (r[3] == 1.f || r[3] == 0.f) {
    p[0] = r[0];
    p[1] = r[1];
    p[2] = r[2];
  } else {
    p[0] = __fdiv_rn(r[0], r[3]);
    p[1] = __fdiv_rn(r[1], r[3]);
    p[2] = __fdiv_rn(r[2], r[3]);
  }
  float* n = nrm + 3ull * i;
  const float nx = n[0], ny = n[1], nz = n[2];
  float q[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float a = __fmul_rn(t.inv[12 + k], 0.f);
    a = __fadd_rn(__fmul_rn(t.inv[8 + k], nz), a);
    a = __fadd_rn(__fmul_rn(t.inv[4 + k], ny), a);
    q[k] = __fadd_rn(__fmul_rn(t.inv[k], nx), a);
  }
  const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(q[0], q[0]), __fmul_rn(q[1], q[1])), __fmul_rn(q[2], q[2])));
  n[0] = __fdiv_rn(q[0], len);
  n[1] = __fdiv_rn(q[1], len);
  n[2] = __fdiv_rn(q[2], len);
}

template <int W>
__global__ void k_intersect(DevScene s, uint64_t n, const float* __restrict__ rays, int any, int32_t* prim,
                            float* tout, float* b1out, float* b2out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* r = rays + 7 * i;
  float3 o = mk(r[0], r[1], r[2]), d = mk(r[3], r[4], r[5]);
  float tmax = r[6], b1 = 0.f, b2 = 0.f;
  int p = any ? (trace<W, true>(s, o, d, tmax, b1, b2) >= 0 ? 1 : 0) : trace<W, false>(s, o, d, tmax, b1, b2);
  if (!any && p >= 0 && p < s.n_tris) p = __float_as_int(__ldg(s.tris + 3 * p).w);
  prim[i] = p;
  if (!any) {
    tout[i] = p >= 0 ? tmax : 0.f;
    b1out[i] = p >= 0 && p < s.n_tris ? b1 : 0.f;
    b2out[i] = p >= 0 && p < s.n_tris ? b2 : 0.f;
  }
}

// One BxDF per case in its local frame, the lobes the shading kernels use:
// sample (u), evaluate and pdf toward a second direction (we). vec holds wo,
// u, we (9 floats per case); out 11 floats: f, wi, pdf of the sample, f and
// pdf toward we.
__global__ void k_bsdf_table(uint64_t n, const float* __restrict__ params, const uint32_t* __restrict__ types,
                             const float* __restrict__ vec, float* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Lobe l = load_lobe(params, types, (uint32_t)i);
  const float* v = vec + 9 * i;
  const float3 wo = mk(v[0], v[1], v[2]), we = mk(v[6], v[7], v[8]);
  float3 wi = mk(0.f, 0.f, 0.f);
  float pdf = 0.f;
  const float3 f = l.sample(wo, &wi, &pdf, v[3], v[4], v[5]);
  const float3 fe = l.eval(wo, we);
  const float pe = l.pdf(wo, we);
  float* o = out + 11 * i;
  o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = wi.x; o[4] = wi.y; o[5] = wi.z; o[6] = pdf;
  o[7] = fe.x; o[8] = fe.y; o[9] = fe.z; o[10] = pe;
}

__global__ void k_sobol(const uint32_t* __restrict__ mat, uint64_t n, const uint32_t* dims, const uint64_t* idx,
                        float* out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = sobol_sample(mat, idx[i], dims[i]);
}

__global__ void k_halton(SamplerTables tab, uint64_t n, const uint32_t* dims, const uint64_t* idx, float* out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = halton_sample(tab, idx[i], dims[i]);
}

__global__ void k_halton_enum(Cam cam, uint64_t n, const uint32_t* sxy, uint64_t* out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = halton_enum_index(cam, sxy[3 * i], sxy[3 * i + 1], sxy[3 * i + 2]);
}

__global__ void k_enum(SamplerTables tab, uint32_t m, uint64_t n, const uint32_t* sxy, uint64_t* out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = enum_index(tab, m, sxy[3 * i], sxy[3 * i + 1], sxy[3 * i + 2]);
}

inline uint32_t grid_for(uint64_t n) { return (uint32_t)((n + kBlock - 1) / kBlock); }

// Persistent traversal kernels and their grid sizes (blocks per SM at full
// occupancy times the SM count), computed once per context.
enum { kPExtend = 0, kPShadow = 1, kPMis = 2 };
constexpr int kPersistentKinds = 3 * 2 * 2;  // kernel x width (2, 8) x counting
inline int pindex(int kind, int w, bool count) { return (kind * 2 + (w == 8 ? 1 : 0)) * 2 + (count ? 1 : 0); }

template <int W, bool C>
const void* persistent_fn(int kind) {
  if (kind == kPExtend) return (const void*)k_extend<W, C>;
  return (const void*)k_connect<W, C>;  // shadow and MIS rays (kPMis: grid of the adjoint's MIS kernel)
}

}  // namespace

// Leaf-order triangle data of a device-built BVH, the same records the host
// path writes: tris[3k + c] = (p_c, triangle id bits for c = 0) and
// tnrm[3k + c] = (vertex normal, or the face normal without normals; material
// bits for c = 0, light bits for c = 1, the packed medium interface for c = 2). The face normal is computed with the
// host's IEEE operations in the host's order (no contraction), so both paths
// store identical floats. leaf_of[t] = k.
__global__ void k_leaf_data(uint32_t nt, const uint32_t* __restrict__ order, const float* __restrict__ V,
                            const uint32_t* __restrict__ I, const float* __restrict__ N,
                            const int2* __restrict__ info, const uint32_t* __restrict__ tmed,
                            const uint32_t* __restrict__ mtype, float4* __restrict__ tris, float4* __restrict__ tnrm,
                            int* __restrict__ leaf_of) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  const uint32_t t = order[k];
  leaf_of[t] = (int)k;
  uint32_t vi[3];
  float3 p[3];
  for (int c = 0; c < 3; ++c) {
    vi[c] = I[3 * (size_t)t + c];
    p[c] = mk(V[3 * (size_t)vi[c]], V[3 * (size_t)vi[c] + 1], V[3 * (size_t)vi[c] + 2]);
  }
  const float3 a = mk(__fsub_rn(p[1].x, p[0].x), __fsub_rn(p[1].y, p[0].y), __fsub_rn(p[1].z, p[0].z));
  const float3 b = mk(__fsub_rn(p[2].x, p[0].x), __fsub_rn(p[2].y, p[0].y), __fsub_rn(p[2].z, p[0].z));
  const float3 cr = mk(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
                       __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
                       __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
  const float len =
      __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(cr.x, cr.x), __fmul_rn(cr.y, cr.y)), __fmul_rn(cr.z, cr.z)));
  const float3 face = mk(__fdiv_rn(cr.x, len), __fdiv_rn(cr.y, len), __fdiv_rn(cr.z, len));
  const int2 in = info[t];
  const uint32_t cls = min(mtype[in.x], 4u) + 1u;
  for (int c = 0; c < 3; ++c) {
    tris[3 * (size_t)k + c] =
        make_float4(p[c].x, p[c].y, p[c].z, c == 0 ? __int_as_float((int)t) : (c == 1 ? __uint_as_float(cls) : 0.f));
    const float3 n = N ? mk(N[3 * (size_t)vi[c]], N[3 * (size_t)vi[c] + 1], N[3 * (size_t)vi[c] + 2]) : face;
    const float w = c == 0 ? __int_as_float(in.x) : (c == 1 ? __int_as_float(in.y) : __uint_as_float(tmed ? tmed[t] : 0u));
    tnrm[3 * (size_t)k + c] = make_float4(n.x, n.y, n.z, w);
  }
}

__global__ void k_gather_int(uint32_t n, const int* __restrict__ index, const int* __restrict__ src,
                             int* __restrict__ dst) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[index[i]];
}

// ------------------------------------------------------------- host side ---
struct gyt_context {
  int device = 0;
  int pgrid[kPersistentKinds] = {};
  cudaStream_t stream = nullptr;
  std::string err;
  uint32_t capacity = 1u << 21;
  uint32_t pool_cap = 0;
  PathBuf pool[2] = {};
  Queues q = {};
  uint32_t* d_counter = nullptr;
  uint32_t* h_counter = nullptr;
  uint32_t* d_sobol = nullptr;
  uint32_t* d_sobol_bits = nullptr;
  uint16_t* d_hperm = nullptr;  // Halton digit-block tables (halton_tables)
  uint4* d_hdesc = nullptr;
  uint64_t* d_vdc = nullptr;
  uint64_t* d_vdc_inv = nullptr;
  double* d_film = nullptr;
  size_t film_bytes = 0;
  float* d_rgb = nullptr;
  size_t rgb_bytes = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_in = nullptr;  // orders a render after the caller's legacy-stream work
  std::vector<void*> pool_allocs;
  int profile = 0;
  int bvh_width = 2;
  int bvh_builder = GYT_BVH_BUILD_DEVICE;
  cudaEvent_t kev[8] = {};
  unsigned long long* d_counters = nullptr;  // node visits and triangle tests per traversal kernel
  GytProfile prof = {};
  int sms = 0;
  // batched renders: device loop state, configuration and the captured graph
  // (rebuilt when its kernels' arguments change)
  IterState* d_iter = nullptr;
  IterState* h_iter = nullptr;  // pinned
  GytBatchConfig bcfg = {0, 0, 0, 1, 0};
  int btrace[2][2] = {};  // occupancy limit (blocks per SM) of the batched extend/shadow, width 2/8
  cudaGraph_t bgraph = nullptr;
  cudaGraphExec_t bexec = nullptr;
  uint64_t bkey[6] = {};
  // adjoint pass: replay state per path slot (two buffers) and queue payloads
  AdjBuf adj[2] = {};
  uint32_t adj_cap = 0;
  std::vector<void*> adj_allocs;
};

struct gyt_scene {
  gyt_context* ctx = nullptr;  // the creating context (may be destroyed before the scene)
  int device = 0;
  DevScene dev = {};
  std::vector<void*> allocs;
  uint64_t n_tris = 0, n_nodes = 0, n_slots = 0, bytes = 0;
  uint32_t bvh_depth = 0;
  // what gyt_scene_set_materials needs to rebuild the light tables
  uint32_t n_materials = 0, n_emission = 0;
  std::vector<float4> ltab;       // host copy of the light records
  std::vector<float> light_area;  // per area light
  std::vector<float> power;       // light powers (area lights, then the environment)
  float* sparams_buf = nullptr;   // device copy of the frozen sampling parameters (gyt_scene_freeze_sampling)
};

namespace {

int32_t fail(gyt_context* ctx, int32_t code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

#define GYT_CK(ctx, call)                                                                          \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? GYT_ERR_OUT_OF_MEMORY : GYT_ERR_CUDA,     \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                             \
  } while (0)

template <typename T>
cudaError_t dalloc(std::vector<void*>& list, T** p, size_t count) {
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e == cudaSuccess) list.push_back(*p);
  return e;
}

// The context's stream does not synchronise with the legacy default stream,
// where callers (and torch) typically clear a film: the render waits for the
// work already queued there.
cudaError_t after_legacy_stream(gyt_context* ctx) {
  cudaError_t e = cudaEventRecord(ctx->ev_in, cudaStreamLegacy);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_in, 0);
  return e;
}

SamplerTables tables(const gyt_context* c) {
  return SamplerTables{c->d_sobol, c->d_vdc, c->d_vdc_inv, c->d_sobol_bits, c->d_hperm, c->d_hdesc};
}

Params make_params(const GytRenderParams* p) {
  return Params{p->spp, p->max_depth, p->rr_depth, (p->flags & GYT_SAMPLER_HALTON) ? 1u : 0u};
}

// ProjectiveCamera::Initialize (camera/Camera.cpp:6-59): RasterToWorld in
// closed form, in double. Raster (x, y, z, 1) -> NDC (2x/W - 1, 1 - 2y/H, z)
// -> camera through the inverse of Transform::Perspective
// (math/Transform.cpp:132-150) -> world through the camera basis.
void raster_to_world(const GytCamera& c, double m[16]) {
  double pos[3] = {c.pos[0], c.pos[1], c.pos[2]};
  double cz[3] = {c.look_at[0] - pos[0], c.look_at[1] - pos[1], c.look_at[2] - pos[2]};
  double l = std::sqrt(cz[0] * cz[0] + cz[1] * cz[1] + cz[2] * cz[2]);
  for (double& v : cz) v /= l;
  double up[3] = {c.up[0], c.up[1], c.up[2]};
  double cx[3] = {-(up[1] * cz[2] - up[2] * cz[1]), -(up[2] * cz[0] - up[0] * cz[2]), -(up[0] * cz[1] - up[1] * cz[0])};
  l = std::sqrt(cx[0] * cx[0] + cx[1] * cx[1] + cx[2] * cx[2]);
  for (double& v : cx) v /= l;
  double cy[3] = {-(cz[1] * cx[2] - cz[2] * cx[1]), -(cz[2] * cx[0] - cz[0] * cx[2]), -(cz[0] * cx[1] - cz[1] * cx[0])};
  double aspect = (double)((float)c.res_x / (float)c.res_y);
  double dis = c.film_distance, n = dis, f = 100000.0;
  double t = dis * std::tan(c.fovy * (3.14159265358979 / 180.0) * 0.5);
  double r = t * aspect;
  double a = dis / r, b = dis / t, A = (f + n) / (f - n), B = -2.0 * f * n / (f - n);
  double r2c[4][4] = {{2.0 / (a * c.res_x), 0, 0, -1.0 / a},
                      {0, -2.0 / (b * c.res_y), 0, 1.0 / b},
                      {0, 0, 0, 1.0},
                      {0, 0, 1.0 / B, -A / B}};
  double c2w[4][4] = {{cx[0], cy[0], cz[0], pos[0]}, {cx[1], cy[1], cz[1], pos[1]}, {cx[2], cy[2], cz[2], pos[2]},
                      {0, 0, 0, 1}};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += c2w[i][k] * r2c[k][j];
      m[4 * i + j] = s;
    }
}

// Digit-block tables of HaltonSampler with Faure permutations
// (sampler/Halton.h:595-625 builds the permutations, :912-1435 the tables).
// Faure's permutation of {0..b-1}: identity for b <= 3; for even b the
// permutation of b/2 doubled into the even and the odd half; for odd b the
// permutation of b - 1 with the middle value c = (b-1)/2 inserted at c (values
// and positions from c on move up by one). Dimension d >= 1 uses the d-th
// prime b, blocks of k digits (the largest k with b^k <= 512) through a table
// of B = b^k entries, as many whole blocks n as keep B^n below 2^32.
void halton_tables(std::vector<uint16_t>* perm_out, std::vector<uint4>* desc_out) {
  constexpr uint32_t kMaxBase = 1619;  // the 256th prime
  std::vector<std::vector<uint16_t>> fp(kMaxBase + 1);
  for (uint32_t b = 1; b <= kMaxBase; ++b) {
    std::vector<uint16_t>& q = fp[b];
    q.resize(b);
    if (b <= 3) {
      for (uint32_t i = 0; i < b; ++i) q[i] = (uint16_t)i;
    } else if (b % 2 == 0) {
      const std::vector<uint16_t>& h = fp[b / 2];
      for (uint32_t i = 0; i < b / 2; ++i) {
        q[i] = (uint16_t)(2 * h[i]);
        q[b / 2 + i] = (uint16_t)(2 * h[i] + 1);
      }
    } else {
      const uint32_t c = b / 2;
      const std::vector<uint16_t>& h = fp[b - 1];
      for (uint32_t i = 0; i < b - 1; ++i) q[i < c ? i : i + 1] = (uint16_t)(h[i] < c ? h[i] : h[i] + 1);
      q[c] = (uint16_t)c;
    }
  }
  perm_out->clear();
  desc_out->assign(kHaltonDims, make_uint4(0, 0, 0, 0));
  uint32_t b = 2;
  for (uint32_t d = 1; d < kHaltonDims; ++d) {
    for (++b;; ++b) {
      bool prime = true;
      for (uint32_t f = 2; f * f <= b && prime; ++f) prime = b % f != 0;
      if (prime) break;
    }
    uint32_t k = 1;
    uint64_t B = b;
    while (B * b <= 512) { B *= b; ++k; }
    uint32_t n = 0;
    uint64_t Bn = 1;
    while (Bn * B < (1ull << 32)) { Bn *= B; ++n; }
    const float scale = (float)(0x1.fffffcp-1 / (double)Bn);
    uint32_t bits;
    std::memcpy(&bits, &scale, 4);
    (*desc_out)[d] = make_uint4((uint32_t)perm_out->size(), (uint32_t)B, n, bits);
    for (uint32_t i = 0; i < B; ++i) {
      uint32_t r = 0, q = i;
      for (uint32_t j = 0; j < k; ++j, q /= b) r = r * b + fp[b][q % b];
      perm_out->push_back((uint16_t)r);
    }
  }
}

// a^-1 mod m in [0, m), 0 for m == 1 (extended Euclidean algorithm)
uint64_t inverse_mod(int64_t a, int64_t m) {
  if (m == 1) return 0;
  int64_t r0 = m, r1 = a % m, s0 = 0, s1 = 1;
  while (r1) {
    const int64_t q = r0 / r1;
    int64_t t = r0 - q * r1;
    r0 = r1;
    r1 = t;
    t = s0 - q * s1;
    s0 = s1;
    s1 = t;
  }
  return (uint64_t)(((s0 % m) + m) % m);
}

// The camera and the sample enumeration of the render's sampler
// (params->flags: GYT_SAMPLER_HALTON selects HaltonSampler + HaltonEnum).
int32_t make_cam(gyt_context* ctx, const GytCamera* c, const GytRenderParams* prm, Cam* out) {
  if (!c || c->res_x == 0 || c->res_y == 0) return fail(ctx, GYT_ERR_INVALID, "camera: empty film");
  if ((uint64_t)c->res_x * c->res_y > kPixMask) return fail(ctx, GYT_ERR_UNSUPPORTED, "camera: film too large");
  *out = Cam{};
  double m[16];
  raster_to_world(*c, m);
  for (int i = 0; i < 16; ++i) out->m[i] = (float)m[i];
  out->pos = mk(c->pos[0], c->pos[1], c->pos[2]);
  out->res_x = c->res_x;
  out->res_y = c->res_y;
  out->sampler = (prm && (prm->flags & GYT_SAMPLER_HALTON)) ? 1u : 0u;
  if (out->sampler) {
    // HaltonEnum::HaltonEnum (sampler/HaltonEnum.h): the film padded to 2^p2 x 3^p3
    uint64_t w = 1, h = 1;
    while (w < c->res_x) { w *= 2; ++out->h_p2; }
    while (h < c->res_y) { h *= 3; ++out->h_p3; }
    if (w * h >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "camera: film too large for HaltonEnum");
    out->h_sx = (float)w;
    out->h_sy = (float)h;
    out->h_inc = w * h;
    out->h_mx = h * inverse_mod((int64_t)h, (int64_t)w);
    out->h_my = w * inverse_mod((int64_t)w, (int64_t)h);
    return GYT_OK;
  }
  uint32_t r = std::max(c->res_x, c->res_y), p = 1, lg = 0;
  while (p < r) { p <<= 1; ++lg; }
  if (lg > GYT_ENUM_M) return fail(ctx, GYT_ERR_UNSUPPORTED, "camera: resolution beyond the Sobol' enumeration tables");
  out->log2_res = lg;
  out->res_pow2 = (float)p;
  return GYT_OK;
}

// Distribution1D over light power (visual/Sampling.h:18-45), in float as the
// reference builds it: returns the integral, fills the n + 1 CDF values.
float light_distribution(const std::vector<float>& power, std::vector<float>* cdf_out) {
  const int nl = (int)power.size();
  std::vector<float>& cdf = *cdf_out;
  cdf.assign(nl + 1, 0.f);
  float fint = 0.f;
  if (nl) {
    for (int i = 1; i < nl + 1; ++i) cdf[i] = cdf[i - 1] + power[i - 1] / nl;
    fint = cdf[nl];
    if (fint == 0.f) {
      for (int i = 1; i < nl + 1; ++i) cdf[i] = (float)i / (float)nl;
    } else {
      for (int i = 1; i < nl + 1; ++i) cdf[i] /= fint;
    }
  }
  return fint;
}

// AreaLight::Power (light/AreaLight.h:45-48)
float area_light_power(const float* em, float area) { return lum(mk(em[0], em[1], em[2]) * area * kPi); }

int32_t check_params(gyt_context* ctx, const GytRenderParams* p, uint32_t extra_flags = 0) {
  if (!p) return fail(ctx, GYT_ERR_INVALID, "params: null");
  if (p->spp == 0) return fail(ctx, GYT_ERR_INVALID, "params: spp must be > 0");
  if (p->max_depth == 0 || p->max_depth > 100)
    return fail(ctx, GYT_ERR_UNSUPPORTED, "params: max_depth must be in [1, 100] (Sobol' has 1024 dimensions)");
  if (p->rr_depth > 255) return fail(ctx, GYT_ERR_INVALID, "params: rr_depth too large");
  if (p->flags & ~(GYT_SAMPLER_HALTON | extra_flags)) return fail(ctx, GYT_ERR_INVALID, "params: unknown flags");
  return GYT_OK;
}

// 4x4 inverse by Gauss-Jordan elimination with partial pivoting (double).
bool invert4(const double a[16], double out[16]) {
  double m[4][8];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 8; ++j) m[i][j] = j < 4 ? a[4 * i + j] : (j - 4 == i ? 1.0 : 0.0);
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(m[r][c]) > std::fabs(m[piv][c])) piv = r;
    if (m[piv][c] == 0.0) return false;
    for (int j = 0; j < 8; ++j) std::swap(m[c][j], m[piv][j]);
    const double d = m[c][c];
    for (int j = 0; j < 8; ++j) m[c][j] /= d;
    for (int r = 0; r < 4; ++r)
      if (r != c) {
        const double f = m[r][c];
        for (int j = 0; j < 8; ++j) m[r][j] -= f * m[c][j];
      }
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) out[4 * i + j] = m[i][4 + j];
  return true;
}

// The camera quantities light tracing reads (camera/Camera.cpp:6-59) in float
// as the reference computes them: mCz = -(pos - look).Norm(), the film plane
// height 2 d tan(fovy / 2) and area; world to raster as the inverse of
// RasterToWorld (in double, then float).
int32_t make_lt_cam(gyt_context* ctx, const GytCamera* c, unsigned long long total, LtCam* out) {
  double m[16], w[16];
  raster_to_world(*c, m);
  if (!invert4(m, w)) return fail(ctx, GYT_ERR_INVALID, "light_tracing: singular camera");
  for (int i = 0; i < 16; ++i) out->w2r[i] = (float)w[i];
  out->pos = mk(c->pos[0], c->pos[1], c->pos[2]);
  const float dx = c->pos[0] - c->look_at[0], dy = c->pos[1] - c->look_at[1], dz = c->pos[2] - c->look_at[2];
  const float len = std::sqrt((dx * dx + dy * dy) + dz * dz);
  out->cz = mk(-(dx / len), -(dy / len), -(dz / len));
  const float pi = (float)3.14159265358979;  // common/Core.h:185
  const float height = c->film_distance * std::tan(c->fovy * 0.5f * pi / 180) * 2.f;
  const float width = height * ((float)c->res_x / (float)c->res_y);
  out->film_dist = c->film_distance;
  out->film_area = width * height;
  out->res_x = c->res_x;
  out->res_y = c->res_y;
  out->fx = (float)c->res_x;
  out->fy = (float)c->res_y;
  out->ftotal = (float)total;
  return GYT_OK;
}

__global__ void k_splat_to_rgb(const double* __restrict__ splat, float* __restrict__ rgb, uint64_t n) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rgb[i] = (float)splat[i];
}

// All photons of LightTracing::Render (n == 0: every photon, splatted into
// d_splat) or the listed ones (ids, records only).
int32_t run_light_tracing(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                          const GytRenderParams* params, uint64_t n, const unsigned long long* ids, double* d_splat,
                          float* d_rec, GytRenderStats* stats) {
  int32_t st = check_params(ctx, params);
  if (st) return st;
  if (scene->dev.has_env)
    return fail(ctx, GYT_ERR_UNSUPPORTED, "light_tracing: environment lights are not sampled (area lights only)");
  if (scene->dev.sparams) return fail(ctx, GYT_ERR_UNSUPPORTED, "light_tracing: the scene's BSDF sampling is frozen");
  Cam cam;
  st = make_cam(ctx, camera, params, &cam);  // validates the film (and the sampler's enumeration limits)
  if (st) return st;
  const unsigned long long total = (unsigned long long)camera->res_x * camera->res_y * params->spp;
  LtCam lc;
  st = make_lt_cam(ctx, camera, total, &lc);
  if (st) return st;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  GYT_CK(ctx, after_legacy_stream(ctx));
  const Params prm = make_params(params);
  const unsigned long long count = n ? n : total;
  const uint32_t grid = (uint32_t)std::min<unsigned long long>((count + kBlock - 1) / kBlock,
                                                                (unsigned long long)std::max(1, ctx->sms) * 8);
  GYT_CK(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
  if (scene->dev.wnodes)
    k_light_trace<8><<<grid, kBlock, 0, ctx->stream>>>(scene->dev, lc, prm, tables(ctx), count, ids, d_splat, d_rec);
  else
    k_light_trace<2><<<grid, kBlock, 0, ctx->stream>>>(scene->dev, lc, prm, tables(ctx), count, ids, d_splat, d_rec);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
  GYT_CK(ctx, cudaEventSynchronize(ctx->ev1));
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    *stats = GytRenderStats{count, 0, 1, 1, ms};
  }
  return GYT_OK;
}

// VolPathTracing (n == 0: every sample of the render into d_film; else the
// listed (x, y, s) samples, radiance and dimensions used out).
int32_t ensure_pool(gyt_context* ctx);
unsigned long long wavefront_bound(unsigned long long total, uint32_t max_depth, uint32_t pool);

int32_t run_volume(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera, const GytRenderParams* params,
                   uint64_t n, const uint32_t* xys, double* d_film, float* L_out, uint32_t* cursor_out,
                   GytRenderStats* stats) {
  int32_t st = check_params(ctx, params, GYT_VOLUME_EQUI_ANGULAR);
  if (st) return st;
  if (scene->dev.has_env)
    return fail(ctx, GYT_ERR_UNSUPPORTED, "render_volume: environment lights are not supported with media");
  if ((params->flags & GYT_VOLUME_EQUI_ANGULAR) && scene->dev.n_area == 0)
    return fail(ctx, GYT_ERR_UNSUPPORTED, "render_volume: equi-angular sampling needs an area light");
  if (scene->dev.sparams) return fail(ctx, GYT_ERR_UNSUPPORTED, "render_volume: the scene's BSDF sampling is frozen");
  Cam cam;
  st = make_cam(ctx, camera, params, &cam);
  if (st) return st;
  const unsigned long long total = (unsigned long long)camera->res_x * camera->res_y * params->spp;
  const unsigned long long count = n ? n : total;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  st = ensure_pool(ctx);
  if (st) return st;
  GYT_CK(ctx, after_legacy_stream(ctx));
  const Params prm = make_params(params);
  const SamplerTables tab = tables(ctx);
  const DevScene& D = scene->dev;
  const int W = D.wnodes ? 8 : 2;
  const bool equi = (params->flags & GYT_VOLUME_EQUI_ANGULAR) != 0;
  const int g_ext = ctx->pgrid[pindex(kPExtend, W, false)];
  const int g_walk = std::max(1, ctx->sms) * 4;  // grid-stride walks over the queues
  const Queues q = ctx->q;
  const DebugOut dbg{L_out, cursor_out, nullptr, nullptr, nullptr};
  cudaStream_t sm = ctx->stream;
  // a crossing of a material-less surface takes a wavefront iteration without a bounce
  const unsigned long long max_iters = wavefront_bound(count, params->max_depth + 65, ctx->capacity);
  unsigned long long generated = 0;
  uint32_t active = 0, iters = 0, launches = 0;
  unsigned long long slots = 0;
  int cur = 0;
  GYT_CK(ctx, cudaEventRecord(ctx->ev0, sm));
  while (generated < count || active > 0) {
    const uint32_t n_new = (uint32_t)std::min<unsigned long long>(ctx->capacity - active, count - generated);
    GYT_CK(ctx, cudaMemsetAsync(q.counts, 0, 8 * sizeof(uint32_t), sm));
    const PathBuf P = ctx->pool[cur], N = ctx->pool[cur ^ 1];
    if (n_new) {
      k_generate<<<grid_for(n_new), kBlock, 0, sm>>>(P, active, n_new, generated, cam, params->spp, xys, tab);
      ++launches;
    }
    generated += n_new;
    active += n_new;
    if (W == 8) {
      k_extend<8, false><<<g_ext, kBlock, 0, sm>>>(P, active, D, q.hit, q.counts + 2, nullptr);
      if (equi) k_vshade<8, true><<<grid_for(active), kBlock, 0, sm>>>(P, active, D, prm, q, tab);
      else k_vshade<8, false><<<grid_for(active), kBlock, 0, sm>>>(P, active, D, prm, q, tab);
      k_vshadow<8><<<g_walk, kBlock, 0, sm>>>(P, D, q);
      k_vmis<8><<<g_walk, kBlock, 0, sm>>>(P, D, q);
    } else {
      k_extend<2, false><<<g_ext, kBlock, 0, sm>>>(P, active, D, q.hit, q.counts + 2, nullptr);
      if (equi) k_vshade<2, true><<<grid_for(active), kBlock, 0, sm>>>(P, active, D, prm, q, tab);
      else k_vshade<2, false><<<grid_for(active), kBlock, 0, sm>>>(P, active, D, prm, q, tab);
      k_vshadow<2><<<g_walk, kBlock, 0, sm>>>(P, D, q);
      k_vmis<2><<<g_walk, kBlock, 0, sm>>>(P, D, q);
    }
    k_finish<<<grid_for(active), kBlock, 0, sm>>>(P, N, active, d_film, cam.res_x, q.counts + 5, q.madd, dbg);
    launches += 5;
    GYT_CK(ctx, cudaGetLastError());
    GYT_CK(ctx, cudaMemcpyAsync(ctx->h_counter, q.counts, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, sm));
    GYT_CK(ctx, cudaStreamSynchronize(sm));
    slots += active;
    active = ctx->h_counter[5];
    cur ^= 1;
    if (++iters > max_iters) return fail(ctx, GYT_ERR_WATCHDOG, "render_volume: wavefront iteration cap reached");
  }
  GYT_CK(ctx, cudaEventRecord(ctx->ev1, sm));
  GYT_CK(ctx, cudaEventSynchronize(ctx->ev1));
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    *stats = GytRenderStats{count, slots, iters, launches, ms};
  }
  return GYT_OK;
}

// Pools changed size: the adjoint buffers follow on their next use.
int32_t ensure_adj_reset(gyt_context* ctx) {
  for (void* p : ctx->adj_allocs) cudaFree(p);
  ctx->adj_allocs.clear();
  ctx->adj_cap = 0;
  ctx->q.sx = ctx->q.mx = nullptr;
  return GYT_OK;
}

int32_t ensure_pool(gyt_context* ctx) {
  if (ctx->pool_cap == ctx->capacity) return GYT_OK;
  for (void* p : ctx->pool_allocs) cudaFree(p);
  ctx->pool_allocs.clear();
  ctx->pool_cap = 0;
  size_t n = ctx->capacity;
  auto& L = ctx->pool_allocs;
  for (int b = 0; b < 2; ++b) {
    PathBuf& P = ctx->pool[b];
    GYT_CK(ctx, dalloc(L, &P.o, n));
    GYT_CK(ctx, dalloc(L, &P.d, n));
    GYT_CK(ctx, dalloc(L, &P.tp, n));
    GYT_CK(ctx, dalloc(L, &P.L, n));
    GYT_CK(ctx, dalloc(L, &P.sidx, n));
    GYT_CK(ctx, dalloc(L, &P.meta, n));
    GYT_CK(ctx, dalloc(L, &P.pix, n));
    GYT_CK(ctx, dalloc(L, &P.pid, n));
    GYT_CK(ctx, dalloc(L, &P.inst, n));
  }
  Queues& q = ctx->q;
  GYT_CK(ctx, dalloc(L, &q.so, n));
  GYT_CK(ctx, dalloc(L, &q.sd, n));
  GYT_CK(ctx, dalloc(L, &q.sc, n));
  GYT_CK(ctx, dalloc(L, &q.mo, n));
  GYT_CK(ctx, dalloc(L, &q.md, n));
  GYT_CK(ctx, dalloc(L, &q.mc, n));
  GYT_CK(ctx, dalloc(L, &q.hit, n));
  GYT_CK(ctx, dalloc(L, &q.madd, n));
  GYT_CK(ctx, dalloc(L, &q.counts, 8));
  ctx->pool_cap = ctx->capacity;
  return ensure_adj_reset(ctx);
}

int32_t ensure_adj(gyt_context* ctx) {
  if (ctx->adj_cap == ctx->pool_cap && ctx->q.sx) return GYT_OK;
  for (void* p : ctx->adj_allocs) cudaFree(p);
  ctx->adj_allocs.clear();
  ctx->adj_cap = 0;
  ctx->q.sx = ctx->q.mx = nullptr;
  const size_t n = ctx->pool_cap;
  auto& L = ctx->adj_allocs;
  for (int b = 0; b < 2; ++b) {
    GYT_CK(ctx, dalloc(L, &ctx->adj[b].delta, n));
    GYT_CK(ctx, dalloc(L, &ctx->adj[b].Ltot, n));
    GYT_CK(ctx, dalloc(L, &ctx->adj[b].pend, n));
  }
  GYT_CK(ctx, dalloc(L, &ctx->q.sx, n));
  GYT_CK(ctx, dalloc(L, &ctx->q.mx, n));
  ctx->adj_cap = ctx->pool_cap;
  return GYT_OK;
}

// Wavefront iterations that a render of `total` paths of at most max_depth
// bounces can take with `pool` paths in flight: a path holds a slot for at
// most max_depth + 1 iterations and a full pool finishes at least
// pool / (max_depth + 1) paths per iteration; doubled, with room for the
// tail. The loops stop with GYT_ERR_WATCHDOG past it.
unsigned long long wavefront_bound(unsigned long long total, uint32_t max_depth, uint32_t pool) {
  return 2ull * (total / std::max(1u, pool) + 2) * ((unsigned long long)max_depth + 2) + 64;
}

// The wavefront loop shared by full renders and explicit path lists.
int32_t run_paths(gyt_context* ctx, const gyt_scene* scene, const Cam& cam, const GytRenderParams* p,
                  unsigned long long total, const uint32_t* d_list, double* d_film, DebugOut dbg,
                  GytRenderStats* stats) {
  int32_t st = ensure_pool(ctx);
  if (st) return st;
  Params prm = make_params(p);
  SamplerTables tab = tables(ctx);
  cudaStream_t s = ctx->stream;
  unsigned long long generated = 0;
  uint32_t active = 0, iters = 0;
  unsigned long long rays = 0;
  int cur = 0;
  const bool prof = ctx->profile > 0, cnt = ctx->profile > 1;
  uint32_t launches = 0;
  unsigned long long slots = 0;
  const int W = scene->dev.wnodes ? 8 : 2;
  const int g_ext = ctx->pgrid[pindex(kPExtend, W, cnt)], g_sh = ctx->pgrid[pindex(kPShadow, W, cnt)];
  Queues q = ctx->q;
  if (cnt) GYT_CK(ctx, cudaMemsetAsync(ctx->d_counters, 0, 6 * sizeof(unsigned long long), s));
  uint32_t hcounts[8];
  GYT_CK(ctx, after_legacy_stream(ctx));
  GYT_CK(ctx, cudaEventRecord(ctx->ev0, s));
  while (generated < total || active > 0) {
    uint32_t n_new = (uint32_t)std::min<unsigned long long>(ctx->capacity - active, total - generated);
    GYT_CK(ctx, cudaMemsetAsync(q.counts, 0, 8 * sizeof(uint32_t), s));
    if (prof) GYT_CK(ctx, cudaEventRecord(ctx->kev[0], s));
    if (n_new) {
      k_generate<<<grid_for(n_new), kBlock, 0, s>>>(ctx->pool[cur], active, n_new, generated, cam, p->spp, d_list, tab);
      ++launches;
    }
    generated += n_new;
    active += n_new;
    const PathBuf P = ctx->pool[cur], N = ctx->pool[cur ^ 1];
    const DevScene& D = scene->dev;
    unsigned long long* C = ctx->d_counters;
    if (prof) GYT_CK(ctx, cudaEventRecord(ctx->kev[1], s));
    if (W == 8) {
      if (cnt) k_extend<8, true><<<g_ext, kBlock, 0, s>>>(P, active, D, q.hit, q.counts + 2, C);
      else k_extend<8, false><<<g_ext, kBlock, 0, s>>>(P, active, D, q.hit, q.counts + 2, nullptr);
    } else {
      if (cnt) k_extend<2, true><<<g_ext, kBlock, 0, s>>>(P, active, D, q.hit, q.counts + 2, C);
      else k_extend<2, false><<<g_ext, kBlock, 0, s>>>(P, active, D, q.hit, q.counts + 2, nullptr);
    }
    if (prof) GYT_CK(ctx, cudaEventRecord(ctx->kev[2], s));
    if (D.sparams) {
      if (prm.sampler) k_shade<true, 1><<<grid_for(active), kBlock, 0, s>>>(P, active, D, prm, q, tab, dbg);
      else k_shade<true, 0><<<grid_for(active), kBlock, 0, s>>>(P, active, D, prm, q, tab, dbg);
    } else {
      if (prm.sampler) k_shade<false, 1><<<grid_for(active), kBlock, 0, s>>>(P, active, D, prm, q, tab, dbg);
      else k_shade<false, 0><<<grid_for(active), kBlock, 0, s>>>(P, active, D, prm, q, tab, dbg);
    }
    if (prof) GYT_CK(ctx, cudaEventRecord(ctx->kev[3], s));
    // shadow and MIS rays in one launch (profile slot 3; slot 4 stays empty)
    if (W == 8) {
      if (cnt) k_connect<8, true><<<g_sh, kBlock, 0, s>>>(P, D, q, dbg, C + 2);
      else k_connect<8, false><<<g_sh, kBlock, 0, s>>>(P, D, q, dbg, nullptr);
    } else {
      if (cnt) k_connect<2, true><<<g_sh, kBlock, 0, s>>>(P, D, q, dbg, C + 2);
      else k_connect<2, false><<<g_sh, kBlock, 0, s>>>(P, D, q, dbg, nullptr);
    }
    if (prof) GYT_CK(ctx, cudaEventRecord(ctx->kev[4], s));
    if (prof) GYT_CK(ctx, cudaEventRecord(ctx->kev[5], s));
    k_finish<<<grid_for(active), kBlock, 0, s>>>(P, N, active, d_film, cam.res_x, q.counts + 5, q.madd, dbg);
    if (prof) GYT_CK(ctx, cudaEventRecord(ctx->kev[6], s));
    launches += 4;
    GYT_CK(ctx, cudaGetLastError());
    GYT_CK(ctx, cudaMemcpyAsync(ctx->h_counter, q.counts, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GYT_CK(ctx, cudaStreamSynchronize(s));
    std::memcpy(hcounts, ctx->h_counter, sizeof(hcounts));
    if (prof) {
      for (int k = 0; k < 6; ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->kev[k], ctx->kev[k + 1]);
        ctx->prof.ms[k] += ms;
        if ((k != 0 || n_new) && k != 4) ctx->prof.launches[k]++;
      }
      ctx->prof.rays[0] += active;
      ctx->prof.rays[1] += hcounts[0];
      ctx->prof.rays[2] += hcounts[1];
    }
    slots += active;
    rays += active;
    active = hcounts[5];
    cur ^= 1;
    if (++iters > wavefront_bound(total, p->max_depth, ctx->capacity))
      return fail(ctx, GYT_ERR_WATCHDOG, "render: wavefront iteration cap reached");
  }
  GYT_CK(ctx, cudaEventRecord(ctx->ev1, s));
  GYT_CK(ctx, cudaEventSynchronize(ctx->ev1));
  if (cnt) {
    unsigned long long c[6];
    GYT_CK(ctx, cudaMemcpy(c, ctx->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 3; ++k) {
      ctx->prof.node_visits[k] += c[2 * k];
      ctx->prof.tri_tests[k] += c[2 * k + 1];
    }
  }
  if (stats) {
    stats->paths = total;
    stats->path_slots = slots;
    stats->iterations = iters;
    stats->launches = launches;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->ms = ms;
  }
  return GYT_OK;
}

// The path replay (adjoint) wavefront: the primal's paths again, with the
// adjoint kernels moving gradient into G.
int32_t run_adjoint(gyt_context* ctx, const gyt_scene* scene, const Cam& cam, const GytRenderParams* p,
                    unsigned long long total, const uint32_t* d_list, const AdjIn& in, GradOut G,
                    GytRenderStats* stats) {
  if (scene->dev.sparams)
    return fail(ctx, GYT_ERR_UNSUPPORTED, "adjoint: the scene's BSDF sampling is frozen (the replay samples as "
                                          "the primal did only without it)");
  int32_t st = ensure_pool(ctx);
  if (st) return st;
  st = ensure_adj(ctx);
  if (st) return st;
  const Params prm = make_params(p);
  const SamplerTables tab = tables(ctx);
  cudaStream_t s = ctx->stream;
  const int W = scene->dev.wnodes ? 8 : 2;
  const int g_ext = ctx->pgrid[pindex(kPExtend, W, false)], g_sh = ctx->pgrid[pindex(kPShadow, W, false)],
            g_mis = ctx->pgrid[pindex(kPMis, W, false)];
  const DevScene& D = scene->dev;
  const Queues q = ctx->q;
  unsigned long long generated = 0;
  uint32_t active = 0, iters = 0, launches = 0;
  int cur = 0;
  GYT_CK(ctx, after_legacy_stream(ctx));
  GYT_CK(ctx, cudaEventRecord(ctx->ev0, s));
  while (generated < total || active > 0) {
    const uint32_t n_new = (uint32_t)std::min<unsigned long long>(ctx->capacity - active, total - generated);
    GYT_CK(ctx, cudaMemsetAsync(q.counts, 0, 8 * sizeof(uint32_t), s));
    const PathBuf P = ctx->pool[cur], N = ctx->pool[cur ^ 1];
    const AdjBuf A = ctx->adj[cur], AN = ctx->adj[cur ^ 1];
    if (n_new) {
      k_generate_adj<<<grid_for(n_new), kBlock, 0, s>>>(P, A, active, n_new, generated, cam, p->spp, d_list, tab, in);
      ++launches;
    }
    generated += n_new;
    active += n_new;
    if (W == 8) k_extend<8, false><<<g_ext, kBlock, 0, s>>>(P, active, D, q.hit, q.counts + 2, nullptr);
    else k_extend<2, false><<<g_ext, kBlock, 0, s>>>(P, active, D, q.hit, q.counts + 2, nullptr);
    k_shade_adj<<<grid_for(active), kBlock, 0, s>>>(P, A, active, D, prm, q, tab, G);
    if (W == 8) k_shadow_adj<8><<<g_sh, kBlock, 0, s>>>(P, A, D, q, G);
    else k_shadow_adj<2><<<g_sh, kBlock, 0, s>>>(P, A, D, q, G);
    if (W == 8) k_mis_adj<8><<<g_mis, kBlock, 0, s>>>(P, A, D, q, G);
    else k_mis_adj<2><<<g_mis, kBlock, 0, s>>>(P, A, D, q, G);
    k_finish_adj<<<grid_for(active), kBlock, 0, s>>>(P, N, A, AN, active, q.counts + 5);
    launches += 5;
    GYT_CK(ctx, cudaGetLastError());
    GYT_CK(ctx, cudaMemcpyAsync(ctx->h_counter, q.counts, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GYT_CK(ctx, cudaStreamSynchronize(s));
    active = ctx->h_counter[5];
    cur ^= 1;
    if (++iters > wavefront_bound(total, p->max_depth, ctx->capacity))
      return fail(ctx, GYT_ERR_WATCHDOG, "adjoint: wavefront iteration cap reached");
  }
  GYT_CK(ctx, cudaEventRecord(ctx->ev1, s));
  GYT_CK(ctx, cudaEventSynchronize(ctx->ev1));
  if (stats) {
    stats->paths = total;
    stats->path_slots = 0;
    stats->iterations = iters;
    stats->launches = launches;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->ms = ms;
  }
  return GYT_OK;
}

}  // namespace

struct gyt_mesh {
  gyt::ObjMesh mesh;
};

extern "C" {

int32_t gyt_context_create(int32_t device, gyt_context** out) {
  if (!out) return GYT_ERR_INVALID;
  *out = nullptr;
  auto* c = new gyt_context();
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_counter, sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_counter, 8 * sizeof(uint32_t));
  const size_t sob = GYT_SOBOL_DIMS * GYT_SOBOL_COLS;
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_sobol, (sob + 64) * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_sobol, 0, (sob + 64) * sizeof(uint32_t), c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->d_sobol, gyt_sobol_matrices, sob * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    // transposed copy: row b = column b of every dimension (see sobol10)
    std::vector<uint32_t> tr((size_t)64 * kSobolRow, 0u);
    for (int b = 0; b < 64; ++b)
      for (int dm = 0; dm < kSobolRow; ++dm) {
        size_t flat = (size_t)dm * 52 + b;
        tr[(size_t)b * kSobolRow + dm] = flat < sob ? gyt_sobol_matrices[flat] : 0u;
      }
    e = cudaMalloc((void**)&c->d_sobol_bits, tr.size() * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->d_sobol_bits, tr.data(), tr.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream);
  }
  std::vector<uint16_t> hperm;
  std::vector<uint4> hdesc;
  halton_tables(&hperm, &hdesc);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_hperm, hperm.size() * sizeof(uint16_t));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->d_hperm, hperm.data(), hperm.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_hdesc, hdesc.size() * sizeof(uint4));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c->d_hdesc, hdesc.data(), hdesc.size() * sizeof(uint4), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_vdc, sizeof(gyt_vdc_sobol));
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->d_vdc, gyt_vdc_sobol, sizeof(gyt_vdc_sobol), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_vdc_inv, sizeof(gyt_vdc_sobol_inv));
  if (e == cudaSuccess) e = cudaMemcpyAsync(c->d_vdc_inv, gyt_vdc_sobol_inv, sizeof(gyt_vdc_sobol_inv), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming);
  for (int k = 0; k < 8 && e == cudaSuccess; ++k) e = cudaEventCreate(&c->kev[k]);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_counters, 6 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // tables resident before the first launch
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_iter, sizeof(IterState));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&c->h_iter, sizeof(IterState));
  if (e == cudaSuccess) {
    const void* fns[2][2] = {{(const void*)k_extend_batch<2>, (const void*)k_connect_batch<2>},
                             {(const void*)k_extend_batch<8>, (const void*)k_connect_batch<8>}};
    for (int w = 0; w < 2 && e == cudaSuccess; ++w)
      for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fns[w][k], kBlock, 0);
        c->btrace[w][k] = std::max(1, nb);
      }
  }
  if (e == cudaSuccess) {
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    c->sms = sms;
    for (int kind = 0; kind < 3 && e == cudaSuccess; ++kind)
      for (int w : {2, 8})
        for (int cntm = 0; cntm < 2 && e == cudaSuccess; ++cntm) {
          const void* fn = w == 8 ? (cntm ? persistent_fn<8, true>(kind) : persistent_fn<8, false>(kind))
                                  : (cntm ? persistent_fn<2, true>(kind) : persistent_fn<2, false>(kind));
          int nb = 0;
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kBlock, 0);
          // MIS rays are rare (only BSDF samples that would reach the sampled
          // light): one block per SM keeps the launch cheap
          if (kind == kPMis) nb = 1;
          c->pgrid[pindex(kind, w, cntm != 0)] = std::max(1, nb) * std::max(1, sms);
        }
  }
  if (e != cudaSuccess) {
    gyt_context_destroy(c);
    return e == cudaErrorMemoryAllocation ? GYT_ERR_OUT_OF_MEMORY : GYT_ERR_CUDA;
  }
  *out = c;
  return GYT_OK;
}

void gyt_context_destroy(gyt_context* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (void* p : c->pool_allocs) cudaFree(p);
  for (void* p : c->adj_allocs) cudaFree(p);
  cudaFree(c->d_counter);
  cudaFreeHost(c->h_counter);
  cudaFree(c->d_sobol);
  cudaFree(c->d_sobol_bits);
  cudaFree(c->d_hperm);
  cudaFree(c->d_hdesc);
  cudaFree(c->d_vdc);
  cudaFree(c->d_vdc_inv);
  cudaFree(c->d_film);
  cudaFree(c->d_rgb);
  if (c->bexec) cudaGraphExecDestroy(c->bexec);
  if (c->bgraph) cudaGraphDestroy(c->bgraph);
  if (c->d_iter) cudaFree(c->d_iter);
  if (c->h_iter) cudaFreeHost(c->h_iter);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev_in) cudaEventDestroy(c->ev_in);
  for (int k = 0; k < 8; ++k)
    if (c->kev[k]) cudaEventDestroy(c->kev[k]);
  cudaFree(c->d_counters);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char* gyt_last_error(const gyt_context* c) { return c ? c->err.c_str() : "null context"; }

int32_t gyt_context_set_capacity(gyt_context* c, uint32_t n) {
  if (!c) return GYT_ERR_INVALID;
  if (n < 1024 || n > (1u << 26)) return fail(c, GYT_ERR_INVALID, "capacity must be in [1024, 2^26]");
  c->capacity = n;
  return GYT_OK;
}

int32_t gyt_context_set_profile(gyt_context* c, int32_t mode) {
  if (!c) return GYT_ERR_INVALID;
  if (mode < 0 || mode > 2) return fail(c, GYT_ERR_INVALID, "profile mode must be 0, 1 or 2");
  c->profile = mode;
  return GYT_OK;
}

int32_t gyt_context_set_bvh_width(gyt_context* c, int32_t width) {
  if (!c) return GYT_ERR_INVALID;
  if (width != 2 && width != 8) return fail(c, GYT_ERR_INVALID, "bvh width must be 2 or 8");
  c->bvh_width = width;
  return GYT_OK;
}

int32_t gyt_context_set_bvh_builder(gyt_context* c, int32_t builder) {
  if (!c) return GYT_ERR_INVALID;
  if (builder != GYT_BVH_BUILD_HOST && builder != GYT_BVH_BUILD_DEVICE)
    return fail(c, GYT_ERR_INVALID, "bvh builder must be GYT_BVH_BUILD_HOST or GYT_BVH_BUILD_DEVICE");
  c->bvh_builder = builder;
  return GYT_OK;
}

int32_t gyt_profile_read(gyt_context* c, GytProfile* out) {
  if (!c || !out) return GYT_ERR_INVALID;
  *out = c->prof;
  c->prof = GytProfile{};
  return GYT_OK;
}

int32_t gyt_scene_create(gyt_context* ctx, const GytSceneDesc* d, gyt_scene** out) {
  if (!ctx || !d || !out) return fail(ctx, GYT_ERR_INVALID, "scene_create: null argument");
  *out = nullptr;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, GYT_ERR_CUDA, "scene_create: cudaSetDevice");
  if (d->n_triangles && (!d->vertices || !d->indices || !d->tri_material || !d->tri_emission))
    return fail(ctx, GYT_ERR_INVALID, "scene_create: triangle arrays missing");
  if (d->n_spheres && (!d->spheres || !d->sphere_material))
    return fail(ctx, GYT_ERR_INVALID, "scene_create: sphere arrays missing");
  if (d->n_materials == 0 || !d->mat_type || !d->mat_params)
    return fail(ctx, GYT_ERR_INVALID, "scene_create: no materials");
  const bool has_env = d->env && d->env_w && d->env_h;
  if (has_env && ((uint64_t)d->env_w * d->env_h > (1ull << 28) || d->env_w < 1 || d->env_h < 1))
    return fail(ctx, GYT_ERR_UNSUPPORTED, "scene_create: environment map too large");
  // closest-hit records keep the primitive in 28 bits (hit_prim)
  if ((uint64_t)d->n_triangles + d->n_spheres >= (1ull << 28))
    return fail(ctx, GYT_ERR_UNSUPPORTED, "scene_create: too many primitives");
  for (uint32_t m = 0; m < d->n_materials; ++m)
    if (d->mat_type[m] > GYT_MAT_NONE) return fail(ctx, GYT_ERR_INVALID, "scene_create: unknown material type");
  if (d->n_media && !d->media) return fail(ctx, GYT_ERR_INVALID, "scene_create: media array missing");
  if (d->n_media >= 0xffffu) return fail(ctx, GYT_ERR_UNSUPPORTED, "scene_create: too many media");
  // the triangles' medium interfaces, packed (inside + 1) | (outside + 1) << 16
  std::vector<uint32_t> tmed;
  if (d->tri_medium) {
    tmed.resize(d->n_triangles);
    for (uint32_t t = 0; t < d->n_triangles; ++t) {
      const int32_t a = d->tri_medium[2 * t], b = d->tri_medium[2 * t + 1];
      if (a < -1 || b < -1 || a >= (int32_t)d->n_media || b >= (int32_t)d->n_media)
        return fail(ctx, GYT_ERR_INVALID, "scene_create: medium index out of range");
      tmed[t] = (uint32_t)(a + 1) | ((uint32_t)(b + 1) << 16);
    }
  }
  std::vector<int2> info(d->n_triangles);
  std::vector<int> light_tris;
  std::vector<float> power;
  const float* V = d->vertices;
  auto vtx = [&](uint32_t i) { return mk(V[3 * i], V[3 * i + 1], V[3 * i + 2]); };
  for (uint32_t t = 0; t < d->n_triangles; ++t) {
    for (int k = 0; k < 3; ++k)
      if (d->indices[3 * t + k] >= d->n_vertices) return fail(ctx, GYT_ERR_INVALID, "scene_create: index out of range");
    if (d->tri_material[t] >= d->n_materials) return fail(ctx, GYT_ERR_INVALID, "scene_create: material out of range");
    int e = d->tri_emission[t];
    info[t].x = (int)d->tri_material[t];
    info[t].y = -1;
    if (e >= 0) {
      if ((uint32_t)e >= d->n_emission || !d->emission) return fail(ctx, GYT_ERR_INVALID, "scene_create: emission out of range");
      info[t].y = (int)light_tris.size();
      light_tris.push_back((int)t);
      const float* em = &d->emission[3 * e];
      const uint32_t* I = &d->indices[3 * t];
      float area = 0.5f * length(cross(vtx(I[1]) - vtx(I[0]), vtx(I[2]) - vtx(I[0])));
      power.push_back(area_light_power(em, area));
    }
  }
  for (uint32_t k = 0; k < d->n_spheres; ++k)
    if (d->sphere_material[k] >= d->n_materials) return fail(ctx, GYT_ERR_INVALID, "scene_create: sphere material out of range");
  const int n_area = (int)power.size();
  // environment light (light/EnvLight.cpp, light/EnvMap.h): texels, the
  // Distribution2D of ConvertImageToPdf (EnvMap.h:75-90) and the light's power,
  // all in float as the reference computes them
  std::vector<float4> env_tex;
  std::vector<float> env_ccdf, env_cfunc, env_cint, env_mcdf, env_mfunc;
  float env_mint = 0.f, env_radius = 0.f;
  if (has_env) {
    const int w = (int)d->env_w, hgt = (int)d->env_h;
    env_tex.resize((size_t)w * hgt);
    for (size_t k = 0; k < env_tex.size(); ++k)
      env_tex[k] = make_float4(d->env[3 * k], d->env[3 * k + 1], d->env[3 * k + 2], 0.f);
    auto dist1d = [](const float* f, int n, float* cdf, float* fint) {
      cdf[0] = 0.f;
      for (int i = 1; i < n + 1; ++i) cdf[i] = cdf[i - 1] + f[i - 1] / n;
      *fint = cdf[n];
      if (*fint == 0.f) {
        for (int i = 1; i < n + 1; ++i) cdf[i] = (float)i / (float)n;
      } else {
        for (int i = 1; i < n + 1; ++i) cdf[i] /= *fint;
      }
    };
    env_cfunc.resize((size_t)w * hgt);
    env_ccdf.resize((size_t)(w + 1) * hgt);
    env_cint.resize(hgt);
    for (int r = 0; r < hgt; ++r) {
      float v = (float)(r + 0.5f) / (float)hgt;
      float st = std::sin(kPi * v);
      for (int c = 0; c < w; ++c) {
        const float* px = &d->env[((size_t)r * w + c) * 3];
        env_cfunc[(size_t)r * w + c] = st * lum(mk(px[0], px[1], px[2]));
      }
      dist1d(&env_cfunc[(size_t)r * w], w, &env_ccdf[(size_t)r * (w + 1)], &env_cint[r]);
    }
    env_mfunc = env_cint;
    env_mcdf.resize(hgt + 1);
    dist1d(env_mfunc.data(), hgt, env_mcdf.data(), &env_mint);
    // AABB::GetBoundingSphere of the accelerator's bounds (math/AABB.h:69-72)
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t t = 0; t < d->n_triangles; ++t)
      for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) {
          float vv = d->vertices[3 * d->indices[3 * t + k] + a];
          lo[a] = std::min(lo[a], vv);
          hi[a] = std::max(hi[a], vv);
        }
    for (uint32_t k = 0; k < d->n_spheres; ++k)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], d->spheres[4 * k + a] - d->spheres[4 * k + 3]);
        hi[a] = std::max(hi[a], d->spheres[4 * k + a] + d->spheres[4 * k + 3]);
      }
    env_radius = length(mk(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2])) * 0.5f;
    // EnvironmentLight::Power (EnvLight.cpp:59-62): Y(LookupRadiance(0.5, 0.5) * PI * R * R)
    auto texel = [&](int x, int y) {
      x = std::min(std::max(x, 0), w - 1);
      y = std::min(std::max(y, 0), hgt - 1);
      const float* px = &d->env[((size_t)(hgt - 1 - y) * w + x) * 3];
      return mk(px[0], px[1], px[2]);
    };
    float su = (float)w * 0.5f - 0.5f, sv = (float)hgt * (1.f - 0.5f) - 0.5f;
    int s0 = (int)std::floor(su), t0 = (int)std::floor(sv);
    float ds = su - s0, dt = sv - t0;
    float3 a = texel(s0, t0) * (1.f - ds) + texel(s0 + 1, t0) * ds;
    float3 b2 = texel(s0, t0 + 1) * (1.f - ds) + texel(s0 + 1, t0 + 1) * ds;
    float3 mid = (a * (1.f - dt) + b2 * dt) * d->env_scale;
    power.push_back(lum(mid * kPi * env_radius * env_radius));
  }
  const int nl = (int)power.size();
  std::vector<float> cdf;
  const float fint = light_distribution(power, &cdf);
  // acceleration structure: binary (two child boxes per 64-byte node) or
  // 8-wide with quantized child boxes (80-byte nodes), built on the device
  // or the host, per context setting
  const bool use_wide = ctx->bvh_width == 8;
  const bool use_dev = ctx->bvh_builder == GYT_BVH_BUILD_DEVICE && d->n_triangles > 0;
  auto* sc = new gyt_scene();
  sc->ctx = ctx;
  sc->device = ctx->device;
  auto bail = [&](int32_t code, const std::string& msg) {
    gyt_scene_destroy(sc);
    return fail(ctx, code, msg);
  };
  auto up = [&](auto** dst, const auto* src, size_t count) -> cudaError_t {
    using T = std::remove_const_t<std::remove_reference_t<decltype(*src)>>;
    cudaError_t e = dalloc(sc->allocs, (T**)dst, count);
    if (e == cudaSuccess && count && src) e = cudaMemcpyAsync((void*)*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    sc->bytes += count * sizeof(T);
    return e;
  };
  auto cuda_code = [](cudaError_t e) { return e == cudaErrorMemoryAllocation ? GYT_ERR_OUT_OF_MEMORY : GYT_ERR_CUDA; };
  DevScene& ds = sc->dev;
  cudaError_t e = cudaSuccess;
  std::vector<int> light_leaf(n_area, -1);  // leaf-order position of each area light's triangle
  auto bits = [](int v) { float f; std::memcpy(&f, &v, 4); return f; };
  if (use_dev) {
    const uint32_t nt = d->n_triangles;
    std::vector<void*> tmp;
    struct Free {
      std::vector<void*>& v;
      ~Free() {
        for (void* q : v) cudaFree(q);
      }
    } tmp_free{tmp};
    auto tup = [&](auto** dst, const auto* src, size_t count) -> cudaError_t {
      using T = std::remove_const_t<std::remove_reference_t<decltype(*src)>>;
      cudaError_t e2 = dalloc(tmp, (T**)dst, count);
      if (e2 == cudaSuccess && count && src)
        e2 = cudaMemcpyAsync((void*)*dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
      return e2;
    };
    float *dV = nullptr, *dN = nullptr;
    uint32_t* dI = nullptr;
    int2* dInfo = nullptr;
    int *dLeafOf = nullptr, *dLights = nullptr, *dLightLeaf = nullptr;
    e = tup(&dV, d->vertices, (size_t)d->n_vertices * 3);
    if (e == cudaSuccess) e = tup(&dI, d->indices, (size_t)nt * 3);
    if (e == cudaSuccess && d->normals) e = tup(&dN, d->normals, (size_t)d->n_vertices * 3);
    if (e == cudaSuccess) e = tup(&dInfo, info.data(), info.size());
    uint32_t* dMtype = nullptr;
    if (e == cudaSuccess) e = tup(&dMtype, d->mat_type, d->n_materials);
    uint32_t* dTmed = nullptr;
    if (e == cudaSuccess && !tmed.empty()) e = tup(&dTmed, tmed.data(), tmed.size());
    if (e == cudaSuccess) e = tup(&dLeafOf, (const int*)nullptr, nt);
    if (e == cudaSuccess && n_area) e = tup(&dLights, light_tris.data(), light_tris.size());
    if (e == cudaSuccess && n_area) e = tup(&dLightLeaf, (const int*)nullptr, light_tris.size());
    if (e != cudaSuccess) return bail(cuda_code(e), std::string("scene_create: ") + cudaGetErrorString(e));
    GpuBvh g;
    GpuWideBvh gw;
    std::string berr;
    const int rc = use_wide ? build_wide_bvh_gpu(ctx->stream, dV, dI, nt, &gw, &berr)
                            : build_bvh_gpu(ctx->stream, dV, dI, nt, &g, &berr);
    if (rc) return bail(rc, "scene_create: " + berr);
    if (use_wide) {
      sc->allocs.push_back(gw.nodes);  // the scene owns the nodes
      tmp.push_back(gw.order);
      g.order = gw.order;
      sc->bytes += (uint64_t)gw.n_nodes * 80;
      if (gw.max_depth >= (uint32_t)kWStack)
        return bail(GYT_ERR_UNSUPPORTED, "scene_create: BVH deeper than the traversal stack");
    } else {
      sc->allocs.push_back(g.nodes);
      tmp.push_back(g.order);
      sc->bytes += (uint64_t)g.n_slots * 64;
      if (g.max_depth >= (uint32_t)kBStack)
        return bail(GYT_ERR_UNSUPPORTED, "scene_create: BVH deeper than the traversal stack");
    }
    float4 *dtris = nullptr, *dn = nullptr;
    e = dalloc(sc->allocs, &dtris, (size_t)nt * 3);
    if (e == cudaSuccess) e = dalloc(sc->allocs, &dn, (size_t)nt * 3);
    if (e != cudaSuccess) return bail(cuda_code(e), std::string("scene_create: ") + cudaGetErrorString(e));
    sc->bytes += (uint64_t)nt * 3 * 2 * sizeof(float4);
    k_leaf_data<<<(nt + 255) / 256, 256, 0, ctx->stream>>>(nt, g.order, dV, dI, dN, dInfo, dTmed, dMtype, dtris, dn,
                                                               dLeafOf);
    if (n_area)
      k_gather_int<<<(n_area + 255) / 256, 256, 0, ctx->stream>>>((uint32_t)n_area, dLights, dLeafOf, dLightLeaf);
    e = cudaGetLastError();
    if (e == cudaSuccess && n_area)
      e = cudaMemcpyAsync(light_leaf.data(), dLightLeaf, n_area * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return bail(cuda_code(e), std::string("scene_create: ") + cudaGetErrorString(e));
    ds.nodes = use_wide ? nullptr : g.nodes;
    ds.wnodes = use_wide ? gw.nodes : nullptr;
    ds.tris = dtris;
    ds.tnrm = dn;
    sc->n_nodes = use_wide ? gw.n_nodes : g.n_inner;
    sc->n_slots = use_wide ? 0 : g.n_slots;
    sc->bvh_depth = use_wide ? gw.max_depth : g.max_depth;
  } else {
    WideBvhHost wide;
    BvhHost bin;
    if (use_wide) {
      if (!build_wide_bvh_host(d->vertices, d->n_vertices, d->indices, d->n_triangles, &wide))
        return bail(GYT_ERR_INVALID, "scene_create: BVH build failed");
      if (wide.max_depth >= (uint32_t)kWStack)
        return bail(GYT_ERR_UNSUPPORTED, "scene_create: BVH deeper than the traversal stack");
    } else {
      if (!build_bvh_host(d->vertices, d->n_vertices, d->indices, d->n_triangles, &bin))
        return bail(GYT_ERR_INVALID, "scene_create: BVH build failed");
      if (bin.max_depth >= (uint32_t)kBStack)
        return bail(GYT_ERR_UNSUPPORTED, "scene_create: BVH deeper than the traversal stack");
    }
    const std::vector<uint32_t>& order = use_wide ? wide.order : bin.order;
    // leaf-order triangle positions and shading data
    std::vector<float4> tris((size_t)order.size() * 3), tnrm((size_t)order.size() * 3);
    std::vector<int> leaf_of(d->n_triangles, -1);
    for (size_t k = 0; k < order.size(); ++k) {
      uint32_t t = order[k];
      leaf_of[t] = (int)k;
      const uint32_t* I = &d->indices[3 * t];
      float3 p[3] = {vtx(I[0]), vtx(I[1]), vtx(I[2])};
      float3 face = norm(cross(p[1] - p[0], p[2] - p[0]));
      for (int c = 0; c < 3; ++c) {
        const int cls = (int)std::min(d->mat_type[info[t].x], 4u) + 1;
        tris[3 * k + c] = make_float4(p[c].x, p[c].y, p[c].z, c == 0 ? bits((int)t) : (c == 1 ? bits(cls) : 0.f));
        float3 n = d->normals ? mk(d->normals[3 * I[c]], d->normals[3 * I[c] + 1], d->normals[3 * I[c] + 2]) : face;
        uint32_t mw = tmed.empty() ? 0u : tmed[t];
        float w = c == 0 ? bits(info[t].x) : (c == 1 ? bits(info[t].y) : bits((int)mw));
        tnrm[3 * k + c] = make_float4(n.x, n.y, n.z, w);
      }
    }
    for (int li = 0; li < n_area; ++li) light_leaf[li] = leaf_of[light_tris[li]];
    if (use_wide) {
      uint4* nodes = nullptr;
      e = up(&nodes, (const uint4*)wide.nodes.data(), wide.nodes.size() / 4);
      ds.wnodes = nodes;
      ds.nodes = nullptr;
    } else {
      float4* nodes = nullptr;
      e = up(&nodes, (const float4*)bin.nodes.data(), bin.nodes.size() / 4);
      ds.nodes = nodes;
      ds.wnodes = nullptr;
    }
    float4* dtris = nullptr;
    if (e == cudaSuccess) e = up(&dtris, tris.data(), tris.size());
    ds.tris = dtris;
    float4* dn = nullptr;
    if (e == cudaSuccess) e = up(&dn, tnrm.data(), tnrm.size());
    ds.tnrm = dn;
    sc->n_nodes = use_wide ? wide.nodes.size() / 20 : bin.nodes.size() / 16;
    sc->n_slots = use_wide ? 0 : bin.nodes.size() / 16;
    sc->bvh_depth = use_wide ? wide.max_depth : bin.max_depth;
  }
  // light records: (p0, Le.r) (p1, Le.g) (p2, Le.b) (n0, area) (n1, leaf) (n2, id) (face, emission row)
  std::vector<float4> ltab((size_t)n_area * kLightRec);
  for (int li = 0; li < n_area; ++li) {
    const int t = light_tris[li];
    const int k = light_leaf[li];
    const uint32_t* I = &d->indices[3 * t];
    const float* em = &d->emission[3 * d->tri_emission[t]];
    float3 p0 = vtx(I[0]), p1 = vtx(I[1]), p2 = vtx(I[2]);
    float area = 0.5f * length(cross(p1 - p0, p2 - p0));
    float3 face = norm(cross(p1 - p0, p2 - p0));
    float3 nc[3];
    for (int c = 0; c < 3; ++c)
      nc[c] = d->normals ? mk(d->normals[3 * I[c]], d->normals[3 * I[c] + 1], d->normals[3 * I[c] + 2]) : face;
    float4* r = &ltab[(size_t)li * kLightRec];
    r[0] = make_float4(p0.x, p0.y, p0.z, em[0]);
    r[1] = make_float4(p1.x, p1.y, p1.z, em[1]);
    r[2] = make_float4(p2.x, p2.y, p2.z, em[2]);
    r[3] = make_float4(nc[0].x, nc[0].y, nc[0].z, area);
    r[4] = make_float4(nc[1].x, nc[1].y, nc[1].z, bits(k));
    r[5] = make_float4(nc[2].x, nc[2].y, nc[2].z, bits(t));
    r[6] = make_float4(face.x, face.y, face.z, bits(d->tri_emission[t]));
  }
  std::vector<float4> sph(d->n_spheres);
  for (uint32_t k = 0; k < d->n_spheres; ++k)
    sph[k] = make_float4(d->spheres[4 * k], d->spheres[4 * k + 1], d->spheres[4 * k + 2], d->spheres[4 * k + 3]);
  float4* dsph = nullptr;
  if (e == cudaSuccess) e = up(&dsph, sph.data(), sph.size());
  ds.spheres = dsph;
  uint32_t* smat = nullptr;
  if (e == cudaSuccess) e = up(&smat, d->sphere_material, d->n_spheres);
  ds.sphere_mat = smat;
  float* mp = nullptr;
  if (e == cudaSuccess) e = up(&mp, d->mat_params, (size_t)d->n_materials * 16);
  ds.mparams = mp;
  uint32_t* mt = nullptr;
  if (e == cudaSuccess) e = up(&mt, d->mat_type, d->n_materials);
  ds.mtypes = mt;
  float4* dl = nullptr;
  if (e == cudaSuccess) e = up(&dl, ltab.data(), ltab.size());
  ds.ltab = dl;
  float* dc = nullptr;
  if (e == cudaSuccess) e = up(&dc, cdf.data(), cdf.size());
  ds.lcdf = dc;
  float* df = nullptr;
  if (e == cudaSuccess) e = up(&df, power.data(), power.size());
  ds.lfunc = df;
  ds.lfunc_int = fint;
  ds.n_lights = nl;
  ds.n_area = n_area;
  ds.media = nullptr;
  ds.n_media = (int)d->n_media;
  if (d->n_media) {
    std::vector<float4> mrec(2 * (size_t)d->n_media);
    for (uint32_t k = 0; k < d->n_media; ++k) {
      const float* q = &d->media[7 * (size_t)k];
      mrec[2 * k] = make_float4(q[0], q[1], q[2], q[6]);
      mrec[2 * k + 1] = make_float4(q[3], q[4], q[5], 0.f);
    }
    float4* dm = nullptr;
    if (e == cudaSuccess) e = up(&dm, mrec.data(), mrec.size());
    ds.media = dm;
  }
  ds.has_env = has_env ? 1 : 0;
  if (has_env) {
    EnvDev& ev = ds.env;
    float4* et = nullptr;
    float *cc = nullptr, *cf = nullptr, *ci = nullptr, *mc = nullptr, *mf = nullptr;
    if (e == cudaSuccess) e = up(&et, env_tex.data(), env_tex.size());
    if (e == cudaSuccess) e = up(&cc, env_ccdf.data(), env_ccdf.size());
    if (e == cudaSuccess) e = up(&cf, env_cfunc.data(), env_cfunc.size());
    if (e == cudaSuccess) e = up(&ci, env_cint.data(), env_cint.size());
    if (e == cudaSuccess) e = up(&mc, env_mcdf.data(), env_mcdf.size());
    if (e == cudaSuccess) e = up(&mf, env_mfunc.data(), env_mfunc.size());
    ev.tex = et; ev.ccdf = cc; ev.cfunc = cf; ev.cint = ci; ev.mcdf = mc; ev.mfunc = mf;
    ev.mint = env_mint;
    ev.w = (int)d->env_w;
    ev.h = (int)d->env_h;
    ev.scale = d->env_scale;
    ev.radius = env_radius;
  }
  ds.n_tris = (int)d->n_triangles;
  ds.n_spheres = (int)d->n_spheres;
  sc->n_tris = d->n_triangles;
  sc->n_materials = d->n_materials;
  sc->n_emission = d->n_emission;
  sc->ltab = ltab;
  sc->power = power;
  sc->light_area.resize(n_area);
  for (int li = 0; li < n_area; ++li) sc->light_area[li] = ltab[(size_t)li * kLightRec + 3].w;
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // uploads are ordered on the context stream
  if (e != cudaSuccess) {
    gyt_scene_destroy(sc);
    return fail(ctx, e == cudaErrorMemoryAllocation ? GYT_ERR_OUT_OF_MEMORY : GYT_ERR_CUDA,
                std::string("scene_create: ") + cudaGetErrorString(e));
  }
  *out = sc;
  return GYT_OK;
}

void gyt_scene_destroy(gyt_scene* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  for (void* p : s->allocs) cudaFree(p);
  delete s;
}

int32_t gyt_scene_info(const gyt_scene* s, uint64_t* nt, uint64_t* nn, uint64_t* bytes) {
  if (!s) return GYT_ERR_INVALID;
  if (nt) *nt = s->n_tris;
  if (nn) *nn = s->n_nodes;
  if (bytes) *bytes = s->bytes;
  return GYT_OK;
}

int32_t gyt_scene_set_materials(gyt_scene* s, const float* mat_params, const float* emission, uint32_t flags) {
  if (!s || !s->ctx) return GYT_ERR_INVALID;
  gyt_context* ctx = s->ctx;
  GYT_CK(ctx, cudaSetDevice(s->device));
  cudaStream_t st = ctx->stream;
  if (mat_params) {
    for (size_t k = 0; k < (size_t)s->n_materials * 16; ++k)
      if (!std::isfinite(mat_params[k])) return fail(ctx, GYT_ERR_INVALID, "set_materials: non-finite parameter");
    GYT_CK(ctx, cudaMemcpyAsync((void*)s->dev.mparams, mat_params, (size_t)s->n_materials * 16 * sizeof(float),
                                cudaMemcpyHostToDevice, st));
  }
  if (emission) {
    for (size_t k = 0; k < (size_t)s->n_emission * 3; ++k)
      if (!(emission[k] >= 0.f) || !std::isfinite(emission[k]))
        return fail(ctx, GYT_ERR_INVALID, "set_materials: emission must be finite and >= 0");
    const int n_area = s->dev.n_area;
    for (int li = 0; li < n_area; ++li) {
      float4* r = &s->ltab[(size_t)li * kLightRec];
      int row;
      std::memcpy(&row, &r[6].w, 4);
      const float* em = emission + 3 * (size_t)row;
      r[0].w = em[0];
      r[1].w = em[1];
      r[2].w = em[2];
      s->power[li] = area_light_power(em, s->light_area[li]);
    }
    if (n_area)
      GYT_CK(ctx, cudaMemcpyAsync((void*)s->dev.ltab, s->ltab.data(), s->ltab.size() * sizeof(float4),
                                  cudaMemcpyHostToDevice, st));
    std::vector<float> cdf;
    const float fint = light_distribution(s->power, &cdf);
    if (!s->power.empty() && !(flags & GYT_KEEP_LIGHT_SAMPLING)) {
      GYT_CK(ctx, cudaMemcpyAsync((void*)s->dev.lcdf, cdf.data(), cdf.size() * sizeof(float), cudaMemcpyHostToDevice, st));
      GYT_CK(ctx, cudaMemcpyAsync((void*)s->dev.lfunc, s->power.data(), s->power.size() * sizeof(float),
                                  cudaMemcpyHostToDevice, st));
      s->dev.lfunc_int = fint;
    }
  }
  GYT_CK(ctx, cudaStreamSynchronize(st));
  return GYT_OK;
}

int32_t gyt_scene_freeze_sampling(gyt_scene* s, const float* mat_params) {
  if (!s || !s->ctx) return GYT_ERR_INVALID;
  gyt_context* ctx = s->ctx;
  GYT_CK(ctx, cudaSetDevice(s->device));
  if (!mat_params) {
    s->dev.sparams = nullptr;
    return GYT_OK;
  }
  const size_t nf = (size_t)s->n_materials * 16;
  for (size_t k = 0; k < nf; ++k)
    if (!std::isfinite(mat_params[k])) return fail(ctx, GYT_ERR_INVALID, "freeze_sampling: non-finite parameter");
  if (!s->sparams_buf) {
    float* p = nullptr;
    GYT_CK(ctx, dalloc(s->allocs, &p, nf));
    s->sparams_buf = p;
  }
  GYT_CK(ctx, cudaMemcpyAsync(s->sparams_buf, mat_params, nf * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  s->dev.sparams = s->sparams_buf;
  return GYT_OK;
}

int32_t gyt_scene_read_bvh(const gyt_scene* s, float* nodes, uint64_t node_capacity, uint32_t* tri_ids,
                           uint64_t tri_capacity, uint64_t* n_slots) {
  if (!s || !n_slots) return GYT_ERR_INVALID;
  gyt_context* ctx = s->ctx;
  if (!s->dev.nodes && s->n_tris) return fail(ctx, GYT_ERR_UNSUPPORTED, "read_bvh: not a binary BVH");
  *n_slots = s->n_slots;
  if (!nodes) return GYT_OK;
  if (node_capacity < s->n_slots * 16 || (tri_ids && tri_capacity < s->n_tris))
    return fail(ctx, GYT_ERR_INVALID, "read_bvh: output arrays too small");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  if (s->n_slots) GYT_CK(ctx, cudaMemcpy(nodes, s->dev.nodes, s->n_slots * 64, cudaMemcpyDeviceToHost));
  if (tri_ids && s->n_tris) {
    std::vector<float4> t0((size_t)s->n_tris * 3);
    GYT_CK(ctx, cudaMemcpy(t0.data(), s->dev.tris, t0.size() * sizeof(float4), cudaMemcpyDeviceToHost));
    for (uint64_t k = 0; k < s->n_tris; ++k) std::memcpy(&tri_ids[k], &t0[3 * k].w, 4);
  }
  return GYT_OK;
}

int32_t gyt_scene_read_wide_bvh(const gyt_scene* s, uint32_t* words, uint64_t word_capacity, uint32_t* tri_ids,
                                uint64_t tri_capacity, uint64_t* n_nodes) {
  if (!s || !n_nodes) return GYT_ERR_INVALID;
  gyt_context* ctx = s->ctx;
  if (!s->dev.wnodes && s->n_tris) return fail(ctx, GYT_ERR_UNSUPPORTED, "read_wide_bvh: not an 8-wide BVH");
  const uint64_t n = s->dev.wnodes ? s->n_nodes : 0;
  *n_nodes = n;
  if (!words) return GYT_OK;
  if (word_capacity < n * 20 || (tri_ids && tri_capacity < s->n_tris))
    return fail(ctx, GYT_ERR_INVALID, "read_wide_bvh: output arrays too small");
  GYT_CK(ctx, cudaSetDevice(s->device));
  if (n) GYT_CK(ctx, cudaMemcpy(words, s->dev.wnodes, n * 80, cudaMemcpyDeviceToHost));
  if (tri_ids && s->n_tris) {
    std::vector<float4> t0((size_t)s->n_tris * 3);
    GYT_CK(ctx, cudaMemcpy(t0.data(), s->dev.tris, t0.size() * sizeof(float4), cudaMemcpyDeviceToHost));
    for (uint64_t k = 0; k < s->n_tris; ++k) std::memcpy(&tri_ids[k], &t0[3 * k].w, 4);
  }
  return GYT_OK;
}

int32_t gyt_render_device(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                          const GytRenderParams* params, double* d_film, GytRenderStats* stats) {
  if (!ctx || !scene || !d_film) return fail(ctx, GYT_ERR_INVALID, "render_device: null argument");
  int32_t st = check_params(ctx, params);
  if (st) return st;
  Cam cam;
  st = make_cam(ctx, camera, params, &cam);
  if (st) return st;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  unsigned long long total = (unsigned long long)camera->res_x * camera->res_y * params->spp;
  if (total >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "render: more than 2^32 paths in one render");
  return run_paths(ctx, scene, cam, params, total, nullptr, d_film, DebugOut{}, stats);
}

// The context's FP64 film and RGB staging buffers of the host-image renders
// (grown to the largest request, kept until the context is destroyed).
int32_t ensure_host_films(gyt_context* ctx, size_t fb, size_t rb) {
  if (fb > ctx->film_bytes) {
    cudaFree(ctx->d_film);
    ctx->d_film = nullptr;
    ctx->film_bytes = 0;
    GYT_CK(ctx, cudaMalloc((void**)&ctx->d_film, fb));
    ctx->film_bytes = fb;
  }
  if (rb > ctx->rgb_bytes) {
    cudaFree(ctx->d_rgb);
    ctx->d_rgb = nullptr;
    ctx->rgb_bytes = 0;
    GYT_CK(ctx, cudaMalloc((void**)&ctx->d_rgb, rb));
    ctx->rgb_bytes = rb;
  }
  return GYT_OK;
}

int32_t gyt_render(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera, const GytRenderParams* params,
                   float* rgb_out) {
  if (!ctx || !scene || !camera || !rgb_out) return fail(ctx, GYT_ERR_INVALID, "render: null argument");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  size_t npix = (size_t)camera->res_x * camera->res_y;
  size_t fb = npix * 4 * sizeof(double), rb = npix * 3 * sizeof(float);
  int32_t st0 = ensure_host_films(ctx, fb, rb);
  if (st0) return st0;
  GYT_CK(ctx, cudaMemsetAsync(ctx->d_film, 0, fb, ctx->stream));
  int32_t st = gyt_render_device(ctx, scene, camera, params, ctx->d_film, nullptr);
  if (st) return st;
  k_resolve<<<grid_for(npix), kBlock, 0, ctx->stream>>>(ctx->d_film, ctx->d_rgb, (uint32_t)npix);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaMemcpyAsync(rgb_out, ctx->d_rgb, rb, cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

int32_t gyt_render_light_tracing_device(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                        const GytRenderParams* params, double* d_splat, GytRenderStats* stats) {
  if (!ctx || !scene || !camera || !d_splat) return fail(ctx, GYT_ERR_INVALID, "light_tracing: null argument");
  return run_light_tracing(ctx, scene, camera, params, 0, nullptr, d_splat, nullptr, stats);
}

int32_t gyt_render_light_tracing(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                 const GytRenderParams* params, float* rgb_out) {
  if (!ctx || !scene || !camera || !rgb_out) return fail(ctx, GYT_ERR_INVALID, "light_tracing: null argument");
  const uint64_t npix = (uint64_t)camera->res_x * camera->res_y;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* q : v) cudaFree(q); }
  } guard{tmp};
  double* d = nullptr;
  float* f = nullptr;
  GYT_CK(ctx, dalloc(tmp, &d, 3 * std::max<uint64_t>(npix, 1)));
  GYT_CK(ctx, dalloc(tmp, &f, 3 * std::max<uint64_t>(npix, 1)));
  GYT_CK(ctx, cudaMemsetAsync(d, 0, 3 * npix * sizeof(double), ctx->stream));
  int32_t st = run_light_tracing(ctx, scene, camera, params, 0, nullptr, d, nullptr, nullptr);
  if (st) return st;
  k_splat_to_rgb<<<grid_for(3 * npix), kBlock, 0, ctx->stream>>>(d, f, 3 * npix);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaMemcpyAsync(rgb_out, f, 3 * npix * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

int32_t gyt_trace_light_paths(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                              const GytRenderParams* params, uint64_t n, const uint64_t* photons, float* records) {
  if (!ctx || !scene || !camera || (n && (!photons || !records)))
    return fail(ctx, GYT_ERR_INVALID, "trace_light_paths: null argument");
  if (n == 0) return GYT_OK;
  int32_t st = check_params(ctx, params);
  if (st) return st;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* q : v) cudaFree(q); }
  } guard{tmp};
  unsigned long long* di = nullptr;
  float* dr = nullptr;
  const uint64_t nrec = 6ull * params->max_depth * n;
  GYT_CK(ctx, dalloc(tmp, &di, n));
  GYT_CK(ctx, dalloc(tmp, &dr, nrec));
  GYT_CK(ctx, cudaMemcpyAsync(di, photons, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  st = run_light_tracing(ctx, scene, camera, params, n, di, nullptr, dr, nullptr);
  if (st) return st;
  GYT_CK(ctx, cudaMemcpyAsync(records, dr, nrec * 4, cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

int32_t gyt_render_volume_device(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                 const GytRenderParams* params, double* d_film, GytRenderStats* stats) {
  if (!ctx || !scene || !camera || !d_film) return fail(ctx, GYT_ERR_INVALID, "render_volume: null argument");
  return run_volume(ctx, scene, camera, params, 0, nullptr, d_film, nullptr, nullptr, stats);
}

int32_t gyt_render_volume(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                          const GytRenderParams* params, float* rgb_out) {
  if (!ctx || !scene || !camera || !rgb_out) return fail(ctx, GYT_ERR_INVALID, "render_volume: null argument");
  const uint64_t npix = (uint64_t)camera->res_x * camera->res_y;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* q : v) cudaFree(q); }
  } guard{tmp};
  double* d = nullptr;
  float* f = nullptr;
  GYT_CK(ctx, dalloc(tmp, &d, 4 * std::max<uint64_t>(npix, 1)));
  GYT_CK(ctx, dalloc(tmp, &f, 3 * std::max<uint64_t>(npix, 1)));
  GYT_CK(ctx, cudaMemsetAsync(d, 0, 4 * npix * sizeof(double), ctx->stream));
  int32_t st = run_volume(ctx, scene, camera, params, 0, nullptr, d, nullptr, nullptr, nullptr);
  if (st) return st;
  k_resolve<<<grid_for(npix), kBlock, 0, ctx->stream>>>(d, f, (uint32_t)npix);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaMemcpyAsync(rgb_out, f, 3 * npix * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

int32_t gyt_trace_volume_paths(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                               const GytRenderParams* params, uint64_t n, const uint32_t* xys, float* L_out,
                               uint32_t* cursor_out) {
  if (!ctx || !scene || !camera || (n && !xys)) return fail(ctx, GYT_ERR_INVALID, "trace_volume_paths: null argument");
  if (n == 0) return GYT_OK;
  for (uint64_t i = 0; i < n; ++i)
    if (xys[3 * i] >= camera->res_x || xys[3 * i + 1] >= camera->res_y)
      return fail(ctx, GYT_ERR_INVALID, "trace_volume_paths: pixel outside the film");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* q : v) cudaFree(q); }
  } guard{tmp};
  uint32_t *dx = nullptr, *dc = nullptr;
  float* dl = nullptr;
  GYT_CK(ctx, dalloc(tmp, &dx, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &dl, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &dc, n));
  GYT_CK(ctx, cudaMemcpyAsync(dx, xys, 3 * n * 4, cudaMemcpyHostToDevice, ctx->stream));
  int32_t st = run_volume(ctx, scene, camera, params, n, dx, nullptr, dl, dc, nullptr);
  if (st) return st;
  if (L_out) GYT_CK(ctx, cudaMemcpyAsync(L_out, dl, 3 * n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  if (cursor_out) GYT_CK(ctx, cudaMemcpyAsync(cursor_out, dc, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

int32_t gyt_mesh_load_obj(const char* path, int32_t reverse_vertices, gyt_mesh** out, char* err, uint32_t err_len) {
  auto report = [&](const std::string& m) {
    if (err && err_len) {
      std::strncpy(err, m.c_str(), err_len - 1);
      err[err_len - 1] = '\0';
    }
  };
  if (!path || !out) {
    report("mesh_load_obj: null argument");
    return GYT_ERR_INVALID;
  }
  *out = nullptr;
  auto* m = new gyt_mesh();
  std::string msg;
  if (!load_obj(path, reverse_vertices != 0, &m->mesh, &msg)) {
    delete m;
    report(msg);
    return GYT_ERR_INVALID;
  }
  *out = m;
  return GYT_OK;
}

int32_t gyt_mesh_size(const gyt_mesh* mesh, uint32_t* n_triangles) {
  if (!mesh || !n_triangles) return GYT_ERR_INVALID;
  *n_triangles = mesh->mesh.triangles();
  return GYT_OK;
}

int32_t gyt_mesh_read(const gyt_mesh* mesh, float* positions, float* normals, float* uvs) {
  if (!mesh) return GYT_ERR_INVALID;
  const ObjMesh& m = mesh->mesh;
  if (positions) std::memcpy(positions, m.pos.data(), m.pos.size() * sizeof(float));
  if (normals) std::memcpy(normals, m.nrm.data(), m.nrm.size() * sizeof(float));
  if (uvs) std::memcpy(uvs, m.uv.data(), m.uv.size() * sizeof(float));
  return GYT_OK;
}

int32_t gyt_mesh_transform(gyt_context* ctx, gyt_mesh* mesh, const float* matrix, const float* inverse) {
  if (!ctx || !mesh || !matrix || !inverse) return fail(ctx, GYT_ERR_INVALID, "mesh_transform: null argument");
  ObjMesh& m = mesh->mesh;
  const uint64_t nvert = 3ull * m.triangles();
  if (nvert == 0) return GYT_OK;
  if (nvert >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "mesh_transform: mesh too large");
  Xform t;
  std::memcpy(t.m, matrix, sizeof(t.m));
  std::memcpy(t.inv, inverse, sizeof(t.inv));
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* q : v) cudaFree(q); }
  } guard{tmp};
  float *dp = nullptr, *dn = nullptr;
  GYT_CK(ctx, dalloc(tmp, &dp, 3 * nvert));
  GYT_CK(ctx, dalloc(tmp, &dn, 3 * nvert));
  GYT_CK(ctx, cudaMemcpyAsync(dp, m.pos.data(), 3 * nvert * 4, cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemcpyAsync(dn, m.nrm.data(), 3 * nvert * 4, cudaMemcpyHostToDevice, ctx->stream));
  k_mesh_transform<<<grid_for(nvert), kBlock, 0, ctx->stream>>>(dp, dn, (uint32_t)nvert, t);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaMemcpyAsync(m.pos.data(), dp, 3 * nvert * 4, cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaMemcpyAsync(m.nrm.data(), dn, 3 * nvert * 4, cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

void gyt_mesh_destroy(gyt_mesh* mesh) { delete mesh; }

int32_t gyt_film_quantize(gyt_context* ctx, const double* d_film, uint32_t res_x, uint32_t res_y, float gamma,
                          uint8_t* rgb8_out) {
  if (!ctx || !d_film || !rgb8_out) return fail(ctx, GYT_ERR_INVALID, "film_quantize: null argument");
  if (!(gamma > 0.f)) return fail(ctx, GYT_ERR_INVALID, "film_quantize: gamma must be positive");
  const uint64_t npix = (uint64_t)res_x * res_y;
  if (npix == 0 || npix > kPixMask) return fail(ctx, GYT_ERR_INVALID, "film_quantize: bad film size");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* q : v) cudaFree(q); }
  } guard{tmp};
  uint8_t* d = nullptr;
  GYT_CK(ctx, dalloc(tmp, &d, 3 * npix));
  GYT_CK(ctx, after_legacy_stream(ctx));
  k_film_rgb8<<<grid_for(npix), kBlock, 0, ctx->stream>>>(d_film, d, (uint32_t)npix, 1.f / gamma);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaMemcpyAsync(rgb8_out, d, 3 * npix, cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

int32_t gyt_film_save(gyt_context* ctx, const double* d_film, uint32_t res_x, uint32_t res_y, const char* path) {
  if (!ctx || !d_film || !path) return fail(ctx, GYT_ERR_INVALID, "film_save: null argument");
  const std::string name(path);
  const std::string suffix = name.size() >= 4 ? name.substr(name.size() - 4) : std::string();
  if (suffix != ".png" && suffix != ".bmp" && suffix != ".hdr")
    return fail(ctx, GYT_ERR_INVALID, "film_save: the file name must end in .png, .bmp or .hdr");
  const uint64_t npix = (uint64_t)res_x * res_y;
  if (npix == 0 || npix > kPixMask) return fail(ctx, GYT_ERR_INVALID, "film_save: bad film size");
  std::vector<uint8_t> host;
  bool ok = false;
  if (suffix == ".hdr") {
    GYT_CK(ctx, cudaSetDevice(ctx->device));
    std::vector<void*> tmp;
    struct Guard {
      std::vector<void*>& v;
      ~Guard() { for (void* q : v) cudaFree(q); }
    } guard{tmp};
    uint8_t* d = nullptr;
    GYT_CK(ctx, dalloc(tmp, &d, 4 * npix));
    GYT_CK(ctx, after_legacy_stream(ctx));
    k_film_rgbe<<<grid_for(npix), kBlock, 0, ctx->stream>>>(d_film, d, (uint32_t)npix);
    GYT_CK(ctx, cudaGetLastError());
    host.resize(4 * npix);
    GYT_CK(ctx, cudaMemcpyAsync(host.data(), d, 4 * npix, cudaMemcpyDeviceToHost, ctx->stream));
    GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
    ok = write_hdr_rgbe(name, host.data(), res_x, res_y);
  } else {
    host.resize(3 * npix);
    // ImageIO::WriteImage's default gamma (image/ImageIO.h:47)
    const int32_t st = gyt_film_quantize(ctx, d_film, res_x, res_y, 2.2f, host.data());
    if (st) return st;
    ok = suffix == ".png" ? write_png_rgb8(name, host.data(), res_x, res_y)
                          : write_bmp_rgb8(name, host.data(), res_x, res_y);
  }
  if (!ok) return fail(ctx, GYT_ERR_INVALID, "film_save: cannot write " + name);
  return GYT_OK;
}

int32_t gyt_trace_paths(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                        const GytRenderParams* params, uint64_t n, const uint32_t* xys, float* L_out,
                        uint32_t* cursor_out, uint64_t* rr_out, uint64_t* occ_out, uint64_t* mis_out) {
  if (!ctx || !scene || !camera || (n && !xys)) return fail(ctx, GYT_ERR_INVALID, "trace_paths: null argument");
  int32_t st = check_params(ctx, params);
  if (st) return st;
  Cam cam;
  st = make_cam(ctx, camera, params, &cam);
  if (st) return st;
  if (n == 0) return GYT_OK;
  if (n >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "trace_paths: too many paths");
  for (uint64_t i = 0; i < n; ++i)
    if (xys[3 * i] >= camera->res_x || xys[3 * i + 1] >= camera->res_y)
      return fail(ctx, GYT_ERR_INVALID, "trace_paths: pixel outside the film");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* p : v) cudaFree(p); }
  } guard{tmp};
  uint32_t* dl = nullptr;
  float* dL = nullptr;
  uint32_t* dc = nullptr;
  unsigned long long* dm = nullptr;
  GYT_CK(ctx, dalloc(tmp, &dl, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &dL, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &dc, n));
  GYT_CK(ctx, dalloc(tmp, &dm, 3 * n));
  GYT_CK(ctx, cudaMemcpyAsync(dl, xys, 3 * n * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemsetAsync(dm, 0, 3 * n * sizeof(unsigned long long), ctx->stream));
  st = run_paths(ctx, scene, cam, params, n, dl, nullptr, DebugOut{dL, dc, dm, dm + n, dm + 2 * n}, nullptr);
  if (st) return st;
  if (L_out) GYT_CK(ctx, cudaMemcpy(L_out, dL, 3 * n * sizeof(float), cudaMemcpyDeviceToHost));
  if (cursor_out) GYT_CK(ctx, cudaMemcpy(cursor_out, dc, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (rr_out) GYT_CK(ctx, cudaMemcpy(rr_out, dm, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  if (occ_out) GYT_CK(ctx, cudaMemcpy(occ_out, dm + n, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  if (mis_out) GYT_CK(ctx, cudaMemcpy(mis_out, dm + 2 * n, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return GYT_OK;
}

int32_t gyt_diff_forward(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                         const GytRenderParams* params, double* d_film, float* d_path_L, GytRenderStats* stats) {
  if (!ctx || !scene || !d_film || !d_path_L) return fail(ctx, GYT_ERR_INVALID, "diff_forward: null argument");
  int32_t st = check_params(ctx, params);
  if (st) return st;
  Cam cam;
  st = make_cam(ctx, camera, params, &cam);
  if (st) return st;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  const unsigned long long total = (unsigned long long)camera->res_x * camera->res_y * params->spp;
  if (total >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "diff_forward: more than 2^32 paths");
  return run_paths(ctx, scene, cam, params, total, nullptr, d_film, DebugOut{d_path_L, nullptr, nullptr, nullptr,
                                                                            nullptr}, stats);
}

int32_t gyt_diff_backward(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                          const GytRenderParams* params, const float* d_image_grad, const double* d_film,
                          const float* d_path_L, double* d_grad_mat, double* d_grad_em, GytRenderStats* stats) {
  if (!ctx || !scene || !d_image_grad || !d_film || !d_path_L || !d_grad_mat || (scene->n_emission && !d_grad_em))
    return fail(ctx, GYT_ERR_INVALID, "diff_backward: null argument");
  int32_t st = check_params(ctx, params);
  if (st) return st;
  Cam cam;
  st = make_cam(ctx, camera, params, &cam);
  if (st) return st;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  const unsigned long long total = (unsigned long long)camera->res_x * camera->res_y * params->spp;
  if (total >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "diff_backward: more than 2^32 paths");
  const AdjIn in{d_image_grad, d_film, nullptr, d_path_L};
  return run_adjoint(ctx, scene, cam, params, total, nullptr, in, GradOut{d_grad_mat, d_grad_em}, stats);
}

int32_t gyt_diff_backward_paths(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                const GytRenderParams* params, uint64_t n, const uint32_t* xys, const float* delta,
                                const float* L_total, double* grad_mat, double* grad_em) {
  if (!ctx || !scene || !camera || !grad_mat || (scene->n_emission && !grad_em) ||
      (n && (!xys || !delta || !L_total)))
    return fail(ctx, GYT_ERR_INVALID, "diff_backward_paths: null argument");
  int32_t st = check_params(ctx, params);
  if (st) return st;
  Cam cam;
  st = make_cam(ctx, camera, params, &cam);
  if (st) return st;
  if (n >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "diff_backward_paths: too many paths");
  for (uint64_t i = 0; i < n; ++i)
    if (xys[3 * i] >= camera->res_x || xys[3 * i + 1] >= camera->res_y)
      return fail(ctx, GYT_ERR_INVALID, "diff_backward_paths: pixel outside the film");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() {
      for (void* p : v) cudaFree(p);
    }
  } guard{tmp};
  const size_t nm = (size_t)scene->n_materials * 4, ne = (size_t)scene->n_emission * 3;
  uint32_t* dl = nullptr;
  float *dd = nullptr, *dL = nullptr;
  double *gm = nullptr, *ge = nullptr;
  GYT_CK(ctx, dalloc(tmp, &dl, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &dd, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &dL, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &gm, nm));
  GYT_CK(ctx, dalloc(tmp, &ge, ne));
  GYT_CK(ctx, cudaMemcpyAsync(dl, xys, 3 * n * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemcpyAsync(dd, delta, 3 * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemcpyAsync(dL, L_total, 3 * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemsetAsync(gm, 0, nm * sizeof(double), ctx->stream));
  GYT_CK(ctx, cudaMemsetAsync(ge, 0, std::max<size_t>(ne, 1) * sizeof(double), ctx->stream));
  if (n) {
    const AdjIn in{nullptr, nullptr, dd, dL};
    st = run_adjoint(ctx, scene, cam, params, n, dl, in, GradOut{gm, ge}, nullptr);
    if (st) return st;
  }
  GYT_CK(ctx, cudaMemcpyAsync(grad_mat, gm, nm * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (ne) GYT_CK(ctx, cudaMemcpyAsync(grad_em, ge, ne * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

int32_t gyt_intersect(gyt_context* ctx, const gyt_scene* scene, uint64_t n, const float* rays, int32_t any_hit,
                      int32_t* prim, float* t, float* b1, float* b2) {
  if (!ctx || !scene || (n && !rays)) return fail(ctx, GYT_ERR_INVALID, "intersect: null argument");
  if (n == 0) return GYT_OK;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* p : v) cudaFree(p); }
  } guard{tmp};
  float* dr = nullptr;
  int32_t* dp = nullptr;
  float *dt = nullptr, *d1 = nullptr, *d2 = nullptr;
  GYT_CK(ctx, dalloc(tmp, &dr, 7 * n));
  GYT_CK(ctx, dalloc(tmp, &dp, n));
  GYT_CK(ctx, dalloc(tmp, &dt, n));
  GYT_CK(ctx, dalloc(tmp, &d1, n));
  GYT_CK(ctx, dalloc(tmp, &d2, n));
  GYT_CK(ctx, cudaMemcpyAsync(dr, rays, 7 * n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  if (scene->dev.wnodes)
    k_intersect<8><<<grid_for(n), kBlock, 0, ctx->stream>>>(scene->dev, n, dr, any_hit ? 1 : 0, dp, dt, d1, d2);
  else
    k_intersect<2><<<grid_for(n), kBlock, 0, ctx->stream>>>(scene->dev, n, dr, any_hit ? 1 : 0, dp, dt, d1, d2);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  if (prim) GYT_CK(ctx, cudaMemcpy(prim, dp, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (!any_hit) {
    if (t) GYT_CK(ctx, cudaMemcpy(t, dt, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (b1) GYT_CK(ctx, cudaMemcpy(b1, d1, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (b2) GYT_CK(ctx, cudaMemcpy(b2, d2, n * sizeof(float), cudaMemcpyDeviceToHost));
  }
  return GYT_OK;
}

int32_t gyt_sobol(gyt_context* ctx, uint64_t n, const uint32_t* dims, const uint64_t* indices, float* out) {
  if (!ctx || (n && (!dims || !indices || !out))) return fail(ctx, GYT_ERR_INVALID, "sobol: null argument");
  if (n == 0) return GYT_OK;
  for (uint64_t i = 0; i < n; ++i)
    if (dims[i] >= GYT_SOBOL_DIMS) return fail(ctx, GYT_ERR_INVALID, "sobol: dimension >= 1024");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* p : v) cudaFree(p); }
  } guard{tmp};
  uint32_t* dd = nullptr;
  uint64_t* di = nullptr;
  float* dout = nullptr;
  GYT_CK(ctx, dalloc(tmp, &dd, n));
  GYT_CK(ctx, dalloc(tmp, &di, n));
  GYT_CK(ctx, dalloc(tmp, &dout, n));
  GYT_CK(ctx, cudaMemcpyAsync(dd, dims, n * 4, cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemcpyAsync(di, indices, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  k_sobol<<<grid_for(n), kBlock, 0, ctx->stream>>>(ctx->d_sobol, n, dd, di, dout);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  GYT_CK(ctx, cudaMemcpy(out, dout, n * 4, cudaMemcpyDeviceToHost));
  return GYT_OK;
}

int32_t gyt_bsdf_table(gyt_context* ctx, uint64_t n, const uint32_t* types, const float* params, const float* vec,
                       float* out) {
  if (!ctx || (n && (!types || !params || !vec || !out))) return fail(ctx, GYT_ERR_INVALID, "bsdf_table: null argument");
  if (n == 0) return GYT_OK;
  if (n >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "bsdf_table: more than 2^32 cases");
  for (uint64_t i = 0; i < n; ++i)
    if (types[i] > GYT_MAT_DIELECTRIC) return fail(ctx, GYT_ERR_INVALID, "bsdf_table: unknown material kind");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* p : v) cudaFree(p); }
  } guard{tmp};
  uint32_t* dt = nullptr;
  float *dp = nullptr, *dv = nullptr, *dout = nullptr;
  GYT_CK(ctx, dalloc(tmp, &dt, n));
  GYT_CK(ctx, dalloc(tmp, &dp, 16 * n));
  GYT_CK(ctx, dalloc(tmp, &dv, 9 * n));
  GYT_CK(ctx, dalloc(tmp, &dout, 11 * n));
  GYT_CK(ctx, cudaMemcpyAsync(dt, types, n * 4, cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemcpyAsync(dp, params, 16 * n * 4, cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemcpyAsync(dv, vec, 9 * n * 4, cudaMemcpyHostToDevice, ctx->stream));
  k_bsdf_table<<<grid_for(n), kBlock, 0, ctx->stream>>>(n, dp, dt, dv, dout);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  GYT_CK(ctx, cudaMemcpy(out, dout, 11 * n * 4, cudaMemcpyDeviceToHost));
  return GYT_OK;
}

int32_t gyt_halton(gyt_context* ctx, uint64_t n, const uint32_t* dims, const uint64_t* indices, float* out) {
  if (!ctx || (n && (!dims || !indices || !out))) return fail(ctx, GYT_ERR_INVALID, "halton: null argument");
  if (n == 0) return GYT_OK;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* p : v) cudaFree(p); }
  } guard{tmp};
  uint32_t* dd = nullptr;
  uint64_t* di = nullptr;
  float* dout = nullptr;
  GYT_CK(ctx, dalloc(tmp, &dd, n));
  GYT_CK(ctx, dalloc(tmp, &di, n));
  GYT_CK(ctx, dalloc(tmp, &dout, n));
  GYT_CK(ctx, cudaMemcpyAsync(dd, dims, n * 4, cudaMemcpyHostToDevice, ctx->stream));
  GYT_CK(ctx, cudaMemcpyAsync(di, indices, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  k_halton<<<grid_for(n), kBlock, 0, ctx->stream>>>(tables(ctx), n, dd, di, dout);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  GYT_CK(ctx, cudaMemcpy(out, dout, n * 4, cudaMemcpyDeviceToHost));
  return GYT_OK;
}

int32_t gyt_halton_enum_index(gyt_context* ctx, uint32_t res_x, uint32_t res_y, uint64_t n, const uint32_t* sxy,
                              uint64_t* out) {
  if (!ctx || (n && (!sxy || !out))) return fail(ctx, GYT_ERR_INVALID, "halton_enum_index: null argument");
  GytCamera c = {};
  c.res_x = res_x;
  c.res_y = res_y;
  c.fovy = 53.13f;
  c.film_distance = 1.f;
  c.look_at[2] = -1.f;
  c.up[1] = 1.f;
  GytRenderParams prm = {1, 1, 0, GYT_SAMPLER_HALTON};
  Cam cam;
  int32_t st = make_cam(ctx, &c, &prm, &cam);
  if (st) return st;
  if (n == 0) return GYT_OK;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* q : v) cudaFree(q); }
  } guard{tmp};
  uint32_t* ds = nullptr;
  uint64_t* dout = nullptr;
  GYT_CK(ctx, dalloc(tmp, &ds, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &dout, n));
  GYT_CK(ctx, cudaMemcpyAsync(ds, sxy, 3 * n * 4, cudaMemcpyHostToDevice, ctx->stream));
  k_halton_enum<<<grid_for(n), kBlock, 0, ctx->stream>>>(cam, n, ds, dout);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  GYT_CK(ctx, cudaMemcpy(out, dout, n * 8, cudaMemcpyDeviceToHost));
  return GYT_OK;
}

int32_t gyt_sobol_enum_index(gyt_context* ctx, uint32_t res_x, uint32_t res_y, uint64_t n, const uint32_t* sxy,
                             uint64_t* out) {
  if (!ctx || (n && (!sxy || !out))) return fail(ctx, GYT_ERR_INVALID, "sobol_enum_index: null argument");
  uint32_t r = std::max(res_x, res_y), p = 1, m = 0;
  while (p < r) { p <<= 1; ++m; }
  if (m > GYT_ENUM_M) return fail(ctx, GYT_ERR_UNSUPPORTED, "sobol_enum_index: resolution too large");
  if (n == 0) return GYT_OK;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() { for (void* q : v) cudaFree(q); }
  } guard{tmp};
  uint32_t* ds = nullptr;
  uint64_t* dout = nullptr;
  GYT_CK(ctx, dalloc(tmp, &ds, 3 * n));
  GYT_CK(ctx, dalloc(tmp, &dout, n));
  GYT_CK(ctx, cudaMemcpyAsync(ds, sxy, 3 * n * 4, cudaMemcpyHostToDevice, ctx->stream));
  k_enum<<<grid_for(n), kBlock, 0, ctx->stream>>>(tables(ctx), m, n, ds, dout);
  GYT_CK(ctx, cudaGetLastError());
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  GYT_CK(ctx, cudaMemcpy(out, dout, n * 8, cudaMemcpyDeviceToHost));
  return GYT_OK;
}

int32_t gyt_camera_raster_to_world(const GytCamera* camera, double* out16) {
  if (!camera || !out16) return GYT_ERR_INVALID;
  raster_to_world(*camera, out16);
  return GYT_OK;
}

}  // extern "C"

// ------------------------------------------------------ no-alloc variant ---
// A render entry point for callers that must not allocate device memory while
// rendering: applications whose GPU memory is owned by another allocator or
// budget (a host engine's pool, a frame loop with a fixed memory plan) and
// code that runs where cudaMalloc is not allowed. Its path pools, queues and
// compaction counter live in the file-scope array below instead of the
// context's lazily allocated pools.
//
// The array is reserved once per device when the library's module is loaded
// on that device and held until the process exits. All calls on a device
// share it and it keeps whatever the last call left; only the compaction
// counter must start at zero and it is cleared every iteration. Two calls
// whose work overlaps on the GPU (different streams or threads) race on the
// array.
// ------------------------------------------------------ batched renders ---
namespace {

struct BatchPlan {
  int W = 2;
  int sampler = -1;  // 0 / 1: every instance samples with Sobol' / Halton (the shade kernel compiled for it)
  uint32_t stride_grid = 0, ext_grid = 0, sh_grid = 0, shade_grid = 0;
};

BatchPlan batch_plan(const gyt_context* ctx, int W, int sampler) {
  BatchPlan b;
  b.W = W;
  b.sampler = sampler;
  const GytBatchConfig& c = ctx->bcfg;
  const int wi = W == 8 ? 1 : 0;
  const uint32_t sms = (uint32_t)std::max(1, ctx->sms);
  b.stride_grid = sms * (c.stride_blocks_per_sm ? c.stride_blocks_per_sm : 8u);
  const uint32_t te = c.trace_blocks_per_sm ? std::min<uint32_t>(c.trace_blocks_per_sm, ctx->btrace[wi][0])
                                            : (uint32_t)ctx->btrace[wi][0];
  const uint32_t ts = c.trace_blocks_per_sm ? std::min<uint32_t>(c.trace_blocks_per_sm, ctx->btrace[wi][1])
                                            : (uint32_t)ctx->btrace[wi][1];
  b.ext_grid = sms * std::max(1u, te);
  b.sh_grid = sms * std::max(1u, ts);
  b.shade_grid = grid_for(ctx->capacity);
  return b;
}

// One half-iteration of the batched wavefront: pool P (current) to N (next).
// ev (profiling, host loop only): six events around generate, extend, shade,
// connect and finish.
cudaError_t enqueue_half(gyt_context* ctx, const BatchPlan& b, const PathBuf& P, const PathBuf& N,
                         cudaGraphConditionalHandle cond, int in_graph, cudaEvent_t* ev = nullptr) {
  cudaStream_t s = ctx->stream;
  const Queues q = ctx->q;
  const SamplerTables tab = tables(ctx);
  IterState* st = ctx->d_iter;
  k_batch_begin<<<1, 32, 0, s>>>(st, q.counts);
  if (ev) cudaEventRecord(ev[0], s);
  k_generate_batch<<<b.stride_grid, kBlock, 0, s>>>(P, st, tab);
  if (ev) cudaEventRecord(ev[1], s);
  if (b.W == 8) k_extend_batch<8><<<b.ext_grid, kBlock, 0, s>>>(P, st, q.hit, q.counts + 2);
  else k_extend_batch<2><<<b.ext_grid, kBlock, 0, s>>>(P, st, q.hit, q.counts + 2);
  if (ev) cudaEventRecord(ev[2], s);
  if (b.sampler == 0) k_shade_batch<0><<<b.shade_grid, kBlock, 0, s>>>(P, st, q, tab);
  else if (b.sampler == 1) k_shade_batch<1><<<b.shade_grid, kBlock, 0, s>>>(P, st, q, tab);
  else k_shade_batch<-1><<<b.shade_grid, kBlock, 0, s>>>(P, st, q, tab);
  if (ev) cudaEventRecord(ev[3], s);
  if (b.W == 8) k_connect_batch<8><<<b.sh_grid, kBlock, 0, s>>>(P, q);
  else k_connect_batch<2><<<b.sh_grid, kBlock, 0, s>>>(P, q);
  if (ev) cudaEventRecord(ev[4], s);
  k_finish_batch<<<b.shade_grid, kBlock, 0, s>>>(P, N, st, q.counts + 5, q.madd);
  if (ev) cudaEventRecord(ev[5], s);
  k_batch_end<<<1, 32, 0, s>>>(st, q.counts, cond, in_graph);
  return cudaGetLastError();
}
constexpr uint32_t kKernelsPerHalf = 7;

// The batched render as one graph: a while-loop node whose body is two
// half-iterations (pool 0 -> 1 -> 0); k_batch_end sets the loop condition.
int32_t ensure_batch_graph(gyt_context* ctx, const BatchPlan& b) {
  const uint64_t key[6] = {(uint64_t)b.W | ((uint64_t)(b.sampler + 1) << 8), (uint64_t)b.stride_grid,
                           ((uint64_t)b.ext_grid << 32) | b.sh_grid, (uint64_t)b.shade_grid,
                           (uint64_t)(uintptr_t)ctx->pool[0].o, (uint64_t)ctx->pool_cap};
  if (ctx->bexec && std::memcmp(key, ctx->bkey, sizeof(key)) == 0) return GYT_OK;
  if (ctx->bexec) cudaGraphExecDestroy(ctx->bexec);
  if (ctx->bgraph) cudaGraphDestroy(ctx->bgraph);
  ctx->bexec = nullptr;
  ctx->bgraph = nullptr;
  cudaGraph_t g = nullptr;
  GYT_CK(ctx, cudaGraphCreate(&g, 0));
  ctx->bgraph = g;
  cudaGraphConditionalHandle cond;
  GYT_CK(ctx, cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = cond;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  GYT_CK(ctx, cudaGraphAddNode(&node, g, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  GYT_CK(ctx, cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = enqueue_half(ctx, b, ctx->pool[0], ctx->pool[1], cond, 1);
  if (e == cudaSuccess) e = enqueue_half(ctx, b, ctx->pool[1], ctx->pool[0], cond, 1);
  cudaGraph_t captured = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &captured);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    cudaGetLastError();
    return fail(ctx, GYT_ERR_CUDA, std::string("batch graph capture: ") +
                                       cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  cudaGraphExec_t ex = nullptr;
  GYT_CK(ctx, cudaGraphInstantiate(&ex, g, 0));
  ctx->bexec = ex;
  std::memcpy(ctx->bkey, key, sizeof(key));
  return GYT_OK;
}

struct BatchInput {
  std::vector<Inst> insts;
  unsigned long long total = 0;
  uint32_t max_depth = 0;
  int W = 2;
};

int32_t batch_input(gyt_context* ctx, uint32_t n, const gyt_scene* const* scenes, const GytCamera* cameras,
                    const GytRenderParams* params, double* const* films, BatchInput* in) {
  if (n && (!scenes || !cameras || !params || !films)) return fail(ctx, GYT_ERR_INVALID, "batch: null array");
  in->insts.resize(n);
  in->total = 0;
  in->max_depth = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const gyt_scene* sc = scenes[i];
    if (!sc || !films[i]) return fail(ctx, GYT_ERR_INVALID, "batch: null scene or film at " + std::to_string(i));
    if (sc->device != ctx->device)
      return fail(ctx, GYT_ERR_INVALID, "batch: scene " + std::to_string(i) + " lives on another device");
    const int W = sc->dev.wnodes ? 8 : 2;
    if (i == 0) in->W = W;
    else if (W != in->W) return fail(ctx, GYT_ERR_UNSUPPORTED, "batch: scenes of different BVH widths");
    if (sc->dev.sparams)
      return fail(ctx, GYT_ERR_UNSUPPORTED, "batch: scene " + std::to_string(i) + " has frozen BSDF sampling");
    int32_t st = check_params(ctx, &params[i]);
    if (st) return st;
    Inst& I = in->insts[i];
    st = make_cam(ctx, &cameras[i], &params[i], &I.cam);
    if (st) return st;
    const unsigned long long np = (unsigned long long)cameras[i].res_x * cameras[i].res_y * params[i].spp;
    if (np >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "batch: more than 2^32 paths in one instance");
    I.s = sc->dev;
    I.prm = make_params(&params[i]);
    I.film = films[i];
    I.first = in->total;
    in->total += np;
    in->max_depth = std::max(in->max_depth, params[i].max_depth);
  }
  return GYT_OK;
}

// Runs a prepared batch: per group of at most kMaxBatch instances, the
// instance table to constant memory and the loop state to the device, then
// the graph (or the host loop); timed with events on the context stream. The
// constant table is shared by every context of the process, so batched
// renders are serialised.
std::mutex g_batch_mutex;

int32_t run_batch(gyt_context* ctx, const BatchInput& in, GytRenderStats* stats) {
  const uint32_t n = (uint32_t)in.insts.size();
  if (stats) *stats = GytRenderStats{};
  if (n == 0 || in.total == 0) return GYT_OK;
  if (ctx->bcfg.paths_in_flight && ctx->bcfg.paths_in_flight != ctx->capacity) {
    if (ctx->bcfg.paths_in_flight < 1024) return fail(ctx, GYT_ERR_INVALID, "batch: paths_in_flight below 1024");
    ctx->capacity = ctx->bcfg.paths_in_flight;
  }
  int32_t st = ensure_pool(ctx);
  if (st) return st;
  int sampler = in.insts.empty() ? 0 : (int)in.insts[0].prm.sampler;
  for (const Inst& I : in.insts)
    if ((int)I.prm.sampler != sampler) sampler = -1;
  const BatchPlan b = batch_plan(ctx, in.W, sampler);
  std::lock_guard<std::mutex> lock(g_batch_mutex);
  // profiling (gyt_context_set_profile) times every kernel: host loop
  const bool prof = ctx->profile > 0;
  const bool graph = ctx->bcfg.use_graph && !prof;
  if (graph) {
    st = ensure_batch_graph(ctx, b);
    if (st) return st;
  }
  cudaStream_t s = ctx->stream;
  GYT_CK(ctx, after_legacy_stream(ctx));
  GYT_CK(ctx, cudaEventRecord(ctx->ev0, s));
  uint32_t halves = 0;
  for (uint32_t g0 = 0; g0 < n; g0 += kMaxBatch) {
    const uint32_t m = std::min(n - g0, kMaxBatch);
    std::vector<Inst> grp(in.insts.begin() + g0, in.insts.begin() + g0 + m);
    const unsigned long long base = grp[0].first;
    const unsigned long long end = g0 + m < n ? in.insts[g0 + m].first : in.total;
    for (Inst& I : grp) I.first -= base;
    GYT_CK(ctx, cudaMemcpyToSymbolAsync(c_insts, grp.data(), m * sizeof(Inst), 0, cudaMemcpyHostToDevice, s));
    IterState is = {};
    is.total = end - base;
    is.n_inst = m;
    is.capacity = ctx->capacity;
    // a path holds a slot for at most max_depth half-iterations and a full
    // pool retires at least one slot per half-iteration: generous bound
    const unsigned long long bound = wavefront_bound(is.total, in.max_depth, ctx->capacity);
    is.max_iter = (uint32_t)std::min<unsigned long long>(bound, 1u << 30);
    *ctx->h_iter = is;
    GYT_CK(ctx, cudaMemcpyAsync(ctx->d_iter, ctx->h_iter, sizeof(IterState), cudaMemcpyHostToDevice, s));
    if (graph) {
      GYT_CK(ctx, cudaGraphLaunch(ctx->bexec, s));
    } else if (prof) {
      // one half at a time, every kernel between events; profile slots as
      // gyt_render_device fills them (3 = connect, 4 unused)
      for (int half = 0;; half ^= 1) {
        GYT_CK(ctx, enqueue_half(ctx, b, ctx->pool[half], ctx->pool[half ^ 1], 0, 0, ctx->kev));
        GYT_CK(ctx, cudaMemcpyAsync(ctx->h_counter, ctx->q.counts, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        GYT_CK(ctx, cudaMemcpyAsync(ctx->h_iter, ctx->d_iter, sizeof(IterState), cudaMemcpyDeviceToHost, s));
        GYT_CK(ctx, cudaStreamSynchronize(s));
        const IterState& h = *ctx->h_iter;
        static const int slot[5] = {0, 1, 2, 3, 5};
        for (int k = 0; k < 5; ++k) {
          float ms = 0.f;
          cudaEventElapsedTime(&ms, ctx->kev[k], ctx->kev[k + 1]);
          ctx->prof.ms[slot[k]] += ms;
          ctx->prof.launches[slot[k]]++;
        }
        ctx->prof.rays[0] += h.n;
        ctx->prof.rays[1] += ctx->h_counter[0];
        ctx->prof.rays[2] += ctx->h_counter[1];
        if (h.watchdog || !(h.generated < h.total || h.active > 0)) break;
        if (h.iter >= h.max_iter) break;
      }
    } else {
      for (;;) {
        GYT_CK(ctx, enqueue_half(ctx, b, ctx->pool[0], ctx->pool[1], 0, 0));
        GYT_CK(ctx, enqueue_half(ctx, b, ctx->pool[1], ctx->pool[0], 0, 0));
        GYT_CK(ctx, cudaMemcpyAsync(ctx->h_iter, ctx->d_iter, sizeof(IterState), cudaMemcpyDeviceToHost, s));
        GYT_CK(ctx, cudaStreamSynchronize(s));
        const IterState& h = *ctx->h_iter;
        if (h.watchdog || !(h.generated < h.total || h.active > 0)) break;
        if (h.iter >= h.max_iter) break;
      }
    }
    GYT_CK(ctx, cudaMemcpyAsync(ctx->h_iter, ctx->d_iter, sizeof(IterState), cudaMemcpyDeviceToHost, s));
    GYT_CK(ctx, cudaStreamSynchronize(s));
    const IterState h = *ctx->h_iter;
    if (h.watchdog || h.generated < h.total || h.active > 0)
      return fail(ctx, GYT_ERR_WATCHDOG, "batch: the device loop hit its iteration bound");
    halves += h.iter;
  }
  GYT_CK(ctx, cudaEventRecord(ctx->ev1, s));
  GYT_CK(ctx, cudaEventSynchronize(ctx->ev1));
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    stats->paths = in.total;
    stats->path_slots = 0;
    stats->iterations = halves;
    stats->launches = halves * kKernelsPerHalf;
    stats->ms = ms;
  }
  return GYT_OK;
}

}  // namespace

int32_t gyt_context_set_batch_config(gyt_context* ctx, const GytBatchConfig* c) {
  if (!ctx) return GYT_ERR_INVALID;
  if (!c) {
    ctx->bcfg = GytBatchConfig{0, 0, 0, 1, 0};
    return GYT_OK;
  }
  if (c->paths_in_flight && c->paths_in_flight < 1024)
    return fail(ctx, GYT_ERR_INVALID, "batch config: paths_in_flight must be 0 or >= 1024");
  if (c->stride_blocks_per_sm > 64 || c->trace_blocks_per_sm > 64)
    return fail(ctx, GYT_ERR_INVALID, "batch config: blocks per SM above 64");
  ctx->bcfg = *c;
  ctx->bcfg.use_graph = c->use_graph ? 1 : 0;
  return GYT_OK;
}

int32_t gyt_context_get_batch_config(const gyt_context* ctx, GytBatchConfig* out) {
  if (!ctx || !out) return GYT_ERR_INVALID;
  *out = ctx->bcfg;
  return GYT_OK;
}

int32_t gyt_render_batch_device(gyt_context* ctx, uint32_t n, const gyt_scene* const* scenes,
                                const GytCamera* cameras, const GytRenderParams* params, double* const* d_films,
                                GytRenderStats* stats) {
  if (!ctx) return GYT_ERR_INVALID;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  BatchInput in;
  int32_t st = batch_input(ctx, n, scenes, cameras, params, d_films, &in);
  if (st) return st;
  return run_batch(ctx, in, stats);
}

int32_t gyt_render_batch(gyt_context* ctx, uint32_t n, const gyt_scene* const* scenes, const GytCamera* cameras,
                         const GytRenderParams* params, float* const* rgb_out) {
  if (!ctx) return GYT_ERR_INVALID;
  if (n && (!cameras || !rgb_out)) return fail(ctx, GYT_ERR_INVALID, "batch: null array");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  std::vector<size_t> off(n + 1, 0);
  for (uint32_t i = 0; i < n; ++i) {
    if (!rgb_out[i]) return fail(ctx, GYT_ERR_INVALID, "batch: null image at " + std::to_string(i));
    off[i + 1] = off[i] + (size_t)cameras[i].res_x * cameras[i].res_y;
  }
  if (off[n] >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "batch: more than 2^32 pixels");
  int32_t st = ensure_host_films(ctx, off[n] * 4 * sizeof(double), off[n] * 3 * sizeof(float));
  if (st) return st;
  double* films = ctx->d_film;
  float* rgb = ctx->d_rgb;
  GYT_CK(ctx, cudaMemsetAsync(films, 0, off[n] * 4 * sizeof(double), ctx->stream));
  std::vector<double*> fp(n);
  for (uint32_t i = 0; i < n; ++i) fp[i] = films + 4 * off[i];
  st = gyt_render_batch_device(ctx, n, scenes, cameras, params, fp.data(), nullptr);
  if (st) return st;
  // the films are contiguous: one resolve for all, then one copy per image
  if (off[n]) k_resolve<<<grid_for(off[n]), kBlock, 0, ctx->stream>>>(films, rgb, (uint32_t)off[n]);
  GYT_CK(ctx, cudaGetLastError());
  for (uint32_t i = 0; i < n; ++i) {
    const size_t npix = off[i + 1] - off[i];
    if (!npix) continue;
    GYT_CK(ctx, cudaMemcpyAsync(rgb_out[i], rgb + 3 * off[i], npix * 3 * sizeof(float), cudaMemcpyDeviceToHost,
                                ctx->stream));
  }
  GYT_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return GYT_OK;
}

int32_t gyt_batch_autotune(gyt_context* ctx, uint32_t n, const gyt_scene* const* scenes,
                           const gyt_scene* const* scenes_alt, const GytCamera* cameras,
                           const GytRenderParams* params, uint32_t sample_spp, GytBatchConfig* best,
                           float* best_mpaths) {
  if (!ctx || !best) return GYT_ERR_INVALID;
  if (n == 0) return fail(ctx, GYT_ERR_INVALID, "autotune: empty batch");
  if (!params || !cameras) return fail(ctx, GYT_ERR_INVALID, "autotune: null array");
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  const uint32_t sspp = sample_spp ? sample_spp : 1u;
  std::vector<GytRenderParams> prm(params, params + n);
  size_t npix = 0;
  uint32_t spp_max = 1;
  for (uint32_t i = 0; i < n; ++i) spp_max = std::max(spp_max, prm[i].spp);
  // the sample keeps the batch's mix: every instance's spp scaled by
  // sample_spp / (the largest spp), at least 1
  for (uint32_t i = 0; i < n; ++i) {
    const uint64_t scaled = ((uint64_t)prm[i].spp * sspp + spp_max / 2) / spp_max;
    prm[i].spp = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(scaled, sspp));
    npix += (size_t)cameras[i].res_x * cameras[i].res_y;
  }
  std::vector<void*> tmp;
  struct Guard {
    std::vector<void*>& v;
    ~Guard() {
      for (void* p : v) cudaFree(p);
    }
  } guard{tmp};
  double* films = nullptr;
  GYT_CK(ctx, dalloc(tmp, &films, npix * 4));
  std::vector<double*> fp(n);
  for (uint32_t i = 0, o = 0; i < n; ++i) {
    fp[i] = films + 4ull * o;
    o += cameras[i].res_x * cameras[i].res_y;
  }
  const GytBatchConfig saved = ctx->bcfg;
  const uint32_t saved_cap = ctx->capacity;
  // per candidate one untimed render, then the median of three timed ones:
  // a single timed render of the short sample varies by several per cent,
  // enough to pick the wrong BVH width
  auto trial = [&](const GytBatchConfig& c, const gyt_scene* const* sc, float* mp, int timed = 3) -> int32_t {
    ctx->bcfg = c;
    BatchInput in;
    int32_t st = batch_input(ctx, n, sc, cameras, prm.data(), fp.data(), &in);
    if (st) return st;
    GytRenderStats rs;
    float ms[3];
    for (int k = 0; k <= timed; ++k) {
      st = run_batch(ctx, in, &rs);
      if (st) return st;
      if (k) ms[k - 1] = rs.ms;
    }
    std::sort(ms, ms + timed);
    const float med = ms[timed / 2];
    *mp = med > 0.f ? (float)(rs.paths / (med * 1e3)) : 0.f;
    return GYT_OK;
  };
  GytBatchConfig cur = {saved_cap, 8, 0, 1, (uint32_t)(scenes[0] && scenes[0]->dev.wnodes ? 8 : 2)};
  const gyt_scene* const* cur_scenes = scenes;
  float cur_mp = 0.f;
  int32_t st = trial(cur, cur_scenes, &cur_mp);
  if (st) { ctx->bcfg = saved; return st; }
  // coordinate search: BVH width, pool size, grid-stride blocks, traversal blocks
  if (scenes_alt) {
    float mp = 0.f;
    st = trial(cur, scenes_alt, &mp);
    if (st) { ctx->bcfg = saved; return st; }
    if (mp > cur_mp) {
      cur_mp = mp;
      cur_scenes = scenes_alt;
      cur.bvh_width = scenes_alt[0] && scenes_alt[0]->dev.wnodes ? 8 : 2;
    }
  }
  // Pool size. Every half-iteration pays a fixed cost (the persistent
  // traversal kernels' last rays, launch gaps), so larger pools win on long
  // renders, while the drain at a render's end grows with the pool: a short
  // sample undervalues them (on the uneven batch 4M, 8M and 16M paths in
  // flight gave 376, 395 and 406 Mpaths/s, while the 1/8 sample preferred 4M).
  // The candidates are therefore timed on a sample four times larger (at most
  // the whole batch), all of them on the same one, one timed render each
  // after an untimed one (a render of that size varies by well under 1%).
  {
    std::vector<GytRenderParams> big(params, params + n);
    const uint32_t bspp = std::min<uint32_t>(spp_max, sspp * 4u);
    uint64_t big_paths = 0;
    for (uint32_t i = 0; i < n; ++i) {
      const uint64_t scaled = ((uint64_t)big[i].spp * bspp + spp_max / 2) / spp_max;
      big[i].spp = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(scaled, bspp));
      big_paths += (uint64_t)cameras[i].res_x * cameras[i].res_y * big[i].spp;
    }
    std::swap(prm, big);
    uint32_t best_cap = cur.paths_in_flight;
    float best_mp = 0.f;
    for (uint32_t cap : {1u << 21, 1u << 22, 1u << 23, 1u << 24, 1u << 25}) {
      if (cap > (1u << 21) && (uint64_t)cap > 2 * big_paths) break;  // a pool the sample cannot fill
      GytBatchConfig c = cur;
      c.paths_in_flight = cap;
      float mp = 0.f;
      st = trial(c, cur_scenes, &mp, 1);
      if (st == GYT_ERR_OUT_OF_MEMORY) { cudaGetLastError(); continue; }
      if (st) { std::swap(prm, big); ctx->bcfg = saved; return st; }
      if (mp > best_mp) { best_mp = mp; best_cap = cap; }
    }
    std::swap(prm, big);
    if (best_cap != cur.paths_in_flight) {
      cur.paths_in_flight = best_cap;
      st = trial(cur, cur_scenes, &cur_mp);  // the baseline of the next steps, on the base sample
      if (st) { ctx->bcfg = saved; return st; }
    }
  }
  for (uint32_t sb : {4u, 16u}) {
    GytBatchConfig c = cur;
    c.stride_blocks_per_sm = sb;
    float mp = 0.f;
    st = trial(c, cur_scenes, &mp);
    if (st) { ctx->bcfg = saved; return st; }
    if (mp > cur_mp) { cur_mp = mp; cur = c; }
  }
  const int wi = cur.bvh_width == 8 ? 1 : 0;
  for (uint32_t tb : {(uint32_t)std::max(1, ctx->btrace[wi][0] / 2), (uint32_t)std::max(1, ctx->btrace[wi][0] * 3 / 4)}) {
    GytBatchConfig c = cur;
    c.trace_blocks_per_sm = tb;
    float mp = 0.f;
    st = trial(c, cur_scenes, &mp);
    if (st) { ctx->bcfg = saved; return st; }
    if (mp > cur_mp) { cur_mp = mp; cur = c; }
  }
  ctx->bcfg = cur;
  *best = cur;
  if (best_mpaths) *best_mpaths = cur_mp;
  return GYT_OK;
}

namespace {

constexpr size_t kNoAllocSlotBytes = 2 * (4 * sizeof(float4) + 8 + 3 * 4) + 8 * sizeof(float4);
constexpr size_t kNoAllocAlign = 256;
constexpr size_t align_up(size_t v) { return (v + kNoAllocAlign - 1) / kNoAllocAlign * kNoAllocAlign; }
// per-array rounding adds at most one alignment unit per array (25 arrays)
constexpr size_t kNoAllocBytes = (size_t)GYT_NOALLOC_MAX_PATHS * kNoAllocSlotBytes + 32 * kNoAllocAlign;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct NoAllocDevice {
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch
  bool ready = false;
};
std::mutex g_noalloc_mutex;
NoAllocDevice g_noalloc_dev[64];

// Device address of the scratch array on the current device. The first call
// on each device looks it up with cudaGetSymbolAddress (in host code the
// array's name is only a host-side stand-in, never a device address).
int32_t noalloc_scratch(gyt_context* ctx, unsigned char** out) {
  int dev = ctx->device;
  if (dev < 0 || dev >= 64) return fail(ctx, GYT_ERR_UNSUPPORTED, "render_device_noalloc: device index >= 64");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(ctx, GYT_ERR_CUDA, std::string("render_device_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    d.base = (unsigned char*)p;
    d.ready = true;
  }
  *out = d.base;
  return GYT_OK;
}

template <typename T>
T* carve(unsigned char*& cursor, size_t count) {
  T* p = (T*)cursor;
  cursor += align_up(count * sizeof(T));
  return p;
}

}  // namespace

extern "C" int32_t gyt_render_device_noalloc(gyt_context* ctx, const gyt_scene* scene, const GytCamera* camera,
                                             const GytRenderParams* params, double* d_film, uint32_t paths_in_flight) {
  if (!ctx || !scene || !d_film) return fail(ctx, GYT_ERR_INVALID, "render_device_noalloc: null argument");
  if (paths_in_flight == 0 || paths_in_flight > GYT_NOALLOC_MAX_PATHS)
    return fail(ctx, GYT_ERR_UNSUPPORTED,
                "render_device_noalloc: paths_in_flight must be in [1, " + std::to_string(GYT_NOALLOC_MAX_PATHS) +
                    "] (the size of the library's built-in scratch array)");
  if (scene->dev.sparams)
    return fail(ctx, GYT_ERR_UNSUPPORTED, "render_device_noalloc: the scene's BSDF sampling is frozen");
  int32_t st = check_params(ctx, params);
  if (st) return st;
  Cam cam;
  st = make_cam(ctx, camera, params, &cam);
  if (st) return st;
  GYT_CK(ctx, cudaSetDevice(ctx->device));
  unsigned long long total = (unsigned long long)camera->res_x * camera->res_y * params->spp;
  if (total >= (1ull << 32)) return fail(ctx, GYT_ERR_UNSUPPORTED, "render_device_noalloc: more than 2^32 paths");
  // every wavefront iteration waits for the GPU once: refuse a pool so small
  // for the render that the loop could run for minutes
  const unsigned long long max_iters = wavefront_bound(total, params->max_depth, paths_in_flight);
  if (max_iters > (1ull << 24))
    return fail(ctx, GYT_ERR_UNSUPPORTED, "render_device_noalloc: paths_in_flight too small for this render (its "
                                          "iteration bound exceeds 2^24 wavefront iterations)");
  unsigned char* base = nullptr;
  st = noalloc_scratch(ctx, &base);
  if (st) return st;
  const size_t n = paths_in_flight;
  unsigned char* c = base;
  PathBuf pool[2];
  for (int b = 0; b < 2; ++b) {
    pool[b].o = carve<float4>(c, n);
    pool[b].d = carve<float4>(c, n);
    pool[b].tp = carve<float4>(c, n);
    pool[b].L = carve<float4>(c, n);
    pool[b].sidx = carve<unsigned long long>(c, n);
    pool[b].meta = carve<uint32_t>(c, n);
    pool[b].pix = carve<uint32_t>(c, n);
    pool[b].pid = carve<uint32_t>(c, n);
  }
  Queues q;
  q.so = carve<float4>(c, n);
  q.sd = carve<float4>(c, n);
  q.sc = carve<float4>(c, n);
  q.mo = carve<float4>(c, n);
  q.md = carve<float4>(c, n);
  q.mc = carve<float4>(c, n);
  q.hit = carve<float4>(c, n);
  q.madd = carve<float4>(c, n);
  q.counts = carve<uint32_t>(c, 8);
  if ((size_t)(c - base) > kNoAllocBytes)
    return fail(ctx, GYT_ERR_UNSUPPORTED, "render_device_noalloc: scratch layout exceeds the array");

  Params prm = make_params(params);
  SamplerTables tab = tables(ctx);
  cudaStream_t s = ctx->stream;
  const int W = scene->dev.wnodes ? 8 : 2;
  const int g_ext = ctx->pgrid[pindex(kPExtend, W, false)], g_sh = ctx->pgrid[pindex(kPShadow, W, false)];
  const DevScene& D = scene->dev;
  unsigned long long generated = 0;
  uint32_t active = 0, iters = 0, live = 0;
  int cur = 0;
  GYT_CK(ctx, after_legacy_stream(ctx));
  while (generated < total || active > 0) {
    uint32_t n_new = (uint32_t)std::min<unsigned long long>(paths_in_flight - active, total - generated);
    GYT_CK(ctx, cudaMemsetAsync(q.counts, 0, 8 * sizeof(uint32_t), s));
    if (n_new)
      k_generate<<<grid_for(n_new), kBlock, 0, s>>>(pool[cur], active, n_new, generated, cam, params->spp, nullptr, tab);
    generated += n_new;
    active += n_new;
    if (W == 8) k_extend<8, false><<<g_ext, kBlock, 0, s>>>(pool[cur], active, D, q.hit, q.counts + 2, nullptr);
    else k_extend<2, false><<<g_ext, kBlock, 0, s>>>(pool[cur], active, D, q.hit, q.counts + 2, nullptr);
    if (prm.sampler) k_shade<false, 1><<<grid_for(active), kBlock, 0, s>>>(pool[cur], active, D, prm, q, tab, DebugOut{});
    else k_shade<false, 0><<<grid_for(active), kBlock, 0, s>>>(pool[cur], active, D, prm, q, tab, DebugOut{});
    if (W == 8) k_connect<8, false><<<g_sh, kBlock, 0, s>>>(pool[cur], D, q, DebugOut{}, nullptr);
    else k_connect<2, false><<<g_sh, kBlock, 0, s>>>(pool[cur], D, q, DebugOut{}, nullptr);
    k_finish<<<grid_for(active), kBlock, 0, s>>>(pool[cur], pool[cur ^ 1], active, d_film, cam.res_x, q.counts + 5,
                                                q.madd,
                                                DebugOut{});
    GYT_CK(ctx, cudaGetLastError());
    // pageable destination: the copy completes before cudaMemcpyAsync returns
    GYT_CK(ctx, cudaMemcpyAsync(&live, q.counts + 5, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GYT_CK(ctx, cudaStreamSynchronize(s));
    active = live;
    cur ^= 1;
    if (++iters > max_iters) return fail(ctx, GYT_ERR_WATCHDOG, "render_device_noalloc: iteration cap reached");
  }
  return GYT_OK;
}
