// Device-side building blocks of the B200 path tracer: vector math, Sobol'
// sampling, camera rays, watertight triangle and sphere tests, BSDF lobes and
// light sampling. FP32 throughout; each function cites the reference routine
// (xiaoyxue/Gyunity, paths inside Gyunity/src) whose results it reproduces.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define GYT_D __device__ __forceinline__
#define GYT_HD __host__ __device__ __forceinline__

namespace gyt {

// ------------------------------------------------------------------ math ---
GYT_HD float3 mk(float x, float y, float z) { return make_float3(x, y, z); }
GYT_HD float3 operator+(float3 a, float3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
GYT_HD float3 operator-(float3 a, float3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
GYT_HD float3 operator-(float3 a) { return mk(-a.x, -a.y, -a.z); }
GYT_HD float3 operator*(float3 a, float3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
GYT_HD float3 operator*(float3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
GYT_HD float3 operator*(float s, float3 a) { return mk(a.x * s, a.y * s, a.z * s); }
GYT_HD float3 operator/(float3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
GYT_HD float3 operator/(float3 a, float3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
GYT_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
GYT_HD float3 cross(float3 a, float3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
GYT_HD float length(float3 a) { return sqrtf(dot(a, a)); }
// Vector::Norm divides by the length (math/Linagl.h:527-531)
GYT_HD float3 norm(float3 a) { return a / length(a); }
GYT_HD float3 vabs(float3 a) { return mk(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
GYT_HD bool is_zero(float3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
GYT_HD float comp(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
// Vector::Y (math/Linagl.h:569-572)
GYT_HD float lum(float3 a) { return 0.212671f * a.x + 0.715160f * a.y + 0.072169f * a.z; }
GYT_HD float sgnf(float v) { return v > 0.f ? 1.f : -1.f; }  // math/MathUtils.h:130
GYT_HD float3 f3(float4 a) { return mk(a.x, a.y, a.z); }

constexpr float kPi = 3.14159265358979f;         // common/Core.h:185-191
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kPiOver2 = 1.57079632679489661923f;
constexpr float kPiOver4 = 0.78539816339744830961f;
constexpr float kRayEps = 1e-4f;                  // common/Core.h:193
constexpr float kShadowEps = 1e-4f;               // common/Core.h:194
constexpr float kMachEps = 5.9604644775390625e-08f;  // numeric_limits<float>::epsilon() * 0.5
GYT_HD constexpr float gammaf(int n) { return (n * kMachEps) / (1.f - n * kMachEps); }  // NumericUtils.h:49-51

// NextFloatUp / NextFloatDown (numeric/NumericUtils.h:22-47)
GYT_D float next_up(float v) {
  if (isinf(v) && v > 0.f) return v;
  if (v == -0.f) v = 0.f;
  uint32_t u = __float_as_uint(v);
  u = v >= 0.f ? u + 1 : u - 1;
  return __uint_as_float(u);
}
GYT_D float next_down(float v) {
  if (isinf(v) && v < 0.f) return v;
  if (v == 0.f) v = -0.f;
  uint32_t u = __float_as_uint(v);
  u = v > 0.f ? u - 1 : u + 1;
  return __uint_as_float(u);
}

// ---------------------------------------------------------------- Sobol ---
struct SamplerTables {
  const uint32_t* matrices;   // 1024 * 52 (+ padding) generator columns
  const uint64_t* vdc;        // m levels * 52
  const uint64_t* vdc_inv;    // m levels * 52
  const uint32_t* bits;       // transposed: column b of every dimension, kSobolRow per b
  const uint16_t* hperm;      // Halton digit-block tables of dimensions 1..255, concatenated
  const uint4* hdesc;         // per Halton dimension: table offset, block size, blocks, scale bits
};

// Transposed generator table: row b holds column b of dimensions 0..1039 (the
// last 16 are padding), so consecutive dimensions of one column are adjacent.
// Column b >= 52 of dimension d is column b - 52 of dimension d + 1, which is
// what sobol::sample reads for indices of 52 bits or more.
constexpr int kSobolRow = 1040;

// Ten consecutive dimensions [c, c + 10) of one Sobol' point at once: one pass
// over the set bits of the index, four 128-bit loads per bit. Same values as
// ten sobol_sample calls (RandomStateSequence's >= 1 -> 0 rule applied).
GYT_D void sobol10(const uint32_t* __restrict__ bits, uint64_t index, uint32_t c, float out[10]) {
  const uint32_t base = c & ~3u, sh = c & 3u;
  uint4 a0 = make_uint4(0, 0, 0, 0), a1 = a0, a2 = a0, a3 = a0;
  while (index) {
    int b = __ffsll((long long)index) - 1;
    const uint4* row = (const uint4*)(bits + (size_t)b * kSobolRow + base);
    uint4 v0 = __ldg(row), v1 = __ldg(row + 1), v2 = __ldg(row + 2), v3 = __ldg(row + 3);
    a0.x ^= v0.x; a0.y ^= v0.y; a0.z ^= v0.z; a0.w ^= v0.w;
    a1.x ^= v1.x; a1.y ^= v1.y; a1.z ^= v1.z; a1.w ^= v1.w;
    a2.x ^= v2.x; a2.y ^= v2.y; a2.z ^= v2.z; a2.w ^= v2.w;
    a3.x ^= v3.x; a3.y ^= v3.y; a3.z ^= v3.z; a3.w ^= v3.w;
    index &= index - 1;
  }
  const uint32_t acc[16] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w,
                            a2.x, a2.y, a2.z, a2.w, a3.x, a3.y, a3.z, a3.w};
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    uint32_t r = sh == 0 ? acc[k] : (sh == 1 ? acc[k + 1] : (sh == 2 ? acc[k + 2] : acc[k + 3]));
    float f = __fmul_rn(__uint2float_rn(r), 2.3283064365386963e-10f);
    out[k] = f >= 1.f ? 0.f : f;
  }
}

// sobol::sample (sampler/Sobol.h:46-61): XOR of the columns selected by the
// set bits of the index, then float(result) * 2^-32 (both steps exact here).
GYT_D float sobol_sample(const uint32_t* __restrict__ mat, uint64_t index, uint32_t dim) {
  const uint32_t* m = mat + dim * 52u;
  uint32_t r = 0;
  while (index) {
    int b = __ffsll((long long)index) - 1;
    r ^= __ldg(m + b);
    index &= index - 1;
  }
  return __fmul_rn(__uint2float_rn(r), 2.3283064365386963e-10f);
}

// SobolEnum::look_up (sampler/SobolEnum.h:42-72), zero scrambles.
GYT_D uint64_t enum_index(const SamplerTables& t, uint32_t m, uint32_t frame, uint32_t px, uint32_t py) {
  if (m == 0) return 0;
  uint64_t index = (uint64_t)frame << (2u * m);
  const uint64_t* fw = t.vdc + (m - 1) * 52u;
  const uint64_t* iv = t.vdc_inv + (m - 1) * 52u;
  uint64_t delta = 0;
  for (uint32_t c = 0; frame; frame >>= 1, ++c)
    if (frame & 1) delta ^= __ldg((const unsigned long long*)fw + c);
  uint64_t b = (((uint64_t)px << m) | py) ^ delta;
  while (b) {
    int c = __ffsll((long long)b) - 1;
    index ^= __ldg((const unsigned long long*)iv + c);
    b &= b - 1;
  }
  return index;
}

// --------------------------------------------------------------- Halton ---
// HaltonSampler with Faure permutations (sampler/Halton.h): dimension d is
// the radical inverse of the index in the d-th prime b with every digit
// mapped through Faure's permutation of {0..b-1}. hdesc[d] = (offset of the
// dimension's table in hperm, block size B = b^k, blocks n, scale bits): the
// table maps k digits at once, least significant index digit to the most
// significant place; the n block values are summed exactly (below 2^32) and
// scaled by float((1 - 2^-23) / B^n). Dimension 0 (base 2) writes the
// reversed index bits into a float mantissa; dimensions >= 256 give 0
// (Halton.h:648-905).
constexpr uint32_t kHaltonDims = 256;

GYT_D float halton_sample(const SamplerTables& t, uint64_t index, uint32_t dim) {
  if (dim == 0) return __fsub_rn(__uint_as_float(0x3f800000u | (uint32_t)(__brevll(index) >> 41)), 1.f);
  if (dim >= kHaltonDims) return 0.f;
  const uint4 d = __ldg(t.hdesc + dim);
  const uint16_t* tab = t.hperm + d.x;
  uint32_t v = 0;
  if ((index >> 32) == 0) {
    uint32_t q = (uint32_t)index;
    for (uint32_t j = 0; j < d.z; ++j) {
      const uint32_t nq = q / d.y;
      v = v * d.y + __ldg(tab + (q - nq * d.y));
      q = nq;
    }
  } else {
    uint64_t q = index;
    for (uint32_t j = 0; j < d.z; ++j) {
      const uint64_t nq = q / d.y;
      v = v * d.y + __ldg(tab + (uint32_t)(q - nq * d.y));
      q = nq;
    }
  }
  return __fmul_rn(__uint2float_rn(v), __uint_as_float(d.w));
}

// Ten consecutive Halton dimensions [c, c + 10) (RandomStateSequence's
// >= 1 -> 0 rule applied).
GYT_D void halton10(const SamplerTables& t, uint64_t index, uint32_t c, float out[10]) {
#pragma unroll 1
  for (int k = 0; k < 10; ++k) {
    const float f = halton_sample(t, index, c + k);
    out[k] = f >= 1.f ? 0.f : f;
  }
}

// RandomStateSequence (sampler/Sampler.h:42-66): one dimension per call,
// values >= 1 become 0.
struct Rng {
  uint64_t index;
  uint32_t cursor;
  GYT_D float next(const SamplerTables& t, uint32_t sampler) {
    float r = sampler ? halton_sample(t, index, cursor) : sobol_sample(t.matrices, index, cursor);
    ++cursor;
    return r >= 1.f ? 0.f : r;
  }
};

// ---------------------------------------------------------------- camera ---
struct Cam {
  float m[16];      // RasterToWorld, row-major (camera/Camera.cpp:38)
  float3 pos;
  uint32_t res_x, res_y, log2_res;
  float res_pow2;   // SobolEnum's padded resolution (SobolEnum.h:17-21)
  uint32_t sampler; // 0 SobolSampler + SobolEnum, 1 HaltonSampler + HaltonEnum
  // HaltonEnum (sampler/HaltonEnum.h): 2^p2 >= res_x, 3^p3 >= res_y, the
  // Chinese-remainder multipliers and the index increment 2^p2 3^p3
  uint32_t h_p2, h_p3;
  float h_sx, h_sy;  // 2^p2, 3^p3
  unsigned long long h_mx, h_my, h_inc;
};

// HaltonEnum::get_index: the index congruent to the base-2 digit reversal of
// x modulo 2^p2 and the base-3 digit reversal of y modulo 3^p3, plus s times
// the increment.
GYT_D uint64_t halton_enum_index(const Cam& c, uint32_t s, uint32_t x, uint32_t y) {
  const uint64_t hx = c.h_p2 ? (__brevll((unsigned long long)x) >> (64u - c.h_p2)) : 0ull;
  uint64_t hy = 0;
  uint32_t q = y;
  for (uint32_t d = 0; d < c.h_p3; ++d) {
    hy = hy * 3u + q % 3u;
    q /= 3u;
  }
  return (hx * c.h_mx + hy * c.h_my) % c.h_inc + (uint64_t)s * c.h_inc;
}

// PinHoleCamera::GenerateRay (camera/PinholeCamera.h:22-29) + the Ray
// constructor's RayEps shift (math/Ray.h:17-18).
GYT_D void camera_ray(const Cam& c, float px, float py, float3* o, float3* d) {
  float x = c.m[0] * px + c.m[1] * py - c.m[2] + c.m[3];
  float y = c.m[4] * px + c.m[5] * py - c.m[6] + c.m[7];
  float z = c.m[8] * px + c.m[9] * py - c.m[10] + c.m[11];
  float w = c.m[12] * px + c.m[13] * py - c.m[14] + c.m[15];
  float3 p = mk(x, y, z);
  if (!(w == 1.f || w == 0.f)) p = p / w;
  *d = norm(p - c.pos);
  *o = c.pos + *d * kRayEps;
}

// ------------------------------------------------------------ geometry ----
// Per-ray constants of the watertight test (Woop, Benthin, Wald 2013).
struct WtRay {
  float3 o, d;
  int kx, ky, kz;
  float Sx, Sy, Sz;
};

GYT_D WtRay wt_setup(float3 o, float3 d) {
  WtRay w;
  w.o = o;
  w.d = d;
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = 0;
  if (ay > ax && ay >= az) kz = 1;
  else if (az > ax && az > ay) kz = 2;
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  float dkz = comp(d, kz);
  if (dkz < 0.f) { int t = kx; kx = ky; ky = t; }
  w.kx = kx; w.ky = ky; w.kz = kz;
  w.Sx = comp(d, kx) / dkz;
  w.Sy = comp(d, ky) / dkz;
  w.Sz = 1.f / dkz;
  return w;
}

// The same test in FP64, used only to settle hits whose FP32 distance lands
// within a few ulps of tmax. Shadow rays end on the light's surface (the Ray
// constructor's RayEps shift cancels ShadowRayEps, visual/Intersection.h:64-72),
// so their fate would otherwise be decided by rounding.
__device__ __noinline__ bool wt_intersect_fp64(const WtRay& r, float3 p0, float3 p1, float3 p2, float tmax) {
  double dx = comp(r.d, r.kx), dy = comp(r.d, r.ky), dz = comp(r.d, r.kz);
  double ox = comp(r.o, r.kx), oy = comp(r.o, r.ky), oz = comp(r.o, r.kz);
  double Sx = dx / dz, Sy = dy / dz, Sz = 1.0 / dz;
  double Akz = comp(p0, r.kz) - oz, Bkz = comp(p1, r.kz) - oz, Ckz = comp(p2, r.kz) - oz;
  double Ax = (comp(p0, r.kx) - ox) - Sx * Akz, Ay = (comp(p0, r.ky) - oy) - Sy * Akz;
  double Bx = (comp(p1, r.kx) - ox) - Sx * Bkz, By = (comp(p1, r.ky) - oy) - Sy * Bkz;
  double Cx = (comp(p2, r.kx) - ox) - Sx * Ckz, Cy = (comp(p2, r.ky) - oy) - Sy * Ckz;
  // edge functions without contraction: a shared edge gives exactly opposite
  // values in its two triangles (see wt_intersect)
  double U = __dsub_rn(__dmul_rn(Cx, By), __dmul_rn(Cy, Bx));
  double V = __dsub_rn(__dmul_rn(Ax, Cy), __dmul_rn(Ay, Cx));
  double W = __dsub_rn(__dmul_rn(Bx, Ay), __dmul_rn(By, Ax));
  if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return false;
  double det = U + V + W;
  if (det == 0) return false;
  double th = (U * (Sz * Akz) + V * (Sz * Bkz) + W * (Sz * Ckz)) / det;
  return th >= 0.0 && th <= (double)tmax;
}

// Watertight ray/triangle test. On a hit returns t and the barycentric
// weights of p1 (b1) and p2 (b2), the convention of Triangle::Intersect
// (shape/Triangle.cpp:71-103). Accepts 0 <= t <= tmax. With SETTLE (segment
// rays: shadow rays) a distance within 2e-6 relative of tmax is settled in FP64.
template <bool SETTLE = false>
GYT_D bool wt_intersect(const WtRay& r, float3 p0, float3 p1, float3 p2, float tmax, float* t, float* b1,
                        float* b2) {
  float3 A = p0 - r.o, B = p1 - r.o, C = p2 - r.o;
  float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
  float Ax = comp(A, r.kx) - r.Sx * Akz, Ay = comp(A, r.ky) - r.Sy * Akz;
  float Bx = comp(B, r.kx) - r.Sx * Bkz, By = comp(B, r.ky) - r.Sy * Bkz;
  float Cx = comp(C, r.kx) - r.Sx * Ckz, Cy = comp(C, r.ky) - r.Sy * Ckz;
  // Edge functions without FMA contraction: the two triangles of a shared
  // edge evaluate it from the same two transformed vertices in swapped order,
  // and only unfused products make the results exact negatives of each other,
  // which is what makes the test watertight (a fused a*b - c*d rounds the
  // two orders differently, and a ray exactly on the edge can miss both).
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.f || V == 0.f || W == 0.f) {
    U = (float)((double)Cx * By - (double)Cy * Bx);
    V = (float)((double)Ax * Cy - (double)Ay * Cx);
    W = (float)((double)Bx * Ay - (double)By * Ax);
  }
  if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
  float det = U + V + W;
  if (det == 0.f) return false;
  float T = U * (r.Sz * Akz) + V * (r.Sz * Bkz) + W * (r.Sz * Ckz);
  float th = T / det;
  if (SETTLE) {
    if (!(th >= 0.f && th <= tmax * 1.000002f)) return false;
    if (th >= tmax * 0.999998f) {
      if (!wt_intersect_fp64(r, p0, p1, p2, tmax)) return false;
      th = fminf(th, tmax);
    }
  } else if (!(th >= 0.f && th <= tmax)) {
    return false;
  }
  *t = th;
  *b1 = V / det;
  *b2 = W / det;
  return true;
}

struct Ray {
  float3 o, d;
  float tmax, tmin;
};

// The identity WorldToObject applied to a ray (math/Transform.h:211-225) and
// the Ray constructor's RayEps shift: Sphere::Intersect tests this re-made ray.
GYT_D Ray sphere_object_ray(float3 o, float3 d, float tmax, float tmin) {
  float3 oerr = vabs(o) * gammaf(3);
  float l2 = dot(d, d);
  if (l2 > 0.f) {
    float dt = dot(vabs(d), oerr) / l2;
    o = o + d * dt;
    tmax -= dt;
    tmin += dt;
  }
  Ray r;
  r.o = o + d * kRayEps;
  r.d = d;
  r.tmax = tmax;
  r.tmin = tmin;
  return r;
}

// Root selection of Sphere::Intersect (shape/Sphere.h:37-56).
GYT_D bool sphere_root(float4 s, const Ray& r, float* th) {
  float3 po = r.o - f3(s);
  float vd = dot(po, r.d), d2 = dot(r.d, r.d), po2 = dot(po, po);
  float det = vd * vd - d2 * po2 + d2 * s.w * s.w;
  if (det < 0.f) return false;
  det = sqrtf(det);
  float t = (-vd - det) / d2;
  if (t < r.tmin || t > r.tmax) {
    t = (-vd + det) / d2;
    if (t < r.tmin || t > r.tmax) return false;
  }
  *th = t;
  return true;
}

// Surface record used by shading (the fields of Intersection that the path
// tracer reads, visual/Intersection.h:12-24).
struct Hit {
  float3 pos, n, abs_n, geo_n, wo, perr, su, sv;
};

// Sphere::Intersect hit record (shape/Sphere.h:70-117, with the written-back
// record) under the identity ObjectToWorld (math/Transform.h:296-308).
GYT_D void sphere_hit(float4 s, const Ray& r, float th, Hit* h) {
  float3 c = f3(s);
  float3 hit = r.o + r.d * th;
  float3 sd = (hit - c) * s.w / length(hit - c);
  hit = c + sd;
  float3 n = norm(hit - c);
  float3 nl = dot(n, r.d) < 0.f ? n : n * -1.f;
  float3 perr = vabs(c) * gammaf(1) + vabs(sd) * gammaf(6);
  float3 ph = hit - c;
  const float phimax = 2.f * kPi;
  float3 dpdu = mk(-phimax * ph.z, 0.f, phimax * ph.x);
  float3 su = norm(dpdu - n * dot(n, dpdu));
  float3 sv = norm(cross(n, su));
  h->pos = hit;
  h->perr = perr * (gammaf(3) + 1.f) + vabs(hit) * gammaf(3);
  h->n = norm(n);
  h->abs_n = norm(nl);
  h->wo = norm(r.d * -1.f);
  h->geo_n = norm(n);
  h->su = norm(su);
  h->sv = norm(sv);
}

// Triangle::QueryIntersectionInfo (shape/Triangle.cpp:6-69) and the hit
// position of Triangle::Intersect (:97).
GYT_D void tri_hit(float3 p0, float3 p1, float3 p2, float3 n0, float3 n1, float3 n2, float3 face, float b1,
                   float b2, float3 ro, float3 rd, Hit* h) {
  float b0 = 1.f - b1 - b2;
  h->pos = p0 * (1.f - b1 - b2) + p1 * b1 + p2 * b2;
  float xs = fabsf(b0 * p0.x) + fabsf(b1 * p1.x) + fabsf(b2 * p2.x);
  float ys = fabsf(b0 * p0.y) + fabsf(b1 * p1.y) + fabsf(b2 * p2.y);
  float zs = fabsf(b0 * p0.z) + fabsf(b1 * p1.z) + fabsf(b2 * p2.z);
  float3 ns = norm(n0 * b0 + n1 * b1 + n2 * b2);
  h->geo_n = dot(face, ns) < 0.f ? -face : face;
  h->abs_n = dot(h->geo_n, rd) < 0.f ? h->geo_n : h->geo_n * -1.f;
  h->wo = -rd;
  h->perr = mk(xs, ys, zs) * gammaf(7);
  float s = dot(ro - p0, ns) > 0.f ? 1.f : -1.f;
  float3 du = norm(p1 - p0);
  float3 dv = norm(cross(ns * s, du));
  du = norm(cross(dv, ns));
  h->n = ns;
  h->su = du;
  h->sv = dv;
}

// OffsetRayOrigin (math/GeometryUtils.h:39-64): the offset distance
// d = |n| . pErr, then the origin moved by d along n (towards w) and rounded
// one float away. A shading kernel that spawns several rays from one point
// computes d once (offset_dist) and calls offset_origin_d.
GYT_D float offset_dist(float3 perr, float3 n) { return dot(vabs(n), perr); }
GYT_D float3 offset_origin_d(float3 p, float d, float3 n, float3 w) {
  float3 off = n * d;
  if (dot(w, n) < 0.f) off = -off;
  float3 po = p + off;
  if (off.x > 0.f) po.x = next_up(po.x); else if (off.x < 0.f) po.x = next_down(po.x);
  if (off.y > 0.f) po.y = next_up(po.y); else if (off.y < 0.f) po.y = next_down(po.y);
  if (off.z > 0.f) po.z = next_up(po.z); else if (off.z < 0.f) po.z = next_down(po.z);
  return po;
}
GYT_D float3 offset_origin(float3 p, float3 perr, float3 n, float3 w) {
  return offset_origin_d(p, offset_dist(perr, n), n, w);
}

// --------------------------------------------------------------- BSDFs ----
enum { kRefl = 1, kTrans = 2 };

// FrDielectric (bsdf/BSDF.cpp:5-26)
GYT_D float fr_dielectric(float cosI, float etaI, float etaT) {
  cosI = fminf(fmaxf(cosI, -1.f), 1.f);
  if (!(cosI > 0.f)) { float t = etaI; etaI = etaT; etaT = t; cosI = fabsf(cosI); }
  float sinI = sqrtf(fmaxf(0.f, 1.f - cosI * cosI));
  float sinT = etaI / etaT * sinI;
  if (sinT >= 1.f) return 1.f;
  float cosT = sqrtf(fmaxf(0.f, 1.f - sinT * sinT));
  float rpar = ((etaT * cosI) - (etaI * cosT)) / ((etaT * cosI) + (etaI * cosT));
  float rper = ((etaI * cosI) - (etaT * cosT)) / ((etaI * cosI) + (etaT * cosT));
  return (rpar * rpar + rper * rper) / 2.f;
}

GYT_D float fr_cond1(float c2, float s2, float eta, float k, float cosI) {
  float eta2 = eta * eta, etak2 = k * k;
  float t0 = eta2 - etak2 - s2;
  float a2b2 = sqrtf(t0 * t0 + 4.f * eta2 * etak2);
  float t1 = a2b2 + c2;
  float a = sqrtf(0.5f * (a2b2 + t0));
  float t2 = 2.f * cosI * a;
  float Rs = (t1 - t2) / (t1 + t2);
  float t3 = c2 * a2b2 + s2 * s2;
  float t4 = t2 * s2;
  float Rp = Rs * (t3 - t4) / (t3 + t4);
  return 0.5f * (Rp + Rs);
}

// FrConductor with etai = 1 (bsdf/BSDF.cpp:29-51)
GYT_D float3 fr_conductor(float cosI, float3 eta, float3 k) {
  cosI = fminf(fmaxf(cosI, -1.f), 1.f);
  float c2 = cosI * cosI, s2 = 1.f - c2;
  return mk(fr_cond1(c2, s2, eta.x, k.x, cosI), fr_cond1(c2, s2, eta.y, k.y, cosI), fr_cond1(c2, s2, eta.z, k.z, cosI));
}

// GGXDistribution with visible-normal sampling (visual/Microfacet.cpp:232-379)
struct GGX {
  float ax, ay;
  GYT_D float D(float3 m) const {
    if (m.z <= 0.f) return 0.f;
    float c2 = m.z * m.z;
    float be = ((m.x * m.x) / (ax * ax) + (m.y * m.y) / (ay * ay)) / c2;
    float root = (1.f + be) * c2;
    float res = 1.f / (kPi * ax * ay * root * root);
    if (res * m.z < 1e-20f) res = 0.f;
    return res;
  }
  GYT_D float project(float3 v) const {
    float inv = 1.f / fmaxf(0.f, 1.f - v.z * v.z);
    if (ax == ay || inv <= 0.f) return ax;
    float c = v.x * v.x * inv, s = v.y * v.y * inv;
    return sqrtf(c * ax * ax + s * ay * ay);
  }
  GYT_D float G1(float3 v, float3 m) const {
    if (dot(v, m) * v.z <= 0.f) return 0.f;
    float tanT = fabsf(sqrtf(fmaxf(0.f, 1.f - v.z * v.z)) / v.z);
    if (tanT == 0.f) return 1.f;
    float root = project(v) * tanT;
    return 2.f / (1.f + sqrtf(1.f + root * root));
  }
  GYT_D float G(float3 wo, float3 wi, float3 wh) const { return G1(wo, wh) * G1(wi, wh); }
  GYT_D float pdf(float3 wo, float3 wh) const {
    if (wo.z == 0.f) return 0.f;
    return G1(wo, wh) * fabsf(dot(wo, wh)) * D(wh) / fabsf(wo.z);
  }
  GYT_D float3 sample(float3 v_, float u0, float u1) const {  // SampleGGXVNDF (Heitz 2018)
    float3 v = norm(mk(ax * v_.x, ay * v_.y, v_.z));
    float3 T1 = (v.z < 0.9999f) ? norm(cross(v, mk(0.f, 0.f, 1.f))) : mk(1.f, 0.f, 0.f);
    float3 T2 = cross(T1, v);
    float a = 1.f / (1.f + v.z);
    float r = sqrtf(u0);
    float phi = (u1 < a) ? u1 / a * kPi : kPi + (u1 - a) / (1.f - a) * kPi;
    float sp, cp;
    sincosf(phi, &sp, &cp);
    float P1 = r * cp;
    float P2 = r * sp * ((u1 < a) ? 1.f : v.z);
    float3 dir = T1 * P1 + T2 * P2 + v * sqrtf(fmaxf(0.f, 1.f - P1 * P1 - P2 * P2));
    return norm(mk(ax * dir.x, ay * dir.y, fmaxf(0.f, dir.z)));
  }
};

GYT_D float3 reflect(float3 w, float3 n) { return n * (2.f * dot(w, n)) - w; }

// TransmissionBSDF::Refract (bsdf/BSDF.h:290-302)
GYT_D bool refract(float3 wi, float3 n, float eta, float3* wt) {
  float cosI = dot(n, wi);
  float sin2I = fmaxf(0.f, 1.f - cosI * cosI);
  float sin2T = eta * eta * sin2I;
  if (sin2T >= 1.f) return false;
  float cosT = sqrtf(1.f - sin2T);
  *wt = (-wi) * eta + n * (eta * cosI - cosT);
  return true;
}

// Material record: the one BxDF each reference material adds.
struct Lobe {
  uint32_t type;
  float3 a, b, ceta, ck;
  float eta, eta1;
  GGX g;
  // TransportMode::Importance (light tracing): no eta^2 radiance scaling in
  // the transmission lobes (bsdf/BSDF.h:266-271, 505, 608)
  bool importance = false;

  GYT_D int flags() const { return (type == 0 || type == 1 || type == 3) ? kRefl : (kRefl | kTrans); }
  GYT_D bool delta() const { return type == 1 || type == 2; }

  GYT_D float3 eval(float3 wo, float3 wi) const {
    if (type == 0) return a * kInvPi;  // DiffuseBSDF::Evaluate (BSDF.h:183-185)
    if (type == 3) {  // MicrofacetReflectionBSDF::Evaluate (BSDF.h:348-368)
      if (!(wo.z * wi.z > 0.f)) return mk(0.f, 0.f, 0.f);
      float co = fabsf(wo.z), ci = fabsf(wi.z);
      float3 wh = wi + wo;
      if (ci == 0.f || co == 0.f || is_zero(wh)) return mk(0.f, 0.f, 0.f);
      wh = norm(wh);
      wh = wh * sgnf(wh.z);
      float3 F = fr_conductor(fabsf(dot(wo, wh)), ceta, ck);
      return a * F * (g.D(wh) * g.G(wo, wi, wh)) / (4.f * ci * co);
    }
    if (type == 4) {  // RoughDielectricBSDF::Evaluate (BSDF.h:466-512)
      if (wo.z * wi.z > 0.f) {
        float co = fabsf(wo.z), ci = fabsf(wi.z);
        float3 wh = wi + wo;
        if (ci == 0.f || co == 0.f || is_zero(wh)) return mk(0.f, 0.f, 0.f);
        wh = norm(wh);
        wh = wh * sgnf(wh.z);
        float F = fr_dielectric(dot(wo, wh), 1.f, eta);
        return a * (F * g.D(wh) * g.G(wo, wi, wh) / (4.f * ci * co));
      }
      float co = wo.z, ci = wi.z;
      if (ci == 0.f || co == 0.f) return mk(0.f, 0.f, 0.f);
      float e = wo.z > 0.f ? eta : 1.f / eta;
      float3 wh = -norm(wo + wi * e);
      wh = wh * sgnf(wh.z);
      float F = fr_dielectric(dot(wo, wh), 1.f, eta);
      float sd = dot(wo, wh) + e * dot(wi, wh);
      float factor = importance ? 1.f : 1.f / e;
      float value = (1.f - F) * g.D(wh) * g.G(wo, wi, wh) * e * e * fabsf(dot(wi, wh)) * fabsf(dot(wo, wh)) /
                    fabsf(ci * co * sd * sd);
      return b * fabsf(value * factor * factor);
    }
    return mk(0.f, 0.f, 0.f);  // mirror and glass have delta lobes only
  }

  GYT_D float pdf(float3 wo, float3 wi) const {
    if (type == 0) return (wo.z * wi.z > 0.f) ? fabsf(wi.z) * kInvPi : 0.f;  // BSDF.h:171-174
    if (type == 3) {  // MicrofacetReflectionBSDF::Pdf (BSDF.h:319-329)
      float3 wh = norm(wo + wi);
      float dwh = 1.f / (4.f * dot(wi, wh));
      wh = wh * sgnf(wh.z);
      return fabsf(g.pdf(wo, wh) * dwh);
    }
    if (type == 4) {  // RoughDielectricBSDF::Pdf (BSDF.h:514-543)
      bool refl = wo.z * wi.z > 0.f;
      float3 wh;
      float dwh;
      if (refl) {
        wh = norm(wo + wi);
        dwh = 1.f / (4.f * dot(wi, wh));
      } else {
        float e = wo.z > 0.f ? eta : 1.f / eta;
        wh = -norm(wo + wi * e);
        float sd = dot(wo, wh) + e * dot(wi, wh);
        dwh = fabsf((e * e * dot(wi, wh)) / (sd * sd));
      }
      wh = wh * sgnf(wh.z);
      float p = fabsf(g.pdf(wo, wh) * dwh);
      float F = fr_dielectric(dot(wo, wh), 1.f, eta);
      return p * (refl ? F : (1.f - F));
    }
    return 0.f;
  }

  // BxDF::Sample with *pdf starting at 0 (bsdf/BSDF.cpp:80)
  GYT_D float3 sample(float3 wo, float3* wi, float* pdf, float u0, float u1, float u2) const {
    *pdf = 0.f;
    const float3 zero = mk(0.f, 0.f, 0.f);
    if (type == 0) {  // DiffuseBSDF::Sample + CosineSampleHemisphere (visual/Sampling.cpp:5-36)
      float ox = 2.f * u0 - 1.f, oy = 2.f * u1 - 1.f;
      float dx = 0.f, dy = 0.f;
      if (!(ox == 0.f && oy == 0.f)) {
        float th, r;
        if (fabsf(ox) > fabsf(oy)) { r = ox; th = kPiOver4 * (oy / ox); }
        else { r = oy; th = kPiOver2 - kPiOver4 * (ox / oy); }
        float s, c;
        sincosf(th, &s, &c);
        dx = r * c;
        dy = r * s;
      }
      float z = sqrtf(fmaxf(0.f, 1.f - dx * dx - dy * dy));
      *wi = mk(dx, dy, z);
      if (wo.z < 0.f) wi->z *= -1.f;
      *pdf = pdf_diffuse(wo, *wi);
      return a * kInvPi;
    }
    if (type == 1) {  // SpecularBSDF::Sample (BSDF.h:200-206)
      *wi = mk(-wo.x, -wo.y, wo.z);
      *pdf = 1.f;
      return a / fabsf(wi->z);
    }
    if (type == 2) {  // TransmissionBSDF::Sample (BSDF.h:239-268)
      float Re = fr_dielectric(wo.z, eta1, eta);
      bool entering = wo.z > 0.f;
      float eI = entering ? eta1 : eta, eT = entering ? eta : eta1;
      float3 nf = wo.z > 0.f ? mk(0.f, 0.f, 1.f) : mk(0.f, 0.f, -1.f);
      float P = Re;
      if (u1 < P) {
        *wi = mk(-wo.x, -wo.y, wo.z);
        *pdf = P;
        return a * Re / fabsf(wi->z);
      }
      if (!refract(wo, nf, eI / eT, wi)) return zero;
      *pdf = 1.f - P;
      float e = eI / eT;
      if (importance) return b * (1.f - Re) / fabsf(wi->z);
      return b * (e * e) * (1.f - Re) / fabsf(wi->z);
    }
    if (type == 3) {  // MicrofacetReflectionBSDF::Sample (BSDF.h:331-346)
      if (wo.z == 0.f) return zero;
      const float3 wh = g.sample(wo * sgnf(wo.z), u0, u1);
      // a non-zero pdf means D(wh) > 0, so wh.z > 0 and the reference's
      // Faceforward of wh to +z leaves it (and this pdf) unchanged
      const float gp = g.pdf(wo, wh);
      if (gp == 0.f) return zero;
      *wi = reflect(wo, wh);
      if (!(wo.z * wi->z > 0.f)) return zero;
      *pdf = fabsf(gp / (4.f * dot(*wi, wh)));
      return eval(wo, *wi);
    }
    if (type == 4) {  // RoughDielectricBSDF::Sample (BSDF.h:545-613)
      float3 wh = g.sample(wo * sgnf(wo.z), u0, u1);
      if (g.pdf(wo, wh) == 0.f) return zero;
      float F = fr_dielectric(dot(wo, wh), 1.f, eta);
      float P = F;
      if (u2 < P) {
        if (wo.z == 0.f) return zero;
        *wi = reflect(wo, wh);
        if (!(wo.z * wi->z > 0.f)) return zero;
        float dwh = 1.f / (4.f * dot(*wi, wh));
        *pdf = P * fabsf(g.pdf(wo, wh) * dwh);
        float co = fabsf(wo.z), ci = fabsf(wi->z);
        return a * (F * g.D(wh) * g.G(wo, *wi, wh) / (4.f * ci * co));
      }
      if (wo.z == 0.f) return zero;
      float er = wo.z > 0.f ? 1.f / eta : eta;
      float3 ff = dot(wh, wo) < 0.f ? -wh : wh;  // Faceforward (GeometryUtils.h:66-68)
      if (!refract(wo, ff, er, wi)) { *pdf = 0.f; return zero; }
      if (wo.z * wi->z >= 0.f) return zero;
      float e = wo.z > 0.f ? eta : 1.f / eta;
      float sd = dot(wo, wh) + e * dot(*wi, wh);
      float dwh = fabsf((e * e * dot(*wi, wh)) / (sd * sd));
      *pdf = fabsf((1.f - P) * g.pdf(wo, wh) * dwh);
      float co = wo.z, ci = wi->z;
      if (ci == 0.f || co == 0.f) return zero;
      float factor = importance ? 1.f : 1.f / e;
      float value = (1.f - F) * g.D(wh) * g.G(wo, *wi, wh) * e * e * fabsf(dot(*wi, wh)) * fabsf(dot(wo, wh)) /
                    fabsf(ci * co * sd * sd);
      return b * fabsf(value * factor * factor);
    }
    return zero;
  }

  GYT_D static float pdf_diffuse(float3 wo, float3 wi) { return (wo.z * wi.z > 0.f) ? fabsf(wi.z) * kInvPi : 0.f; }
};

GYT_D Lobe load_lobe(const float* __restrict__ params, const uint32_t* __restrict__ types, uint32_t m) {
  const float4* p = (const float4*)(params + 16u * m);
  float4 q0 = __ldg(p), q1 = __ldg(p + 1), q2 = __ldg(p + 2), q3 = __ldg(p + 3);
  Lobe l;
  l.type = __ldg(types + m);
  l.a = mk(q0.x, q0.y, q0.z);
  l.b = mk(q0.w, q1.x, q1.y);
  l.g.ax = q1.z;
  l.g.ay = q1.w;
  l.eta = q2.x;
  l.ceta = mk(q2.y, q2.z, q2.w);
  l.ck = mk(q3.x, q3.y, q3.z);
  l.eta1 = q3.w;
  return l;
}

// BSDF wrapper for one lobe in the shading frame (bsdf/BSDF.cpp:58-119)
struct Bsdf {
  Lobe lobe;
  float3 su, sv, n, gn;
  GYT_D float3 local(float3 v) const { return mk(dot(v, su), dot(v, sv), dot(v, n)); }
  GYT_D float3 world(float3 v) const { return su * v.x + sv * v.y + n * v.z; }
  GYT_D float pdf(float3 wo, float3 wi) const { return lobe.pdf(local(wo), local(wi)); }
  GYT_D float3 eval(float3 wo, float3 wi) const {
    bool refl = dot(wi, gn) * dot(wo, gn) > 0.f;
    int f = lobe.flags();
    if ((refl && (f & kRefl)) || (!refl && (f & kTrans))) return lobe.eval(local(wo), local(wi));
    return mk(0.f, 0.f, 0.f);
  }
  // Not inlined: the shading kernel samples the BSDF twice (the MIS half of
  // direct lighting and the continuation), and one out-of-line copy keeps its
  // instruction footprint small (it is instruction-bound).
  __device__ __noinline__ float3 sample(float3 wo, float3* wi, float* pdf, float u0, float u1, float u2) const {
    float3 wl;
    float3 f = lobe.sample(local(wo), &wl, pdf, u0, u1, u2);
    *wi = world(wl);
    return f;
  }
};

GYT_D float power_heuristic(float f, float g) { return (f * f) / (f * f + g * g); }  // Integrator.h:11-15

// d log f / d alpha of the GGX reflection lobe (MicrofacetReflectionBSDF,
// bsdf/BSDF.h:308-370) at local directions wo, wi, for ax = ay = alpha: the
// factors that depend on alpha are D (Microfacet.cpp:232-252),
//   D = 1 / (pi a^2 (c^2 + s^2 / a^2)^2),  d log D / da = -2/a + 4 s^2 / (a (a^2 c^2 + s^2)),
// and the Smith terms G1 = 2 / (1 + S), S = sqrt(1 + a^2 tan^2) (:357-373),
//   d log G1 / da = -a tan^2 / (S (1 + S)).
// Where f = 0 (a grazing or back-facing direction) the derivative is 0.
GYT_D float ggx_dlog_alpha(const GGX& g, float3 wo, float3 wi) {
  float3 wh = wi + wo;
  if (is_zero(wh)) return 0.f;
  wh = norm(wh);
  wh = wh * sgnf(wh.z);
  const float a = g.ax;
  const float c2 = wh.z * wh.z, s2 = wh.x * wh.x + wh.y * wh.y;
  float d = -2.f / a + 4.f * s2 / (a * (a * a * c2 + s2));
  const float3 vs[2] = {wo, wi};
  for (int k = 0; k < 2; ++k) {
    const float3 v = vs[k];
    const float tanT = fabsf(sqrtf(fmaxf(0.f, 1.f - v.z * v.z)) / v.z);
    if (tanT > 0.f && isfinite(tanT)) {
      const float r = a * tanT;
      const float S = sqrtf(1.f + r * r);
      d -= a * tanT * tanT / (S * (1.f + S));
    }
  }
  return isfinite(d) ? d : 0.f;
}
// The lobe's alpha derivative (0 for lobes without a differentiable alpha).
GYT_D float lobe_dlog_alpha(const Lobe& l, float3 wo, float3 wi) { return l.type == 3 ? ggx_dlog_alpha(l.g, wo, wi) : 0.f; }

// ----------------------------------------------------- environment light ---
// EnvironmentMap (light/EnvMap.h) over a lat-long RGB image with the
// Distribution2D of ConvertImageToPdf (EnvMap.h:75-90, visual/Sampling.h:101-150).
struct EnvDev {
  const float4* tex;   // w*h texels in file order (row 0 = theta 0)
  const float* ccdf;   // h rows of w+1 conditional CDF entries
  const float* cfunc;  // h rows of w function values
  const float* cint;   // h row integrals
  const float* mcdf;   // h+1 marginal CDF
  const float* mfunc;  // h marginal function values (the row integrals)
  float mint;          // marginal integral
  int w, h;
  float scale, radius; // radiance scale; bounding-sphere radius (EnvLight.cpp:6-9)
};

// ImageTexture::Texel with CLAMP (texture/ImageTexture.h:48-54); the texture
// holds the file rows bottom-up (image/ImageIO.cpp:100-114).
GYT_D float3 env_texel(const EnvDev& e, int x, int y) {
  x = min(max(x, 0), e.w - 1);
  y = min(max(y, 0), e.h - 1);
  return f3(__ldg(e.tex + (size_t)(e.h - 1 - y) * e.w + x));
}

// ImageTexture::Triangle, bilinear (ImageTexture.h:58-69)
GYT_D float3 env_bilinear(const EnvDev& e, float u, float v) {
  float s = __fsub_rn(__fmul_rn((float)e.w, u), 0.5f), t = __fsub_rn(__fmul_rn((float)e.h, v), 0.5f);
  int s0 = (int)floorf(s), t0 = (int)floorf(t);
  float ds = s - s0, dt = t - t0;
  float3 a = env_texel(e, s0, t0) * (1.f - ds) + env_texel(e, s0 + 1, t0) * ds;
  float3 b = env_texel(e, s0, t0 + 1) * (1.f - ds) + env_texel(e, s0 + 1, t0 + 1) * ds;
  return a * (1.f - dt) + b * dt;
}

GYT_D float3 env_radiance(const EnvDev& e, float u, float v) {  // LookupRadiance (EnvMap.h:63-65)
  return env_bilinear(e, u, 1.f - v) * e.scale;
}

GYT_D void env_dir_to_uv(float3 d, float* u, float* v) {  // DirToLatLong (EnvMap.h:102-116)
  float phi = (d.x != 0.f || d.z != 0.f) ? atan2f(d.z, d.x) : 0.f;
  float theta = acosf(d.y);
  phi = phi < 0.f ? phi + 2.f * kPi : phi;
  *u = phi * kInvPi * 0.5f;
  *v = fminf(fmaxf(theta * kInvPi, 0.f), 1.f);
}

GYT_D float env_sin_theta(const EnvDev& e, float v) {  // SinTheta (EnvMap.h:119-127)
  if (v < 1.f) return sinf(kPi * (float)(int)(v * (float)e.h + 0.5f) / (float)e.h);
  return sinf(kPi * ((float)(e.h - 1) + 0.5f) / (float)e.h);
}

GYT_D float3 env_lookup(const EnvDev& e, float3 d) {  // Lookup (EnvMap.h:30-51)
  float u, v;
  env_dir_to_uv(norm(d), &u, &v);
  return env_radiance(e, u, v);
}

GYT_D float env_pdf_dir(const EnvDev& e, float3 d) {  // PdfDir (EnvMap.h:53-61)
  float u, v;
  env_dir_to_uv(norm(d), &u, &v);
  float st = env_sin_theta(e, v);
  if (st == 0.f) return 0.f;
  int iu = min(max((int)(u * e.w), 0), e.w - 1), iv = min(max((int)(v * e.h), 0), e.h - 1);
  float ci = __ldg(e.cint + iv);
  if (ci * e.mint == 0.f) return 0.f;
  float p = (__ldg(e.cfunc + (size_t)iv * e.w + iu) * __ldg(e.mfunc + iv)) / (ci * e.mint);
  return p / (2.f * kPi * kPi * st);
}

// Distribution1D::SampleContinuous (visual/Sampling.h:53-84)
GYT_D float dist_sample(const float* cdf, const float* func, int n, float fint, float u, float* pdf, int* off) {
  int lo = 0, hi = n + 1;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(cdf + mid) > u) hi = mid; else lo = mid + 1;
  }
  int o = min(max(lo - 1, 0), n - 1);
  if (__ldg(cdf + o) == __ldg(cdf + o + 1)) {
    do { o--; } while (o > 0 && __ldg(cdf + o) == __ldg(cdf + o + 1));
    o = max(o, 0);
  }
  *off = o;
  float c0 = __ldg(cdf + o), c1 = __ldg(cdf + o + 1);
  float du = (u - c0) / (c1 - c0);
  *pdf = __ldg(func + o) / fint;
  return ((float)o + du) / (float)n;
}

// EnvironmentMap::Sample (EnvMap.h:16-28)
GYT_D float3 env_sample(const EnvDev& e, float u0, float u1, float3* dir, float* pdfW) {
  float p0, p1;
  int row, col;
  float v = dist_sample(e.mcdf, e.mfunc, e.h, e.mint, u1, &p1, &row);
  float u = dist_sample(e.ccdf + (size_t)row * (e.w + 1), e.cfunc + (size_t)row * e.w, e.w, __ldg(e.cint + row), u0,
                        &p0, &col);
  float pdf = p0 * p1;
  float st = env_sin_theta(e, v);
  *pdfW = st == 0.f ? 0.f : pdf / (2.f * kPi * kPi * st);
  float phi = u * 2.f * kPi, theta = v * kPi;  // LatLongToDir (EnvMap.h:92-100)
  float sth = sinf(theta);
  *dir = mk(sth * cosf(phi), cosf(theta), sth * sinf(phi));
  return env_radiance(e, u, v);
}

}  // namespace gyt
