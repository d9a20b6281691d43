// CPU restatement of the reference PathTracing route (xiaoyxue/Gyunity),
// templated on the arithmetic type so the same code runs in FP32 and FP64.
//
// TEST INFRASTRUCTURE ONLY. It is the checker of the CUDA path: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it. It shares
// no code with the product (gyunity_b200/csrc); the Sobol' tables are the
// reference's data, generated into gyunity_b200/_gen by gen_tables.py.
//
// Reference citations are file:line inside Gyunity/src unless noted.
// Deliberate differences from the reference, all shared with the CUDA path:
//   * ray/triangle: watertight test (Woop, Benthin, Wald 2013) instead of
//     Moller-Trumbore (shape/Triangle.cpp:71-103);
//   * acceleration structure: any exact closest-hit structure gives the same
//     answer up to equal-t ties; this file uses its own binary BVH.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "../../gyunity_b200/_gen/sobol_tables.h"

namespace gyo {
int g_trace = 0;  // debugging aid: per-bounce trace of gyo_paths on stderr

// ------------------------------------------------------------------ math ---
template <typename T> struct V3 {
  T x = 0, y = 0, z = 0;
  V3() = default;
  V3(T a, T b, T c) : x(a), y(b), z(c) {}
  T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  T& at(int i) { return i == 0 ? x : (i == 1 ? y : z); }
  V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
  V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
  V3 operator-() const { return V3(-x, -y, -z); }
  V3 operator*(const V3& o) const { return V3(x * o.x, y * o.y, z * o.z); }
  V3 operator*(T s) const { return V3(x * s, y * s, z * s); }
  V3 operator/(T s) const { return V3(x / s, y / s, z / s); }
  V3 operator/(const V3& o) const { return V3(x / o.x, y / o.y, z / o.z); }
  bool zero() const { return x == 0 && y == 0 && z == 0; }
};
template <typename T> V3<T> operator*(T s, const V3<T>& v) { return v * s; }
template <typename T> T dot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> V3<T> cross(const V3<T>& a, const V3<T>& b) {
  return V3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T> T length(const V3<T>& a) { return std::sqrt(dot(a, a)); }
// Vector::Norm divides by the length (math/Linagl.h:527-531)
template <typename T> V3<T> norm(const V3<T>& a) { return a / length(a); }
template <typename T> V3<T> vabs(const V3<T>& a) { return V3<T>(std::abs(a.x), std::abs(a.y), std::abs(a.z)); }
// Vector::Y (math/Linagl.h:569-572)
template <typename T> T lum(const V3<T>& a) {
  return (T)0.212671 * a.x + (T)0.715160 * a.y + (T)0.072169f * a.z;
}
template <typename T> T sgn(T v) { return v > 0 ? (T)1 : (T)-1; }  // math/MathUtils.h:130
template <typename T> T clampv(T v, T lo, T hi) { return v < lo ? lo : (v > hi ? hi : v); }
template <typename T> V3<T> v3f(const float* p) { return V3<T>((T)p[0], (T)p[1], (T)p[2]); }

template <typename T> struct K {
  static constexpr T PI = (T)3.14159265358979;           // common/Core.h:185
  static constexpr T INV_PI = (T)0.31830988618379067154;
  static constexpr T PI_OVER_2 = (T)1.57079632679489661923;
  static constexpr T PI_OVER_4 = (T)0.78539816339744830961;
  static constexpr T RAY_EPS = (T)1e-4;                  // common/Core.h:193
  static constexpr T SHADOW_EPS = (T)1e-4;               // common/Core.h:194
  static T gamma(int n) {                                 // numeric/NumericUtils.h:49-51
    T e = std::numeric_limits<T>::epsilon() * (T)0.5;
    return (n * e) / (1 - n * e);
  }
};

// numeric/NumericUtils.h:22-47 (one ulp of T)
template <typename T> T next_up(T v) {
  if (std::isinf(v) && v > 0) return v;
  if (v == (T)-0.) v = (T)0.;
  return std::nextafter(v, std::numeric_limits<T>::infinity());
}
template <typename T> T next_down(T v) {
  if (std::isinf(v) && v < 0) return v;
  if (v == (T)0.) v = (T)-0.;
  return std::nextafter(v, -std::numeric_limits<T>::infinity());
}

// ---------------------------------------------------------------- Sobol ---
// sobol::sample (sampler/Sobol.h:46-61): XOR of generator columns, then
// float(result) * 2^-32.
inline float sobol_sample(uint64_t index, uint32_t dim) {
  uint32_t result = 0;
  for (uint32_t i = dim * GYT_SOBOL_COLS; index; index >>= 1, ++i)
    if (index & 1) result ^= gyt_sobol_matrices[i];
  return (float)result * (1.f / (float)(1ULL << 32));
}

// SobolEnum::look_up (sampler/SobolEnum.h:42-72) with zero scrambles.
inline uint64_t enum_index(uint32_t m, uint32_t frame, uint32_t px, uint32_t py) {
  if (m == 0) return 0;
  const uint32_t m2 = m << 1;
  uint64_t index = (uint64_t)frame << m2;
  uint64_t delta = 0;
  for (uint32_t c = 0; frame; frame >>= 1, ++c)
    if (frame & 1) delta ^= gyt_vdc_sobol[m - 1][c];
  uint64_t b = (((uint64_t)px << m) | py) ^ delta;
  for (uint32_t c = 0; b; b >>= 1, ++c)
    if (b & 1) index ^= gyt_vdc_sobol_inv[m - 1][c];
  return index;
}

inline uint32_t log2_pow2_res(uint32_t rx, uint32_t ry) {  // SobolEnum ctor, SobolEnum.h:17-21
  uint32_t r = std::max(rx, ry), p = 1, m = 0;
  while (p < r) { p <<= 1; ++m; }
  return m;
}

// --------------------------------------------------------------- Halton ---
// HaltonSampler with Faure permutations (sampler/Halton.h, generated code):
// dimension d is the radical inverse in the d-th prime b with every digit
// mapped through Faure's permutation of {0..b-1}. The digits are processed k
// at a time through a table of b^k entries (k = 5, 3, 3, 2, 2, 2, 2 for
// b = 3..19, else 1: the largest k with b^k <= 512, Halton.h:925-1435), n
// blocks of k digits in all (the most whole blocks with b^(n k) < 2^32),
// summed exactly in integers and scaled by float((1 - 2^-23) / b^(n k))
// (Halton.h:1455-3308). Base 2 writes the reversed index bits into a float
// mantissa (Halton.h:1441-1452). Dimensions >= 256 give 0 (Halton.h:648-905).
struct HaltonDim {
  uint32_t base = 0, block = 0, blocks = 0;
  float scale = 0.f;
  std::vector<uint16_t> table;
};

struct HaltonTables {
  std::vector<HaltonDim> dims;
  HaltonTables() {
    const uint32_t max_base = 1619;  // the 256th prime
    // Faure permutations (Halton.h:595-625): identity for b <= 3; an even b
    // doubles the permutation of b/2 into its even and odd halves, an odd b
    // inserts the middle digit into the permutation of b - 1
    std::vector<std::vector<uint16_t>> perm(max_base + 1);
    for (uint32_t b = 1; b <= 3; ++b)
      for (uint32_t i = 0; i < b; ++i) perm[b].push_back((uint16_t)i);
    for (uint32_t b = 4; b <= max_base; ++b) {
      perm[b].assign(b, 0);
      const uint32_t c = b / 2;
      if (b % 2 == 0) {
        for (uint32_t i = 0; i < c; ++i) {
          perm[b][i] = (uint16_t)(2 * perm[c][i]);
          perm[b][c + i] = (uint16_t)(2 * perm[c][i] + 1);
        }
      } else {
        for (uint32_t i = 0; i + 1 < b; ++i) {
          const uint32_t v = perm[b - 1][i];
          perm[b][i + (i >= c ? 1 : 0)] = (uint16_t)(v + (v >= c ? 1 : 0));
        }
        perm[b][c] = (uint16_t)c;
      }
    }
    dims.resize(256);
    uint32_t b = 1;
    for (uint32_t d = 0; d < 256; ++d) {
      do {
        ++b;
      } while (!is_prime(b));
      HaltonDim& h = dims[d];
      h.base = b;
      if (b == 2) continue;
      uint32_t k = 1;
      while (pow_u64(b, k + 1) <= 512) ++k;
      uint32_t digits = 0;
      while (pow_u64(b, digits + 1) < (1ull << 32)) ++digits;
      h.blocks = digits / k;
      h.block = (uint32_t)pow_u64(b, k);
      h.scale = (float)(0x1.fffffcp-1 / (double)pow_u64(b, k * h.blocks));
      h.table.resize(h.block);
      for (uint32_t i = 0; i < h.block; ++i) {  // HaltonSampler::invert (Halton.h:912-923)
        uint32_t r = 0, q = i;
        for (uint32_t j = 0; j < k; ++j) {
          r = r * b + perm[b][q % b];
          q /= b;
        }
        h.table[i] = (uint16_t)r;
      }
    }
  }
  static bool is_prime(uint32_t n) {
    for (uint32_t q = 2; q * q <= n; ++q)
      if (n % q == 0) return false;
    return n >= 2;
  }
  static uint64_t pow_u64(uint64_t b, uint32_t e) {
    uint64_t r = 1;
    while (e--) r *= b;
    return r;
  }
};

const HaltonTables& halton_tables() {
  static const HaltonTables t;
  return t;
}

inline uint64_t reverse_bits64(uint64_t v) {
  uint64_t r = 0;
  for (int i = 0; i < 64; ++i, v >>= 1) r = (r << 1) | (v & 1);
  return r;
}

inline float halton_sample(uint64_t index, uint32_t dim) {
  if (dim == 0) {
    const uint32_t bits = 0x3f800000u | (uint32_t)(reverse_bits64(index) >> 41);
    float f;
    std::memcpy(&f, &bits, 4);
    return f - 1.f;
  }
  if (dim >= 256) return 0.f;
  const HaltonDim& h = halton_tables().dims[dim];
  uint64_t v = 0, q = index;
  for (uint32_t j = 0; j < h.blocks; ++j) {
    v = v * h.block + h.table[q % h.block];
    q /= h.block;
  }
  return (float)v * h.scale;
}

// HaltonEnum (sampler/HaltonEnum.h): the film is padded to 2^p2 x 3^p3 and
// sample i of pixel (x, y) is the index congruent to the base-2 digit
// reversal of x modulo 2^p2 and the base-3 digit reversal of y modulo 3^p3
// (Chinese remainder theorem), plus i times 2^p2 3^p3.
struct HaltonEnumC {
  uint32_t p2 = 0, p3 = 0, w = 1, h = 1;
  uint64_t mx = 0, my = 0, inc = 1;
  HaltonEnumC(uint32_t width, uint32_t height) {
    while (w < width) { w *= 2; ++p2; }
    while (h < height) { h *= 3; ++p3; }
    inc = (uint64_t)(uint32_t)(w * h);
    mx = (uint64_t)h * inverse_mod(h, w);
    my = (uint64_t)w * inverse_mod(w, h);
  }
  // a^-1 mod m in [0, m) (0 when m == 1), by the extended Euclidean algorithm
  static uint64_t inverse_mod(int64_t a, int64_t m) {
    if (m == 1) return 0;
    int64_t r0 = m, r1 = a % m, s0 = 0, s1 = 1;
    while (r1) {
      const int64_t qq = r0 / r1;
      int64_t t = r0 - qq * r1; r0 = r1; r1 = t;
      t = s0 - qq * s1; s0 = s1; s1 = t;
    }
    return (uint64_t)(((s0 % m) + m) % m);
  }
  uint64_t index(uint32_t i, uint32_t x, uint32_t y) const {
    const uint64_t hx = p2 ? reverse_bits64(x) >> (64 - p2) : 0;
    uint64_t hy = 0;
    for (uint32_t d = 0, q = y; d < p3; ++d, q /= 3) hy = hy * 3 + q % 3;
    return (hx * mx + hy * my) % inc + (uint64_t)i * inc;
  }
};

// RandomStateSequence::Sample (sampler/Sampler.h:52-64): cursor++ per call,
// values >= 1 become 0. halton selects HaltonSampler instead of SobolSampler.
struct Rand {
  uint64_t index;
  int cursor = 0;
  bool halton = false;
  float next() {
    const uint32_t d = (uint32_t)cursor++;
    float r = halton ? halton_sample(index, d) : sobol_sample(index, d);
    return r >= 1.f ? 0.f : r;
  }
};

// --------------------------------------------------------------- scene ----
struct SceneIn {
  uint32_t n_vertices, n_triangles, n_spheres, n_materials, n_emission;
  const float* vertices;       // nv*3
  const float* normals;        // nv*3 or null
  const uint32_t* indices;     // nt*3
  const uint32_t* tri_material;
  const int32_t* tri_emission;
  const float* spheres;        // ns*4
  const uint32_t* sphere_material;
  const uint32_t* mat_type;
  const float* mat_params;     // nm*16
  const float* emission;       // ne*3
  uint32_t env_w, env_h;
  const float* env;            // h*w*3, row 0 = top
  float env_scale;
};

struct CameraIn {
  float pos[3], look_at[3], up[3];
  float fovy, film_distance;
  uint32_t res_x, res_y;
};

struct ParamsIn {
  uint32_t spp, max_depth, rr_depth;
  uint32_t sampler;  // 0 Sobol' + SobolEnum, 1 Halton (Faure) + HaltonEnum
};

struct Material {
  uint32_t type;
  float p[16];
};

template <typename T> struct Tri {
  V3<T> p0, p1, p2, n0, n1, n2, face;
  uint32_t mat;
  int light;  // index into lights or -1
};

template <typename T> struct Sph {
  V3<T> c;
  T r;
  uint32_t mat;
};

// Distribution1D (visual/Sampling.h:8-99)
template <typename T> struct Dist1D {
  std::vector<T> func, cdf;
  T funcInt = 0;
  int count = 0;
  void init(const T* f, int n) {
    count = n;
    func.assign(f, f + n);
    cdf.assign(n + 1, (T)0);
    for (int i = 1; i < n + 1; ++i) cdf[i] = cdf[i - 1] + func[i - 1] / n;
    funcInt = cdf[n];
    if (funcInt == 0) {
      for (int i = 1; i < n + 1; ++i) cdf[i] = T(i) / T(n);
    } else {
      for (int i = 1; i < n + 1; ++i) cdf[i] /= funcInt;
    }
  }
  T sample_continuous(T u, T* pdf, int* off) const {
    int offset = (int)(std::upper_bound(cdf.begin(), cdf.begin() + count + 1, u) - cdf.begin()) - 1;
    offset = clampv(offset, 0, count - 1);
    if (cdf[offset] == cdf[offset + 1]) {
      do { offset--; } while (cdf[offset] == cdf[offset + 1] && offset > 0);
    }
    if (off) *off = offset;
    T du = (u - cdf[offset]) / (cdf[offset + 1] - cdf[offset]);
    if (pdf) *pdf = func[offset] / funcInt;
    return (offset + du) / count;
  }
  int sample_discrete(T u, T* pdf) const {
    int offset = std::max(0, (int)(std::upper_bound(cdf.begin(), cdf.begin() + count + 1, u) - cdf.begin()) - 1);
    if (pdf) *pdf = func[offset] / (funcInt * count);
    return offset;
  }
};

// EnvironmentMap (light/EnvMap.h) over an RGB lat-long image, plus the
// Distribution2D built by ConvertImageToPdf (EnvMap.h:75-90).
template <typename T> struct Env {
  int w = 0, h = 0;
  T scale = 1;
  std::vector<float> file;  // row 0 = top; ImageTexture stores it flipped
  std::vector<Dist1D<T>> cond;
  Dist1D<T> marg;
  T radius = 0;  // bounding-sphere radius (EnvLight.cpp:6-9)

  V3<T> file_px(int x, int y) const { return v3f<T>(&file[((size_t)y * w + x) * 3]); }
  // ImageTexture::Texel with CLAMP (texture/ImageTexture.h:48-54): mTexture[v] is file row h-1-v
  V3<T> texel(int u, int v) const {
    u = clampv(u, 0, w - 1);
    v = clampv(v, 0, h - 1);
    return file_px(u, h - 1 - v);
  }
  // ImageTexture::Triangle (bilinear, ImageTexture.h:58-69), in float as the reference
  V3<T> bilinear(float u, float v) const {
    float s = w * u - 0.5f, t = h * v - 0.5f;
    int s0 = (int)std::floor(s), t0 = (int)std::floor(t);
    T ds = (T)(s - s0), dt = (T)(t - t0);
    auto lerp = [](T a, V3<T> x0, V3<T> x1) { return x0 * ((T)1 - a) + x1 * a; };
    return lerp(dt, lerp(ds, texel(s0, t0), texel(s0 + 1, t0)), lerp(ds, texel(s0, t0 + 1), texel(s0 + 1, t0 + 1)));
  }
  V3<T> lookup_radiance(T u, T v) const { return bilinear((float)u, (float)(1 - v)) * scale; }  // EnvMap.h:63-65
  void init(const float* data, int width, int height, float sc) {
    w = width; h = height; scale = sc;
    file.assign(data, data + (size_t)w * h * 3);
    std::vector<T> f((size_t)w * h);
    for (int r = 0; r < h; ++r) {
      float v = (float)(r + 0.5f) / (float)h;
      T st = std::sin(K<T>::PI * (T)v);
      for (int c = 0; c < w; ++c) f[(size_t)r * w + c] = st * lum(file_px(c, r));
    }
    cond.resize(h);
    std::vector<T> mf(h);
    for (int r = 0; r < h; ++r) { cond[r].init(&f[(size_t)r * w], w); mf[r] = cond[r].funcInt; }
    marg.init(mf.data(), h);
  }
  T sin_theta(T v) const {  // EnvMap.h:119-127
    if (v < 1) return std::sin(K<T>::PI * (T)(int)((v * h) + (T)0.5f) / (T)h);
    return std::sin(K<T>::PI * (T)((h - 1) + 0.5f) / (T)h);
  }
  V3<T> latlong_to_dir(T u, T v) const {  // EnvMap.h:92-100
    T phi = u * 2 * K<T>::PI, theta = v * K<T>::PI;
    T st = std::sin(theta);
    return V3<T>(st * std::cos(phi), std::cos(theta), st * std::sin(phi));
  }
  void dir_to_latlong(const V3<T>& d, T* u, T* v) const {  // EnvMap.h:102-116
    T phi = (d.x != 0 || d.z != 0) ? std::atan2(d.z, d.x) : (T)0;
    T theta = std::acos(d.y);
    phi = phi < 0 ? phi + 2 * K<T>::PI : phi;
    *u = phi * K<T>::INV_PI * (T)0.5;
    *v = clampv(theta * K<T>::INV_PI, (T)0, (T)1);
  }
  T pdf2d(T u, T v) const {  // Distribution2D::Pdf (Sampling.h:140-149)
    int iu = clampv((int)(u * cond[0].count), 0, cond[0].count - 1);
    int iv = clampv((int)(v * marg.count), 0, marg.count - 1);
    if (cond[iv].funcInt * marg.funcInt == 0) return 0;
    return (cond[iv].func[iu] * marg.func[iv]) / (cond[iv].funcInt * marg.funcInt);
  }
  V3<T> sample(V3<T>* dir, T* pdfW, T u0, T u1) const {  // EnvMap.h:16-28
    T p0, p1;
    int vi;
    T uv1 = marg.sample_continuous(u1, &p1, &vi);
    T uv0 = cond[vi].sample_continuous(u0, &p0, nullptr);
    T pdf = p0 * p1;
    T st = sin_theta(uv1);
    *pdfW = st == 0 ? (T)0 : pdf / (2 * K<T>::PI * K<T>::PI * st);
    *dir = latlong_to_dir(uv0, uv1);
    return lookup_radiance(uv0, uv1);
  }
  V3<T> lookup(const V3<T>& dir) const {  // EnvMap.h:30-51
    T u, v;
    dir_to_latlong(norm(dir), &u, &v);
    return lookup_radiance(u, v);
  }
  T pdf_dir(const V3<T>& dir) const {  // EnvMap.h:53-61
    T u, v;
    dir_to_latlong(norm(dir), &u, &v);
    T st = sin_theta(v);
    return st == 0 ? (T)0 : pdf2d(u, v) / (2 * K<T>::PI * K<T>::PI * st);
  }
};

struct BNode {
  double lo[3], hi[3];
  int left, right;   // children, or -1
  int start, count;  // leaf range into order
};

template <typename T> struct Scene {
  std::vector<Tri<T>> tris;
  std::vector<Sph<T>> sph;
  std::vector<Material> mats;
  // test hook: when not empty, BSDF sampling and pdfs use these materials
  // while BSDF values use mats (sampling held fixed under a parameter change)
  std::vector<Material> smats;
  std::vector<V3<T>> emission;     // per light (area lights only)
  std::vector<int> light_tri;      // light index -> triangle, -1 = environment
  std::vector<int> light_row;      // light index -> emission row, -1 = environment
  Dist1D<T> light_power;
  bool has_env = false;
  Env<T> env;
  std::vector<BNode> nodes;
  std::vector<uint32_t> order;
};

// -------------------------------------------------------------- camera ----
struct M4 { double m[4][4]; };
inline M4 mul(const M4& a, const M4& b) {
  M4 r{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += a.m[i][k] * b.m[k][j];
      r.m[i][j] = s;
    }
  return r;
}
inline M4 inverse(const M4& a) {  // Gauss-Jordan with partial pivoting
  double w[4][8];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 8; ++j) w[i][j] = j < 4 ? a.m[i][j] : (j - 4 == i ? 1.0 : 0.0);
  for (int c = 0; c < 4; ++c) {
    int p = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::abs(w[r][c]) > std::abs(w[p][c])) p = r;
    for (int j = 0; j < 8; ++j) std::swap(w[c][j], w[p][j]);
    double d = w[c][c];
    for (int j = 0; j < 8; ++j) w[c][j] /= d;
    for (int r = 0; r < 4; ++r)
      if (r != c) {
        double f = w[r][c];
        for (int j = 0; j < 8; ++j) w[r][j] -= f * w[c][j];
      }
  }
  M4 r{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r.m[i][j] = w[i][j + 4];
  return r;
}

// ProjectiveCamera::Initialize (camera/Camera.cpp:6-59) with
// Transform::Perspective (math/Transform.cpp:132-150): RasterToWorld.
inline M4 raster_to_world(const CameraIn& c) {
  V3<double> pos(c.pos[0], c.pos[1], c.pos[2]), look(c.look_at[0], c.look_at[1], c.look_at[2]),
      up(c.up[0], c.up[1], c.up[2]);
  V3<double> cz = -norm(pos - look);
  V3<double> cx = -norm(cross(up, cz));
  V3<double> cy = -cross(cz, cx);
  M4 c2w = {{{cx.x, cy.x, cz.x, pos.x}, {cx.y, cy.y, cz.y, pos.y}, {cx.z, cy.z, cz.z, pos.z}, {0, 0, 0, 1}}};
  double aspect = (double)(float)((float)c.res_x / (float)c.res_y);
  double dis = c.film_distance, n = dis, f = 100000.0;
  double t = dis * std::tan(c.fovy * (3.14159265358979 / 180.0) * 0.5);
  double r = t * aspect;
  M4 persp = {{{dis / r, 0, 0, 0}, {0, dis / t, 0, 0}, {0, 0, (f + n) / (f - n), -2 * f * n / (f - n)}, {0, 0, 1, 0}}};
  M4 scale1 = {{{(double)c.res_x, 0, 0, 0}, {0, (double)c.res_y, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}}};
  M4 scale2 = {{{0.5, 0, 0, 0}, {0, -0.5, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}}};
  M4 trans = {{{1, 0, 0, 1}, {0, 1, 0, -1}, {0, 0, 1, 0}, {0, 0, 0, 1}}};
  M4 ndc_to_raster = mul(mul(scale1, scale2), trans);
  M4 raster_to_camera = mul(inverse(persp), inverse(ndc_to_raster));
  return mul(c2w, raster_to_camera);
}

// ----------------------------------------------------------- geometry ----
template <typename T> struct Ray {
  V3<T> o, d;
  T tmax, tmin;
};

// Ray constructor (math/Ray.h:17-18): the origin is moved by RayEps along d.
template <typename T> Ray<T> make_ray(const V3<T>& o, const V3<T>& d, T tmax, T tmin) {
  return Ray<T>{o + d * K<T>::RAY_EPS, d, tmax, tmin};
}

template <typename T> struct Isect {
  V3<T> pos, n, abs_n, geo_n, wo, perr;
  V3<T> su, sv;  // shading frame x, y (z = n)
  T b1 = 0, b2 = 0;
  int prim = -1;
};

// Watertight ray/triangle test (Woop, Benthin, Wald 2013). Returns t and the
// barycentric weights of p1 (b1) and p2 (b2), as Triangle::Intersect reports.
template <typename T> bool tri_intersect(const Tri<T>& tr, const Ray<T>& r, T* t, T* b1, T* b2) {
  int kz = 0;
  T ax = std::abs(r.d.x), ay = std::abs(r.d.y), az = std::abs(r.d.z);
  if (ay > ax && ay >= az) kz = 1;
  else if (az > ax && az > ay) kz = 2;
  int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
  if (r.d[kz] < 0) std::swap(kx, ky);
  T Sx = r.d[kx] / r.d[kz], Sy = r.d[ky] / r.d[kz], Sz = (T)1 / r.d[kz];
  V3<T> A = tr.p0 - r.o, B = tr.p1 - r.o, C = tr.p2 - r.o;
  T Ax = A[kx] - Sx * A[kz], Ay = A[ky] - Sy * A[kz];
  T Bx = B[kx] - Sx * B[kz], By = B[ky] - Sy * B[kz];
  T Cx = C[kx] - Sx * C[kz], Cy = C[ky] - Sy * C[kz];
  T U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
  if (U == 0 || V == 0 || W == 0) {
    long double cxby = (long double)Cx * By, cybx = (long double)Cy * Bx;
    long double axcy = (long double)Ax * Cy, aycx = (long double)Ay * Cx;
    long double bxay = (long double)Bx * Ay, byax = (long double)By * Ax;
    U = (T)(cxby - cybx); V = (T)(axcy - aycx); W = (T)(bxay - byax);
  }
  if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return false;
  T det = U + V + W;
  if (det == 0) return false;
  T Az = Sz * A[kz], Bz = Sz * B[kz], Cz = Sz * C[kz];
  T Tn = U * Az + V * Bz + W * Cz;
  T th = Tn / det;
  if (!(th >= r.tmin && th <= r.tmax)) return false;
  *t = th;
  *b1 = V / det;
  *b2 = W / det;
  return true;
}

// Transform::operator()(Ray) of the identity object transform
// (math/Transform.h:211-225) followed by the Ray constructor's RayEps shift:
// Sphere::Intersect works on this re-made ray (shape/Sphere.h:35, 134 with P7).
template <typename T> Ray<T> sphere_object_ray(const Ray<T>& r) {
  V3<T> oerr = vabs(r.o) * K<T>::gamma(3);
  T l2 = dot(r.d, r.d);
  V3<T> o = r.o;
  T tmax = r.tmax, tmin = r.tmin;
  if (l2 > 0) {
    T dt = dot(vabs(r.d), oerr) / l2;
    o = o + r.d * dt;
    tmax -= dt;
    tmin += dt;
  }
  return make_ray(o, r.d, tmax, tmin);
}

template <typename T> bool sphere_root(const Sph<T>& s, const Ray<T>& r, T* th) {
  V3<T> po = r.o - s.c;
  T vd = dot(po, r.d), d2 = dot(r.d, r.d), po2 = dot(po, po);
  T det = vd * vd - d2 * po2 + d2 * s.r * s.r;
  if (det < 0) return false;
  det = std::sqrt(det);
  T t = (-vd - det) / d2;
  if (t < r.tmin || t > r.tmax) {
    t = (-vd + det) / d2;
    if (t < r.tmin || t > r.tmax) return false;
  }
  *th = t;
  return true;
}

// Sphere::Intersect with P6 (shape/Sphere.h:29-125) and ObjectToWorld of the
// hit record under the identity transform (math/Transform.h:296-308).
template <typename T> bool sphere_intersect(const Sph<T>& s, const Ray<T>& wr, T* tout, Isect<T>* is) {
  Ray<T> r = sphere_object_ray(wr);
  T th;
  if (!sphere_root(s, r, &th)) return false;
  V3<T> hit = r.o + r.d * th;
  V3<T> sd = (hit - s.c) * s.r / length(hit - s.c);
  hit = s.c + sd;
  V3<T> n = norm(hit - s.c);
  V3<T> nl = dot(n, r.d) < 0 ? n : n * (T)-1;
  V3<T> wo = r.d * (T)-1;
  V3<T> perr = vabs(s.c) * K<T>::gamma(1) + vabs(sd) * K<T>::gamma(6);
  V3<T> ph = hit - s.c;
  const T phimax = 2 * K<T>::PI;
  V3<T> dpdu(-phimax * ph.z, 0, phimax * ph.x);
  V3<T> su = norm(dpdu - n * dot(n, dpdu));
  V3<T> sv = norm(cross(n, su));
  is->pos = hit;
  is->perr = perr * (K<T>::gamma(3) + 1) + vabs(hit) * K<T>::gamma(3);
  is->n = norm(n);
  is->abs_n = norm(nl);
  is->wo = norm(wo);
  is->geo_n = norm(n);
  is->su = norm(su);
  is->sv = norm(sv);
  *tout = th;
  return true;
}

template <typename T> bool sphere_occludes(const Sph<T>& s, const Ray<T>& wr) {
  T th;
  return sphere_root(s, sphere_object_ray(wr), &th);
}

inline bool box_hit(const BNode& nd, const double o[3], const double inv[3], double tmax) {
  double t0 = 0, t1 = tmax;
  for (int a = 0; a < 3; ++a) {
    double tn = (nd.lo[a] - o[a]) * inv[a], tf = (nd.hi[a] - o[a]) * inv[a];
    if (tn > tf) std::swap(tn, tf);
    tf *= 1 + 1e-9;
    tn -= std::abs(tn) * 1e-9;
    t0 = tn > t0 ? tn : t0;
    t1 = tf < t1 ? tf : t1;
    if (t0 > t1) return false;
  }
  return true;
}

// Closest hit over triangles (BVH) and spheres (linear). Returns the primitive
// id (triangles first, then spheres) and fills the hit record for spheres;
// triangles fill t/b1/b2 only (QueryIntersectionInfo completes them).
template <typename T> int closest_hit(const Scene<T>& sc, Ray<T>& r, Isect<T>* is) {
  int best = -1;
  if (!sc.nodes.empty()) {
    double o[3] = {(double)r.o.x, (double)r.o.y, (double)r.o.z};
    double inv[3] = {1.0 / (double)r.d.x, 1.0 / (double)r.d.y, 1.0 / (double)r.d.z};
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const BNode& nd = sc.nodes[stack[--sp]];
      if (!box_hit(nd, o, inv, (double)r.tmax)) continue;
      if (nd.left < 0) {
        for (int k = 0; k < nd.count; ++k) {
          uint32_t ti = sc.order[nd.start + k];
          T t, b1, b2;
          if (tri_intersect(sc.tris[ti], r, &t, &b1, &b2)) {
            r.tmax = t;
            is->b1 = b1;
            is->b2 = b2;
            best = (int)ti;
          }
        }
      } else {
        stack[sp++] = nd.right;
        stack[sp++] = nd.left;
      }
    }
  }
  for (size_t s = 0; s < sc.sph.size(); ++s) {
    T t;
    Isect<T> tmp;
    if (sphere_intersect(sc.sph[s], r, &t, &tmp)) {
      r.tmax = t;
      *is = tmp;
      best = (int)(sc.tris.size() + s);
    }
  }
  is->prim = best;
  return best;
}

template <typename T> bool occluded(const Scene<T>& sc, const Ray<T>& r) {
  if (!sc.nodes.empty()) {
    double o[3] = {(double)r.o.x, (double)r.o.y, (double)r.o.z};
    double inv[3] = {1.0 / (double)r.d.x, 1.0 / (double)r.d.y, 1.0 / (double)r.d.z};
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const BNode& nd = sc.nodes[stack[--sp]];
      if (!box_hit(nd, o, inv, (double)r.tmax)) continue;
      if (nd.left < 0) {
        for (int k = 0; k < nd.count; ++k) {
          T t, b1, b2;
          if (tri_intersect(sc.tris[sc.order[nd.start + k]], r, &t, &b1, &b2)) {
            if (g_trace)
              std::fprintf(stderr, "      occluder tri %u t %.9g tmax %.9g o (%.9g %.9g %.9g) d (%.9g %.9g %.9g)\n",
                           sc.order[nd.start + k], (double)t, (double)r.tmax, (double)r.o.x, (double)r.o.y,
                           (double)r.o.z, (double)r.d.x, (double)r.d.y, (double)r.d.z);
            return true;
          }
        }
      } else {
        stack[sp++] = nd.right;
        stack[sp++] = nd.left;
      }
    }
  }
  for (const auto& s : sc.sph)
    if (sphere_occludes(s, r)) return true;
  return false;
}

// Triangle::QueryIntersectionInfo (shape/Triangle.cpp:6-69) plus the hit
// position of Triangle::Intersect (:97).
template <typename T> void tri_info(const Tri<T>& tr, const Ray<T>& r, Isect<T>* is) {
  T b1 = is->b1, b2 = is->b2, b0 = 1 - b1 - b2;
  is->pos = tr.p0 * (1 - b1 - b2) + tr.p1 * b1 + tr.p2 * b2;
  T xs = std::abs(b0 * tr.p0.x) + std::abs(b1 * tr.p1.x) + std::abs(b2 * tr.p2.x);
  T ys = std::abs(b0 * tr.p0.y) + std::abs(b1 * tr.p1.y) + std::abs(b2 * tr.p2.y);
  T zs = std::abs(b0 * tr.p0.z) + std::abs(b1 * tr.p1.z) + std::abs(b2 * tr.p2.z);
  V3<T> ns = norm(tr.n0 * b0 + tr.n1 * b1 + tr.n2 * b2);
  is->geo_n = dot(tr.face, ns) < 0 ? -tr.face : tr.face;
  is->abs_n = dot(is->geo_n, r.d) < 0 ? is->geo_n : is->geo_n * (T)-1;
  is->wo = -r.d;
  is->perr = V3<T>(xs, ys, zs) * K<T>::gamma(7);
  T s = dot(r.o - tr.p0, ns) > 0 ? (T)1 : (T)-1;
  V3<T> du = norm(tr.p1 - tr.p0);
  V3<T> dv = norm(cross(ns * s, du));
  du = norm(cross(dv, ns));
  is->n = ns;
  is->su = du;
  is->sv = dv;
}

// OffsetRayOrigin (math/GeometryUtils.h:39-64)
template <typename T> V3<T> offset_origin(const V3<T>& p, const V3<T>& perr, const V3<T>& n, const V3<T>& w) {
  T d = dot(vabs(n), perr);
  V3<T> off = n * d;
  if (dot(w, n) < 0) off = -off;
  V3<T> po = p + off;
  for (int i = 0; i < 3; ++i) {
    if (off[i] > 0) po.at(i) = next_up(po[i]);
    else if (off[i] < 0) po.at(i) = next_down(po[i]);
  }
  return po;
}

// Intersection::SpawnRay (visual/Intersection.h:74-78)
template <typename T> Ray<T> spawn_ray(const Isect<T>& it, const V3<T>& d) {
  return make_ray(offset_origin(it.pos, it.perr, it.abs_n, d), d, std::numeric_limits<T>::infinity(), (T)0);
}

// Intersection::SpawnTo (visual/Intersection.h:64-72)
template <typename T> Ray<T> spawn_to(const Isect<T>& a, const V3<T>& bpos, const V3<T>& bperr, const V3<T>& babs) {
  V3<T> origin = offset_origin(a.pos, a.perr, a.abs_n, bpos - a.pos);
  V3<T> target = offset_origin(bpos, bperr, babs, origin - bpos);
  V3<T> d = target - origin;
  T dis = length(d);
  d = d / dis;
  return make_ray(origin, d, dis - K<T>::SHADOW_EPS, (T)0);
}

// ---------------------------------------------------------------- BSDF ----
enum { REFL = 1, TRANS = 2 };

// FrDielectric (bsdf/BSDF.cpp:5-26)
template <typename T> T fr_dielectric(T cosI, T etaI, T etaT) {
  cosI = clampv(cosI, (T)-1, (T)1);
  if (!(cosI > 0)) { std::swap(etaI, etaT); cosI = std::abs(cosI); }
  T sinI = std::sqrt(std::max((T)0, 1 - cosI * cosI));
  T sinT = etaI / etaT * sinI;
  if (sinT >= 1) return 1;
  T cosT = std::sqrt(std::max((T)0, 1 - sinT * sinT));
  T rpar = ((etaT * cosI) - (etaI * cosT)) / ((etaT * cosI) + (etaI * cosT));
  T rper = ((etaI * cosI) - (etaT * cosT)) / ((etaI * cosI) + (etaT * cosT));
  return (rpar * rpar + rper * rper) / 2;
}

// FrConductor (bsdf/BSDF.cpp:29-51) with etai = 1
template <typename T> V3<T> fr_conductor(T cosI, const V3<T>& etat, const V3<T>& k) {
  cosI = clampv(cosI, (T)-1, (T)1);
  V3<T> eta = etat, etak = k;
  T c2 = cosI * cosI, s2 = 1 - c2;
  V3<T> eta2 = eta * eta, etak2 = etak * etak;
  V3<T> t0 = eta2 - etak2 - V3<T>(s2, s2, s2);
  V3<T> sq = t0 * t0 + eta2 * etak2 * (T)4;
  V3<T> a2b2(std::sqrt(sq.x), std::sqrt(sq.y), std::sqrt(sq.z));
  V3<T> t1 = a2b2 + V3<T>(c2, c2, c2);
  V3<T> ha = (a2b2 + t0) * (T)0.5f;
  V3<T> a(std::sqrt(ha.x), std::sqrt(ha.y), std::sqrt(ha.z));
  V3<T> t2 = a * ((T)2 * cosI);
  V3<T> Rs = (t1 - t2) / (t1 + t2);
  V3<T> t3 = a2b2 * c2 + V3<T>(s2 * s2, s2 * s2, s2 * s2);
  V3<T> t4 = t2 * s2;
  V3<T> Rp = Rs * (t3 - t4) / (t3 + t4);
  return (Rp + Rs) * (T)0.5;
}

// GGXDistribution (visual/Microfacet.cpp:232-379), visible-normal sampling
template <typename T> struct GGX {
  T ax, ay;
  T D(const V3<T>& m) const {
    if (m.z <= 0) return 0;
    T c2 = m.z * m.z;
    T be = ((m.x * m.x) / (ax * ax) + (m.y * m.y) / (ay * ay)) / c2;
    T root = ((T)1 + be) * c2;
    T res = (T)1 / (K<T>::PI * ax * ay * root * root);
    if (res * m.z < (T)1e-20f) res = 0;
    return res;
  }
  T project(const V3<T>& v) const {
    T inv = 1 / std::max((T)0, 1 - v.z * v.z);
    if (ax == ay || inv <= 0) return ax;
    T c = v.x * v.x * inv, s = v.y * v.y * inv;
    return std::sqrt(c * ax * ax + s * ay * ay);
  }
  T G1(const V3<T>& v, const V3<T>& m) const {
    if (dot(v, m) * v.z <= 0) return 0;
    T tanT = std::abs(std::sqrt(std::max((T)0, 1 - v.z * v.z)) / v.z);
    if (tanT == 0) return 1;
    T alpha = project(v);
    T root = alpha * tanT;
    return (T)2 / ((T)1 + std::sqrt(1 + root * root));
  }
  T G(const V3<T>& wo, const V3<T>& wi, const V3<T>& wh) const { return G1(wo, wh) * G1(wi, wh); }
  T pdf(const V3<T>& wo, const V3<T>& wh) const {
    if (wo.z == 0) return 0;
    return G1(wo, wh) * std::abs(dot(wo, wh)) * D(wh) / std::abs(wo.z);
  }
  V3<T> sample(const V3<T>& v_, T u0, T u1) const {  // SampleGGXVNDF (Heitz 2018)
    V3<T> v = norm(V3<T>(ax * v_.x, ay * v_.y, v_.z));
    V3<T> T1 = (v.z < (T)0.9999) ? norm(cross(v, V3<T>(0, 0, 1))) : V3<T>(1, 0, 0);
    V3<T> T2 = cross(T1, v);
    T a = 1 / ((T)1.f + v.z);
    T r = std::sqrt(u0);
    T phi = (u1 < a) ? u1 / a * K<T>::PI : K<T>::PI + (u1 - a) / ((T)1.f - a) * K<T>::PI;
    T P1 = r * std::cos(phi);
    T P2 = r * std::sin(phi) * ((u1 < a) ? (T)1.0f : v.z);
    V3<T> dir = T1 * P1 + T2 * P2 + v * std::sqrt(std::max((T)0, 1 - P1 * P1 - P2 * P2));
    return norm(V3<T>(ax * dir.x, ay * dir.y, std::max((T)0, dir.z)));
  }
};

template <typename T> V3<T> reflect(const V3<T>& w, const V3<T>& n) { return n * ((T)2.f * dot(w, n)) - w; }

// TransmissionBSDF::Refract (bsdf/BSDF.h:290-302)
template <typename T> bool refract(const V3<T>& wi, const V3<T>& n, T eta, V3<T>* wt) {
  T cosI = dot(n, wi);
  T sin2I = std::max((T)0, (T)(1 - cosI * cosI));
  T sin2T = eta * eta * sin2I;
  if (sin2T >= 1) return false;
  T cosT = std::sqrt(1 - sin2T);
  *wt = (-wi) * eta + n * (eta * cosI - cosT);
  return true;
}

// One-lobe BSDF of a material (every reference material adds one BxDF).
template <typename T> struct Lobe {
  uint32_t type;
  V3<T> a, b, ceta, ck;
  T eta, eta1;
  GGX<T> g;
  int flags() const {
    switch (type) {
      case 0: case 1: case 3: return REFL;
      default: return REFL | TRANS;
    }
  }
  bool delta() const { return type == 1 || type == 2; }

  V3<T> eval(const V3<T>& wo, const V3<T>& wi) const {
    switch (type) {
      case 0: return a * K<T>::INV_PI;  // DiffuseBSDF::Evaluate (BSDF.h:183-185)
      case 1: case 2: return V3<T>();
      case 3: {  // MicrofacetReflectionBSDF::Evaluate (BSDF.h:348-368)
        if (!(wo.z * wi.z > 0)) return V3<T>();
        T co = std::abs(wo.z), ci = std::abs(wi.z);
        V3<T> wh = wi + wo;
        if (ci == 0 || co == 0) return V3<T>();
        if (wh.zero()) return V3<T>();
        wh = norm(wh);
        wh = wh * sgn(wh.z);
        V3<T> F = fr_conductor(std::abs(dot(wo, wh)), ceta, ck);
        T D = g.D(wh), G = g.G(wo, wi, wh);
        return a * F * D * G / (4 * ci * co);
      }
      case 4: {  // RoughDielectricBSDF::Evaluate (BSDF.h:466-512)
        bool refl = wo.z * wi.z > 0;
        if (refl) {
          T co = std::abs(wo.z), ci = std::abs(wi.z);
          V3<T> wh = wi + wo;
          if (ci == 0 || co == 0) return V3<T>();
          if (wh.zero()) return V3<T>();
          wh = norm(wh);
          wh = wh * sgn(wh.z);
          T F = fr_dielectric(dot(wo, wh), (T)1.f, eta);
          T D = g.D(wh), G = g.G(wo, wi, wh);
          return a * F * D * G / (4 * ci * co);
        }
        T co = wo.z, ci = wi.z;
        if (ci == 0 || co == 0) return V3<T>();
        T e = wo.z > 0 ? (eta / (T)1.f) : ((T)1.f / eta);
        V3<T> wh = -norm(wo + wi * e);
        wh = wh * sgn(wh.z);
        T F = fr_dielectric(dot(wo, wh), (T)1.f, eta);
        T D = g.D(wh), G = g.G(wo, wi, wh);
        T sd = dot(wo, wh) + e * dot(wi, wh);
        T factor = 1 / e;
        T value = (1 - F) * D * G * e * e * std::abs(dot(wi, wh)) * std::abs(dot(wo, wh)) /
                  std::abs(ci * co * sd * sd);
        return b * std::abs(value * factor * factor);
      }
    }
    return V3<T>();
  }

  T pdf(const V3<T>& wo, const V3<T>& wi) const {
    switch (type) {
      case 0: return (wo.z * wi.z > 0) ? std::abs(wi.z) * K<T>::INV_PI : (T)0.f;  // BSDF.h:171-174
      case 1: case 2: return 0;
      case 3: {  // MicrofacetReflectionBSDF::Pdf (BSDF.h:319-329)
        V3<T> wh = norm(wo + wi);
        T dwh = 1.f / (4 * dot(wi, wh));
        wh = wh * sgn(wh.z);
        return std::abs(g.pdf(wo, wh) * dwh);
      }
      case 4: {  // RoughDielectricBSDF::Pdf (BSDF.h:514-543)
        bool refl = wo.z * wi.z > 0;
        V3<T> wh;
        T dwh;
        if (refl) {
          wh = norm(wo + wi);
          dwh = 1.f / (4 * dot(wi, wh));
        } else {
          T e = wo.z > 0 ? (eta / (T)1.f) : ((T)1.f / eta);
          wh = -norm(wo + wi * e);
          T sd = dot(wo, wh) + e * dot(wi, wh);
          dwh = std::abs((e * e * dot(wi, wh)) / (sd * sd));
        }
        wh = wh * sgn(wh.z);
        T p = std::abs(g.pdf(wo, wh) * dwh);
        T F = fr_dielectric(dot(wo, wh), (T)1.f, eta);
        return p * (refl ? F : (1 - F));
      }
    }
    return 0;
  }

  // BxDF::Sample; *pdf starts at 0 (BSDF::Sample sets it, bsdf/BSDF.cpp:80)
  V3<T> sample(const V3<T>& wo, V3<T>* wi, T* pdf, T u0, T u1, T u2) const {
    *pdf = 0;
    switch (type) {
      case 0: {  // DiffuseBSDF::Sample (BSDF.h:176-181) + CosineSampleHemisphere
        T ox = 2.0 * u0 - 1, oy = 2.0 * u1 - 1;  // ConcentricSampleDisk (visual/Sampling.cpp:5-23)
        T dx = 0, dy = 0;
        if (!(ox == 0 && oy == 0)) {
          T th, r;
          if (std::abs(ox) > std::abs(oy)) { r = ox; th = K<T>::PI_OVER_4 * (oy / ox); }
          else { r = oy; th = K<T>::PI_OVER_2 - K<T>::PI_OVER_4 * (ox / oy); }
          dx = r * std::cos(th); dy = r * std::sin(th);
        }
        T z = std::sqrt(std::max((T)0, 1 - dx * dx - dy * dy));
        *wi = V3<T>(dx, dy, z);
        if (wo.z < 0) wi->z *= -1;
        *pdf = this->pdf(wo, *wi);
        return eval(wo, *wi);
      }
      case 1: {  // SpecularBSDF::Sample (BSDF.h:200-206)
        *wi = V3<T>(-wo.x, -wo.y, wo.z);
        *pdf = 1.0;
        return a / std::abs(wi->z);
      }
      case 2: {  // TransmissionBSDF::Sample (BSDF.h:239-268)
        T Re = fr_dielectric(wo.z, eta1, eta);
        bool entering = wo.z > 0;
        T eI = entering ? eta1 : eta, eT = entering ? eta : eta1;
        V3<T> nf = wo.z > 0 ? V3<T>(0, 0, 1) : V3<T>(0, 0, -1);
        T P = Re;
        if (u1 < P) {
          *wi = V3<T>(-wo.x, -wo.y, wo.z);
          *pdf = P;
          return a * Re / std::abs(wi->z);
        }
        if (!refract(wo, nf, eI / eT, wi)) return V3<T>();
        *pdf = 1 - P;
        T e = eI / eT;
        return b * (e * e) * (1.f - Re) / std::abs(wi->z);
      }
      case 3: {  // MicrofacetReflectionBSDF::Sample (BSDF.h:331-346)
        if (wo.z == 0) return V3<T>();
        V3<T> wh = g.sample(wo * sgn(wo.z), u0, u1);
        if (g.pdf(wo, wh) == 0) return V3<T>();
        *wi = reflect(wo, wh);
        if (!(wo.z * wi->z > 0)) return V3<T>();
        wh = wh * sgn(wh.z);
        *pdf = std::abs(g.pdf(wo, wh) / (4 * dot(*wi, wh)));
        return eval(wo, *wi);
      }
      case 4: {  // RoughDielectricBSDF::Sample (BSDF.h:545-613)
        V3<T> wh = g.sample(wo * sgn(wo.z), u0, u1);
        if (g.pdf(wo, wh) == 0) return V3<T>();
        T F = fr_dielectric(dot(wo, wh), (T)1.f, eta);
        T P = F;
        if (u2 < P) {
          if (wo.z == 0) return V3<T>();
          *wi = reflect(wo, wh);
          if (!(wo.z * wi->z > 0)) return V3<T>();
          T dwh = 1.f / (4 * dot(*wi, wh));
          *pdf = P * std::abs(g.pdf(wo, wh) * dwh);
          T co = std::abs(wo.z), ci = std::abs(wi->z);
          T D = g.D(wh), G = g.G(wo, *wi, wh);
          return a * F * D * G / (4 * ci * co);
        }
        if (wo.z == 0) return V3<T>();
        T er = wo.z > 0 ? ((T)1.f / eta) : (eta / (T)1.f);
        V3<T> ff = dot(wh, wo) < 0.f ? -wh : wh;  // Faceforward (GeometryUtils.h:66-68)
        if (!refract(wo, ff, er, wi)) { *pdf = 0; return V3<T>(); }
        if (wo.z * wi->z >= 0) return V3<T>();
        T e = wo.z > 0 ? (eta / (T)1.f) : ((T)1.f / eta);
        T sd = dot(wo, wh) + e * dot(*wi, wh);
        T dwh = std::abs((e * e * dot(*wi, wh)) / (sd * sd));
        *pdf = std::abs((1 - P) * g.pdf(wo, wh) * dwh);
        T co = wo.z, ci = wi->z;
        if (ci == 0 || co == 0) return V3<T>();
        T D = g.D(wh), G = g.G(wo, *wi, wh);
        T factor = 1 / e;
        T value = (1 - F) * D * G * e * e * std::abs(dot(*wi, wh)) * std::abs(dot(wo, wh)) /
                  std::abs(ci * co * sd * sd);
        return b * std::abs(value * factor * factor);
      }
    }
    return V3<T>();
  }
};

template <typename T> Lobe<T> make_lobe(const Material& m) {
  Lobe<T> l;
  l.type = m.type;
  l.a = v3f<T>(&m.p[0]);
  l.b = v3f<T>(&m.p[3]);
  l.g = GGX<T>{(T)m.p[6], (T)m.p[7]};
  l.eta = (T)m.p[8];
  l.ceta = v3f<T>(&m.p[9]);
  l.ck = v3f<T>(&m.p[12]);
  l.eta1 = (T)m.p[15];
  return l;
}

// BSDF wrapper (bsdf/BSDF.cpp:58-119) for one lobe in the shading frame.
template <typename T> struct Bsdf {
  Lobe<T> lobe;
  Lobe<T> slobe;       // sampling lobe (the same as lobe unless the scene's smats are set)
  bool split = false;
  V3<T> su, sv, n, gn;
  V3<T> to_local(const V3<T>& v) const { return V3<T>(dot(v, su), dot(v, sv), dot(v, n)); }
  V3<T> to_world(const V3<T>& v) const { return su * v.x + sv * v.y + n * v.z; }
  T pdf(const V3<T>& wo, const V3<T>& wi) const { return slobe.pdf(to_local(wo), to_local(wi)); }
  V3<T> eval(const V3<T>& wo, const V3<T>& wi) const {
    bool refl = dot(wi, gn) * dot(wo, gn) > 0;
    int f = lobe.flags();
    if ((refl && (f & REFL)) || (!refl && (f & TRANS))) return lobe.eval(to_local(wo), to_local(wi));
    return V3<T>();
  }
  V3<T> sample(const V3<T>& wo, V3<T>* wi, T* pdf, T u0, T u1, T u2) const {
    V3<T> wl;
    V3<T> f = slobe.sample(to_local(wo), &wl, pdf, u0, u1, u2);
    if (split && slobe.type == 3 && !f.zero()) f = lobe.eval(to_local(wo), wl);
    *wi = to_world(wl);
    return f;
  }
};

template <typename T> Bsdf<T> make_bsdf(const Scene<T>& sc, const Isect<T>& is, uint32_t mat) {
  Bsdf<T> b;
  b.lobe = make_lobe<T>(sc.mats[mat]);
  b.split = !sc.smats.empty();
  b.slobe = b.split ? make_lobe<T>(sc.smats[mat]) : b.lobe;
  b.su = is.su; b.sv = is.sv; b.n = is.n; b.gn = is.geo_n;
  return b;
}

template <typename T> T power_heuristic(T f, T g) { return (f * f) / (f * f + g * g); }  // Integrator.h:11-15

// d log f / d alpha of the GGX reflection lobe for ax = ay = alpha at local
// directions: D = 1 / (pi a^2 (c^2 + s^2/a^2)^2) and the Smith terms
// G1 = 2 / (1 + sqrt(1 + a^2 tan^2)) are the factors that depend on alpha.
template <typename T> T ggx_dlog_alpha(const GGX<T>& g, const V3<T>& wo, const V3<T>& wi) {
  V3<T> wh = wi + wo;
  if (wh.zero()) return 0;
  wh = norm(wh);
  wh = wh * sgn(wh.z);
  const T a = g.ax;
  const T c2 = wh.z * wh.z, s2 = wh.x * wh.x + wh.y * wh.y;
  T d = -2 / a + 4 * s2 / (a * (a * a * c2 + s2));
  const V3<T> vs[2] = {wo, wi};
  for (const V3<T>& v : vs) {
    const T tanT = std::abs(std::sqrt(std::max((T)0, 1 - v.z * v.z)) / v.z);
    if (tanT > 0 && std::isfinite(tanT)) {
      const T r = a * tanT, S = std::sqrt(1 + r * r);
      d -= a * tanT * tanT / (S * (1 + S));
    }
  }
  return std::isfinite(d) ? d : 0;
}
template <typename T> T lobe_dlog_alpha(const Lobe<T>& l, const V3<T>& wo, const V3<T>& wi) {
  return l.type == 3 ? ggx_dlog_alpha(l.g, wo, wi) : (T)0;
}

// Path replay adjoint of one path (detached sampling: pdfs, MIS weights, light
// selection and roulette are constants). Every radiance contribution C moves
// gradient to each BSDF factor it contains: the continuation factors of the
// earlier vertices, the own factor of a light or MIS sample, and the emitter.
// f is linear in the albedo a of the diffuse and GGX lobes (dC/da_c = C_c/a_c)
// and d log f / d alpha is the GGX term above.
template <typename T> struct AdjAcc {
  V3<T> delta;
  std::vector<std::pair<uint32_t, T>> conts;
  const Scene<T>* sc = nullptr;
  double* gm = nullptr;  // per material: a.r, a.g, a.b, alpha
  double* ge = nullptr;  // per emission row: r, g, b
  void mat(uint32_t m, T da, const V3<T>& Cd) const {
    const Material& mt = sc->mats[m];
    if (mt.type != 0 && mt.type != 3) return;
    for (int c = 0; c < 3; ++c)
      if (mt.p[c] != 0.f) gm[4 * m + c] += (double)Cd[c] / (double)mt.p[c];
    gm[4 * m + 3] += ((double)Cd.x + (double)Cd.y + (double)Cd.z) * (double)da;
  }
  void add(const V3<T>& C, int own_m, T own_da, int row, const V3<T>& Le) const {
    const V3<T> Cd = delta * C;
    for (const auto& k : conts) mat(k.first, k.second, Cd);
    if (own_m >= 0) mat((uint32_t)own_m, own_da, Cd);
    if (row >= 0)
      for (int c = 0; c < 3; ++c)
        if (Le[c] != 0) ge[3 * row + c] += (double)Cd[c] / (double)Le[c];
  }
};

// The two halves of DirectIllumination for the adjoint.
template <typename T> struct DirectParts {
  bool has1 = false, has2 = false;
  V3<T> C1, C2;  // (L1 w1 + L2 w2) / lightSel split into its halves
  T da1 = 0, da2 = 0;
  int row = -1;
  V3<T> Le;
};

template <typename T> uint32_t prim_material(const Scene<T>& sc, int prim) {
  return prim < (int)sc.tris.size() ? sc.tris[prim].mat : sc.sph[prim - sc.tris.size()].mat;
}
template <typename T> int prim_light(const Scene<T>& sc, int prim) {
  return prim < (int)sc.tris.size() ? sc.tris[prim].light : -1;
}

template <typename T> void complete_hit(const Scene<T>& sc, const Ray<T>& r, Isect<T>* is) {
  if (is->prim >= 0 && is->prim < (int)sc.tris.size()) tri_info(sc.tris[is->prim], r, is);
}

// Shape::Pdf (shape/Shape.h:34-47) for a triangle light
template <typename T> T tri_light_pdf(const Tri<T>& tr, const Isect<T>& it, const V3<T>& wi) {
  Ray<T> r = spawn_ray(it, wi);
  T t, b1, b2;
  if (!tri_intersect(tr, r, &t, &b1, &b2)) return 0;
  Isect<T> lp;
  lp.b1 = b1; lp.b2 = b2;
  tri_info(tr, r, &lp);
  V3<T> d = lp.pos - it.pos;
  T area = (T)0.5 * length(cross(tr.p1 - tr.p0, tr.p2 - tr.p0));
  T pdf = dot(d, d) / (std::abs(dot(lp.n, -wi)) * area);
  if (std::isinf(pdf)) return 0;
  return pdf;
}

// Discrete decisions of one path for a replay (bit i = bounce i < 64).
struct Replay {
  int bounce = 0;
  const uint64_t* force_occ = nullptr;  // shadow ray occluded
  const uint64_t* force_mis = nullptr;  // MIS ray reached the sampled light
  uint64_t occ = 0, mis = 0;            // decisions taken
  bool forced(const uint64_t* m) const { return m && bounce < 64; }
  bool bit(const uint64_t* m) const { return ((*m) >> bounce) & 1ull; }
};

// Integrator::DirectIllumination (integrator/Integrator.cpp:9-107), surfaces only
template <typename T> V3<T> direct(const Scene<T>& sc, const Isect<T>& is, const Bsdf<T>& bsdf, T uLight,
                                   T u0, T u1, T v0, T v1, T v2, Replay* rp, DirectParts<T>* parts = nullptr) {
  T lightSel;
  int li = sc.light_power.sample_discrete(uLight, &lightSel);
  if (lightSel == 0) return V3<T>();
  int ltri = sc.light_tri[li];
  V3<T> wi1, wi2;
  T w1 = 1, w2 = 1;
  V3<T> L1, L2;
  {
    V3<T> wi, lpos, lerr, labs, Li;
    T pdf = 0;
    if (ltri >= 0) {
      // AreaLight::Sample_Li -> Shape::Sample(isect) -> Triangle::Sample
      const Tri<T>& tr = sc.tris[ltri];
      T su0 = std::sqrt(u0);
      T bb0 = 1 - su0, bb1 = u1 * su0;  // UniformSampleTriangle (Sampling.cpp:38-41)
      lpos = tr.p0 * bb0 + tr.p1 * bb1 + tr.p2 * (1 - bb0 - bb1);
      V3<T> ln = tr.n0 * bb0 + tr.n1 * bb1 + tr.n2 * (1 - bb0 - bb1);
      lerr = (vabs(tr.p0 * bb0) + vabs(tr.p1 * bb1) + vabs(tr.p2 * (1 - bb0 - bb1))) * K<T>::gamma(6);
      labs = tr.face;
      T area = (T)0.5 * length(cross(tr.p1 - tr.p0, tr.p2 - tr.p0));
      pdf = 1 / area;
      V3<T> w = is.pos - lpos;
      if (length(w) == 0) {
        pdf = 0;
      } else {
        w = norm(w);
        V3<T> dd = is.pos - lpos;
        pdf *= dot(dd, dd) / std::abs(dot(ln, -w));
        if (std::isinf(pdf)) pdf = 0;
      }
      wi = norm(lpos - is.pos);
      Li = dot(ln, -wi) > 0 ? sc.emission[li] : V3<T>();
    } else {
      // EnvironmentLight::Sample_Li (light/EnvLight.cpp:41-51)
      V3<T> sd;
      Li = sc.env.sample(&sd, &pdf, u0, u1);
      wi = norm(sd);
      lpos = is.pos + wi * (2 * sc.env.radius);
      lerr = V3<T>();
      labs = wi;
    }
    if (pdf > 0 && !Li.zero()) {
      T spdf = bsdf.pdf(is.wo, wi);
      V3<T> f = bsdf.eval(is.wo, wi);
      T cosT = std::abs(dot(is.n, wi));
      if (!f.zero()) {
        Ray<T> sr = spawn_to(is, lpos, lerr, labs);
        bool occ = rp->forced(rp->force_occ) ? rp->bit(rp->force_occ) : occluded(sc, sr);
        if (occ) {
          Li = V3<T>();
          if (rp->bounce < 64) rp->occ |= 1ull << rp->bounce;
        }
        w1 = power_heuristic(pdf, spdf);
        L1 = Li * f * cosT / pdf;
        wi1 = wi;
      }
    }
  }
  {
    V3<T> wi;
    T pdf;
    V3<T> f = bsdf.sample(is.wo, &wi, &pdf, v0, v1, v2);
    T cosT = std::abs(dot(is.n, wi));
    wi2 = wi;
    if (pdf != 0 && !f.zero()) {
      T lpdf = ltri >= 0 ? tri_light_pdf(sc.tris[ltri], is, wi) : sc.env.pdf_dir(wi);
      if (lpdf == 0) {
        w2 = 0;
      } else {
        w2 = power_heuristic(pdf, lpdf);
        Ray<T> r = spawn_ray(is, wi);
        Isect<T> h;
        int prim = closest_hit(sc, r, &h);
        bool reach = ltri >= 0 ? (prim >= 0 && prim_light(sc, prim) == li) : prim < 0;
        if (rp->forced(rp->force_mis)) {
          bool want = rp->bit(rp->force_mis);
          if (want && !reach && ltri >= 0) {
            // the replayed path reached the light: take the hit on the light triangle itself
            Ray<T> rl = spawn_ray(is, wi);
            T t, b1, b2;
            if (tri_intersect(sc.tris[ltri], rl, &t, &b1, &b2)) {
              h = Isect<T>();
              h.b1 = b1; h.b2 = b2; h.prim = ltri;
              r = rl;
              prim = ltri;
            } else {
              want = false;
            }
          }
          reach = want;
        }
        if (reach && rp->bounce < 64) rp->mis |= 1ull << rp->bounce;
        if (reach) {
          if (ltri >= 0) {
            complete_hit(sc, r, &h);
            V3<T> e = dot(h.n, -wi) > 0 ? sc.emission[li] : V3<T>();
            L2 = e * f * cosT / pdf;
          } else {
            L2 = sc.env.lookup(wi) * f * cosT / pdf;
          }
        }
      }
    }
  }
  if (g_trace)
    std::fprintf(stderr, "    light %d sel %.9g L1 %.9g w1 %.9g L2 %.9g w2 %.9g\n", li, (double)lightSel, (double)L1.x,
                 (double)w1, (double)L2.x, (double)w2);
  if (parts) {
    parts->row = sc.light_row[li];
    parts->Le = sc.emission[li];
    parts->has1 = !L1.zero();
    parts->has2 = !L2.zero();
    parts->C1 = L1 * w1 / lightSel;
    parts->C2 = L2 * w2 / lightSel;
    parts->da1 = lobe_dlog_alpha(bsdf.lobe, bsdf.to_local(is.wo), bsdf.to_local(wi1));
    parts->da2 = lobe_dlog_alpha(bsdf.lobe, bsdf.to_local(is.wo), bsdf.to_local(wi2));
  }
  return (L1 * w1 + L2 * w2) / lightSel;
}

template <typename T> struct CamT {
  double m[4][4];
  V3<T> pos;
};

// PinHoleCamera::GenerateRay (camera/PinholeCamera.h:22-29)
template <typename T> Ray<T> camera_ray(const CamT<T>& c, T px, T py) {
  double p[4] = {(double)px, (double)py, -1.0, 1.0}, q[4];
  for (int i = 0; i < 4; ++i) q[i] = c.m[i][0] * p[0] + c.m[i][1] * p[1] + c.m[i][2] * p[2] + c.m[i][3] * p[3];
  V3<T> sp((T)q[0], (T)q[1], (T)q[2]);
  if (!(q[3] == 1 || q[3] == 0)) sp = sp / (T)q[3];
  V3<T> d = norm(sp - c.pos);
  return make_ray(c.pos, d, std::numeric_limits<T>::infinity(), (T)0);
}

// PathTracing::Li (integrator/PT.cpp:10-67) preceded by the per-sample set-up
// of TiledIntegrator::Render (integrator/TiledIntegrator.cpp:40-45).
template <typename T> V3<T> trace_path(const Scene<T>& sc, const CamT<T>& cam, const CameraIn& ci,
                                       const ParamsIn& pr, uint32_t x, uint32_t y, uint32_t s, int* cursor_out,
                                       float* u_out = nullptr, float* v_out = nullptr,
                                       const uint64_t* force_rr = nullptr, uint64_t* rr_out = nullptr,
                                       Replay* rp_in = nullptr, AdjAcc<T>* adj = nullptr) {
  Replay rp_local;
  Replay* rp = rp_in ? rp_in : &rp_local;
  float u, v;
  Rand rnd{0};
  if (pr.sampler == 1) {
    // HaltonEnum::SampleX/Y (sampler/HaltonEnum.h): scale by 2^p2 and 3^p3
    const HaltonEnumC he(ci.res_x, ci.res_y);
    rnd = Rand{he.index(s, x, y), 0, true};
    u = (float)he.w * rnd.next() - (float)x;
    v = (float)he.h * rnd.next() - (float)y;
  } else {
    uint32_t m = log2_pow2_res(ci.res_x, ci.res_y);
    rnd = Rand{enum_index(m, s, x, y)};
    float res = (float)(1u << m);
    u = res * rnd.next() - (float)x;  // SobolEnum::SampleX (SobolEnum.h:30-32)
    v = res * rnd.next() - (float)y;
  }
  if (u_out) *u_out = u;
  if (v_out) *v_out = v;
  Ray<T> ray = camera_ray(cam, (T)((float)x + u), (T)((float)y + v));
  bool delta = false;
  uint64_t rr_mask = 0;
  V3<T> tp(1, 1, 1), L;
  for (int i = 0; i < (int)pr.max_depth; ++i) {
    Isect<T> is;
    int prim = closest_hit(sc, ray, &is);
    if (prim < 0) {
      if ((i == 0 || delta) && sc.has_env) {
        L = L + tp * sc.env.lookup(ray.d);
        if (adj) adj->add(tp * sc.env.lookup(ray.d), -1, 0, -1, V3<T>());
      }
      break;
    }
    complete_hit(sc, ray, &is);
    Bsdf<T> bsdf = make_bsdf(sc, is, prim_material(sc, prim));
    int pl = prim_light(sc, prim);
    if ((i == 0 || delta) && pl >= 0) {
      V3<T> e = dot(is.n, is.wo) > 0 ? sc.emission[pl] : V3<T>();  // AreaLight::Emission (AreaLight.h:40-43)
      L = L + tp * e;
      if (adj && !e.zero()) adj->add(tp * e, -1, 0, sc.light_row[pl], sc.emission[pl]);
    } else {
      // argument evaluation order of PT.cpp:38 as compiled by GCC: v.z, v.y, v.x, u.y, u.x, uLight
      T vz = rnd.next(), vy = rnd.next(), vx = rnd.next();
      T uy = rnd.next(), ux = rnd.next();
      T ul = rnd.next();
      rp->bounce = i;
      DirectParts<T> parts;
      V3<T> di = direct(sc, is, bsdf, ul, ux, uy, vx, vy, vz, rp, adj ? &parts : nullptr);
      if (adj) {
        const int m = (int)prim_material(sc, prim);
        if (parts.has1) adj->add(tp * parts.C1, m, parts.da1, parts.row, parts.Le);
        if (parts.has2) adj->add(tp * parts.C2, m, parts.da2, parts.row, parts.Le);
      }
      if (g_trace)
        std::fprintf(stderr, "  bounce %d prim %d pos (%.9g %.9g %.9g) DI (%.9g %.9g %.9g) tp %.9g\n", i, prim,
                     (double)is.pos.x, (double)is.pos.y, (double)is.pos.z, (double)di.x, (double)di.y, (double)di.z,
                     (double)tp.x);
      L = L + tp * di;
    }
    T rz = rnd.next(), ry = rnd.next(), rx = rnd.next();  // PT.cpp:47, same order
    V3<T> wi;
    T pdf;
    V3<T> f = bsdf.sample(is.wo, &wi, &pdf, rx, ry, rz);
    if (f.zero() || pdf == 0) break;
    V3<T> est = f * std::abs(dot(is.n, wi)) / pdf;
    delta = bsdf.lobe.delta();
    T q = lum(est * tp) / lum(tp);
    T p = (q < (T)1.0) ? q : (T)1.0;  // std::min((real)1, q) keeps 1 when q is NaN
    // Replay: p is exactly 1 in exact arithmetic after a delta lobe, so whether
    // a roulette number is drawn there depends on rounding; a replay can take
    // that decision from the recorded path instead (bit i = drawn at bounce i).
    bool draw = force_rr ? (((*force_rr) >> i) & 1ull) != 0 : (p < 1 && i > (int)pr.rr_depth);
    if (draw) rr_mask |= 1ull << i;
    if (draw) {
      if (rnd.next() < p) tp = tp / p;
      else break;
    }
    tp = tp * est;
    ray = spawn_ray(is, wi);
    if (adj)
      adj->conts.push_back({prim_material(sc, prim), lobe_dlog_alpha(bsdf.lobe, bsdf.to_local(is.wo), bsdf.to_local(wi))});
  }
  if (cursor_out) *cursor_out = rnd.cursor;
  if (rr_out) *rr_out = rr_mask;
  return L;
}

// ----------------------------------------------------------- BVH build ----
template <typename T> void build_bvh(Scene<T>& sc) {
  size_t n = sc.tris.size();
  sc.nodes.clear();
  sc.order.resize(n);
  if (!n) return;
  std::vector<double> lo(n * 3), hi(n * 3), ce(n * 3);
  for (size_t i = 0; i < n; ++i) {
    sc.order[i] = (uint32_t)i;
    const Tri<T>& t = sc.tris[i];
    for (int a = 0; a < 3; ++a) {
      double v0 = (double)t.p0[a], v1 = (double)t.p1[a], v2 = (double)t.p2[a];
      lo[i * 3 + a] = std::min(v0, std::min(v1, v2));
      hi[i * 3 + a] = std::max(v0, std::max(v1, v2));
      ce[i * 3 + a] = 0.5 * (lo[i * 3 + a] + hi[i * 3 + a]);
    }
  }
  struct Job { int node, start, count; };
  std::vector<Job> stack;
  sc.nodes.push_back(BNode{});
  stack.push_back({0, 0, (int)n});
  while (!stack.empty()) {
    Job j = stack.back();
    stack.pop_back();
    BNode nd;
    double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
    for (int a = 0; a < 3; ++a) { nd.lo[a] = 1e300; nd.hi[a] = -1e300; }
    for (int k = j.start; k < j.start + j.count; ++k) {
      uint32_t i = sc.order[k];
      for (int a = 0; a < 3; ++a) {
        nd.lo[a] = std::min(nd.lo[a], lo[i * 3 + a]);
        nd.hi[a] = std::max(nd.hi[a], hi[i * 3 + a]);
        clo[a] = std::min(clo[a], ce[i * 3 + a]);
        chi[a] = std::max(chi[a], ce[i * 3 + a]);
      }
    }
    int axis = 0;
    for (int a = 1; a < 3; ++a)
      if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
    if (j.count <= 4 || chi[axis] - clo[axis] <= 0) {
      nd.left = nd.right = -1;
      nd.start = j.start;
      nd.count = j.count;
      sc.nodes[j.node] = nd;
      continue;
    }
    int mid = j.start + j.count / 2;
    std::nth_element(sc.order.begin() + j.start, sc.order.begin() + mid, sc.order.begin() + j.start + j.count,
                     [&](uint32_t a, uint32_t b) { return ce[a * 3 + axis] < ce[b * 3 + axis]; });
    nd.left = (int)sc.nodes.size();
    nd.right = nd.left + 1;
    nd.start = nd.count = 0;
    sc.nodes[j.node] = nd;
    sc.nodes.push_back(BNode{});
    sc.nodes.push_back(BNode{});
    stack.push_back({nd.left, j.start, mid - j.start});
    stack.push_back({nd.right, mid, j.start + j.count - mid});
  }
}

template <typename T> Scene<T>* make_scene(const SceneIn& in) {
  auto* sc = new Scene<T>();
  for (uint32_t m = 0; m < in.n_materials; ++m) {
    Material mt;
    mt.type = in.mat_type[m];
    std::memcpy(mt.p, &in.mat_params[m * 16], sizeof(mt.p));
    sc->mats.push_back(mt);
  }
  std::vector<T> power;
  double blo[3] = {1e300, 1e300, 1e300}, bhi[3] = {-1e300, -1e300, -1e300};
  for (uint32_t t = 0; t < in.n_triangles; ++t) {
    Tri<T> tr;
    const uint32_t* ix = &in.indices[3 * t];
    // the reference stores vertices as float; T-precision arithmetic starts from them
    tr.p0 = v3f<T>(&in.vertices[3 * ix[0]]);
    tr.p1 = v3f<T>(&in.vertices[3 * ix[1]]);
    tr.p2 = v3f<T>(&in.vertices[3 * ix[2]]);
    tr.face = norm(cross(tr.p1 - tr.p0, tr.p2 - tr.p0));  // Triangle ctor (shape/Triangle.h:52)
    if (in.normals) {
      tr.n0 = v3f<T>(&in.normals[3 * ix[0]]);
      tr.n1 = v3f<T>(&in.normals[3 * ix[1]]);
      tr.n2 = v3f<T>(&in.normals[3 * ix[2]]);
    } else {
      tr.n0 = tr.n1 = tr.n2 = tr.face;
    }
    tr.mat = in.tri_material[t];
    tr.light = -1;
    for (int k = 0; k < 3; ++k)
      for (int a = 0; a < 3; ++a) {
        double v = in.vertices[3 * ix[k] + a];
        blo[a] = std::min(blo[a], v);
        bhi[a] = std::max(bhi[a], v);
      }
    if (in.tri_emission[t] >= 0) {
      tr.light = (int)sc->light_tri.size();
      sc->light_tri.push_back((int)t);
      sc->light_row.push_back(in.tri_emission[t]);
      V3<T> e = v3f<T>(&in.emission[3 * in.tri_emission[t]]);
      sc->emission.push_back(e);
      T area = (T)0.5 * length(cross(tr.p1 - tr.p0, tr.p2 - tr.p0));
      power.push_back(lum(e * area * K<T>::PI));  // AreaLight::Power (AreaLight.h:45-48)
    }
    sc->tris.push_back(tr);
  }
  for (uint32_t s = 0; s < in.n_spheres; ++s) {
    Sph<T> sp;
    sp.c = v3f<T>(&in.spheres[4 * s]);
    sp.r = (T)in.spheres[4 * s + 3];
    sp.mat = in.sphere_material[s];
    for (int a = 0; a < 3; ++a) {
      blo[a] = std::min(blo[a], (double)in.spheres[4 * s + a] - in.spheres[4 * s + 3]);
      bhi[a] = std::max(bhi[a], (double)in.spheres[4 * s + a] + in.spheres[4 * s + 3]);
    }
    sc->sph.push_back(sp);
  }
  if (in.env_w && in.env_h && in.env) {
    sc->has_env = true;
    sc->env.init(in.env, (int)in.env_w, (int)in.env_h, in.env_scale);
    // AABB::GetBoundingSphere of the accelerator's world bound (math/AABB.h:69-72)
    V3<T> d((T)(bhi[0] - blo[0]), (T)(bhi[1] - blo[1]), (T)(bhi[2] - blo[2]));
    sc->env.radius = length(d) * (T)0.5;
    sc->light_tri.push_back(-1);
    sc->light_row.push_back(-1);
    sc->emission.push_back(V3<T>());
    // EnvironmentLight::Power (EnvLight.cpp:59-62)
    power.push_back(lum(sc->env.lookup_radiance((T)0.5, (T)0.5) * K<T>::PI * sc->env.radius * sc->env.radius));
  }
  if (!power.empty()) sc->light_power.init(power.data(), (int)power.size());
  build_bvh(*sc);
  return sc;
}

template <typename T> CamT<T> make_cam(const CameraIn& c) {
  CamT<T> ct;
  M4 m = raster_to_world(c);
  std::memcpy(ct.m, m.m, sizeof(ct.m));
  ct.pos = V3<T>((T)c.pos[0], (T)c.pos[1], (T)c.pos[2]);
  return ct;
}

struct Handle {
  Scene<float>* sf = nullptr;
  Scene<double>* sd = nullptr;
};

template <typename T> Scene<T>* get(Handle* h);
template <> Scene<float>* get<float>(Handle* h) { return h->sf; }
template <> Scene<double>* get<double>(Handle* h) { return h->sd; }

template <typename Fn> void parallel_rows(int n, int threads, Fn fn) {
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        int i = next.fetch_add(1);
        if (i >= n) break;
        fn(i);
      }
    });
  for (auto& th : pool) th.join();
}

template <typename T> void paths_impl(Handle* h, const CameraIn* c, const ParamsIn* p, int64_t n, const uint32_t* x,
                                      const uint32_t* y, const uint32_t* s, double* L, int32_t* cursor, int threads,
                                      const uint64_t* force_rr, uint64_t* rr_out, const uint64_t* force_occ,
                                      const uint64_t* force_mis, uint64_t* occ_out, uint64_t* mis_out) {
  Scene<T>* sc = get<T>(h);
  CamT<T> cam = make_cam<T>(*c);
  int chunks = (int)((n + 255) / 256);
  parallel_rows(chunks, threads, [&](int ch) {
    for (int64_t i = (int64_t)ch * 256; i < std::min<int64_t>(n, (int64_t)ch * 256 + 256); ++i) {
      int cur = 0;
      Replay rp;
      rp.force_occ = force_occ ? &force_occ[i] : nullptr;
      rp.force_mis = force_mis ? &force_mis[i] : nullptr;
      V3<T> l = trace_path(*sc, cam, *c, *p, x[i], y[i], s[i], &cur, nullptr, nullptr,
                           force_rr ? &force_rr[i] : nullptr, rr_out ? &rr_out[i] : nullptr, &rp);
      if (occ_out) occ_out[i] = rp.occ;
      if (mis_out) mis_out[i] = rp.mis;
      L[3 * i] = (double)l.x; L[3 * i + 1] = (double)l.y; L[3 * i + 2] = (double)l.z;
      if (cursor) cursor[i] = cur;
    }
  });
}

// Film::AddSample with the box filter (visual/Film.h:61-87; math/Filter.h:26-38):
// the sample lands on every pixel whose centre is within 0.5, so samples on
// a pixel edge also reach the neighbour.
inline void film_add(double* film, int rx, int ry, float fx, float fy, const double L[3]) {
  float x = fx - 0.5f, y = fy - 0.5f;
  int x0 = std::max(0, (int)std::ceil(x - 0.5f)), x1 = std::min((int)std::floor(x + 0.5f), rx - 1);
  int y0 = std::max(0, (int)std::ceil(y - 0.5f)), y1 = std::min((int)std::floor(y + 0.5f), ry - 1);
  for (int i = y0; i <= y1; ++i)
    for (int j = x0; j <= x1; ++j) {
      double* px = &film[((size_t)i * rx + j) * 4];
      px[0] += L[0]; px[1] += L[1]; px[2] += L[2]; px[3] += 1.0;
    }
}

template <typename T> void render_impl(Handle* h, const CameraIn* c, const ParamsIn* p, uint32_t row0, uint32_t row1,
                                       double* film, int threads) {
  Scene<T>* sc = get<T>(h);
  CamT<T> cam = make_cam<T>(*c);
  int rx = (int)c->res_x, ry = (int)c->res_y;
  std::vector<double> tmp((size_t)rx * ry * 4, 0.0);
  // rows are processed independently; edge samples that spill into a
  // neighbouring row are merged afterwards from per-row buffers
  int nrows = (int)(row1 - row0);
  std::vector<std::vector<double>> spill(nrows);
  parallel_rows(nrows, threads, [&](int ri) {
    int yy = (int)row0 + ri;
    std::vector<double> local((size_t)rx * 3 * 4, 0.0);  // rows yy-1, yy, yy+1
    for (int xx = 0; xx < rx; ++xx)
      for (uint32_t s = 0; s < p->spp; ++s) {
        float u, v;
        int cur;
        V3<T> l = trace_path(*sc, cam, *c, *p, (uint32_t)xx, (uint32_t)yy, s, &cur, &u, &v);
        double L[3] = {(double)l.x, (double)l.y, (double)l.z};
        float fx = (float)xx + u, fy = (float)yy + v;
        float xm = fx - 0.5f, ym = fy - 0.5f;
        int x0 = std::max(0, (int)std::ceil(xm - 0.5f)), x1 = std::min((int)std::floor(xm + 0.5f), rx - 1);
        int y0 = std::max(0, (int)std::ceil(ym - 0.5f)), y1 = std::min((int)std::floor(ym + 0.5f), ry - 1);
        for (int i = y0; i <= y1; ++i)
          for (int j = x0; j <= x1; ++j) {
            double* px = &local[((size_t)(i - yy + 1) * rx + j) * 4];
            px[0] += L[0]; px[1] += L[1]; px[2] += L[2]; px[3] += 1.0;
          }
      }
    spill[ri] = std::move(local);
  });
  for (int ri = 0; ri < nrows; ++ri) {
    int yy = (int)row0 + ri;
    for (int k = 0; k < 3; ++k) {
      int row = yy - 1 + k;
      if (row < 0 || row >= ry) continue;
      for (int j = 0; j < rx * 4; ++j) film[(size_t)row * rx * 4 + j] += spill[ri][(size_t)k * rx * 4 + j];
    }
  }
}

}  // namespace gyo

using namespace gyo;

extern "C" {

const char* gyo_tables_digest() { return GYT_TABLES_DIGEST; }

void gyo_set_trace(int on) { g_trace = on; }

float gyo_sobol(uint32_t dim, uint64_t index) { return sobol_sample(index, dim); }
float gyo_halton(uint32_t dim, uint64_t index) { return halton_sample(index, dim); }
uint64_t gyo_halton_enum_index(uint32_t res_x, uint32_t res_y, uint32_t s, uint32_t x, uint32_t y) {
  return HaltonEnumC(res_x, res_y).index(s, x, y);
}

uint64_t gyo_enum_index(uint32_t res_x, uint32_t res_y, uint32_t s, uint32_t x, uint32_t y) {
  return enum_index(log2_pow2_res(res_x, res_y), s, x, y);
}

void gyo_raster_to_world(const CameraIn* c, double* out16) {
  M4 m = raster_to_world(*c);
  std::memcpy(out16, m.m, sizeof(m.m));
}

void* gyo_scene_create(const SceneIn* in) {
  auto* h = new Handle();
  h->sf = make_scene<float>(*in);
  h->sd = make_scene<double>(*in);
  return h;
}

void gyo_scene_destroy(void* p) {
  auto* h = (Handle*)p;
  delete h->sf;
  delete h->sd;
  delete h;
}

// rays: n records of (o[3], d[3], tmax) as float. precision 32 or 64.
int gyo_closest_hit(void* p, int64_t n, const float* rays, int precision, int32_t* prim, double* t, double* b1,
                    double* b2) {
  auto* h = (Handle*)p;
  for (int64_t i = 0; i < n; ++i) {
    const float* r = &rays[7 * i];
    if (precision == 64) {
      Ray<double> ray{V3<double>(r[0], r[1], r[2]), V3<double>(r[3], r[4], r[5]), (double)r[6], 0.0};
      Isect<double> is;
      prim[i] = closest_hit(*h->sd, ray, &is);
      t[i] = ray.tmax; b1[i] = is.b1; b2[i] = is.b2;
    } else {
      Ray<float> ray{V3<float>(r[0], r[1], r[2]), V3<float>(r[3], r[4], r[5]), r[6], 0.f};
      Isect<float> is;
      prim[i] = closest_hit(*h->sf, ray, &is);
      t[i] = ray.tmax; b1[i] = is.b1; b2[i] = is.b2;
    }
    if (prim[i] < 0) t[i] = b1[i] = b2[i] = 0;
  }
  return 0;
}

int gyo_any_hit(void* p, int64_t n, const float* rays, int32_t* out) {
  auto* h = (Handle*)p;
  for (int64_t i = 0; i < n; ++i) {
    const float* r = &rays[7 * i];
    Ray<double> ray{V3<double>(r[0], r[1], r[2]), V3<double>(r[3], r[4], r[5]), (double)r[6], 0.0};
    out[i] = occluded(*h->sd, ray) ? 1 : 0;
  }
  return 0;
}

// force_rr (optional): per-path roulette-draw masks to replay; rr_out
// (optional) receives the masks this run produced.
// force_occ / force_mis (optional) replay recorded shadow-occlusion and
// MIS-hit decisions; occ_out / mis_out receive the decisions taken.
int gyo_paths(void* p, const CameraIn* c, const ParamsIn* pr, int64_t n, const uint32_t* x, const uint32_t* y,
              const uint32_t* s, int precision, double* L, int32_t* cursor, int threads, const uint64_t* force_rr,
              uint64_t* rr_out, const uint64_t* force_occ, const uint64_t* force_mis, uint64_t* occ_out,
              uint64_t* mis_out) {
  auto* h = (Handle*)p;
  if (precision == 64)
    paths_impl<double>(h, c, pr, n, x, y, s, L, cursor, threads, force_rr, rr_out, force_occ, force_mis, occ_out,
                       mis_out);
  else
    paths_impl<float>(h, c, pr, n, x, y, s, L, cursor, threads, force_rr, rr_out, force_occ, force_mis, occ_out,
                      mis_out);
  return 0;
}

// Path replay adjoint of n explicit paths with adjoint weights delta (n*3),
// replaying the given decisions (any may be null): gradient sums into
// grad_mat (n_materials*4: a.rgb, alpha) and grad_em (n_emission*3), path
// radiance into L (n*3). Chunks of 256 paths accumulate separately and are
// summed in chunk order, so the result does not depend on the thread count.
int gyo_adjoint(void* p, const CameraIn* c, const ParamsIn* pr, int64_t n, const uint32_t* x, const uint32_t* y,
                const uint32_t* s, int precision, const float* delta, int threads, const uint64_t* force_rr,
                const uint64_t* force_occ, const uint64_t* force_mis, uint32_t n_materials, uint32_t n_emission,
                double* grad_mat, double* grad_em, double* L) {
  auto* h = (Handle*)p;
  const int chunks = (int)((n + 255) / 256);
  std::vector<double> gm((size_t)chunks * n_materials * 4, 0.0), ge((size_t)chunks * n_emission * 3, 0.0);
  auto run = [&](auto tag) {
    using T = decltype(tag);
    Scene<T>* sc = get<T>(h);
    CamT<T> cam = make_cam<T>(*c);
    parallel_rows(chunks, threads, [&](int ch) {
      for (int64_t i = (int64_t)ch * 256; i < std::min<int64_t>(n, (int64_t)ch * 256 + 256); ++i) {
        int cur = 0;
        Replay rp;
        rp.force_occ = force_occ ? &force_occ[i] : nullptr;
        rp.force_mis = force_mis ? &force_mis[i] : nullptr;
        AdjAcc<T> adj;
        adj.delta = V3<T>((T)delta[3 * i], (T)delta[3 * i + 1], (T)delta[3 * i + 2]);
        adj.sc = sc;
        adj.gm = &gm[(size_t)ch * n_materials * 4];
        adj.ge = n_emission ? &ge[(size_t)ch * n_emission * 3] : nullptr;
        V3<T> l = trace_path(*sc, cam, *c, *pr, x[i], y[i], s[i], &cur, nullptr, nullptr,
                             force_rr ? &force_rr[i] : nullptr, nullptr, &rp, &adj);
        if (L) { L[3 * i] = (double)l.x; L[3 * i + 1] = (double)l.y; L[3 * i + 2] = (double)l.z; }
      }
    });
  };
  if (precision == 64) run(double());
  else run(float());
  for (size_t k = 0; k < (size_t)n_materials * 4; ++k) {
    double v = 0;
    for (int ch = 0; ch < chunks; ++ch) v += gm[(size_t)ch * n_materials * 4 + k];
    grad_mat[k] = v;
  }
  for (size_t k = 0; k < (size_t)n_emission * 3; ++k) {
    double v = 0;
    for (int ch = 0; ch < chunks; ++ch) v += ge[(size_t)ch * n_emission * 3 + k];
    grad_em[k] = v;
  }
  return 0;
}

// Test hook: BSDF sampling and pdfs from these material parameters (n*16,
// the scene's material count) while BSDF values keep the scene's; null
// restores the scene's own. A finite difference in a BSDF parameter with the
// sampling held fixed is the derivative that path replay computes.
int gyo_set_sampling_materials(void* p, const float* mat_params) {
  auto* h = (Handle*)p;
  auto set = [&](auto* sc) {
    if (!sc) return;
    sc->smats.clear();
    if (!mat_params) return;
    sc->smats = sc->mats;
    for (size_t m = 0; m < sc->smats.size(); ++m) std::memcpy(sc->smats[m].p, &mat_params[m * 16], 16 * sizeof(float));
  };
  set(h->sf);
  set(h->sd);
  return 0;
}

// d log f / d alpha of the GGX lobe (alpha, local wo, wi), for a CPU check of
// the derivative against finite differences of the lobe's value.
double gyo_ggx_dlog_alpha(double alpha, const double* wo, const double* wi) {
  GGX<double> g{alpha, alpha};
  return ggx_dlog_alpha(g, V3<double>(wo[0], wo[1], wo[2]), V3<double>(wi[0], wi[1], wi[2]));
}

// log of the GGX lobe's value f (first channel) for alpha at local wo, wi
// (eta = k = 1.5, a = 1), the function whose derivative the above is.
double gyo_ggx_log_f(double alpha, const double* wo, const double* wi) {
  Material m;
  m.type = 3;
  std::memset(m.p, 0, sizeof(m.p));
  m.p[0] = m.p[1] = m.p[2] = 1.f;
  Lobe<double> l = make_lobe<double>(m);
  l.g = GGX<double>{alpha, alpha};
  l.ceta = V3<double>(1.5, 1.5, 1.5);
  l.ck = V3<double>(1.5, 1.5, 1.5);
  V3<double> f = l.eval(V3<double>(wo[0], wo[1], wo[2]), V3<double>(wi[0], wi[1], wi[2]));
  return std::log(f.x);
}

// Accumulates rows [row0, row1) of the image into film (res_x*res_y*4 doubles:
// colour sum and weight), exactly as Film::AddSample would.
int gyo_render(void* p, const CameraIn* c, const ParamsIn* pr, uint32_t row0, uint32_t row1, int precision,
               double* film, int threads) {
  auto* h = (Handle*)p;
  if (precision == 64) render_impl<double>(h, c, pr, row0, row1, film, threads);
  else render_impl<float>(h, c, pr, row0, row1, film, threads);
  return 0;
}

// BxDF tables in the local frame; same record layout as the reference harness's
// "bsdf" command (u32 type, f32 params[16], wo[3], u[3], we[3]) -> 11 floats.
int gyo_bsdf(int64_t n, const void* cases, double* out) {
  const char* base = (const char*)cases;
  const size_t rec = 4 + 4 * 25;
  for (int64_t i = 0; i < n; ++i) {
    Material m;
    std::memcpy(&m.type, base + i * rec, 4);
    float f[25];
    std::memcpy(f, base + i * rec + 4, sizeof(f));
    std::memcpy(m.p, f, sizeof(m.p));
    Lobe<double> l = make_lobe<double>(m);
    V3<double> wo(f[16], f[17], f[18]), we(f[22], f[23], f[24]), wi;
    double pdf;
    V3<double> fs = l.sample(wo, &wi, &pdf, f[19], f[20], f[21]);
    V3<double> fe = l.eval(wo, we);
    double pe = l.pdf(wo, we);
    double* o = &out[i * 11];
    o[0] = fs.x; o[1] = fs.y; o[2] = fs.z; o[3] = wi.x; o[4] = wi.y; o[5] = wi.z; o[6] = pdf;
    o[7] = fe.x; o[8] = fe.y; o[9] = fe.z; o[10] = pe;
  }
  return 0;
}

}  // extern "C"
