// Wavefront OBJ ingestion (see gyt_obj.h). The arithmetic follows the
// reference build exactly (float, unfused), so that positions, normals and
// the triangulation of polygons agree bit for bit with Mesh::LoadFromFile.
#include "gyt_obj.h"

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace gyt {
namespace {

struct Idx {
  int v = -1, vt = -1, vn = -1;
};

bool is_digit(char c) { return c >= '0' && c <= '9'; }

// tinyobjloader's tryParseDouble (tiny_obj_loader.h:807-931): the integer
// digits accumulate as mantissa * 10 + d, the decimal digits as d * 10^-k
// (k < 8 from a table of the double literals 0.1 ... 0.0000001, else
// pow(10, -k)), the decimal exponent applies as ldexp(m * 5^e, e). Parsing
// stops at the first character that does not fit; no digit at all fails.
bool parse_double(const char* s, const char* end, double* out) {
  if (s >= end) return false;
  static const double kLut[] = {1.0, 0.1, 0.01, 0.001, 0.0001, 0.00001, 0.000001, 0.0000001};
  double mantissa = 0.0;
  int exponent = 0, read = 0;
  char sign = '+', exp_sign = '+';
  const char* c = s;
  bool leading_dot = false;
  if (*c == '+' || *c == '-') {
    sign = *c++;
    if (c != end && *c == '.') leading_dot = true;
  } else if (*c == '.') {
    leading_dot = true;
  } else if (!is_digit(*c)) {
    return false;
  }
  if (!leading_dot) {
    while (c != end && is_digit(*c)) {
      mantissa *= 10;
      mantissa += (int)(*c - '0');
      ++c;
      ++read;
    }
    if (read == 0) return false;
  }
  if (c != end) {
    bool exp_part = false;
    if (*c == '.') {
      ++c;
      read = 1;
      while (c != end && is_digit(*c)) {
        mantissa += (int)(*c - '0') * (read < 8 ? kLut[read] : std::pow(10.0, -read));
        ++read;
        ++c;
      }
      exp_part = c != end && (*c == 'e' || *c == 'E');
    } else {
      exp_part = *c == 'e' || *c == 'E';
    }
    if (exp_part) {
      ++c;
      if (c != end && (*c == '+' || *c == '-')) {
        exp_sign = *c++;
      } else if (!(c != end && is_digit(*c))) {
        return false;  // an empty exponent
      }
      read = 0;
      while (c != end && is_digit(*c)) {
        exponent *= 10;
        exponent += (int)(*c - '0');
        ++c;
        ++read;
      }
      exponent *= exp_sign == '+' ? 1 : -1;
      if (read == 0) return false;
    }
  }
  *out = (sign == '+' ? 1 : -1) * (exponent ? std::ldexp(mantissa * std::pow(5.0, exponent), exponent) : mantissa);
  return true;
}

// parseReal: the next blank-separated token as a float, `def` when absent or
// not a number.
float parse_real(const char*& p, double def) {
  p += std::strspn(p, " \t");
  const char* end = p + std::strcspn(p, " \t\r");
  double v = def;
  parse_double(p, end, &v);
  p = end;
  return (float)v;
}

// fixIndex: 1-based from the start, negative from the end (the count of
// elements read so far); 0 is invalid.
bool fix_index(int i, int n, int* out) {
  if (i > 0) {
    *out = i - 1;
    return true;
  }
  if (i < 0) {
    *out = n + i;
    return true;
  }
  return false;
}

// parseTriple: v, v/vt, v//vn or v/vt/vn, each number read as atoi does.
bool parse_triple(const char*& p, int nv, int nvn, int nvt, Idx* out) {
  Idx r;
  if (!fix_index(std::atoi(p), nv, &r.v)) return false;
  p += std::strcspn(p, "/ \t\r");
  if (*p != '/') {
    *out = r;
    return true;
  }
  ++p;
  if (*p == '/') {
    ++p;
    if (!fix_index(std::atoi(p), nvn, &r.vn)) return false;
    p += std::strcspn(p, "/ \t\r");
    *out = r;
    return true;
  }
  if (!fix_index(std::atoi(p), nvt, &r.vt)) return false;
  p += std::strcspn(p, "/ \t\r");
  if (*p != '/') {
    *out = r;
    return true;
  }
  ++p;
  if (!fix_index(std::atoi(p), nvn, &r.vn)) return false;
  p += std::strcspn(p, "/ \t\r");
  *out = r;
  return true;
}

// Crossing-number point-in-polygon test (W. R. Franklin's pnpoly), as the
// triangulation below uses it.
bool inside(const float* vx, const float* vy, float tx, float ty) {
  bool c = false;
  for (int i = 0, j = 2; i < 3; j = i++)
    if (((vy[i] > ty) != (vy[j] > ty)) && (tx < (vx[j] - vx[i]) * (ty - vy[i]) / (vy[j] - vy[i]) + vx[i])) c = !c;
  return c;
}

// tinyobjloader's polygon triangulation (exportGroupsToShape,
// tiny_obj_loader.h:1364-1573): project onto the two axes other than the
// largest component of the first non-degenerate corner's cross product, take
// the signed area, then clip ears: the triangle of three consecutive
// vertices is cut off when it turns like the polygon and holds no other
// vertex, else the start moves on; a pass without progress ends it (the
// rest is dropped). Triangles keep the face's vertex order.
void triangulate(const std::vector<Idx>& face, const std::vector<float>& v, std::vector<Idx>* tris) {
  size_t np = face.size();
  if (np < 3) return;
  auto ok3 = [&](const Idx& a) { return (size_t)(3 * (size_t)a.v + 2) < v.size(); };
  size_t axes[2] = {1, 2};
  for (size_t k = 0; k < np; ++k) {
    const Idx &i0 = face[k % np], &i1 = face[(k + 1) % np], &i2 = face[(k + 2) % np];
    if (!ok3(i0) || !ok3(i1) || !ok3(i2)) continue;
    const float* a = &v[3 * (size_t)i0.v];
    const float* b = &v[3 * (size_t)i1.v];
    const float* c = &v[3 * (size_t)i2.v];
    const float e0x = b[0] - a[0], e0y = b[1] - a[1], e0z = b[2] - a[2];
    const float e1x = c[0] - b[0], e1y = c[1] - b[1], e1z = c[2] - b[2];
    const float cx = std::fabs(e0y * e1z - e0z * e1y);
    const float cy = std::fabs(e0z * e1x - e0x * e1z);
    const float cz = std::fabs(e0x * e1y - e0y * e1x);
    if (cx > FLT_EPSILON || cy > FLT_EPSILON || cz > FLT_EPSILON) {
      if (!(cx > cy && cx > cz)) {
        axes[0] = 0;
        if (cz > cx && cz > cy) axes[1] = 1;
      }
      break;
    }
  }
  auto coord = [&](const Idx& a, size_t axis, float* out) {
    const size_t i = 3 * (size_t)a.v + axis;
    if (i >= v.size()) return false;
    *out = v[i];
    return true;
  };
  float area = 0.f;
  for (size_t k = 0; k < np; ++k) {
    const Idx &i0 = face[k], &i1 = face[(k + 1) % np];
    float x0, y0, x1, y1;
    if (!coord(i0, axes[0], &x0) || !coord(i0, axes[1], &y0) || !coord(i1, axes[0], &x1) || !coord(i1, axes[1], &y1))
      continue;
    area += (x0 * y1 - y0 * x1) * 0.5f;
  }
  std::vector<Idx> rem = face;
  size_t guess = 0, iterations = face.size(), previous = rem.size();
  while (rem.size() > 3 && iterations > 0) {
    np = rem.size();
    if (guess >= np) guess -= np;
    if (previous != np) {
      previous = np;
      iterations = np;
    } else {
      --iterations;
    }
    Idx ind[3];
    float vx[3], vy[3];
    for (size_t k = 0; k < 3; ++k) {
      ind[k] = rem[(guess + k) % np];
      if (!coord(ind[k], axes[0], &vx[k]) || !coord(ind[k], axes[1], &vy[k])) vx[k] = vy[k] = 0.f;
    }
    const float e0x = vx[1] - vx[0], e0y = vy[1] - vy[0], e1x = vx[2] - vx[1], e1y = vy[2] - vy[1];
    const float cross = e0x * e1y - e0y * e1x;
    if (cross * area < 0.f) {
      ++guess;
      continue;
    }
    bool overlap = false;
    for (size_t o = 3; o < np; ++o) {
      const size_t idx = (guess + o) % np;
      float tx, ty;
      if (idx >= rem.size() || !coord(rem[idx], axes[0], &tx) || !coord(rem[idx], axes[1], &ty)) continue;
      if (inside(vx, vy, tx, ty)) {
        overlap = true;
        break;
      }
    }
    if (overlap) {
      ++guess;
      continue;
    }
    tris->insert(tris->end(), {ind[0], ind[1], ind[2]});
    for (size_t r = (guess + 1) % np; r + 1 < np; ++r) rem[r] = rem[r + 1];
    rem.pop_back();
  }
  if (rem.size() == 3) tris->insert(tris->end(), {rem[0], rem[1], rem[2]});
}

}  // namespace

bool load_obj(const std::string& path, bool reverse, ObjMesh* out, std::string* err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    *err = "cannot open " + path;
    return false;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  std::vector<float> v, vn, vt;
  std::vector<Idx> tri;  // triangulated faces, three indices each
  size_t pos = 0, line_no = 0;
  while (pos < text.size()) {
    // a line ends at \n, \r\n or \r
    size_t e = text.find_first_of("\r\n", pos);
    if (e == std::string::npos) e = text.size();
    std::string line = text.substr(pos, e - pos);
    pos = e < text.size() && text[e] == '\r' && e + 1 < text.size() && text[e + 1] == '\n' ? e + 2 : e + 1;
    ++line_no;
    const char* p = line.c_str();
    p += std::strspn(p, " \t");
    if (p[0] == 'v' && (p[1] == ' ' || p[1] == '\t')) {
      p += 2;
      const float x = parse_real(p, 0.0), y = parse_real(p, 0.0), z = parse_real(p, 0.0);
      v.insert(v.end(), {x, y, z});
    } else if (p[0] == 'v' && p[1] == 'n' && (p[2] == ' ' || p[2] == '\t')) {
      p += 3;
      const float x = parse_real(p, 0.0), y = parse_real(p, 0.0), z = parse_real(p, 0.0);
      vn.insert(vn.end(), {x, y, z});
    } else if (p[0] == 'v' && p[1] == 't' && (p[2] == ' ' || p[2] == '\t')) {
      p += 3;
      const float x = parse_real(p, 0.0), y = parse_real(p, 0.0);
      vt.insert(vt.end(), {x, y});
    } else if (p[0] == 'f' && (p[1] == ' ' || p[1] == '\t')) {
      p += 2;
      p += std::strspn(p, " \t");
      std::vector<Idx> face;
      while (!(*p == '\r' || *p == '\n' || *p == '\0')) {
        Idx idx;
        if (!parse_triple(p, (int)(v.size() / 3), (int)(vn.size() / 3), (int)(vt.size() / 2), &idx)) {
          *err = path + ":" + std::to_string(line_no) + ": bad face index (zero or not a number)";
          return false;
        }
        face.push_back(idx);
        p += std::strspn(p, " \t\r");
      }
      triangulate(face, v, &tri);
    }
  }
  // Mesh::LoadFromFile's records: three new vertices per triangle; normals
  // from the file or the face normal Cross(p1 - p0, p2 - p0), normalised
  // when its length exceeds 1e-6; the second and third vertex swapped when
  // reverse_vertices is set.
  out->pos.clear();
  out->nrm.clear();
  out->uv.clear();
  const size_t nt = tri.size() / 3;
  out->pos.reserve(9 * nt);
  out->nrm.reserve(9 * nt);
  out->uv.reserve(6 * nt);
  for (size_t t = 0; t < nt; ++t) {
    const Idx* f3 = &tri[3 * t];
    float P[3][3], N[3][3], U[3][2];
    int with_normal = 0;
    for (int k = 0; k < 3; ++k) {
      const Idx& a = f3[k];
      if (a.v < 0 || 3 * (size_t)a.v + 2 >= v.size()) {
        *err = path + ": vertex index out of range";
        return false;
      }
      for (int c = 0; c < 3; ++c) P[k][c] = v[3 * (size_t)a.v + c];
      if (a.vn != -1) {
        if (a.vn < 0 || 3 * (size_t)a.vn + 2 >= vn.size()) {
          *err = path + ": normal index out of range";
          return false;
        }
        for (int c = 0; c < 3; ++c) N[k][c] = vn[3 * (size_t)a.vn + c];
        ++with_normal;
      }
      U[k][0] = U[k][1] = 0.f;
      if (a.vt != -1) {
        if (a.vt < 0 || 2 * (size_t)a.vt + 1 >= vt.size()) {
          *err = path + ": texture coordinate index out of range";
          return false;
        }
        U[k][0] = vt[2 * (size_t)a.vt];
        U[k][1] = vt[2 * (size_t)a.vt + 1];
      }
    }
    if (with_normal != 0 && with_normal != 3) {
      *err = path + ": a face gives normals for some of its vertices only";
      return false;
    }
    if (with_normal == 0) {
      const float ax = P[1][0] - P[0][0], ay = P[1][1] - P[0][1], az = P[1][2] - P[0][2];
      const float bx = P[2][0] - P[0][0], by = P[2][1] - P[0][1], bz = P[2][2] - P[0][2];
      float g[3] = {ay * bz - az * by, az * bx - ax * bz, ax * by - ay * bx};
      const float len = std::sqrt((g[0] * g[0] + g[1] * g[1]) + g[2] * g[2]);
      if (len > 1e-6f)
        for (float& c : g) c = c / len;
      for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c) N[k][c] = g[c];
    }
    const int order[3] = {0, reverse ? 2 : 1, reverse ? 1 : 2};
    for (int k : order) {
      out->pos.insert(out->pos.end(), P[k], P[k] + 3);
      out->nrm.insert(out->nrm.end(), N[k], N[k] + 3);
      out->uv.insert(out->uv.end(), U[k], U[k] + 2);
    }
  }
  return true;
}

}  // namespace gyt
