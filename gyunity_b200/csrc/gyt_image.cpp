// Image file containers (see gyt_image.h). The reference writes through
// stb_image_write (image/ImageIO.cpp:117-149); these are independent encoders
// of the same formats: the decoded pixels are what must agree, not the bytes.
#include "gyt_image.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

namespace gyt {
namespace {

struct File {
  FILE* f;
  explicit File(const std::string& path) : f(std::fopen(path.c_str(), "wb")) {}
  ~File() {
    if (f) std::fclose(f);
  }
  bool put(const void* p, size_t n) { return f && std::fwrite(p, 1, n, f) == n; }
};

void be32(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back((uint8_t)(x >> 24));
  v.push_back((uint8_t)(x >> 16));
  v.push_back((uint8_t)(x >> 8));
  v.push_back((uint8_t)x);
}

void le16(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back((uint8_t)x);
  v.push_back((uint8_t)(x >> 8));
}

void le32(std::vector<uint8_t>& v, uint32_t x) {
  le16(v, x & 0xffffu);
  le16(v, x >> 16);
}

// CRC-32 of PNG chunks (ISO 3309 polynomial, reflected: 0xEDB88320).
uint32_t crc32(const uint8_t* p, size_t n, uint32_t c = 0xffffffffu) {
  static uint32_t table[256];
  static bool init = false;
  if (!init) {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t r = i;
      for (int k = 0; k < 8; ++k) r = (r & 1u) ? 0xEDB88320u ^ (r >> 1) : r >> 1;
      table[i] = r;
    }
    init = true;
  }
  for (size_t i = 0; i < n; ++i) c = table[(c ^ p[i]) & 0xffu] ^ (c >> 8);
  return c;
}

void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
  be32(out, (uint32_t)data.size());
  const size_t start = out.size();
  out.insert(out.end(), type, type + 4);
  out.insert(out.end(), data.begin(), data.end());
  be32(out, crc32(&out[start], out.size() - start) ^ 0xffffffffu);
}

}  // namespace

// PNG (RFC 2083): 8-bit truecolour, every row with filter 0, the zlib stream
// (RFC 1950) made of stored deflate blocks (RFC 1951, type 0) and closed by
// the Adler-32 of the raw rows.
bool write_png_rgb8(const std::string& path, const uint8_t* rgb, uint32_t w, uint32_t h) {
  std::vector<uint8_t> raw;
  raw.reserve((size_t)h * (3 * (size_t)w + 1));
  for (uint32_t y = 0; y < h; ++y) {
    raw.push_back(0);
    raw.insert(raw.end(), rgb + 3 * (size_t)w * y, rgb + 3 * (size_t)w * (y + 1));
  }
  std::vector<uint8_t> z = {0x78, 0x01};
  uint32_t a = 1, b = 0;
  for (uint8_t v : raw) {
    a = (a + v) % 65521u;
    b = (b + a) % 65521u;
  }
  size_t pos = 0;
  do {
    const size_t n = std::min<size_t>(65535, raw.size() - pos);
    z.push_back(pos + n == raw.size() ? 1 : 0);
    le16(z, (uint32_t)n);
    le16(z, (uint32_t)(~n & 0xffffu));
    z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
    pos += n;
  } while (pos < raw.size());
  be32(z, (b << 16) | a);
  std::vector<uint8_t> ihdr;
  be32(ihdr, w);
  be32(ihdr, h);
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});
  std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
  chunk(out, "IHDR", ihdr);
  chunk(out, "IDAT", z);
  chunk(out, "IEND", {});
  File f(path);
  return f.put(out.data(), out.size());
}

// BMP: BITMAPFILEHEADER + BITMAPINFOHEADER, 24 bits per pixel, rows bottom
// up in BGR order, each padded to a multiple of 4 bytes.
bool write_bmp_rgb8(const std::string& path, const uint8_t* rgb, uint32_t w, uint32_t h) {
  const uint32_t row = (3 * w + 3) & ~3u;
  std::vector<uint8_t> out = {'B', 'M'};
  le32(out, 54 + row * h);
  le32(out, 0);
  le32(out, 54);
  le32(out, 40);
  le32(out, w);
  le32(out, h);
  le16(out, 1);
  le16(out, 24);
  le32(out, 0);
  le32(out, row * h);
  le32(out, 2835);
  le32(out, 2835);
  le32(out, 0);
  le32(out, 0);
  for (uint32_t k = 0; k < h; ++k) {
    const uint8_t* src = rgb + 3 * (size_t)w * (h - 1 - k);
    for (uint32_t x = 0; x < w; ++x) out.insert(out.end(), {src[3 * x + 2], src[3 * x + 1], src[3 * x]});
    out.insert(out.end(), row - 3 * w, 0);
  }
  File f(path);
  return f.put(out.data(), out.size());
}

// Radiance .hdr (Ward's RGBE). Scanlines of width 8..32767 use the run-length
// layout (four channel planes), here as literal runs of at most 128 bytes,
// which a reader cannot mistake for flat pixels; other widths are flat.
bool write_hdr_rgbe(const std::string& path, const uint8_t* rgbe, uint32_t w, uint32_t h) {
  char head[128];
  const int hn = std::snprintf(head, sizeof(head), "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %u +X %u\n", h, w);
  std::vector<uint8_t> out(head, head + hn);
  const bool rle = w >= 8 && w <= 32767;
  for (uint32_t y = 0; y < h; ++y) {
    const uint8_t* s = rgbe + 4 * (size_t)w * y;
    if (!rle) {
      out.insert(out.end(), s, s + 4 * (size_t)w);
      continue;
    }
    out.insert(out.end(), {2, 2, (uint8_t)(w >> 8), (uint8_t)(w & 0xffu)});
    for (int c = 0; c < 4; ++c)
      for (uint32_t x = 0; x < w;) {
        const uint32_t n = std::min<uint32_t>(128, w - x);
        out.push_back((uint8_t)n);
        for (uint32_t k = 0; k < n; ++k) out.push_back(s[4 * (size_t)(x + k) + c]);
        x += n;
      }
  }
  File f(path);
  return f.put(out.data(), out.size());
}

}  // namespace gyt
