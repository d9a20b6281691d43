// Image file containers for Film::SaveImage (visual/Film.cpp:6-9 ->
// image/ImageIO.cpp:117-149): the per-pixel work (colour / weight, gamma
// quantisation, RGBE) runs on the GPU; these functions only wrap finished
// bytes into a file.
#pragma once
#include <stdint.h>
#include <string>

namespace gyt {

// 8-bit RGB, row 0 = top image row (rgb: w*h*3 bytes). Return false on I/O errors.
bool write_png_rgb8(const std::string& path, const uint8_t* rgb, uint32_t w, uint32_t h);
bool write_bmp_rgb8(const std::string& path, const uint8_t* rgb, uint32_t w, uint32_t h);
// Radiance RGBE (rgbe: w*h*4 bytes, row 0 = top).
bool write_hdr_rgbe(const std::string& path, const uint8_t* rgbe, uint32_t w, uint32_t h);

}  // namespace gyt
