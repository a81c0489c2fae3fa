// Image loading for manifest textures.  Upstream loads with stb_image forcing 4
// components (libopenntc.cpp:1302); this loader returns the same RGBA8 expansion for
// binary PNM (P5 grey -> g,g,g,255; P6 RGB -> r,g,b,255) and PNG (grey, grey+alpha, RGB,
// RGBA, palette; 1/2/4/8/16-bit as the format allows; non-interlaced or Adam7).  Other
// formats stb_image reads (JPEG, TGA, BMP, PSD, GIF, HDR, PIC) are not decoded here.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ontc {

// Returns false if the file cannot be opened or decoded.
bool load_image_rgba8(const std::string& path, std::vector<uint8_t>& rgba, int& width, int& height);

}  // namespace ontc
