// Image loading for manifest textures.  Upstream loads with stb_image forcing 4
// components (libopenntc.cpp:1302); this loader returns the same RGBA8 expansion for
// binary PNM (P5 grey -> g,g,g,255; P6 RGB -> r,g,b,255) and 8-bit PNG (grey, grey+alpha,
// RGB, RGBA, palette; non-interlaced).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ontc {

// Returns false if the file cannot be opened or decoded.
bool load_image_rgba8(const std::string& path, std::vector<uint8_t>& rgba, int& width, int& height);

}  // namespace ontc
