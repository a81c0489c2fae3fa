// PNM and PNG decoding to RGBA8 (see image.h).  PNG per RFC 2083 with zlib inflate.
#include "image.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>

#include <zlib.h>

namespace ontc {

namespace {

bool read_file(const std::string& path, std::vector<uint8_t>& out)
{
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return true;
}

// ---- PNM (P5 / P6, maxval <= 255) ---------------------------------------------------------
bool pnm_token(const std::vector<uint8_t>& d, size_t& p, int& v)
{
  while (p < d.size()) {
    if (d[p] == '#') {
      while (p < d.size() && d[p] != '\n' && d[p] != '\r') p++;
    } else if (d[p] == ' ' || d[p] == '\t' || d[p] == '\n' || d[p] == '\r' || d[p] == '\v' || d[p] == '\f') {
      p++;
    } else {
      break;
    }
  }
  if (p >= d.size() || d[p] < '0' || d[p] > '9') return false;
  long long x = 0;
  while (p < d.size() && d[p] >= '0' && d[p] <= '9') {
    x = x * 10 + (d[p] - '0');
    if (x > (1 << 30)) return false;
    p++;
  }
  v = (int)x;
  return true;
}

bool decode_pnm(const std::vector<uint8_t>& d, std::vector<uint8_t>& rgba, int& w, int& h)
{
  if (d.size() < 2 || d[0] != 'P' || (d[1] != '5' && d[1] != '6')) return false;
  const int comps = d[1] == '5' ? 1 : 3;
  size_t p = 2;
  int maxval;
  if (!pnm_token(d, p, w) || !pnm_token(d, p, h) || !pnm_token(d, p, maxval)) return false;
  if (w <= 0 || h <= 0 || maxval <= 0 || maxval > 255) return false;
  p++;  // single whitespace after maxval
  const size_t n = (size_t)w * h;
  if (d.size() < p + n * comps) return false;
  rgba.resize(n * 4);
  for (size_t i = 0; i < n; i++) {
    const uint8_t* s = &d[p + i * comps];
    rgba[i * 4 + 0] = s[0];
    rgba[i * 4 + 1] = comps == 3 ? s[1] : s[0];
    rgba[i * 4 + 2] = comps == 3 ? s[2] : s[0];
    rgba[i * 4 + 3] = 255;
  }
  return true;
}

// ---- PNG ----------------------------------------------------------------------------------
uint32_t be32(const uint8_t* p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }

int paeth(int a, int b, int c)
{
  const int p = a + b - c;
  const int pa = p > a ? p - a : a - p;
  const int pb = p > b ? p - b : b - p;
  const int pc = p > c ? p - c : c - p;
  if (pa <= pb && pa <= pc) return a;
  if (pb <= pc) return b;
  return c;
}

bool decode_png(const std::vector<uint8_t>& d, std::vector<uint8_t>& rgba, int& w, int& h)
{
  static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (d.size() < 8 || memcmp(d.data(), sig, 8) != 0) return false;
  size_t p = 8;
  int depth = 0, ctype = -1, interlace = 0;
  std::vector<uint8_t> idat, plte, trns;
  bool have_ihdr = false;
  while (p + 12 <= d.size()) {
    const uint32_t len = be32(&d[p]);
    if (p + 12 + (size_t)len > d.size()) return false;
    const uint8_t* type = &d[p + 4];
    const uint8_t* data = &d[p + 8];
    if (!memcmp(type, "IHDR", 4) && len >= 13) {
      w = (int)be32(data);
      h = (int)be32(data + 4);
      depth = data[8];
      ctype = data[9];
      interlace = data[12];
      have_ihdr = true;
    } else if (!memcmp(type, "PLTE", 4)) {
      plte.assign(data, data + len);
    } else if (!memcmp(type, "tRNS", 4)) {
      trns.assign(data, data + len);
    } else if (!memcmp(type, "IDAT", 4)) {
      idat.insert(idat.end(), data, data + len);
    } else if (!memcmp(type, "IEND", 4)) {
      break;
    }
    p += 12 + (size_t)len;
  }
  if (!have_ihdr || interlace != 0 || (depth != 8 && depth != 16) || w <= 0 || h <= 0) return false;
  int comps;
  switch (ctype) {
    case 0: comps = 1; break;
    case 2: comps = 3; break;
    case 3: comps = 1; if (depth != 8 || plte.empty()) return false; break;
    case 4: comps = 2; break;
    case 6: comps = 4; break;
    default: return false;
  }
  const size_t bpp = (size_t)comps * (depth / 8);
  const size_t stride = (size_t)w * bpp;
  std::vector<uint8_t> raw((stride + 1) * h);
  uLongf out_len = (uLongf)raw.size();
  if (uncompress(raw.data(), &out_len, idat.data(), (uLong)idat.size()) != Z_OK || out_len != raw.size()) return false;
  std::vector<uint8_t> img(stride * h);
  for (int y = 0; y < h; y++) {
    const uint8_t* src = &raw[(stride + 1) * y + 1];
    const int filter = raw[(stride + 1) * y];
    uint8_t* cur = &img[stride * y];
    const uint8_t* prev = y > 0 ? &img[stride * (y - 1)] : nullptr;
    for (size_t i = 0; i < stride; i++) {
      const int a = i >= bpp ? cur[i - bpp] : 0;
      const int b = prev ? prev[i] : 0;
      const int c = (prev && i >= bpp) ? prev[i - bpp] : 0;
      int v = src[i];
      switch (filter) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += b; break;
        case 3: v += (a + b) >> 1; break;
        case 4: v += paeth(a, b, c); break;
        default: return false;
      }
      cur[i] = (uint8_t)v;
    }
  }
  const size_t n = (size_t)w * h;
  rgba.resize(n * 4);
  const int sb = depth / 8;  // 16-bit samples keep their high byte
  auto sample = [&](size_t px, int comp) -> int { return img[px * bpp + (size_t)comp * sb]; };
  auto sample16 = [&](size_t px, int comp) -> int {
    return sb == 2 ? (img[px * bpp + comp * 2] << 8) | img[px * bpp + comp * 2 + 1] : img[px * bpp + comp];
  };
  for (size_t i = 0; i < n; i++) {
    uint8_t* o = &rgba[i * 4];
    switch (ctype) {
      case 0: {
        o[0] = o[1] = o[2] = (uint8_t)sample(i, 0);
        o[3] = 255;
        if (trns.size() >= 2 && sample16(i, 0) == (int)((trns[0] << 8) | trns[1])) o[3] = 0;
        break;
      }
      case 2: {
        o[0] = (uint8_t)sample(i, 0);
        o[1] = (uint8_t)sample(i, 1);
        o[2] = (uint8_t)sample(i, 2);
        o[3] = 255;
        if (trns.size() >= 6 && sample16(i, 0) == (int)((trns[0] << 8) | trns[1]) &&
            sample16(i, 1) == (int)((trns[2] << 8) | trns[3]) && sample16(i, 2) == (int)((trns[4] << 8) | trns[5]))
          o[3] = 0;
        break;
      }
      case 3: {
        const int idx = img[i];
        if ((size_t)idx * 3 + 2 >= plte.size()) return false;
        o[0] = plte[idx * 3];
        o[1] = plte[idx * 3 + 1];
        o[2] = plte[idx * 3 + 2];
        o[3] = (size_t)idx < trns.size() ? trns[idx] : 255;
        break;
      }
      case 4: {
        o[0] = o[1] = o[2] = (uint8_t)sample(i, 0);
        o[3] = (uint8_t)sample(i, 1);
        break;
      }
      default: {
        o[0] = (uint8_t)sample(i, 0);
        o[1] = (uint8_t)sample(i, 1);
        o[2] = (uint8_t)sample(i, 2);
        o[3] = (uint8_t)sample(i, 3);
      }
    }
  }
  return true;
}

}  // namespace

bool load_image_rgba8(const std::string& path, std::vector<uint8_t>& rgba, int& width, int& height)
{
  std::vector<uint8_t> d;
  if (!read_file(path, d)) return false;
  if (decode_png(d, rgba, width, height)) return true;
  return decode_pnm(d, rgba, width, height);
}

}  // namespace ontc
