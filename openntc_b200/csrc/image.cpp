// PNM and PNG decoding to RGBA8 (see image.h).  PNG per RFC 2083 with zlib inflate.
#include "image.h"

#include <algorithm>
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

// Bytes of one filtered row of a (sub-)image w pixels wide at `bits` bits per pixel.
size_t row_bytes(size_t w, int bits) { return (w * (size_t)bits + 7) / 8; }

// Reverses the per-row filters (RFC 2083 section 6) of one h-row sub-image in place in `rows`
// (each row: a filter byte then rb bytes), writing the unfiltered rows to out[h][rb].
bool unfilter(const uint8_t* rows, size_t rb, size_t h, size_t bpp, std::vector<uint8_t>& out)
{
  out.assign(rb * h, 0);
  for (size_t y = 0; y < h; y++) {
    const uint8_t* src = rows + (rb + 1) * y + 1;
    const int filter = rows[(rb + 1) * y];
    uint8_t* cur = &out[rb * y];
    const uint8_t* prev = y > 0 ? &out[rb * (y - 1)] : nullptr;
    for (size_t i = 0; i < rb; i++) {
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
  return true;
}

// Sample `comp` of pixel x of an unfiltered row at bit depth `depth` (1, 2, 4, 8 or 16).
int row_sample(const uint8_t* row, size_t x, int comps, int comp, int depth)
{
  if (depth == 16) return (row[(x * comps + comp) * 2] << 8) | row[(x * comps + comp) * 2 + 1];
  if (depth == 8) return row[x * comps + comp];
  const size_t bit = (x * comps + comp) * (size_t)depth;  // sub-byte samples: one component
  return (row[bit >> 3] >> (8 - depth - (int)(bit & 7))) & ((1 << depth) - 1);
}

// PNG to RGBA8 with stb_image's expansion (what upstream's stbi_load(..., 4) returns,
// libopenntc.cpp:1302): grey g -> (g, g, g, 255), grey+alpha -> (g, g, g, a), palette via
// PLTE/tRNS, 16-bit samples keep their high byte, 1/2/4-bit grey scaled to 8 bits (x 255 / 85 /
// 17), tRNS colour keys give alpha 0.  Non-interlaced and Adam7-interlaced images.
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
  if (!have_ihdr || interlace > 1 || w <= 0 || h <= 0 || w > (1 << 24) || h > (1 << 24)) return false;
  int comps;
  bool depth_ok;
  switch (ctype) {
    case 0: comps = 1; depth_ok = depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16; break;
    case 2: comps = 3; depth_ok = depth == 8 || depth == 16; break;
    case 3: comps = 1; depth_ok = (depth == 1 || depth == 2 || depth == 4 || depth == 8) && !plte.empty(); break;
    case 4: comps = 2; depth_ok = depth == 8 || depth == 16; break;
    case 6: comps = 4; depth_ok = depth == 8 || depth == 16; break;
    default: return false;
  }
  if (!depth_ok) return false;
  const int bits = comps * depth;
  const size_t bpp = std::max<size_t>(1, (size_t)bits / 8);  // filter distance in bytes
  // passes: x0, y0, dx, dy (Adam7, or one pass over the whole image)
  static const int adam7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                                  {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
  static const int whole[1][4] = {{0, 0, 1, 1}};
  const int (*passes)[4] = interlace ? adam7 : whole;
  const int npass = interlace ? 7 : 1;
  size_t pw[7], ph[7], total = 0;
  for (int k = 0; k < npass; k++) {
    const int x0 = passes[k][0], y0 = passes[k][1], dx = passes[k][2], dy = passes[k][3];
    pw[k] = (size_t)w > (size_t)x0 ? ((size_t)w - x0 + dx - 1) / dx : 0;
    ph[k] = (size_t)h > (size_t)y0 ? ((size_t)h - y0 + dy - 1) / dy : 0;
    if (pw[k] && ph[k]) total += ph[k] * (row_bytes(pw[k], bits) + 1);
  }
  std::vector<uint8_t> raw(total);
  uLongf out_len = (uLongf)raw.size();
  if (uncompress(raw.data(), &out_len, idat.data(), (uLong)idat.size()) != Z_OK || out_len != raw.size()) return false;
  // raw samples per pixel, unscaled (up to 16 bits)
  const size_t n = (size_t)w * h;
  std::vector<uint16_t> px(n * comps);
  size_t off = 0;
  std::vector<uint8_t> rows;
  for (int k = 0; k < npass; k++) {
    if (!pw[k] || !ph[k]) continue;
    const size_t rb = row_bytes(pw[k], bits);
    if (!unfilter(&raw[off], rb, ph[k], bpp, rows)) return false;
    off += ph[k] * (rb + 1);
    for (size_t yy = 0; yy < ph[k]; yy++) {
      const size_t y = passes[k][1] + yy * passes[k][3];
      for (size_t xx = 0; xx < pw[k]; xx++) {
        const size_t x = passes[k][0] + xx * passes[k][2];
        for (int c = 0; c < comps; c++)
          px[(y * w + x) * comps + c] = (uint16_t)row_sample(&rows[rb * yy], xx, comps, c, depth);
      }
    }
  }
  // 8-bit value of a sample: the high byte of 16-bit samples, grey scaled up from 1/2/4 bits
  const int scale = depth == 1 ? 255 : depth == 2 ? 85 : depth == 4 ? 17 : 1;
  auto to8 = [&](int v) -> uint8_t { return (uint8_t)(depth == 16 ? v >> 8 : v * scale); };
  // whether sample v of component c equals the tRNS colour key: 16-bit samples against the whole
  // key, others (as stb_image compares them) in the 8-bit domain against the key's low byte scaled
  auto keyed = [&](int c, int v) -> bool {
    const int k = (trns[2 * c] << 8) | trns[2 * c + 1];
    return depth == 16 ? v == k : to8(v) == (uint8_t)((k & 255) * scale);
  };
  rgba.resize(n * 4);
  for (size_t i = 0; i < n; i++) {
    const uint16_t* s = &px[i * comps];
    uint8_t* o = &rgba[i * 4];
    switch (ctype) {
      case 0:
        o[0] = o[1] = o[2] = to8(s[0]);
        o[3] = (trns.size() >= 2 && keyed(0, s[0])) ? 0 : 255;
        break;
      case 2:
        o[0] = to8(s[0]);
        o[1] = to8(s[1]);
        o[2] = to8(s[2]);
        o[3] = (trns.size() >= 6 && keyed(0, s[0]) && keyed(1, s[1]) && keyed(2, s[2])) ? 0 : 255;
        break;
      case 3: {
        const int idx = s[0];
        if ((size_t)idx * 3 + 2 >= plte.size()) return false;
        o[0] = plte[idx * 3];
        o[1] = plte[idx * 3 + 1];
        o[2] = plte[idx * 3 + 2];
        o[3] = (size_t)idx < trns.size() ? trns[idx] : 255;
        break;
      }
      case 4:
        o[0] = o[1] = o[2] = to8(s[0]);
        o[3] = to8(s[1]);
        break;
      default:
        o[0] = to8(s[0]);
        o[1] = to8(s[1]);
        o[2] = to8(s[2]);
        o[3] = to8(s[3]);
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

#include "ontc_debug.h"

extern "C" int ontc_debug_load_image(const char* path, int32_t* width, int32_t* height, uint8_t* rgba)
{
  if (!path || !width || !height) return ONTC_INVALID_STATE;
  std::vector<uint8_t> px;
  int w = 0, h = 0;
  if (!ontc::load_image_rgba8(path, px, w, h)) return ONTC_FILE_NOT_FOUND;
  *width = w;
  *height = h;
  if (rgba) memcpy(rgba, px.data(), px.size());
  return ONTC_SUCCESS;
}
