// Shared definitions of libontc's device code: the per-step record, the model
// description handed to kernels, the texel enumeration, the feature gather and the
// counter-based quantisation noise.
//
// Arithmetic that must agree bit-for-bit with upstream (feature construction,
// ntc_kernel.cu:92-176) is written with explicit fused/unfused intrinsics so the
// compiler cannot re-associate it.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#if defined(__CUDACC__)
#define ONTC_HD __host__ __device__ __forceinline__
#else
#define ONTC_HD inline
#endif

namespace ontc {

constexpr int kHidden = 64;    // libopenntc.cpp:338 hidden_dim_
constexpr int kOutPad = 16;    // libopenntc.cpp:335 out_dim_padded_ (= kMaxChannels)
constexpr int kTile = 128;     // texels per CTA work unit
constexpr int kMaxLevels = 6;
constexpr int kMaxMips = 12;
constexpr int kMaxGrids = 8;   // libopenntc.cpp:336 max_batch_
constexpr int kMaxF = 96;      // largest feature_dim_padded_ (Bpp_0_5 / Bpp_2_25)

// Everything a kernel needs to know about one optimisation step, built on the host
// from the same std::mt19937 draws upstream makes (libopenntc.cpp:564-585).
struct StepRec {
  int32_t lod, level, mip_dim, tile_dim;
  int32_t n_grids, texels, noise, grid_update;
  uint32_t seed;        // quantisation-noise stream of this step
  float norm_lod;       // lod / (mip_count - 1), libopenntc.cpp:630
  float lr_grid, lr_dec;
  float b1, b2;         // decoder Adam bias factors (global step)
  float gb1, gb2;       // latent Adam bias factors (per-level step counter)
  int32_t ox[kMaxGrids], oy[kMaxGrids];
  int32_t step;         // global step index (batch_i_)
  int32_t gstep;        // step index within the level (grid_batch_i_ before the step)
  int32_t gfloor;       // deferred optimiser: every latent of the level has had >= gfloor steps
  int32_t sweep_from;   // host only: floor before the level sweep that precedes this step, or -1
  int32_t exact_grad;   // test mode: latent gradients as exactly-summable dyadic values (see train_tc.cu)
};

// Latent cells a step can touch, as DISJOINT rectangles per pyramid: the union of every
// tile's cell range (texel ranges that wrap around the mip edge split in two per axis),
// conservative by one cell.  Each cell of the footprint belongs to exactly one rectangle, so
// the deferred latent optimiser can give every one its own thread with no claiming.
constexpr int kMaxFootRects = 40;
struct FootRec {
  int32_t n[2];                     // rectangles per pyramid
  int32_t cells[2];                 // cells over the rectangles
  int32_t start[2][kMaxFootRects];  // first cell of each rectangle within its pyramid
  int16_t r[2][kMaxFootRects][4];   // x0, y0, w, h in cells
};

// Ring of per-level-step Adam scalars (lr, bias1, bias2) replayed by the deferred optimiser.
// A cell lags its level by at most 64 level steps (the sweep interval); entries are written
// from the step records up to a batch of steps ahead, so the ring holds twice that.
constexpr int kHistRing = 128;

// One latent pyramid (g0 or g1), fp32 master copy plus Adam state, [dim][dim][C] row-major
// per level, exactly upstream's layout (ntc_kernel.cu:127-129).
struct Pyramid {
  float* p[kMaxLevels];
  float* m[kMaxLevels];
  float* v[kMaxLevels];
  float* g[kMaxLevels];
  int32_t dim[kMaxLevels];
  int32_t channels;
  int32_t bits;
  float delta;
};

struct Model {
  int32_t C0, C1, F, Fp, C;  // channels, feature dim, padded feature dim, output channels
  int32_t mips, levels;
  int32_t mip_dim[kMaxMips];
  const uint8_t* package[kMaxMips];  // targets, u8 [dim][dim][C] per mip
  Pyramid g0, g1;
  // decoder, fp32 master: W0 [64][F] | W1 [64][64] | Wout [16][64]
  float* W;
  float* Wm;
  float* Wv;
  int32_t nW;  // 64*F + 64*64 + 16*64
  // upstream-compatible noise buffers (StepRec::noise == 2), indexed like the level's latents
  const float* noise0;
  const float* noise1;
  // deferred latent optimiser: level steps applied per cell, and the per-level ring of
  // (lr, bias1, bias2) of the level's recent steps
  int32_t* applied[2][kMaxLevels];
  float4* hist[kMaxLevels];
};

ONTC_HD int w0_off() { return 0; }
ONTC_HD int w1_off(int F) { return kHidden * F; }
ONTC_HD int wo_off(int F) { return kHidden * F + kHidden * kHidden; }
ONTC_HD int n_weights(int F) { return kHidden * F + kHidden * kHidden + kOutPad * kHidden; }

ONTC_HD int clampi(int x, int a, int b) { return x > b ? b : (x < a ? a : x); }

// log2 of a power of two, and its exact reciprocal: every texture, grid and tile dimension
// here is a power of two, so x / n == x * rcp_pow2(n) bit for bit and the divisions and
// modulos become shifts and masks.
ONTC_HD int log2_pow2(int n)
{
#if defined(__CUDA_ARCH__)
  return __ffs(n) - 1;
#else
  return __builtin_ctz((unsigned)n);
#endif
}
ONTC_HD float rcp_pow2(int n)
{
  const uint32_t bits = (uint32_t)(127 - log2_pow2(n)) << 23;
#if defined(__CUDA_ARCH__)
  return __uint_as_float(bits);
#else
  float f;
  __builtin_memcpy(&f, &bits, 4);
  return f;
#endif
}

// Texel b of a step's batch -> mip-space (x, y).  Tiles are tile_dim x tile_dim blocks at
// the drawn origins, wrapping mod mip_dim (ntc_kernel.cu:94-99); inside a tile, 128-texel
// work units are 16x8 texel blocks (tile_dim >= 16) so one unit's latent footprint is
// compact, or plain rows for the 4x4 and 8x8 tiles of the smallest mips.
ONTC_HD void texel_xy(const StepRec& s, int b, int& x, int& y)
{
  const int lt = log2_pow2(s.tile_dim);  // tile_dim and mip_dim are powers of two
  const int gi = b >> (2 * lt);
  const int r = b & ((1 << (2 * lt)) - 1);
  int lx, ly;
  if (lt >= 4) {
    const int blk = r >> 7, i = r & 127, lb = lt - 4;  // 2^lb 16-wide blocks per block row
    lx = ((blk & ((1 << lb) - 1)) << 4) + (i & 15);
    ly = ((blk >> lb) << 3) + (i >> 4);
  } else {
    lx = r & ((1 << lt) - 1);
    ly = r >> lt;
  }
  const int mask = s.mip_dim - 1;
  x = (lx + s.ox[gi]) & mask;
  y = (ly + s.oy[gi]) & mask;
}

// Quantisation-noise surrogate U(-delta/2, delta/2) for latent element e of pyramid
// `which` (0 = g0, 1 = g1) in the step whose stream is `seed`.  Counter-based: any
// thread touching the element in that step gets the same value, so no per-level noise
// buffer is written (upstream fills one with cuRAND XORWOW, ntc_kernel.cu:427-446).
// The mixer is the 32-bit "lowbias32" finaliser (xorshift-multiply, constants from
// C. Wellons' hash-prospector search).
ONTC_HD uint32_t noise_bits(uint32_t seed, uint32_t which, uint32_t e)
{
  uint32_t x = e * 0x9E3779B1u + seed;
  x ^= which * 0x85EBCA77u;
  x ^= x >> 16;
  x *= 0x7FEB352Du;
  x ^= x >> 15;
  x *= 0x846CA68Bu;
  x ^= x >> 16;
  return x;
}

ONTC_HD float noise_value(uint32_t seed, uint32_t which, uint32_t e, float delta)
{
  // u in (0, 1) on a 2^-24 lattice, then u*delta - delta/2 (exact for power-of-two delta)
  const float u = ((float)(noise_bits(seed, which, e) >> 8) + 0.5f) * (1.0f / 16777216.0f);
  return u * delta - 0.5f * delta;
}

// Noise added to latent element e of pyramid `which` in step s: none (noise == 0), the
// counter-based surrogate (noise == 1), or upstream's cuRAND buffers (noise == 2).
#if defined(__CUDACC__)
__device__ __forceinline__ float latent_noise(const Model& M, const StepRec& s, uint32_t which, uint32_t e)
{
  if (s.noise == 1) return noise_value(s.seed, which, e, which == 0 ? M.g0.delta : M.g1.delta);
  if (s.noise == 2) return which == 0 ? M.noise0[e] : M.noise1[e];
  return 0.0f;
}
#endif

// hardgelu and its derivative (ntc_kernel.cu:50-62)
ONTC_HD float hardgelu(float x)
{
  if (x < -1.5f) return 0.0f;
  if (x > 1.5f) return x;
  return (x / 3.0f) * (x + 1.5f);
}
ONTC_HD float hardgelu_grad(float x)
{
  if (x < -1.5f) return 0.0f;
  if (x < 1.5f) return (2.0f * x + 1.5f) / 3.0f;
  return 1.0f;
}

// Geometry of one texel's gather (ntc_kernel.cu:100-115).  Corner k = 0..3 is
// (x0 + k%2, y0 + k/2), clamped into the grid; g1 weights are bilinear.
struct Gather {
  int c0[4];   // g0 cell index (y*dim + x) per corner
  int c1[4];   // g1 cell index per corner
  float w1[4]; // g1 bilinear weight per corner
};

ONTC_HD void gather_geometry(int x, int y, int mip_dim, int g0_dim, int g1_dim, Gather& G)
{
  const float rm = rcp_pow2(mip_dim);  // exact: (x + 0.5) / mip_dim
  const float u = ((float)x + 0.5f) * rm;
  const float v = ((float)y + 0.5f) * rm;
  // u * dim is exact (power-of-two dims), so fused and unfused forms agree here
  const float g0x = u * (float)g0_dim - 0.5f;
  const float g0y = v * (float)g0_dim - 0.5f;
  const float g1x = u * (float)g1_dim - 0.5f;
  const float g1y = v * (float)g1_dim - 0.5f;
  const float fx0 = floorf(g0x), fy0 = floorf(g0y), fx1 = floorf(g1x), fy1 = floorf(g1y);
  const int g0x0 = (int)fx0, g0y0 = (int)fy0, g1x0 = (int)fx1, g1y0 = (int)fy1;
  const float g1xf = g1x - fx1;
  const float g1yf = g1y - fy1;
  G.w1[0] = (1.0f - g1xf) * (1.0f - g1yf);
  G.w1[1] = g1xf * (1.0f - g1yf);
  G.w1[2] = (1.0f - g1xf) * g1yf;
  G.w1[3] = g1xf * g1yf;
  for (int k = 0; k < 4; k++) {
    const int j = k & 1, i = k >> 1;
    G.c0[k] = clampi(g0y0 + i, 0, g0_dim - 1) * g0_dim + clampi(g0x0 + j, 0, g0_dim - 1);
    G.c1[k] = clampi(g1y0 + i, 0, g1_dim - 1) * g1_dim + clampi(g1x0 + j, 0, g1_dim - 1);
  }
}

// The corner cells (lower and upper, clamped into the grid) that texels a..b of a mip of size
// `mip` reach in a grid of size gd, along one axis: gather_geometry's arithmetic.  First cell
// lo, count n.
ONTC_HD void foot_span(int a, int b, int mip, int gd, int& lo, int& n)
{
  const float rm = rcp_pow2(mip);
  const float ua = ((float)a + 0.5f) * rm, ub = ((float)b + 0.5f) * rm;
  const int l = (int)floorf(ua * (float)gd - 0.5f), h = (int)floorf(ub * (float)gd - 0.5f) + 1;
  lo = clampi(l, 0, gd - 1);
  n = clampi(h, 0, gd - 1) - lo + 1;
}

// Triangle-wave positional encoding, periods 8/4/2 x (x, y) x phase (0, P/4)
// (ntc_kernel.cu:145-165).  All intermediate values are exact in fp32.
ONTC_HD float pos_enc(int x, int y, int idx)
{
  const int p = idx >> 2, a = (idx >> 1) & 1, h = idx & 1;
  const float P = (float)(8 >> p);
  const float c = (float)(a == 0 ? x : y);
  const float phase = h == 0 ? 0.0f : 0.25f * P;
  const float t = (c + 0.5f + phase) * (0.125f * (float)(1 << p));  // exact: / P
  const float s = t - floorf(t);
  return 1.0f - 4.0f * fabsf(s - 0.5f);
}

}  // namespace ontc
