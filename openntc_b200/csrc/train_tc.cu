// BF16 tensor-core tile kernel for one training step (sm_100a, tcgen05 + TMEM).
//
// A CTA (one per SM, persistent) runs two independent 8-warp groups.  Each group owns one
// 128-texel work unit at a time (two threads per texel row = TMEM lane, each taking half of
// the row's columns) and takes it through the whole per-texel pipeline of upstream's step:
//
//   gather (ntc_kernel.cu:75-177)             -> X    [128 x Kp]  bf16, shared memory
//   H0 = X  W0^T          (M128 N64  K=Kp)    -> TMEM, epilogue: A0 = hg(H0)
//   H1 = A0 W1^T          (M128 N64  K=64)    -> TMEM, epilogue: A1 = hg(H1)
//   Y  = A1 Wout^T        (M128 N16  K=64)    -> TMEM, epilogue: dY = -2(t-y)/(C B), loss
//   dA1 = dY Wout         (M128 N64  K=16)    -> TMEM, epilogue: dH1 = dA1 hg'(H1)
//   dA0 = dH1 W1          (M128 N64  K=64)    -> TMEM, epilogue: dH0 = dA0 hg'(H0)
//   dX  = dH0 W0          (M128 N=Kp K=64)    -> TMEM, epilogue: scatter-add into the latent
//                                                gradients (ntc_kernel.cu:280-341)
// while the weight gradients of both groups accumulate in shared TMEM accumulators:
//   dWout^T += A1^T dY (M64 N16), dW1 += dH1^T A0 (M64 N64), dW0 += dH0^T X (M64 N=Kp),
// K = 128 texels each, written once per CTA to its partial-sum slot (libopenntc.cpp:672-693).
//
// The two groups synchronise only with themselves (named barriers, one mbarrier each), so
// one group's epilogue math runs while the other's MMAs execute.  Operands sit in shared
// memory in the no-swizzle canonical layout; a [128 texels][n] activation tile is the
// K-major A operand of the next layer and, unchanged, the MN-major operand of the
// weight-gradient products.  A0 and dH0 share a buffer, as do A1 and dH1 (each is dead
// before its partner is written).  The latent footprint of a unit is staged once in shared
// memory (noise added once per latent) and its gradient reduced there before one global add
// per latent.  Every wait is bounded and reports a timeout through the error word.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"
#include "tc_ptx.cuh"

namespace ontc {

namespace {

constexpr int kGroupThreads = 256; // 2 threads per texel row: half 0 / half 1 of the columns
constexpr uint32_t kTmemCols = 512;
// TMEM column map: per group a 128-column window [128 g, 128 g + 128) holding
//   H0/H1/dA1/dA0 at +0 (64), Y at +64 (16), and later dX at +0 (<= 96);
// the shared weight-gradient accumulators (M=64 layout) follow.
constexpr uint32_t kColW0 = 256;   // dW0     (<= 96 columns)
constexpr uint32_t kColW1 = 352;   // dW1     (64)
constexpr uint32_t kColWo = 416;   // dWout^T (16)
constexpr int kFootFloats = 7168;  // per group, 28 KB: two staging buffers
constexpr int kFootBuf = kFootFloats / 2;
constexpr int kMaxBoxW = 64;       // latent box limits of the owner-computes scatter
constexpr int kMaxBoxH = 32;

// Operand tiles of the MMAs, all bf16 (tcgen05 kind::f16, fp32 accumulate).
//   EBf16:  one bf16 tile per operand; two 8-warp groups per CTA.
//   ESplit: each fp32 operand value v kept as a bf16 high part h = bf16(v) and low part
//           l = bf16(v - h) in two tiles (the low tile right after the high one), and each
//           product formed as h.h + h.l + l.h by three MMAs into the same fp32 accumulator:
//           about 16 mantissa bits per product, more than the tf32 products of upstream's
//           cuBLAS GEMMs (libopenntc.cpp:374).  Its tiles are twice as large: one group per CTA.
// (kind::tf32 itself reads MN-major operands only in a 32-byte-granule 128-byte swizzle, which
// the same tile cannot share with its K-major use in the next layer.)
struct EBf16 {
  static constexpr bool kSplit = false;
  static constexpr int kGroups = 2, kTileMul = 1;
};
struct ESplit {
  static constexpr bool kSplit = true;
  static constexpr int kGroups = 1, kTileMul = 2;
};
// byte stride between 8-row groups of a [*][cols] bf16 operand tile in the canonical layout
constexpr uint32_t row8(int cols) { return (uint32_t)(cols / 8) * 128; }

template <int C0_, int C1_, int KP_>
struct Shape {
  static constexpr int C0 = C0_, C1 = C1_, Kp = KP_;
  static constexpr int F = ((4 * C0 + C1 + 13 + 3) / 4) * 4;
};

// a [rows][cols] operand tile: the bf16 tile and, split, its low-part tile after it
template <class E>
constexpr uint32_t tile_bytes(int rows, int cols)
{
  return (uint32_t)(rows * cols * 2 * E::kTileMul);
}

template <class SH, class E>
struct GroupSmem {
  static constexpr size_t kX = tile_bytes<E>(128, SH::Kp), kP = tile_bytes<E>(128, 64), kY = tile_bytes<E>(128, 16);
  static constexpr size_t kFoot = kFootFloats * 4;
  static constexpr size_t kBytes = kX + 2 * kP + kY + kFoot;
};

template <class SH, class E>
constexpr size_t smem_bytes()
{
  return E::kGroups * GroupSmem<SH, E>::kBytes + tile_bytes<E>(64, SH::Kp) + tile_bytes<E>(64, 64) +
         tile_bytes<E>(16, 64) + 1024;
}

struct GroupPtrs {
  uint8_t* X;    // [128][Kp]
  uint8_t* P0;   // [128][64]  A0, later dH0
  uint8_t* P1;   // [128][64]  A1, later dH1
  uint8_t* dY;   // [128][16]
  float* foot;   // [2][kFootBuf]: the current unit's latent boxes and the next one's
};

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// Stores 8 consecutive values (columns c0..c0+7, c0 % 8 == 0) of row r of a [rows][cols]
// operand tile as one 16-byte bf16 chunk; split, also their low parts in the low-part tile.
template <class E>
__device__ __forceinline__ void st_chunk(uint8_t* base, int r, int c0, int rows, int cols, const float* v)
{
  uint4 q;
  q.x = pack_bf16(v[0], v[1]);
  q.y = pack_bf16(v[2], v[3]);
  q.z = pack_bf16(v[4], v[5]);
  q.w = pack_bf16(v[6], v[7]);
  const uint32_t off = ptx::cm_off16(r, c0, cols);
  *reinterpret_cast<uint4*>(base + off) = q;
  if constexpr (E::kSplit) {
    const uint32_t* h = &q.x;
    float lo[8];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const __nv_bfloat162 hb = *reinterpret_cast<const __nv_bfloat162*>(&h[i]);
      lo[2 * i] = v[2 * i] - __low2float(hb);  // exact: the high part is v rounded to bf16
      lo[2 * i + 1] = v[2 * i + 1] - __high2float(hb);
    }
    uint4 l;
    l.x = pack_bf16(lo[0], lo[1]);
    l.y = pack_bf16(lo[2], lo[3]);
    l.z = pack_bf16(lo[4], lo[5]);
    l.w = pack_bf16(lo[6], lo[7]);
    *reinterpret_cast<uint4*>(base + rows * cols * 2 + off) = l;
  }
}

// D (+)= A B, operands given by descriptor bases and byte offsets; split, the low parts of A and
// B lie a_lo / b_lo bytes after the high ones and D += A.h B.h + A.h B.l + A.l B.h.  Executed by
// a whole warp (one elected lane issues).
template <class E>
__device__ __forceinline__ void mma(uint32_t d, const ptx::DescBase& A, uint32_t a_off, uint32_t a_lo,
                                    const ptx::DescBase& B, uint32_t b_off, uint32_t b_lo, uint32_t idesc,
                                    uint32_t acc)
{
  ptx::mma_bf16_warp(d, A.at(a_off), B.at(b_off), idesc, acc);
  if constexpr (E::kSplit) {
    ptx::mma_bf16_warp(d, A.at(a_off), B.at(b_off + b_lo), idesc, 1);
    ptx::mma_bf16_warp(d, A.at(a_off + a_lo), B.at(b_off), idesc, 1);
  }
}

// upstream's hardgelu and its derivative in fp32 (the split epilogues), as 8-column chunks
__device__ __forceinline__ void hg_chunk_f32(const float* x, float* a, uint32_t* pre)
{
#pragma unroll
  for (int i = 0; i < 8; i++) {
    pre[i] = __float_as_uint(x[i]);
    a[i] = hardgelu(x[i]);
  }
}
__device__ __forceinline__ void dhg_chunk_f32(const float* da, const uint32_t* pre, float* d)
{
#pragma unroll
  for (int i = 0; i < 8; i++) d[i] = da[i] * hardgelu_grad(__uint_as_float(pre[i]));
}

__device__ __forceinline__ void bar_group(int g) { asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kGroupThreads) : "memory"); }

// The step's level as the tile kernel uses it: resolved once per CTA into shared memory (the
// Model's per-level arrays are kernel parameters indexed by a runtime level), and passed by
// value to the out-of-line paths.
struct LevelArgs {
  const float* p0;
  const float* p1;
  float* g0;
  float* g1;
  const float* n0;  // upstream-mode noise buffers
  const float* n1;
  float delta0, delta1, norm_lod;
  uint32_t seed;
  int d0, d1, mip_dim, noise;
};

__device__ __forceinline__ LevelArgs level_args(const Model& M, const StepRec& s)
{
  LevelArgs L;
  L.p0 = M.g0.p[s.level];
  L.p1 = M.g1.p[s.level];
  L.g0 = M.g0.g[s.level];
  L.g1 = M.g1.g[s.level];
  L.n0 = M.noise0;
  L.n1 = M.noise1;
  L.delta0 = M.g0.delta;
  L.delta1 = M.g1.delta;
  L.norm_lod = s.norm_lod;
  L.seed = s.seed;
  L.d0 = M.g0.dim[s.level];
  L.d1 = M.g1.dim[s.level];
  L.mip_dim = s.mip_dim;
  L.noise = s.noise;
  return L;
}

// latent_noise (common.cuh) for the out-of-line paths
__device__ __forceinline__ float level_noise(const LevelArgs& L, uint32_t which, uint32_t e)
{
  if (L.noise == 1) return noise_value(L.seed, which, e, which == 0 ? L.delta0 : L.delta1);
  if (L.noise == 2) return which == 0 ? L.n0[e] : L.n1[e];
  return 0.0f;
}

// hardgelu of 8 fp32 accumulator values, computed on packed bf16 pairs (the results feed the next
// bf16 MMA, so they are bf16 either way), as one 16-byte chunk of activations:
//   c = clamp(x, -1.5, 1.5);  hg = c * (c + 1.5) * (1/3) + relu(x - 1.5)
// (the second term is x - 1.5 above the knee, where c = 1.5 and the first term is 1.5).
__device__ __forceinline__ uint4 hg_chunk_bf16(const float* x, uint32_t* pre)
{
  const __nv_bfloat162 lo = __floats2bfloat162_rn(-1.5f, -1.5f), hi = __floats2bfloat162_rn(1.5f, 1.5f);
  const __nv_bfloat162 third = __floats2bfloat162_rn(1.0f / 3.0f, 1.0f / 3.0f);
  const __nv_bfloat162 one = __floats2bfloat162_rn(1.0f, 1.0f), mhi = __floats2bfloat162_rn(-1.5f, -1.5f);
  uint32_t w[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
    pre[i] = *reinterpret_cast<const uint32_t*>(&v);  // kept for the backward pass
    const __nv_bfloat162 c = __hmin2(__hmax2(v, lo), hi);
    const __nv_bfloat162 mid = __hmul2(__hmul2(c, __hadd2(c, hi)), third);
    // max(v - 1.5, 0) in one fused operation: v * 1 is exact, so the one rounding is that of v - 1.5
    const __nv_bfloat162 r = __hadd2(mid, __hfma2_relu(v, one, mhi));
    w[i] = *reinterpret_cast<const uint32_t*>(&r);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// dA * hardgelu'(h) for 8 columns on packed bf16 pairs (pre: the packed pre-activations of the
// forward pass), as one 16-byte chunk:
//   hg'(x) = x < -1.5 ? 0 : x < 1.5 ? (2x + 1.5) / 3 : 1
//          = [x >= -1.5] * (c * 2/3 + 0.5 - 0.5 * [x >= 1.5]),  c = clamp(x, -1.5, 1.5)
__device__ __forceinline__ uint4 dhg_chunk_bf16(const float* da, const uint32_t* pre)
{
  const __nv_bfloat162 lo = __floats2bfloat162_rn(-1.5f, -1.5f), hi = __floats2bfloat162_rn(1.5f, 1.5f);
  const __nv_bfloat162 two3 = __floats2bfloat162_rn(2.0f / 3.0f, 2.0f / 3.0f);
  const __nv_bfloat162 half = __floats2bfloat162_rn(0.5f, 0.5f), mhalf = __floats2bfloat162_rn(-0.5f, -0.5f);
  uint32_t w[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const __nv_bfloat162 x = *reinterpret_cast<const __nv_bfloat162*>(&pre[i]);
    const __nv_bfloat162 c = __hmin2(__hmax2(x, lo), hi);
    const __nv_bfloat162 d = __hfma2(__hge2(x, hi), mhalf, __hfma2(c, two3, half));
    const __nv_bfloat162 gr = __hmul2(__hge2(x, lo), d);
    const __nv_bfloat162 r = __hmul2(__floats2bfloat162_rn(da[2 * i], da[2 * i + 1]), gr);
    w[i] = *reinterpret_cast<const uint32_t*>(&r);
  }
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// ---- latent footprint of a unit ---------------------------------------------------------
struct Foot {
  int x0, y0, w, h;
};

// True when the unit is a 16x8 texel block that does not wrap and whose g0/g1 footprints fit the
// lod's staging boxes (the g1 box may start one cell before the footprint, see stage_issue).
template <class SH>
__device__ __forceinline__ bool unit_footprint(const LevelArgs& L, const StepRec& s, const LatentBoxes& B, int unit,
                                               Foot& f0, Foot& f1)
{
  if (B.w0 == 0) return false;
  const int lt = log2_pow2(s.tile_dim);
  if (lt < 4) return false;
  const int b0 = unit * kTile, gi = b0 >> (2 * lt), r0 = b0 & ((1 << (2 * lt)) - 1);
  const int blk = r0 >> 7, lb = lt - 4;
  const int mask = s.mip_dim - 1;
  const int xa = (((blk & ((1 << lb) - 1)) << 4) + s.ox[gi]) & mask;
  const int ya = (((blk >> lb) << 3) + s.oy[gi]) & mask;
  if (xa + 16 > s.mip_dim || ya + 8 > s.mip_dim) return false;
  const int d0 = L.d0, d1 = L.d1;
  foot_span(xa, xa + 15, s.mip_dim, d0, f0.x0, f0.w);
  foot_span(ya, ya + 7, s.mip_dim, d0, f0.y0, f0.h);
  foot_span(xa, xa + 15, s.mip_dim, d1, f1.x0, f1.w);
  foot_span(ya, ya + 7, s.mip_dim, d1, f1.y0, f1.h);
  return f0.w <= B.w0 && f0.h <= B.h0 && f1.w + (f1.x0 & B.g1_shift) <= B.w1 && f1.h <= B.h1;
}

// Which texel columns / rows of a unit touch each box column / row, per corner side: bit t
// of lo[i] is set when texel t's lower corner cell is box cell i, of hi[i] for its upper one.
// With these, the owner of a latent element sums exactly the texel-corner contributions
// the per-texel scatter would have added (ntc_kernel.cu:317-340), without atomics.
struct CornerMasks {
  uint32_t xlo[2][kMaxBoxW], xhi[2][kMaxBoxW];  // [g0/g1][box column]
  uint32_t ylo[2][kMaxBoxH], yhi[2][kMaxBoxH];
  float fx[16], fy[8];                          // g1 bilinear fractions of the unit's columns / rows
};

__device__ __forceinline__ void build_masks(const StepRec& s, int d0, int d1, const Foot& f0, const Foot& f1,
                                            int unit, CornerMasks& cm, int gt)
{
  // thread 0..15: texel column xa + gt; 16..23: texel row ya + gt - 16
  const int lt = log2_pow2(s.tile_dim);
  const int b0 = unit * kTile, gi = b0 >> (2 * lt), r0 = b0 & ((1 << (2 * lt)) - 1);
  const int blk = r0 >> 7, lb = lt - 4;
  const int mask = s.mip_dim - 1;
  const float rm = rcp_pow2(s.mip_dim);
  if (gt < 24) {
    const bool col = gt < 16;
    const int t = col ? gt : gt - 16;
    const int p = col ? ((((blk & ((1 << lb) - 1)) << 4) + s.ox[gi]) & mask) + t
                      : ((((blk >> lb) << 3) + s.oy[gi]) & mask) + t;
    const float u = ((float)p + 0.5f) * rm;  // gather_geometry's arithmetic
    for (int g = 0; g < 2; g++) {
      const int gd = g == 0 ? d0 : d1;
      const float q = u * (float)gd - 0.5f;
      const float fq = floorf(q);
      const int lo = clampi((int)fq, 0, gd - 1), hi = clampi((int)fq + 1, 0, gd - 1);
      const Foot& f = g == 0 ? f0 : f1;
      if (col) {
        atomicOr(&cm.xlo[g][lo - f.x0], 1u << t);
        atomicOr(&cm.xhi[g][hi - f.x0], 1u << t);
        if (g == 1) cm.fx[t] = q - fq;
      } else {
        atomicOr(&cm.ylo[g][lo - f.y0], 1u << t);
        atomicOr(&cm.yhi[g][hi - f.y0], 1u << t);
        if (g == 1) cm.fy[t] = q - fq;
      }
    }
  }
}

// Test mode (StepRec::exact_grad): a feature gradient replaced by n * 2^-24 with
// n = clamp(rint(v * 2^24), -15, 15).  Every latent-gradient term is then such a value times a
// bilinear weight with at most 8 fractional bits (the mip-to-g1 cell ratio is at most 8 in
// every profile), so each latent's gradient is a multiple of 2^-32 below 2^-12 in magnitude
// (at most 256 texels reach a g1 cell): every partial sum is exact, and the float atomics give
// the same bits in any order.  Lets a test compare two optimiser schedules bit for bit.
__device__ __forceinline__ float exact_dyadic(float v)
{
  const float n = fminf(fmaxf(rintf(v * 16777216.0f), -15.0f), 15.0f);
  return n * (1.0f / 16777216.0f);
}

// v / d for the small operands of the box loops (v < 2^20, d >= 1) with one multiply: with
// inv = RN(1/d), (v + 0.5) * inv stays within 2^-3 / d of v / d + 0.5 / d, strictly between the
// two integers around it, so its floor is the quotient (replaces a 32-bit division per item).
__device__ __forceinline__ int div_small(int v, float inv)
{
  return (int)(((float)v + 0.5f) * inv);
}

// Starts the TMA loads of a unit's latent boxes into a staging buffer (one thread): the g0 box
// {C0, w0, h0} at the footprint's first cell, the g1 box {w1 * C1, h1} at its first cell or,
// when a g1 cell is not a multiple of 16 bytes (C1 = 10), at the even cell at or below it (the
// innermost TMA coordinate must be a multiple of 16 bytes); both complete on `bar`.
template <class SH>
__device__ __forceinline__ void stage_issue(const LatentBoxes& B, const Foot& f0, const Foot& f1, float* foot,
                                            uint64_t* bar)
{
  ptx::fence_proxy_async();  // earlier generic-proxy reads of this buffer before the async writes
  ptx::mbar_arrive_expect_tx(bar, B.bytes);
  ptx::tma_load_3d(foot, &B.g0, 0, f0.x0, f0.y0, bar);
  ptx::tma_load_2d(foot + B.g1_off, &B.g1, (f1.x0 - (f1.x0 & B.g1_shift)) * SH::C1, f1.y0, bar);
}

// Adds this step's quantisation noise to the staged latents of the unit's footprint (rows of
// the boxes are B.w0 / B.w1 cells apart): the g0 box rows [r0, r1) ...
template <class SH>
__device__ __forceinline__ void stage_noise_g0(const LevelArgs& L, const LatentBoxes& B, const Foot& f0, int r0, int r1,
                                               float* foot, int gt)
{
  constexpr int C0 = SH::C0;
  const int d0 = L.d0;
  const int rowq = f0.w * (C0 / 4);
  const float inv = 1.0f / (float)rowq;
  for (int v = r0 * rowq + gt; v < r1 * rowq; v += kGroupThreads) {
    const int r = div_small(v, inv), q = v - r * rowq;
    const int e = ((f0.y0 + r) * d0 + f0.x0) * C0 + q * 4;
    float4* dst = reinterpret_cast<float4*>(foot + r * B.w0 * C0 + q * 4);
    float4 val = *dst;
    val.x += level_noise(L, 0u, (uint32_t)e);
    val.y += level_noise(L, 0u, (uint32_t)(e + 1));
    val.z += level_noise(L, 0u, (uint32_t)(e + 2));
    val.w += level_noise(L, 0u, (uint32_t)(e + 3));
    *dst = val;
  }
}
// ... and the whole g1 box.
template <class SH>
__device__ __forceinline__ void stage_noise_g1(const LevelArgs& L, const LatentBoxes& B, const Foot& f1, float* foot,
                                               int gt)
{
  constexpr int C1 = SH::C1;
  const int d1 = L.d1;
  const int rowh = f1.w * (C1 / 2);
  const float inv = 1.0f / (float)rowh;
  float* foot1 = foot + B.g1_off + (f1.x0 & B.g1_shift) * C1;
  for (int v = gt; v < f1.h * rowh; v += kGroupThreads) {
    const int r = div_small(v, inv), q = v - r * rowh;
    const int e = ((f1.y0 + r) * d1 + f1.x0) * C1 + q * 2;
    float2* dst = reinterpret_cast<float2*>(foot1 + r * B.w1 * C1 + q * 2);
    float2 val = *dst;
    val.x += level_noise(L, 1u, (uint32_t)e);
    val.y += level_noise(L, 1u, (uint32_t)(e + 1));
    *dst = val;
  }
}

// Buffered stores of a feature row half: 8 values per 16-byte chunk.
struct RowWriter {
  uint8_t* sX;
  int row, col0, f;
  float buf[8];
};

// Half of one texel's feature row (draw_features arithmetic, ntc_kernel.cu:75-177): half 0 the
// 4 C0 g0 corner features, half 1 the C1 bilinear g1 features, positional encoding, lod and
// padding.  `staged`: the latents (noise already added) come from the shared-memory boxes.
// Otherwise gather_half_direct reads them, and adds the noise, from global memory.
template <class SH, class E>
__device__ __noinline__ void gather_half_direct(LevelArgs L, int x, int y, int row, int half, uint8_t* sX)
{
  constexpr int C0 = SH::C0, C1 = SH::C1, Kp = SH::Kp;
  constexpr int kSplit = 4 * C0;
  const int col0 = half ? kSplit : 0;
  Gather G;
  gather_geometry(x, y, L.mip_dim, L.d0, L.d1, G);
  float buf[8];
  int f = 0;
  auto put = [&](float v) {
    buf[f & 7] = v;
    f++;
    if ((f & 7) == 0) st_chunk<E>(sX, row, col0 + f - 8, 128, Kp, buf);
  };
  // vector loads: a cell's C0 (a multiple of 4) / C1 (even) floats start 16 / 8-byte aligned
  if (half == 0) {
    float4 q[4][C0 / 4];
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int c = 0; c < C0; c += 4) q[k][c / 4] = *reinterpret_cast<const float4*>(L.p0 + G.c0[k] * C0 + c);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int base = G.c0[k] * C0;
#pragma unroll
      for (int c = 0; c < C0; c += 4) {
        put(q[k][c / 4].x + level_noise(L, 0u, (uint32_t)(base + c)));
        put(q[k][c / 4].y + level_noise(L, 0u, (uint32_t)(base + c + 1)));
        put(q[k][c / 4].z + level_noise(L, 0u, (uint32_t)(base + c + 2)));
        put(q[k][c / 4].w + level_noise(L, 0u, (uint32_t)(base + c + 3)));
      }
    }
    return;
  }
  float acc[C1];
#pragma unroll
  for (int c = 0; c < C1; c++) acc[c] = 0.0f;
  float2 q[4][C1 / 2];
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int c = 0; c < C1; c += 2) q[k][c / 2] = *reinterpret_cast<const float2*>(L.p1 + G.c1[k] * C1 + c);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int base = G.c1[k] * C1;
#pragma unroll
    for (int c = 0; c < C1; c += 2) {
      acc[c] = __fmaf_rn(G.w1[k], q[k][c / 2].x + level_noise(L, 1u, (uint32_t)(base + c)), acc[c]);
      acc[c + 1] = __fmaf_rn(G.w1[k], q[k][c / 2].y + level_noise(L, 1u, (uint32_t)(base + c + 1)), acc[c + 1]);
    }
  }
#pragma unroll
  for (int c = 0; c < C1; c++) put(acc[c]);
#pragma unroll
  for (int i = 0; i < 12; i++) put(pos_enc(x, y, i));
  put(L.norm_lod);
#pragma unroll
  for (int i = 4 * C0 + C1 + 13; i < Kp; i++) put(0.0f);
}

template <class SH, class E>
__device__ __forceinline__ void gather_half(const LevelArgs& L, const LatentBoxes& B, int x, int y, bool valid, int row,
                                           int half, bool staged, const Foot& f0, const Foot& f1, const float* foot,
                                           const float (*penc)[8], uint8_t* sX)
{
  constexpr int C0 = SH::C0, C1 = SH::C1, Kp = SH::Kp;
  constexpr int kSplit = 4 * C0;  // a multiple of 8: chunk-aligned
  static_assert(kSplit % 8 == 0, "feature split must be chunk-aligned");
  const int col0 = half ? kSplit : 0, col1 = half ? Kp : kSplit;
  if (!valid) {
    const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = col0; c < col1; c += 8) st_chunk<E>(sX, row, c, 128, Kp, z);
    return;
  }
  if (!staged) {
    gather_half_direct<SH, E>(L, x, y, row, half, sX);
    return;
  }
  const int d0 = L.d0, d1 = L.d1;
  // gather_geometry's arithmetic, each half for its own grid only: the corner cells' (x, y),
  // clamped into the grid, and for g1 the bilinear weights
  const float rm = rcp_pow2(L.mip_dim);  // exact: (x + 0.5) / mip_dim
  const float u = ((float)x + 0.5f) * rm, v = ((float)y + 0.5f) * rm;
  float buf[8];
  int f = 0;  // features put so far (compile-time after unrolling, so buf stays in registers)
  auto put = [&](float val) {
    buf[f & 7] = val;
    f++;
    if ((f & 7) == 0) st_chunk<E>(sX, row, col0 + f - 8, 128, Kp, buf);
  };
  if (half == 0) {
    const int gx = (int)floorf(u * (float)d0 - 0.5f), gy = (int)floorf(v * (float)d0 - 0.5f);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int cx = clampi(gx + (k & 1), 0, d0 - 1), cy = clampi(gy + (k >> 1), 0, d0 - 1);
      const float* src = foot + ((cy - f0.y0) * B.w0 + (cx - f0.x0)) * C0;
#pragma unroll
      for (int c = 0; c < C0; c += 4) {
        const float4 q = *reinterpret_cast<const float4*>(src + c);
        put(q.x);
        put(q.y);
        put(q.z);
        put(q.w);
      }
    }
    return;
  }
  const float g1x = u * (float)d1 - 0.5f, g1y = v * (float)d1 - 0.5f;
  const float fx1 = floorf(g1x), fy1 = floorf(g1y);
  const int gx = (int)fx1, gy = (int)fy1;
  const float g1xf = g1x - fx1, g1yf = g1y - fy1;
  const float w1[4] = {(1.0f - g1xf) * (1.0f - g1yf), g1xf * (1.0f - g1yf), (1.0f - g1xf) * g1yf, g1xf * g1yf};
  float acc[C1];
#pragma unroll
  for (int c = 0; c < C1; c++) acc[c] = 0.0f;
  const float* foot1 = foot + B.g1_off + (f1.x0 & B.g1_shift) * C1;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int cx = clampi(gx + (k & 1), 0, d1 - 1), cy = clampi(gy + (k >> 1), 0, d1 - 1);
    const float* src = foot1 + ((cy - f1.y0) * B.w1 + (cx - f1.x0)) * C1;
#pragma unroll
    for (int c = 0; c < C1; c += 2) {
      const float2 q = *reinterpret_cast<const float2*>(src + c);
      acc[c] = __fmaf_rn(w1[k], q.x, acc[c]);
      acc[c + 1] = __fmaf_rn(w1[k], q.y, acc[c + 1]);
    }
  }
#pragma unroll
  for (int c = 0; c < C1; c++) put(acc[c]);
  // the 12 triangle waves from the per-CTA table (their values depend on the coordinate mod 8 only):
  // per period, x phase 0, x phase 1, y phase 0, y phase 1 (pos_enc's feature order)
  {
    const float4 ax = *reinterpret_cast<const float4*>(penc[x & 7]), ay = *reinterpret_cast<const float4*>(penc[y & 7]);
    const float2 bx = *reinterpret_cast<const float2*>(penc[x & 7] + 4), by = *reinterpret_cast<const float2*>(penc[y & 7] + 4);
    put(ax.x), put(ax.y), put(ay.x), put(ay.y);
    put(ax.z), put(ax.w), put(ay.z), put(ay.w);
    put(bx.x), put(bx.y), put(by.x), put(by.y);
  }
  put(L.norm_lod);
#pragma unroll
  for (int i = 4 * C0 + C1 + 13; i < Kp; i++) put(0.0f);
}

// Direct per-texel scatter of one row half (wrapped blocks, tiny tiles, oversized boxes):
// half 0 the g0 corners, half 1 the bilinear g1 corners (ntc_kernel.cu:280-341).
template <class SH>
__device__ __noinline__ void scatter_direct(LevelArgs L, int x, int y, int half, const float* dxr)
{
  constexpr int C0 = SH::C0, C1 = SH::C1;
  Gather G;
  gather_geometry(x, y, L.mip_dim, L.d0, L.d1, G);
  // vector reductions (cells 16 / 8-byte aligned as in the gather); a group of exact zeros
  // (a corner of zero bilinear weight) is left out: adding +0 changes no gradient
  if (half == 0) {
#pragma unroll
    for (int kk = 0; kk < 4; kk++)
#pragma unroll
      for (int c = 0; c < C0; c += 4) {
        const float4 v = *reinterpret_cast<const float4*>(dxr + kk * C0 + c);
        if (v.x != 0.0f || v.y != 0.0f || v.z != 0.0f || v.w != 0.0f)
          atomicAdd(reinterpret_cast<float4*>(L.g0 + G.c0[kk] * C0 + c), v);
      }
  } else {
#pragma unroll
    for (int kk = 0; kk < 4; kk++)
#pragma unroll
      for (int c = 0; c < C1; c += 2) {
        const float2 d = *reinterpret_cast<const float2*>(dxr + 4 * C0 + c);
        const float2 v = make_float2(G.w1[kk] * d.x, G.w1[kk] * d.y);
        if (v.x != 0.0f || v.y != 0.0f) atomicAdd(reinterpret_cast<float2*>(L.g1 + G.c1[kk] * C1 + c), v);
      }
  }
}

// ---- separable latent-gradient scatter of a staged unit ------------------------------------
// Where a latent cell spans two or more texels each way, the corner sums factor into a pass
// along x (texel columns -> box columns, one sum per texel row) and a pass along y (texel rows
// -> box rows).  Pass 1 writes the x sums into an intermediate in shared memory:
//   g0: T0[ty][bx][sy][C0] = sum over corner sides sx of the texels (ty, tx) whose side-sx
//       corner column is bx, of their corner (sx, sy) feature gradient;
//   g1: T1[ty][bx][C1]     = sum over sx of wx(sx, tx) times their g1 feature gradient,
// and pass 2 sums T over the texel rows of each box row (weights wy for g1).  The products
// and sums are those of the per-texel scatter (ntc_kernel.cu:317-340) regrouped.
// dxs: the unit's feature gradients [128 texels][ld]; item i of the pass-1 index space.
template <int C0>
__device__ __forceinline__ void sep_pass1_g0(const float* dxs, int ld, const CornerMasks& cm, int w0, float inv0, int i,
                                             float* T0)
{
  constexpr int Q0 = C0 / 4;
  const int q = i % Q0, r = i / Q0;  // r = (ty * w0 + bx) * 2 + sy
  const int sy = r & 1, tyb = r >> 1;
  const int ty = div_small(tyb, inv0), bx = tyb - ty * w0;
  const float* base = dxs + (ty << 4) * ld + 2 * sy * C0 + 4 * q;
  float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
  for (uint32_t m = cm.xlo[0][bx]; m; m &= m - 1) {
    const float4 v = *reinterpret_cast<const float4*>(base + (__ffs(m) - 1) * ld);
    sum.x += v.x, sum.y += v.y, sum.z += v.z, sum.w += v.w;
  }
  for (uint32_t m = cm.xhi[0][bx]; m; m &= m - 1) {
    const float4 v = *reinterpret_cast<const float4*>(base + (__ffs(m) - 1) * ld + C0);
    sum.x += v.x, sum.y += v.y, sum.z += v.z, sum.w += v.w;
  }
  *reinterpret_cast<float4*>(T0 + r * C0 + 4 * q) = sum;
}

template <int C0, int C1>
__device__ __forceinline__ void sep_pass1_g1(const float* dxs, int ld, const CornerMasks& cm, int w1, float inv1, int j,
                                             float* T1)
{
  constexpr int Q1 = C1 / 2;
  const int q = j % Q1, r = j / Q1;  // r = ty * w1 + bx
  const int ty = div_small(r, inv1), bx = r - ty * w1;
  const float* base = dxs + (ty << 4) * ld + 4 * C0 + 2 * q;
  float2 sum = make_float2(0.f, 0.f);
  for (uint32_t m = cm.xlo[1][bx]; m; m &= m - 1) {
    const int tx = __ffs(m) - 1;
    const float w = 1.0f - cm.fx[tx];
    const float2 v = *reinterpret_cast<const float2*>(base + tx * ld);
    sum.x += w * v.x, sum.y += w * v.y;
  }
  for (uint32_t m = cm.xhi[1][bx]; m; m &= m - 1) {
    const int tx = __ffs(m) - 1;
    const float w = cm.fx[tx];
    const float2 v = *reinterpret_cast<const float2*>(base + tx * ld);
    sum.x += w * v.x, sum.y += w * v.y;
  }
  *reinterpret_cast<float2*>(T1 + r * C1 + 2 * q) = sum;
}

// Loads the fp32 master weights into the canonical operand tiles (zero padding past F / C).  A
// thread's 8-column chunks are all loaded (16-byte loads: F and the row offsets are multiples of
// 4 floats) before any is converted, so the CTA waits for one round trip, not one per chunk.
template <class SH, class E>
__device__ void load_weights(const Model& M, uint8_t* W0, uint8_t* W1, uint8_t* Wo)
{
  constexpr int F = SH::F, Kp = SH::Kp, kThreads = E::kGroups * kGroupThreads;
  static_assert(F % 4 == 0, "16-byte weight loads");
  constexpr int n0 = 64 * (Kp / 8), n1 = n0 + 64 * 8, n2 = n1 + 16 * 8;  // chunk ranges: W0, W1, Wout
  constexpr int kPer = (n2 + kThreads - 1) / kThreads;
  const int C = M.C;
  const float* __restrict__ W = M.W;
  float4 v[kPer][2];
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    const int i = (int)threadIdx.x + j * kThreads;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    v[j][0] = z;
    v[j][1] = z;
    const float* src = nullptr;
    int valid = 0;  // floats of the chunk inside the matrix (0, 4 or 8)
    if (i < n0) {
      const int r = i / (Kp / 8), c0 = (i % (Kp / 8)) * 8;
      src = W + w0_off() + r * F + c0;
      valid = c0 + 8 <= F ? 8 : (c0 < F ? 4 : 0);
    } else if (i < n1) {
      const int r = (i - n0) >> 3, c0 = ((i - n0) & 7) * 8;
      src = W + w1_off(F) + r * 64 + c0;
      valid = 8;
    } else if (i < n2) {
      const int r = (i - n1) >> 3, c0 = ((i - n1) & 7) * 8;
      src = W + wo_off(F) + r * 64 + c0;
      valid = r < C ? 8 : 0;
    }
    if (valid >= 4) v[j][0] = __ldg(reinterpret_cast<const float4*>(src));
    if (valid == 8) v[j][1] = __ldg(reinterpret_cast<const float4*>(src + 4));
  }
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    const int i = (int)threadIdx.x + j * kThreads;
    const float c[8] = {v[j][0].x, v[j][0].y, v[j][0].z, v[j][0].w, v[j][1].x, v[j][1].y, v[j][1].z, v[j][1].w};
    if (i < n0)
      st_chunk<E>(W0, i / (Kp / 8), (i % (Kp / 8)) * 8, 64, Kp, c);
    else if (i < n1)
      st_chunk<E>(W1, (i - n0) >> 3, ((i - n0) & 7) * 8, 64, 64, c);
    else if (i < n2)
      st_chunk<E>(Wo, (i - n1) >> 3, ((i - n1) & 7) * 8, 16, 64, c);
  }
}

// Forward epilogue of one layer, this thread's 32 columns (from hc): activations into the next
// operand tile P, pre-activations kept in `pre` (packed bf16 pairs, or fp32 bits) for the
// backward pass.
template <class E>
__device__ __forceinline__ void epi_fwd(const float* hx, uint32_t* pre, uint8_t* P, int row, int hc)
{
#pragma unroll
  for (int c = 0; c < 32; c += 8) {
    if constexpr (!E::kSplit) {
      *reinterpret_cast<uint4*>(P + ptx::cm_off16(row, hc + c, 64)) = hg_chunk_bf16(hx + c, pre + c / 2);
    } else {
      float a[8];
      hg_chunk_f32(hx + c, a, pre + c);
      st_chunk<E>(P, row, hc + c, 128, 64, a);
    }
  }
}
// Backward epilogue: dA * hardgelu'(pre) for this thread's 32 columns into the operand tile P.
template <class E>
__device__ __forceinline__ void epi_bwd(const float* da, const uint32_t* pre, uint8_t* P, int row, int hc)
{
#pragma unroll
  for (int c = 0; c < 32; c += 8) {
    if constexpr (!E::kSplit) {
      *reinterpret_cast<uint4*>(P + ptx::cm_off16(row, hc + c, 64)) = dhg_chunk_bf16(da + c, pre + c / 2);
    } else {
      float d[8];
      dhg_chunk_f32(da + c, pre + c, d);
      st_chunk<E>(P, row, hc + c, 128, 64, d);
    }
  }
}

template <int kThreads>
__device__ __forceinline__ double block_sum_d_tc(double v, double* red)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (kThreads / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

__device__ __forceinline__ void tmem_st_zero16(uint32_t taddr)
{
  const uint32_t z = 0;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
      "r"(z));
}

// One material's share of a tile launch: CTAs [cta_begin, cta_begin + cta_count) run its step.
template <int kMats>
struct TileJob {
  TileMat mat[kMats];
  int32_t n;
};

template <class SH, class E, int kMats>
__global__ void __launch_bounds__(E::kGroups * kGroupThreads, 1) tc_unit_kernel(const __grid_constant__ TileJob<kMats> J)
{
  // this CTA's material (materials in CTA order) and its place among the material's CTAs
  int mi = 0;
  if constexpr (kMats > 1) {
    for (int i = 1; i < J.n; i++)
      if ((int)blockIdx.x >= J.mat[i].cta_begin) mi = i;
  }
  const TileMat& T = J.mat[mi];
  const Model& M = T.M;
  const LatentBoxes& boxes = T.boxes;
  const TileOut& out = T.out;
  int* __restrict__ err = T.err;
  const int cta = (int)blockIdx.x - T.cta_begin, ncta = T.cta_count;
  constexpr int C0 = SH::C0, C1 = SH::C1, Kp = SH::Kp, F = SH::F;
  constexpr int kThreads = E::kGroups * kGroupThreads;
  constexpr int kParts = E::kGroups * 2;  // splits of the per-CTA epilogue work
  // 8-row group strides of the [*][Kp], [*][64] and [*][16] operand tiles
  constexpr uint32_t SX = row8(Kp), S64 = row8(64), S16 = row8(16);
  constexpr int kK = 16;         // K elements per bf16 MMA instruction
  constexpr uint32_t kKS = 2;    // MN-major operands: 8-row groups per MMA K step
  // bytes from a tile's high part to its low part (split operands)
  constexpr uint32_t kLoX = 128 * Kp * 2, kLoP = 128 * 64 * 2, kLoY = 128 * 16 * 2;
  constexpr uint32_t kLoW0 = 64 * Kp * 2, kLoW1 = 64 * 64 * 2, kLoWo = 16 * 64 * 2;
  constexpr int KH = Kp / 2;  // dX columns per half row (a multiple of 8)
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ __align__(8) uint64_t tma_bars[2][2];  // [group][staging buffer]: latent boxes landed
  __shared__ uint32_t tmem_base_s;
  __shared__ int fail_s;
  __shared__ double red[kThreads / 32];
  __shared__ float u8_to_unit[256];  // v / 255 as upstream computes it (libopenntc draw_targets)
  // triangle-wave features of a texel coordinate c, by c mod 8: [period p][phase h] at 2p + h,
  // pos_enc's exact values (its periods 8, 4, 2 divide 8)
  __shared__ __align__(16) float penc_s[8][8];
  __shared__ CornerMasks masks_s[2];
  __shared__ StepRec step_s;
  __shared__ LevelArgs level_s;

  // The step record lives in shared memory: every group barrier (a memory clobber) makes the
  // compiler re-read the fields it uses, and there that costs a shared load, not an L1/L2 trip.
  const StepRec& s = step_s;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int g = tid >> 8;          // group
  const int gt = tid & 255;        // thread within the group
  const int row = gt & 127;        // texel row == TMEM lane
  const int half = gt >> 7;        // which half of the row's columns this thread takes
  const int part = g * 2 + half;   // 0 .. kParts - 1: splits the per-CTA epilogue work
  const int quad = warp & 3;       // TMEM lane quadrant this warp may access
  const int C = M.C;

  using GS = GroupSmem<SH, E>;
  uint8_t* base = smem_raw + g * GS::kBytes;
  GroupPtrs gp;
  gp.X = base;
  gp.P0 = gp.X + GS::kX;
  gp.P1 = gp.P0 + GS::kP;
  gp.dY = gp.P1 + GS::kP;
  gp.foot = reinterpret_cast<float*>(gp.dY + GS::kY);
  uint8_t* sW0 = smem_raw + E::kGroups * GS::kBytes;
  uint8_t* sW1 = sW0 + tile_bytes<E>(64, Kp);
  uint8_t* sWo = sW1 + tile_bytes<E>(64, 64);

  // prologue: the barriers, the step record and its level first; then the first unit's
  // latent-box loads, in flight while the weights load and the accumulators are zeroed
  static_assert(sizeof(StepRec) % 4 == 0 && sizeof(StepRec) / 4 <= kThreads, "step record copy");
  if (tid < (int)(sizeof(StepRec) / 4))
    reinterpret_cast<int32_t*>(&step_s)[tid] = reinterpret_cast<const int32_t*>(T.step)[tid];
  if (tid == 0) {
    ptx::mbar_init(&bars[0], 1);
    ptx::mbar_init(&bars[1], 1);
    for (int i = 0; i < 4; i++) ptx::mbar_init(&tma_bars[i >> 1][i & 1], 1);
    ptx::fence_mbar_init();
    fail_s = 0;
    level_s = level_args(M, *T.step);
  }
  __syncwarp();
  if (warp == 0) ptx::tmem_alloc(&tmem_base_s, kTmemCols);
  __syncthreads();
  const LevelArgs& L = level_s;
  const int ntiles = (s.texels + kTile - 1) / kTile;
  // latent boxes: unit k's were loaded (TMA, asynchronously) while unit k-1 ran, into the
  // staging buffer the previous unit did not use; tph holds each buffer's next wait parity and
  // inflight which buffers have loads not yet waited for
  const int ustride = ncta * E::kGroups;
  Foot nf0 = {}, nf1 = {};
  bool nstaged = false;
  int pb = 0;
  uint32_t tph = 0, inflight = 0;
  {
    const int u0 = cta * E::kGroups + g;
    nstaged = u0 < ntiles && unit_footprint<SH>(L, s, boxes, u0, nf0, nf1);
    if (nstaged) {
      if (gt == 0) stage_issue<SH>(boxes, nf0, nf1, gp.foot, &tma_bars[g][0]);
      inflight |= 1u;
    }
  }
  load_weights<SH, E>(M, sW0, sW1, sWo);
  if (tid < 256) u8_to_unit[tid] = (float)tid / 255.0f;
  if (tid < 48) {
    const int m = tid / 6, k = tid % 6;                 // coordinate mod 8, 2 x period + phase
    penc_s[m][k] = pos_enc(m, m, 4 * (k >> 1) + (k & 1));  // feature 4p + h: the x wave of period p
  }
  // corner masks start zeroed (each unit zeroes its own after its scatter)
  static_assert(sizeof(CornerMasks) % 4 == 0, "mask words");
  for (int i = tid; i < (int)(sizeof(masks_s) / 4); i += kThreads) reinterpret_cast<uint32_t*>(masks_s)[i] = 0u;
  ptx::fence_proxy_async();
  ptx::fence_before_sync();
  __syncthreads();
  ptx::fence_after_sync();
  const uint32_t tbase = tmem_base_s;
  const uint32_t lane_off = (uint32_t)(quad * 32) << 16;
  // zero the shared weight-gradient accumulators (columns kColW0 .. kColWo + 16): each part
  // takes every kParts-th 16-column chunk of its quadrant's lanes
  for (uint32_t c = kColW0 + 16 * (uint32_t)part; c < kColWo + 16; c += 16 * kParts)
    tmem_st_zero16(tbase + lane_off + c);
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  ptx::fence_before_sync();
  __syncthreads();
  ptx::fence_after_sync();

  const uint32_t win = tbase + 128u * (uint32_t)g;    // this group's TMEM window (MMA address)
  const uint32_t lwin = win + lane_off;                // ... as seen by this thread's lane
  const float inv = -2.0f / ((float)C * (float)s.texels);  // libopenntc.cpp:666
  const uint8_t* target = M.package[s.lod];
  uint64_t* bar = &bars[g];
  uint32_t phase = 0;
  double loss = 0.0;
  // the group's first warp issues its MMAs and commits, from one elected lane
  const bool mma_warp = (gt >> 5) == 0;

  // one warp of the group polls the mbarrier; the others sleep at the group barrier
  const bool poller = (gt >> 5) == 0;
  auto wait_mma = [&]() -> bool {
    if (poller && !ptx::mbar_wait(bar, phase)) atomicExch(&fail_s, 1);
    phase ^= 1u;
    bar_group(g);
    ptx::fence_after_sync();
    return *(volatile int*)&fail_s == 0;
  };
  // this group's shared-memory stores and TMEM reads done -> its issuer may start MMAs
  auto handoff = [&]() {
    ptx::fence_proxy_async();
    ptx::fence_before_sync();
    bar_group(g);
  };

  constexpr uint32_t FM = 1;  // bf16 operands
  constexpr uint32_t I_M128_N64_K = ptx::idesc_f32acc(FM, 128, 64, false, false);
  constexpr uint32_t I_M128_N16_K = ptx::idesc_f32acc(FM, 128, 16, false, false);
  constexpr uint32_t I_M128_N64_BMN = ptx::idesc_f32acc(FM, 128, 64, false, true);
  constexpr uint32_t I_M128_NKP_BMN = ptx::idesc_f32acc(FM, 128, Kp, false, true);
  constexpr uint32_t I_M64_N16_MN = ptx::idesc_f32acc(FM, 64, 16, true, true);
  constexpr uint32_t I_M64_N64_MN = ptx::idesc_f32acc(FM, 64, 64, true, true);
  constexpr uint32_t I_M64_NKP_MN = ptx::idesc_f32acc(FM, 64, Kp, true, true);
  const uint32_t aX = ptx::smem_addr(gp.X), aP0 = ptx::smem_addr(gp.P0), aP1 = ptx::smem_addr(gp.P1);
  const uint32_t adY = ptx::smem_addr(gp.dY);
  const uint32_t aW0 = ptx::smem_addr(sW0), aW1 = ptx::smem_addr(sW1), aWo = ptx::smem_addr(sWo);
  // matrix descriptors of this group's operand tiles and the shared weight tiles, K-major (k)
  // and MN-major (m) views; a tile further on is one add (DescBase::at)
  const ptx::DescBase dXk = ptx::desc_base(aX, 128, SX), dXm = ptx::desc_base(aX, SX, 128);
  const ptx::DescBase dP0k = ptx::desc_base(aP0, 128, S64), dP0m = ptx::desc_base(aP0, S64, 128);
  const ptx::DescBase dP1k = ptx::desc_base(aP1, 128, S64), dP1m = ptx::desc_base(aP1, S64, 128);
  const ptx::DescBase dYk = ptx::desc_base(adY, 128, S16), dYm = ptx::desc_base(adY, S16, 128);
  const ptx::DescBase dW0k = ptx::desc_base(aW0, 128, SX), dW0m = ptx::desc_base(aW0, SX, 128);
  const ptx::DescBase dW1k = ptx::desc_base(aW1, 128, S64), dW1m = ptx::desc_base(aW1, S64, 128);
  const ptx::DescBase dWok = ptx::desc_base(aWo, 128, S64), dWom = ptx::desc_base(aWo, S64, 128);
  const int hc = half * 32;  // this thread's first column of a 64-column tile

  // buffer `buf`'s boxes landed (bounded wait; a timeout is reported, the buffer stays in
  // flight and is waited for again before exit); the noise is added afterwards, in parts
  auto land_wait = [&](int buf) {
    if (ptx::mbar_wait(&tma_bars[g][buf], (tph >> buf) & 1u)) {
      tph ^= 1u << buf;
      inflight &= ~(1u << buf);
    } else {
      atomicExch(&fail_s, 1);
    }
  };
  if (nstaged) {  // the first unit's boxes before its gather
    land_wait(0);
    if (s.noise) {
      stage_noise_g0<SH>(L, boxes, nf0, 0, nf0.h, gp.foot, gt);
      stage_noise_g1<SH>(L, boxes, nf1, gp.foot, gt);
    }
  }
  bar_group(g);

  for (int unit = cta * E::kGroups + g; unit < ntiles; unit += ustride) {
    // ------------------------------------------------------------------ gather
    const int b = unit * kTile + row;
    const bool valid = b < s.texels;
    int x = 0, y = 0;
    if (valid) texel_xy(s, b, x, y);
    // this unit's boxes landed (and took their noise) during the previous unit, or in the
    // prologue; its corner masks are built during its first MMAs
    const Foot f0 = nf0, f1 = nf1;
    const bool staged = nstaged;
    const int cur = pb;
    float* foot = gp.foot + cur * kFootBuf;
    CornerMasks& cm = masks_s[g];
    gather_half<SH, E>(L, boxes, x, y, valid, row, half, staged, f0, f1, foot, penc_s, gp.X);
    handoff();
    if (mma_warp) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < Kp / kK; k++) mma<E>(win, dXk, k * 256, kLoX, dW0k, k * 256, kLoW0, I_M128_N64_K, k > 0);
      ptx::commit_warp(bar);
    }
    // in the shadow of the MMAs: this thread's target channels [8 half, 8 half + 8) (first
    // used after layer 2), and the next unit's box loads into the other staging buffer (its
    // last readers, the previous unit's gather and scatter, finished before this unit began)
    uint32_t tb[8];
#pragma unroll
    for (int j = 0; j < 8; j++) tb[j] = 0u;
    if (valid) {
      const uint8_t* tp = target + ((size_t)y * s.mip_dim + x) * C;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (half * 8 + j < C) tb[j] = tp[half * 8 + j];
    }
    {
      const int nu = unit + ustride;
      nstaged = nu < ntiles && unit_footprint<SH>(L, s, boxes, nu, nf0, nf1);
      if (nstaged) {
        // issued by the group's second warp: the first one issues the MMAs and polls for them
        if (gt == 32) stage_issue<SH>(boxes, nf0, nf1, gp.foot + (cur ^ 1) * kFootBuf, &tma_bars[g][cur ^ 1]);
        inflight |= 2u >> cur;
      }
      pb ^= 1;
    }
    if (!wait_mma()) break;

    // ------------------------------------------------------------------ layer 0 epilogue
    constexpr int kPre = E::kSplit ? 32 : 16;
    uint32_t h0[kPre], h1[kPre];  // pre-activations of this thread's 32 columns (bf16 pairs or fp32)
    float hx[32];
    ptx::ld16(lwin + hc, hx);
    ptx::ld16(lwin + hc + 16, hx + 16);
    ptx::ld_wait();
    epi_fwd<E>(hx, h0, gp.P0, row, hc);
    handoff();
    if (mma_warp) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < 64 / kK; k++) mma<E>(win, dP0k, k * 256, kLoP, dW1k, k * 256, kLoW1, I_M128_N64_K, k > 0);
      ptx::commit_warp(bar);
    }
    // this unit's corner masks (zeroed at the end of the previous unit), by the group's second
    // warp while the first polls the MMA barrier
    if (staged && (gt >> 5) == 1) build_masks(s, L.d0, L.d1, f0, f1, unit, cm, gt - 32);
    if (!wait_mma()) break;

    // ------------------------------------------------------------------ layer 1 epilogue
    ptx::ld16(lwin + hc, hx);
    ptx::ld16(lwin + hc + 16, hx + 16);
    ptx::ld_wait();
    epi_fwd<E>(hx, h1, gp.P1, row, hc);
    handoff();
    if (mma_warp) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < 64 / kK; k++)
        mma<E>(win + 64, dP1k, k * 256, kLoP, dWok, k * 256, kLoWo, I_M128_N16_K, k > 0);
      ptx::commit_warp(bar);
    }
    if (!wait_mma()) break;

    // ------------------------------------------------------------------ output, residual, dY
    {
      float yv[8], d[8];
      ptx::ld8(lwin + 64 + half * 8, yv);
      ptx::ld_wait();
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int c = half * 8 + j;
        d[j] = 0.0f;
        if (valid && c < C) {
          const float r = u8_to_unit[tb[j]] - yv[j];
          loss += (double)r * (double)r;
          d[j] = inv * r;
        }
      }
      st_chunk<E>(gp.dY, row, half * 8, 128, 16, d);
    }
    handoff();
    if (mma_warp) {
      ptx::fence_after_sync();
      // dA1 = dY Wout: B = Wout viewed [c][h] as MN-major (N = h), K = c
#pragma unroll
      for (int k = 0; k < 16 / kK; k++)
        mma<E>(win, dYk, k * 256, kLoY, dWom, k * kKS * S64, kLoWo, I_M128_N64_BMN, k > 0);
      // dWout^T += A1^T dY : A = A1 (M = h), B = dY (N = c), K = texels
#pragma unroll
      for (int k = 0; k < 128 / kK; k++)
        mma<E>(tbase + kColWo, dP1m, k * kKS * S64, kLoP, dYm, k * kKS * S16, kLoY, I_M64_N16_MN, 1);
      ptx::commit_warp(bar);
    }
    // the next unit's boxes (loads issued with this unit's first layer) landed, then their noise,
    // spread over this and the next two MMA waits: the g1 box here, the g0 box's rows in halves
    if (nstaged) {
      land_wait(cur ^ 1);
      if (s.noise) stage_noise_g1<SH>(L, boxes, nf1, gp.foot + (cur ^ 1) * kFootBuf, gt);
    }
    if (!wait_mma()) break;

    // ------------------------------------------------------------------ dH1 (into P1)
    {
      float da[32];
      ptx::ld16(lwin + hc, da);
      ptx::ld16(lwin + hc + 16, da + 16);
      ptx::ld_wait();
      epi_bwd<E>(da, h1, gp.P1, row, hc);
    }
    handoff();
    if (mma_warp) {
      ptx::fence_after_sync();
      // dA0 = dH1 W1 : B = W1 viewed [i][h] as MN-major (N = h), K = i
#pragma unroll
      for (int k = 0; k < 64 / kK; k++)
        mma<E>(win, dP1k, k * 256, kLoP, dW1m, k * kKS * S64, kLoW1, I_M128_N64_BMN, k > 0);
      // dW1 += dH1^T A0
#pragma unroll
      for (int k = 0; k < 128 / kK; k++)
        mma<E>(tbase + kColW1, dP1m, k * kKS * S64, kLoP, dP0m, k * kKS * S64, kLoP, I_M64_N64_MN, 1);
      ptx::commit_warp(bar);
    }
    if (nstaged && s.noise) stage_noise_g0<SH>(L, boxes, nf0, 0, nf0.h / 2, gp.foot + (cur ^ 1) * kFootBuf, gt);
    if (!wait_mma()) break;

    // ------------------------------------------------------------------ dH0 (into P0)
    {
      float da[32];
      ptx::ld16(lwin + hc, da);
      ptx::ld16(lwin + hc + 16, da + 16);
      ptx::ld_wait();
      epi_bwd<E>(da, h0, gp.P0, row, hc);
    }
    handoff();
    if (mma_warp) {
      ptx::fence_after_sync();
      // dX = dH0 W0 : B = W0 viewed [h][f] as MN-major (N = f), K = h
#pragma unroll
      for (int k = 0; k < 64 / kK; k++)
        mma<E>(win, dP0k, k * 256, kLoP, dW0m, k * kKS * SX, kLoW0, I_M128_NKP_BMN, k > 0);
      // dW0 += dH0^T X
#pragma unroll
      for (int k = 0; k < 128 / kK; k++)
        mma<E>(tbase + kColW0, dP0m, k * kKS * S64, kLoP, dXm, k * kKS * SX, kLoX, I_M64_NKP_MN, 1);
      ptx::commit_warp(bar);
    }
    if (nstaged && s.noise)
      stage_noise_g0<SH>(L, boxes, nf0, nf0.h / 2, nf0.h, gp.foot + (cur ^ 1) * kFootBuf, gt);
    if (!wait_mma()) break;

    // ------------------------------------------------------------------ scatter dX
    if (s.grid_update) {
      const int d0 = L.d0, d1 = L.d1;
      // dX rows to shared memory (the group's operand tiles are free now), half a row per thread
      constexpr int LD = Kp + 4;
      float* dxs = reinterpret_cast<float*>(gp.X);
      {
        float dx[KH];
#pragma unroll
        for (int c = 0; c < KH; c += 8) ptx::ld8(lwin + half * KH + c, dx + c);
        ptx::ld_wait();
        if (s.exact_grad) {
#pragma unroll
          for (int c = 0; c < KH; c++) dx[c] = exact_dyadic(dx[c]);
        }
#pragma unroll
        for (int c = 0; c < KH; c += 4)
          *reinterpret_cast<float4*>(dxs + row * LD + half * KH + c) = make_float4(dx[c], dx[c + 1], dx[c + 2], dx[c + 3]);
      }
      bar_group(g);
      float* g0p = L.g0;
      float* g1p = L.g1;
      if (staged) {
        // A work item is one box cell and a group of its channels (4 of g0, 2 of g1), whose
        // thread sums every texel-corner contribution to them and adds the sum with one vector
        // reduction.  Per grid, where a cell spans two or more texels each way, the sums go
        // through the separable passes (the intermediate in this unit's staging buffer, which
        // nothing reads after the gather and the next unit's loads do not target); elsewhere
        // the item's thread walks the corner masks itself.
        constexpr int Q0 = C0 / 4, Q1 = C1 / 2;
        const int w0 = f0.w, w1 = f1.w;
        const float inv0 = 1.0f / (float)w0, inv1 = 1.0f / (float)w1;
        const int n0 = 8 * w0 * 2 * C0, n1 = 8 * w1 * C1;  // intermediate floats
        const bool sep1 = s.mip_dim >= 2 * d1 && n1 <= kFootBuf;
        const bool sep0 = s.mip_dim >= 2 * d0 && n0 + (sep1 ? n1 : 0) <= kFootBuf;
        float* T0 = foot;
        float* T1 = foot + (sep0 ? n0 : 0);
        const int p0 = sep0 ? 8 * w0 * 2 * Q0 : 0;
        const int np = p0 + (sep1 ? 8 * w1 * Q1 : 0);
        if (np > 0) {
          for (int i = gt; i < np; i += kGroupThreads) {
            if (i < p0)
              sep_pass1_g0<C0>(dxs, LD, cm, w0, inv0, i, T0);
            else
              sep_pass1_g1<C0, C1>(dxs, LD, cm, w1, inv1, i - p0, T1);
          }
          bar_group(g);
        }
        const int ni0 = w0 * f0.h * Q0;
        const int ni = ni0 + w1 * f1.h * Q1;
        for (int i = gt; i < ni; i += kGroupThreads) {
          if (i < ni0) {
            const int cell = i / Q0, q = i - cell * Q0;
            const int by = div_small(cell, inv0), bx = cell - by * w0;
            float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
            if (sep0) {
              // T0[ty][bx][sy]: rows whose side-sy corner row is by
#pragma unroll
              for (int sy = 0; sy < 2; sy++) {
                const float* t = T0 + (bx * 2 + sy) * C0 + 4 * q;
                for (uint32_t ym = sy ? cm.yhi[0][by] : cm.ylo[0][by]; ym; ym &= ym - 1) {
                  const float4 v = *reinterpret_cast<const float4*>(t + (__ffs(ym) - 1) * (w0 * 2 * C0));
                  sum.x += v.x, sum.y += v.y, sum.z += v.z, sum.w += v.w;
                }
              }
            } else {
#pragma unroll
              for (int kk = 0; kk < 4; kk++) {
                const uint32_t mx = (kk & 1) ? cm.xhi[0][bx] : cm.xlo[0][bx];
                const uint32_t my = (kk & 2) ? cm.yhi[0][by] : cm.ylo[0][by];
                for (uint32_t ym = my; ym; ym &= ym - 1) {
                  const float* srow = dxs + ((__ffs(ym) - 1) << 4) * LD + kk * C0 + 4 * q;
                  for (uint32_t xm = mx; xm; xm &= xm - 1) {
                    const float4 v = *reinterpret_cast<const float4*>(srow + (__ffs(xm) - 1) * LD);
                    sum.x += v.x, sum.y += v.y, sum.z += v.z, sum.w += v.w;
                  }
                }
              }
            }
            // one 16-byte vector reduction per item (C0 % 4 == 0, latent buffers 256-byte aligned);
            // adding +0 leaves a gradient unchanged, so a group with some zero sums adds them too
            float* dst = g0p + ((f0.y0 + by) * d0 + f0.x0 + bx) * C0 + 4 * q;
            if (sum.x != 0.0f || sum.y != 0.0f || sum.z != 0.0f || sum.w != 0.0f)
              atomicAdd(reinterpret_cast<float4*>(dst), sum);
          } else {
            const int j = i - ni0;
            const int cell = j / Q1, q = j - cell * Q1;
            const int by = div_small(cell, inv1), bx = cell - by * w1;
            float2 sum = make_float2(0.f, 0.f);
            if (sep1) {
              // T1[ty][bx]: weighted by the rows' side-sy fractions
              const float* t = T1 + bx * C1 + 2 * q;
#pragma unroll
              for (int sy = 0; sy < 2; sy++) {
                for (uint32_t ym = sy ? cm.yhi[1][by] : cm.ylo[1][by]; ym; ym &= ym - 1) {
                  const int ty = __ffs(ym) - 1;
                  const float wy = sy ? cm.fy[ty] : 1.0f - cm.fy[ty];
                  const float2 v = *reinterpret_cast<const float2*>(t + ty * (w1 * C1));
                  sum.x += wy * v.x, sum.y += wy * v.y;
                }
              }
            } else {
#pragma unroll
              for (int kk = 0; kk < 4; kk++) {
                const uint32_t mx = (kk & 1) ? cm.xhi[1][bx] : cm.xlo[1][bx];
                const uint32_t my = (kk & 2) ? cm.yhi[1][by] : cm.ylo[1][by];
                for (uint32_t ym = my; ym; ym &= ym - 1) {
                  const int ty = __ffs(ym) - 1;
                  const float fy = cm.fy[ty];
                  const float wy = (kk & 2) ? fy : (1.0f - fy);
                  const float* srow = dxs + (ty << 4) * LD + 4 * C0 + 2 * q;
                  for (uint32_t xm = mx; xm; xm &= xm - 1) {
                    const int tx = __ffs(xm) - 1;
                    const float fx = cm.fx[tx];
                    // the bilinear weight exactly as gather_geometry forms it
                    const float w = ((kk & 1) ? fx : (1.0f - fx)) * wy;
                    const float2 v = *reinterpret_cast<const float2*>(srow + tx * LD);
                    sum.x += w * v.x, sum.y += w * v.y;
                  }
                }
              }
            }
            float* dst = g1p + ((f1.y0 + by) * d1 + f1.x0 + bx) * C1 + 2 * q;
            if (sum.x != 0.0f || sum.y != 0.0f) atomicAdd(reinterpret_cast<float2*>(dst), sum);
          }
        }
        // the intermediate's generic writes before the staging buffer's next asynchronous load
        if (np > 0) ptx::fence_proxy_async();
      } else if (valid) {
        scatter_direct<SH>(L, x, y, half, dxs + row * LD);
      }
    }
    if (staged) {
      if (s.grid_update) bar_group(g);  // every read of the masks done
      uint32_t* m = &cm.xlo[0][0];      // xlo, xhi, ylo, yhi: contiguous words
      for (int i = gt; i < 2 * (2 * kMaxBoxW + 2 * kMaxBoxH); i += kGroupThreads) m[i] = 0u;
    }
    ptx::fence_before_sync();
    bar_group(g);
  }

  // no load may still target shared memory at exit (loads in flight only after an early exit)
  for (int b = 0; b < 2; b++)
    if (inflight & (1u << b)) {
      if (!ptx::mbar_wait(&tma_bars[g][b], (tph >> b) & 1u)) atomicExch(&fail_s, 1);
    }

  // ------------------------------------------------------------------ weight gradients out
  const double ls = block_sum_d_tc<kThreads>(loss, red);
  if (tid == 0) out.loss_partial[cta] = ls;
  ptx::fence_after_sync();
  if (*(volatile int*)&fail_s == 0) {
    // every CTA adds its gradient into the one accumulated row (the optimiser reads and zeroes
    // it); F and the column steps are multiples of 4, so the 4-float runs are 16-byte aligned
    static_assert(F % 4 == 0, "4-float gradient runs");
    float* dst = out.dW_partial;
    const int lane = tid & 31;
    const int h = quad * 16 + lane;  // M=64 accumulators: row = lane of the quadrant's first 16
    const uint32_t la = tbase + lane_off;
    for (int c = part * 8; c < Kp; c += 8 * kParts) {  // dW0 [64][F], 8-column steps split by part
      float v[8];
      ptx::ld8(la + kColW0 + c, v);
      ptx::ld_wait();
      if (lane < 16)
        for (int j = 0; j < 8; j += 4)
          if (c + j < F) ptx::red_add4(dst + w0_off() + h * F + c + j, v[j], v[j + 1], v[j + 2], v[j + 3]);
    }
    for (int c = part * 16; c < 64; c += 16 * kParts) {
      float v[16];  // dW1[i][h]: accumulator row i, columns h, 16 per step
      ptx::ld16(la + kColW1 + c, v);
      ptx::ld_wait();
      if (lane < 16)
        for (int j = 0; j < 16; j += 4)
          ptx::red_add4(dst + w1_off(F) + h * 64 + c + j, v[j], v[j + 1], v[j + 2], v[j + 3]);
    }
    for (int c = part * 8; c < 16; c += 8 * kParts) {
      float v[8];  // dWout^T[h][c] -> dWout[c][h]; output rows past C carry no gradient
      ptx::ld8(la + kColWo + c, v);
      ptx::ld_wait();
      if (lane < 16)
        for (int j = 0; j < 8; j++)
          if (c + j < M.C) atomicAdd(dst + wo_off(F) + (c + j) * 64 + h, v[j]);
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  ptx::fence_before_sync();
  __syncthreads();
  if (warp == 0) ptx::tmem_dealloc(tbase, kTmemCols);
}

template <class SH, class E, int kMats>
cudaError_t launch_shape(const TileJob<kMats>& job, int grid, cudaStream_t stream)
{
  constexpr size_t smem = smem_bytes<SH, E>();
  static_assert(smem <= 227 * 1024 - 6 * 1024, "shared memory budget (dynamic + static)");
  cudaError_t e = cudaFuncSetAttribute(tc_unit_kernel<SH, E, kMats>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  tc_unit_kernel<SH, E, kMats><<<grid, E::kGroups * kGroupThreads, smem, stream>>>(job);
  return cudaGetLastError();
}

template <class E, int kMats>
cudaError_t launch_elem(const Model& M, const TileJob<kMats>& job, int grid, cudaStream_t stream)
{
  // profile shapes (libopenntc.cpp:289-333): C0, C1, padded feature dim
  if (M.C0 == 8 && M.C1 == 12 && M.Fp == 64) return launch_shape<Shape<8, 12, 64>, E>(job, grid, stream);
  if (M.C0 == 12 && M.C1 == 20 && M.Fp == 96) return launch_shape<Shape<12, 20, 96>, E>(job, grid, stream);
  if (M.C0 == 12 && M.C1 == 10 && M.Fp == 80) return launch_shape<Shape<12, 10, 80>, E>(job, grid, stream);
  if (M.C0 == 16 && M.C1 == 12 && M.Fp == 96) return launch_shape<Shape<16, 12, 96>, E>(job, grid, stream);
  return cudaErrorNotSupported;
}

}  // namespace

int tc_max_grid()
{
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

cudaError_t launch_tc_units(const Model& M, const StepRec* d_steps, int step_idx, int grid, TileOut out, int* d_error,
                            const LatentBoxes& boxes, bool split, cudaStream_t stream)
{
  TileJob<1> job;
  job.mat[0].boxes = boxes;
  job.mat[0].M = M;
  job.mat[0].step = d_steps + step_idx;
  job.mat[0].out = out;
  job.mat[0].err = d_error;
  job.mat[0].cta_begin = 0;
  job.mat[0].cta_count = grid;
  job.n = 1;
  return split ? launch_elem<ESplit, 1>(M, job, grid, stream) : launch_elem<EBf16, 1>(M, job, grid, stream);
}

cudaError_t launch_tc_multi(const TileMat* mats, int n, cudaStream_t stream)
{
  if (n < 1 || n > kMaxTileMats) return cudaErrorInvalidValue;
  TileJob<kMaxTileMats> job;
  memset(&job, 0, sizeof(job));
  int grid = 0;
  for (int i = 0; i < n; i++) {
    const Model& a = mats[i].M;
    if (a.C0 != mats[0].M.C0 || a.C1 != mats[0].M.C1 || a.Fp != mats[0].M.Fp) return cudaErrorInvalidValue;
    if (mats[i].cta_begin != grid || mats[i].cta_count < 1) return cudaErrorInvalidValue;
    job.mat[i] = mats[i];
    grid += mats[i].cta_count;
  }
  job.n = n;
  return launch_elem<EBf16, kMaxTileMats>(mats[0].M, job, grid, stream);
}

int tc_groups_per_cta(bool split) { return split ? ESplit::kGroups : EBf16::kGroups; }

int tc_box_capacity() { return kFootBuf; }

}  // namespace ontc
