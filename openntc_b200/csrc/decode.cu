// Decode kernel: upstream's SampleMaterial (ntc_decode.hlsli:605-623) for a batch of
// (uv, lod) samples, with the arithmetic of its DP4A inference path (:410-502).
//
// A CTA (one per SM, persistent) runs kGroups independent 4-warp groups; a group owns a tile
// of 128 samples at a time (thread = sample = TMEM lane):
//
//   features (GetFeaturesPacked, :196-342)  -> X  [128 x Kp] int8, shared memory
//   acc0 = X  W0^T   (M128 N64 K=Kp, tcgen05 kind::i8, s32 in TMEM)
//   a0   = q8(hg(acc0 * s0) / s_a1)          -> A  [128 x 64] int8 (over X)
//   acc1 = a0 W1^T   (M128 N64 K=64)
//   a1   = q8(hg(acc1 * s1) / s_a2)          -> A
//   acc2 = a1 Wout^T (M128 N16 K=64)
//   out  = saturate(acc2 * so)               -> global [n][C] f32
//
// The int8 products and int32 sums are exact, so the tensor cores reproduce the DP4A dot
// products bit for bit (each sum accumulated onto a float bias, kAccBias, so that it reads back
// as a float without a conversion); every float operation of the epilogues is written with
// explicit round-to-nearest intrinsics in upstream's order, so outputs are bit-identical to the
// HLSL semantics (as restated by the CPU oracle).  Every wait is bounded and reports a
// timeout through the error word.
#include <cstdint>

#include "common.cuh"
#include "decode_cells.cuh"
#include "kernels.h"
#include "tc_ptx.cuh"

namespace ontc {

namespace {

constexpr int kGroups = 8;  // 1024 threads, 64 registers each; 8 x 64 TMEM columns
constexpr int kGroupThreads = 128;
constexpr int kThreads = kGroups * kGroupThreads;
constexpr int kHid = 64;
constexpr int kOutRows = 16;  // upstream's padded output rows (OUTP)
static_assert(64 * kGroups == 512 || 64 * kGroups == 256 || 64 * kGroups == 128, "TMEM allocations are powers of two");

// Compile-time profile shape (ntc_decode.hlsli:60-86): channels, bits, first-level mips.
template <int C0_, int C1_, int B0_, int B1_, int L0MIPS_>
struct DShape {
  static constexpr int C0 = C0_, C1 = C1_, B0 = B0_, B1 = B1_, L0MIPS = L0MIPS_;
  static constexpr int Fp = ((4 * C0 + C1 + 13 + 15) / 16) * 16;  // the blob's W0 row stride
  static constexpr int Kp = ((Fp + 31) / 32) * 32;                // K of the i8 MMA (32 per step)
};

struct DecodeSmem {
  static constexpr size_t kTile = 128 * 96;  // per group: X, then a0, then a1 (largest Kp = 96)
};

__device__ __forceinline__ uint32_t group_bar_id(int g) { return 1u + (uint32_t)g; }
__device__ __forceinline__ void bar_group(int g)
{
  asm volatile("bar.sync %0, %1;" ::"r"(group_bar_id(g)), "r"(kGroupThreads) : "memory");
}

// Four consecutive B-bit codes starting at channel c (4 | c) as four signed feature bytes,
// (code << (8 - B)) ^ 0x80 each, built with word-wide shifts and byte permutes.
template <int B>
__device__ __forceinline__ uint32_t code_bytes4(const uint32_t* s, int c)
{
  const uint32_t t = s[(c * B) >> 5] >> ((c * B) & 31);  // codes c..c+3 in the low 4B bits
  if constexpr (B == 4) {
    const uint32_t lo = t & 0x0F0Fu, hi = (t >> 4) & 0x0F0Fu;   // n0 n2 | n1 n3
    const uint32_t n = __byte_perm(lo, hi, 0x5140);             // n0 n1 n2 n3
    return ((n << 4) & 0xF0F0F0F0u) ^ 0x80808080u;
  } else {
    static_assert(B == 2, "2- or 4-bit g0 codes");
    const uint32_t t8 = t & 0xFFu;  // exactly the four codes: higher ones would land on the targets
    const uint32_t u = (t8 << 6) | (t8 << 12) | (t8 << 18) | (t8 << 24);  // code k -> bits 8k+6..8k+7
    return (u & 0xC0C0C0C0u) ^ 0x80808080u;
  }
}

// ClampS8(round(f)) with HLSL round = nearest, ties to even.  Clamping first leaves the
// result unchanged (rounding is monotonic and the bounds are integers) and keeps |f| < 2^22,
// where adding 1.5 * 2^23 rounds to an integer in the low mantissa bits.
__device__ __forceinline__ int q8(float f)
{
  f = fminf(fmaxf(f, -128.0f), 127.0f);
  return __float_as_int(__fadd_rn(f, 12582912.0f)) - 0x4B400000;
}
// ClampS8(round(f)), HLSL round = nearest, ties to even, in one conversion (round to nearest
// even, saturate to [-128, 127]): rounding then saturating equals clamping then rounding, the
// bounds being integers.  The byte is the low byte of the result.
__device__ __forceinline__ uint32_t s8_rne_sat(float f)
{
  uint32_t r;
  asm("cvt.rni.sat.s8.f32 %0, %1;" : "=r"(r) : "f"(f));
  return r;
}

// The s32 accumulators of the int8 MMAs start from kAccBias (the bits of the float 1.5 * 2^23),
// so an accumulated sum s with |s| < 2^22 reads back as the float 12582912 + s exactly: one
// packed subtraction gives (float)s, with no integer-to-float conversion.  The int8 products
// bound every sum here: |s| <= 96 x 128 x 128 < 2^21.
constexpr uint32_t kAccBias = 0x4B400000u;
__device__ __forceinline__ void tmem_st_bias16(uint32_t taddr)
{
  const uint32_t v = kAccBias;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
      "r"(v));
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Low bytes of four words -> one word (byte i from word i).
__device__ __forceinline__ uint32_t pack4(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
  return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

// x / 3 correctly rounded: RN(x * RN(1/3)) corrected once with the exact remainder
// (division by a constant known in advance; checked against IEEE division for every float
// with |x| <= 1.5, the only range hardgelu divides in).
__device__ __forceinline__ float div3(float x)
{
  const float y = 1.0f / 3.0f;
  const float q = __fmul_rn(x, y);
  const float r = __fmaf_rn(-q, 3.0f, x);
  return __fmaf_rn(r, y, q);
}

// hardgelu4 (ntc_decode.hlsli:400-403): x < -1.5 ? 0 : x < 1.5 ? (x / 3) * (x + 1.5) : x.
// Below -1.5 the middle formula at -1.5 gives (-0.5) * 0 = -0, which scales and rounds to the
// same 0, so the lower branch is a max.
__device__ __forceinline__ float hg_hlsl(float x)
{
  const float c = fmaxf(x, -1.5f);
  const float mid = __fmul_rn(div3(c), __fadd_rn(c, 1.5f));
  return x < 1.5f ? mid : x;
}

__device__ __forceinline__ void put_byte(uint32_t* w, int f, int v)
{
  w[f >> 2] |= ((uint32_t)v & 0xFFu) << (8 * (f & 3));
}

// One triangle-wave feature byte (ntc_decode.hlsli:300-330): wave p (period 8 >> p) of texel
// coordinate c, phase h.  For an integer-valued |c| < 2^22 every step is exact (c + 0.5 and the
// quarter-period phase are representable, the period is a power of two), so the byte depends
// only on c mod 8: the decode reads it from a table built with this function.
__device__ __forceinline__ int tri_q8(float c, int p, int h)
{
  const float P = (float)(8 >> p), rP = 1.0f / P;  // P = 8, 4, 2: dividing = exact scaling
  const float ph = h == 0 ? 0.0f : __fmul_rn(0.25f, P);
  const float t = __fmul_rn(__fadd_rn(__fadd_rn(c, 0.5f), ph), rP);
  const float pe = __fsub_rn(1.0f, __fmul_rn(4.0f, fabsf(__fsub_rn(__fsub_rn(t, floorf(t)), 0.5f))));
  return q8(__fmul_rn(pe, 128.0f));
}

// The normalised-lod feature byte of lod l.
__device__ __forceinline__ int lod_q8(int l, int mip_count)
{
  return q8(__fmul_rn(__fdiv_rn((float)l, (float)(mip_count - 1)), 128.0f));
}

// Per-CTA tables of the features that depend only on (texel coordinate mod 8) and on lod:
// tri[a][p][m] holds wave p's two phase bytes of axis a (x: bytes 0-1, y: bytes 2-3 of the
// feature word p) at coordinate m; lodb[l] the lod byte.
struct FeatureTables {
  uint32_t tri[2][3][8];
  uint32_t lodb[32];
};

__device__ __forceinline__ void build_feature_tables(FeatureTables& T, int mip_count, int tid)
{
  if (tid < 48) {
    const int a = tid / 24, p = (tid / 8) % 3, m = tid & 7;
    const uint32_t v = ((uint32_t)tri_q8((float)m, p, 0) & 0xFFu) | (((uint32_t)tri_q8((float)m, p, 1) & 0xFFu) << 8);
    T.tri[a][p][m] = v << (16 * a);
  } else if (tid < 80) {
    T.lodb[tid - 48] = (uint32_t)lod_q8(tid - 48, mip_count) & 0xFFu;
  }
}

// Four feature bytes starting at byte f (a compile-time offset) into w[].
__device__ __forceinline__ void put_word(uint32_t* w, int f, uint32_t v)
{
  const int sh = 8 * (f & 3);
  w[f >> 2] |= v << sh;
  if (sh != 0) w[(f >> 2) + 1] |= v >> (32 - sh);
}

// GetFeaturesPacked (ntc_decode.hlsli:196-342) for one sample -> Kp signed bytes in w[].
template <class SH>
__device__ __forceinline__ void features(const DecodeArgs& A, float u, float v, int lod, uint32_t* w,
                                         const FeatureTables& T)
{
  constexpr int C0 = SH::C0, C1 = SH::C1, B0 = SH::B0, B1 = SH::B1;
  const ontc_constants& k = A.k;
#pragma unroll
  for (int i = 0; i < SH::Kp / 4; i++) w[i] = 0u;
  lod = clampi(lod, 0, k.mip_count - 1);
  const int lvl = lod < SH::L0MIPS ? 0 : 1 + (lod - SH::L0MIPS) / 2;
  const int d0 = k.g0_grid_dim[lvl], d1 = k.g1_grid_dim[lvl];
  const uint32_t o0 = k.g0_offset[lvl] >> 2, o1 = k.g1_offset[lvl] >> 2;
  // g0: the 4 nearest cells, codes re-centred to signed bytes
  {
    const int gx = (int)floorf(__fsub_rn(__fmul_rn(u, (float)d0), 0.5f));
    const int gy = (int)floorf(__fsub_rn(__fmul_rn(v, (float)d0), 0.5f));
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int cx = clampi(gx + (q & 1), 0, d0 - 1), cy = clampi(gy + (q >> 1), 0, d0 - 1);
      uint32_t st[(C0 * B0 + 31) / 32];
      cell_stream<C0 * B0>(A.g0, A.g0_words, o0, (uint32_t)(cy * d0 + cx), st);
      static_assert(C0 % 4 == 0, "g0 features fill whole words");
      if constexpr (B0 == 4) {
        // a whole word of eight codes at once: even codes into the high nibble of each byte, odd
        // ones likewise, each byte (code << 4) ^ 0x80, interleaved by two byte permutes
#pragma unroll
        for (int c = 0; c + 8 <= C0; c += 8) {
          const uint32_t t = st[c >> 3];
          const uint32_t ev = ((t << 4) & 0xF0F0F0F0u) ^ 0x80808080u, od = (t & 0xF0F0F0F0u) ^ 0x80808080u;
          w[(q * C0 + c) >> 2] = __byte_perm(ev, od, 0x5140);
          w[(q * C0 + c + 4) >> 2] = __byte_perm(ev, od, 0x7362);
        }
        if constexpr (C0 % 8 == 4) w[(q * C0 + C0 - 4) >> 2] = code_bytes4<B0>(st, C0 - 4);
      } else {
        // 2-bit codes (C0 <= 16: one word): plane i holds code 4k + i in byte k, already as
        // (code << 6) ^ 0x80; a 4 x 4 byte transpose by byte permutes gives feature word k =
        // codes 4k .. 4k + 3
        static_assert(B0 == 2 && C0 <= 16, "2-bit g0 codes in one word");
        const uint32_t t = st[0];
        const uint32_t p0 = ((t << 6) & 0xC0C0C0C0u) ^ 0x80808080u, p1 = ((t << 4) & 0xC0C0C0C0u) ^ 0x80808080u;
        const uint32_t p2 = ((t << 2) & 0xC0C0C0C0u) ^ 0x80808080u, p3 = (t & 0xC0C0C0C0u) ^ 0x80808080u;
        const uint32_t a = __byte_perm(p0, p1, 0x5140), c2 = __byte_perm(p2, p3, 0x5140);  // bytes 0, 1
        w[(q * C0) >> 2] = __byte_perm(a, c2, 0x5410);
        if constexpr (C0 > 4) w[(q * C0 + 4) >> 2] = __byte_perm(a, c2, 0x7632);
        if constexpr (C0 > 8) {
          const uint32_t b = __byte_perm(p0, p1, 0x7362), d = __byte_perm(p2, p3, 0x7362);  // bytes 2, 3
          w[(q * C0 + 8) >> 2] = __byte_perm(b, d, 0x5410);
          if constexpr (C0 > 12) w[(q * C0 + 12) >> 2] = __byte_perm(b, d, 0x7632);
        }
      }
    }
  }
  // g1: bilinear blend of the dequantised codes, then *128 to a signed byte
  {
    const float g1x = __fsub_rn(__fmul_rn(u, (float)d1), 0.5f);
    const float g1y = __fsub_rn(__fmul_rn(v, (float)d1), 0.5f);
    const float flx = floorf(g1x), fly = floorf(g1y);
    const int hx = (int)flx, hy = (int)fly;
    const float fx = __fsub_rn(g1x, flx), fy = __fsub_rn(g1y, fly);
    const float ofx = __fsub_rn(1.0f, fx), ofy = __fsub_rn(1.0f, fy);
    const float mult[4] = {__fmul_rn(ofx, ofy), __fmul_rn(fx, ofy), __fmul_rn(ofx, fy), __fmul_rn(fx, fy)};
    // mult * (((float)code - half) / half): code - half is exact, and half is a power of two,
    // so the exact product is (mult / half) * (code - half) with mult / half exact too
    const float half = (float)(1u << (B1 - 1)), rhalf = 1.0f / half;
    const float mh[4] = {__fmul_rn(mult[0], rhalf), __fmul_rn(mult[1], rhalf), __fmul_rn(mult[2], rhalf),
                         __fmul_rn(mult[3], rhalf)};
    static_assert(C1 % 2 == 0, "g1 channels blend in pairs");
    float2 blend[C1 / 2];
#pragma unroll
    for (int c = 0; c < C1 / 2; c++) blend[c] = make_float2(0.0f, 0.0f);
    const float2 off = make_float2(-(8388608.0f + half), -(8388608.0f + half));
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int cx = clampi(hx + (q & 1), 0, d1 - 1), cy = clampi(hy + (q >> 1), 0, d1 - 1);
      uint32_t st[(C1 * B1 + 31) / 32];
      cell_stream<C1 * B1>(A.g1, A.g1_words, o1, (uint32_t)(cy * d1 + cx), st);
      const float2 m2 = make_float2(mh[q], mh[q]);
      static_assert(B1 == 4, "4-bit g1 codes (every profile)");
      // each word's even and odd codes as bytes, masked once per word: code c (nibble c mod 8 of
      // word c / 8) is byte (c mod 8) / 2 of lo (c even) or hi (c odd)
      constexpr int NW1 = (C1 * B1 + 31) / 32;
      uint32_t lo[NW1], hi[NW1];
#pragma unroll
      for (int j = 0; j < NW1; j++) {
        lo[j] = st[j] & 0x0F0F0F0Fu;
        hi[j] = (st[j] >> 4) & 0x0F0F0F0Fu;
      }
#pragma unroll
      for (int c = 0; c < C1; c += 2) {
        // the float bits 0x4B000000 | code by one byte permute (byte 0 the code, bytes 1-2 zero,
        // byte 3 0x4B), then code - half, exactly, for the two channels; then the weighted blend
        const uint32_t sel = 0x7540u | (uint32_t)((c & 7) >> 1);
        const float2 centred =
            ptx::add2(make_float2(__uint_as_float(__byte_perm(lo[c >> 3], 0x4B000000u, sel)),
                                  __uint_as_float(__byte_perm(hi[c >> 3], 0x4B000000u, sel))),
                      off);
        blend[c / 2] = ptx::fma2(m2, centred, blend[c / 2]);
      }
    }
    // the g1 bytes start on a word boundary (4 C0): whole words by byte permutes, a last pair
    // (C1 = 10) byte by byte
    static_assert((4 * C0) % 4 == 0 && C1 % 2 == 0, "g1 feature bytes");
    uint32_t b[C1];
#pragma unroll
    for (int c = 0; c < C1; c += 2) {
      b[c] = s8_rne_sat(__fmul_rn(blend[c / 2].x, 128.0f));
      b[c + 1] = s8_rne_sat(__fmul_rn(blend[c / 2].y, 128.0f));
    }
#pragma unroll
    for (int c = 0; c + 4 <= C1; c += 4) w[(4 * C0 + c) >> 2] = pack4(b[c], b[c + 1], b[c + 2], b[c + 3]);
#pragma unroll
    for (int c = C1 & ~3; c < C1; c++) put_byte(w, 4 * C0 + c, (int)b[c]);
  }
  // 12 triangle waves of the texel coordinate at this lod, then the normalised lod
  {
    const float cdim = (float)(k.dim >> lod);
    const float tcx = floorf(__fmul_rn(u, cdim)), tcy = floorf(__fmul_rn(v, cdim));
    constexpr int base = 4 * C0 + C1;
    if (fabsf(tcx) < 4194304.0f && fabsf(tcy) < 4194304.0f) {
      const int mx = (int)tcx & 7, my = (int)tcy & 7;  // floor-mod, negative coordinates too
#pragma unroll
      for (int p = 0; p < 3; p++) put_word(w, base + 4 * p, T.tri[0][p][mx] | T.tri[1][p][my]);
    } else {
#pragma unroll
      for (int p = 0; p < 3; p++)
#pragma unroll
        for (int a = 0; a < 2; a++)
#pragma unroll
          for (int h = 0; h < 2; h++) put_byte(w, base + p * 4 + a * 2 + h, tri_q8(a == 0 ? tcx : tcy, p, h));
    }
    put_byte(w, base + 12, lod < 32 ? (int)T.lodb[lod] : lod_q8(lod, k.mip_count));
  }
}

// Stores 16 consecutive int8 values (columns c0..c0+15, c0 % 16 == 0) of row r.
__device__ __forceinline__ void st16(uint8_t* base, int r, int c0, int cols, uint32_t a, uint32_t b, uint32_t c,
                                     uint32_t d)
{
  *reinterpret_cast<uint4*>(base + ptx::cm_off8(r, c0, cols)) = make_uint4(a, b, c, d);
}

// 16 accumulator columns of this thread's row -> 16 requantised activations (4 words).  The
// arithmetic of hg_hlsl and q8, two columns at a time on packed fp32 pairs (each lane rounds
// exactly as the scalar operation); the accumulators hold kAccBias + sum (see kAccBias).
//
// kFast (for 1.6e-5 <= rcp <= 600) forms the same bytes with fewer select / compare steps:
// hardgelu as mid(max(min(x, 1.5), -1.5)) + (x - min(x, 1.5)), where the remainder is exact
// for |x| < 2^23 and mid(1.5) = 1.5, so the sum is x above 1.5 and mid below (equal to the
// select form for every float with |x| < 2^23, checked exhaustively on the CPU); from 2^23 up
// both forms give at least 2^23, which saturates to 127 at rcp >= 1.6e-5.
template <bool kFast>
__device__ __forceinline__ void requant16(uint32_t taddr, const float* __restrict__ scale, float rcp, uint32_t* out)
{
  float acc[16];
  ptx::ld16(taddr, acc);
  ptx::ld_wait();
  const float2 third = make_float2(1.0f / 3.0f, 1.0f / 3.0f), m3 = make_float2(-3.0f, -3.0f);
  const float2 h15 = make_float2(1.5f, 1.5f), r2 = make_float2(rcp, rcp), m1 = make_float2(-1.0f, -1.0f);
  const float2 unbias = make_float2(-12582912.0f, -12582912.0f);
  uint32_t b[16];
#pragma unroll
  for (int j = 0; j < 16; j += 2) {
    // (float)sum exactly, then times the row scale: as the conversion and multiply did
    const float2 x =
        ptx::mul2(ptx::add2(make_float2(acc[j], acc[j + 1]), unbias), *reinterpret_cast<const float2*>(scale + j));
    float2 hg;
    if constexpr (kFast) {
      const float2 hi = make_float2(fminf(x.x, 1.5f), fminf(x.y, 1.5f));
      const float2 c = make_float2(fmaxf(hi.x, -1.5f), fmaxf(hi.y, -1.5f));
      const float2 q = ptx::mul2(c, third);
      const float2 q1 = ptx::fma2(ptx::fma2(q, m3, c), third, q);
      const float2 mid = ptx::mul2(q1, ptx::add2(c, h15));
      hg = ptx::add2(mid, ptx::fma2(hi, m1, x));
    } else {
      const float2 c = make_float2(fmaxf(x.x, -1.5f), fmaxf(x.y, -1.5f));
      const float2 q = ptx::mul2(c, third);                        // div3: RN(c * RN(1/3)),
      const float2 q1 = ptx::fma2(ptx::fma2(q, m3, c), third, q);  // corrected by the exact remainder
      const float2 mid = ptx::mul2(q1, ptx::add2(c, h15));
      hg = make_float2(x.x < 1.5f ? mid.x : x.x, x.y < 1.5f ? mid.y : x.y);
    }
    const float2 f = ptx::mul2(hg, r2);
    b[j] = s8_rne_sat(f.x);
    b[j + 1] = s8_rne_sat(f.y);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) out[i] = pack4(b[4 * i], b[4 * i + 1], b[4 * i + 2], b[4 * i + 3]);
}

// One hidden layer's 64 columns of this thread's row, requantised into the next operand tile.
__device__ __forceinline__ void requant_row(uint32_t taddr, const float* __restrict__ scale, float rcp, bool fast,
                                            uint8_t* X, int row, int next_cols)
{
  if (fast) {
#pragma unroll
    for (int c = 0; c < kHid; c += 16) {
      uint32_t q[4];
      requant16<true>(taddr + c, scale + c, rcp, q);
      st16(X, row, c, kHid, q[0], q[1], q[2], q[3]);
    }
  } else {
#pragma unroll
    for (int c = 0; c < kHid; c += 16) {
      uint32_t q[4];
      requant16<false>(taddr + c, scale + c, rcp, q);
      st16(X, row, c, kHid, q[0], q[1], q[2], q[3]);
    }
  }
  // the next layer accumulates into the same columns, from the bias
  for (int c = 0; c < next_cols; c += 16) tmem_st_bias16(taddr + c);
  tmem_st_wait();
}

template <class SH>
__device__ void load_decoder(const uint8_t* __restrict__ blob, uint8_t* W0, uint8_t* W1, uint8_t* Wo, float* s0,
                             float* s1, float* so)
{
  constexpr int Fp = SH::Fp, Kp = SH::Kp;
  // W0 [64][Fp] row-major in the blob -> canonical [64][Kp], zero past Fp
  for (int i = threadIdx.x; i < kHid * Kp; i += kThreads) {
    const int r = i / Kp, c = i - r * Kp;
    W0[ptx::cm_off8(r, c, Kp)] = c < Fp ? blob[r * Fp + c] : 0;
  }
  const uint8_t* b1 = blob + kHid * Fp;
  for (int i = threadIdx.x; i < kHid * kHid; i += kThreads) W1[ptx::cm_off8(i >> 6, i & 63, kHid)] = b1[i];
  const uint8_t* bo = b1 + kHid * kHid;
  for (int i = threadIdx.x; i < kOutRows * kHid; i += kThreads) Wo[ptx::cm_off8(i >> 6, i & 63, kHid)] = bo[i];
  const float* sc = reinterpret_cast<const float*>(bo + kOutRows * kHid);
  for (int i = threadIdx.x; i < kHid; i += kThreads) {
    s0[i] = sc[i];
    s1[i] = sc[kHid + i];
  }
  for (int i = threadIdx.x; i < kOutRows; i += kThreads) so[i] = sc[2 * kHid + i];
}

// InterleavedGradientNoise (ntc_decode.hlsli:143-146), each operation rounded on its own.
__device__ __forceinline__ float ign(float x, float y)
{
  const float t = __fadd_rn(__fmul_rn(0.06711056f, x), __fmul_rn(0.00583715f, y));
  const float r = __fmul_rn(52.9829189f, __fsub_rn(t, floorf(t)));
  return __fsub_rn(r, floorf(r));
}

// HLSL's coarse ddx (axis 0) or ddy (axis 1) of the uv image at the quad whose top-left pixel
// is `c0` = (x0, y0): the forward difference along the quad's first row / column, the backward
// one where the image ends inside the quad, 0 in a one-pixel dimension.
__device__ __forceinline__ float2 quad_delta(const float2* __restrict__ img, int64_t c0, float2 c, int64_t pos,
                                             int64_t extent, int64_t step)
{
  if (pos + 1 < extent) {
    const float2 n = img[c0 + step];
    return make_float2(__fsub_rn(n.x, c.x), __fsub_rn(n.y, c.y));
  }
  if (pos > 0) {
    const float2 n = img[c0 - step];
    return make_float2(__fsub_rn(c.x, n.x), __fsub_rn(c.y, n.y));
  }
  return make_float2(0.0f, 0.0f);
}

// The NTC pixel shaders' stochastic filter (flat_ntc.hlsl:78-84) for pixel i of the uv image:
// ComputeLod (ntc_decode.hlsli:152-168), StochasticFilterLod (:172-177), StochasticFilterUv
// (:181-185).  Returns false for a pixel the shader discards (flat_ntc.hlsl:76-77).
__device__ __forceinline__ bool screen_sample(const DecodeArgs& A, int64_t i, float& u, float& v, int& lod)
{
  const int64_t W = A.screen_w, H = A.screen_h;
  const int64_t y = i / W, x = i - y * W;
  const float2* __restrict__ img = reinterpret_cast<const float2*>(A.uv);
  const float2 p = img[i];
  const int64_t x0 = x & ~1ll, y0 = y & ~1ll, c0 = y0 * W + x0;
  const float2 c = img[c0];
  const float dim = (float)A.k.dim;
  const float2 dx = quad_delta(img, c0, c, x0, W, 1), dy = quad_delta(img, c0, c, y0, H, W);
  const float2 du = make_float2(__fmul_rn(dx.x, dim), __fmul_rn(dx.y, dim));
  const float2 dv = make_float2(__fmul_rn(dy.x, dim), __fmul_rn(dy.y, dim));
  const float gu = __fadd_rn(__fmul_rn(du.x, du.x), __fmul_rn(du.y, du.y));
  const float gv = __fadd_rn(__fmul_rn(dv.x, dv.x), __fmul_rn(dv.y, dv.y));
  const float2 major_d = gu > gv ? du : dv;
  const float2 foot = make_float2(__fdiv_rn(major_d.x, dim), __fdiv_rn(major_d.y, dim));
  const float major = __fsqrt_rn(fmaxf(gu, gv));
  const float minor = fmaxf(__fsqrt_rn(fminf(gu, gv)), __fdiv_rn(major, 8.0f));  // max_aniso 8
  const float lodab = fminf(fmaxf(log2f(minor), 0.0f), (float)(A.k.mip_count - 1));
  // noise position: pixel centre + 5.588238 * noise_frame
  const float nf = __fmul_rn(5.588238f, A.noise_frame);
  const float px = __fadd_rn(__fadd_rn((float)x, 0.5f), nf), py = __fadd_rn(__fadd_rn((float)y, 0.5f), nf);
  lod = (int)lodab + (ign(px, py) < __fsub_rn(lodab, floorf(lodab)) ? 1 : 0);
  const float jitter = __fsub_rn(ign(__fadd_rn(px, 61.0f), __fadd_rn(py, 37.0f)), 0.5f);
  u = __fadd_rn(p.x, __fmul_rn(foot.x, jitter));
  v = __fadd_rn(p.y, __fmul_rn(foot.y, jitter));
  return !(A.discard_outside && (p.x < 0.0f || p.y < 0.0f || p.x > 1.0f || p.y > 1.0f));
}

// DefaultMaterialParams (ntc_decode.hlsli:524-540) in ontc_material_params order.
__device__ __forceinline__ void store_material(float* o, const float* y, int C, const DecodeArgs& A)
{
  float2* o2 = reinterpret_cast<float2*>(o);  // records are 72 bytes: 8-byte aligned
  o2[0] = make_float2(0.5f, 0.5f);                        // albedo
  o2[1] = make_float2(0.5f, 1.0f);                        // albedo.z, alpha
  o2[2] = make_float2(0.5f, 0.0f);                        // displacement, emissive
  o2[3] = make_float2(0.0f, 0.0f);                        // gloss, metallic
  o2[4] = make_float2(0.5f, 0.5f);                        // normal.xy
  o2[5] = make_float2(1.0f, 1.0f);                        // normal.z, ao
  o2[6] = make_float2(1.0f, 0.5f);                        // roughness, specular.x
  o2[7] = make_float2(0.5f, 0.5f);                        // specular.yz
  o2[8] = make_float2(0.0f, __uint_as_float(A.material_present));  // transmission, present
  // DecodeMaterial (:544-603): channel c into its field; a later channel of the same scalar
  // field overwrites an earlier one (same thread, program order)
#pragma unroll
  for (int c = 0; c < kOutRows; c++)
    if (c < C && A.material_dst[c] >= 0) o[A.material_dst[c]] = y[c];
}

template <class SH>
__global__ void __launch_bounds__(kThreads, 1) decode_kernel(const __grid_constant__ DecodeArgs A)
{
  constexpr int Kp = SH::Kp;
  constexpr uint32_t SX = (Kp / 16) * 128;  // 8-row group stride of a [*][Kp] int8 tile
  constexpr uint32_t S64 = (kHid / 16) * 128;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[kGroups];
  __shared__ uint32_t tmem_base_s;
  __shared__ int fail_s;
  __shared__ __align__(16) float s0[kHid], s1[kHid], so[kOutRows];  // read as float2 pairs
  __shared__ FeatureTables tables_s;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int g = tid >> 7;
  const int row = tid & 127;
  const int quad = warp & 3;
  uint8_t* X = smem_raw + (size_t)g * DecodeSmem::kTile;
  uint8_t* sW0 = smem_raw + (size_t)kGroups * DecodeSmem::kTile;
  uint8_t* sW1 = sW0 + kHid * Kp;
  uint8_t* sWo = sW1 + kHid * kHid;

  if (tid == 0) {
    for (int i = 0; i < kGroups; i++) ptx::mbar_init(&bars[i], 1);
    ptx::fence_mbar_init();
    fail_s = 0;
  }
  if (warp == 0) ptx::tmem_alloc(&tmem_base_s, 64 * kGroups);  // a power of two: 512
  load_decoder<SH>(A.blob, sW0, sW1, sWo, s0, s1, so);
  build_feature_tables(tables_s, A.k.mip_count, tid);
  ptx::fence_proxy_async();
  ptx::fence_before_sync();
  __syncthreads();
  ptx::fence_after_sync();
  const uint32_t tbase = tmem_base_s;
  const uint32_t win = tbase + 64u * (uint32_t)g;
  const uint32_t lwin = win + ((uint32_t)(quad * 32) << 16);
  uint64_t* bar = &bars[g];
  uint32_t phase = 0;
  // the group's first warp issues its MMAs (one elected lane) and polls for them
  const bool issuer = (row >> 5) == 0, poller = issuer;
  const int C = A.k.channel_count;
  const float rcp1 = A.k.rcp_s_a1, rcp2 = A.k.rcp_s_a2;
  const bool fast1 = rcp1 >= 1.6e-5f && rcp1 <= 600.0f, fast2 = rcp2 >= 1.6e-5f && rcp2 <= 600.0f;

  constexpr uint32_t I_L01 = ptx::idesc_s8(128, kHid, false, false);
  constexpr uint32_t I_L2 = ptx::idesc_s8(128, kOutRows, false, false);
  const uint32_t aX = ptx::smem_addr(X), aW0 = ptx::smem_addr(sW0), aW1 = ptx::smem_addr(sW1),
                 aWo = ptx::smem_addr(sWo);

  auto wait_mma = [&]() -> bool {
    if (poller && !ptx::mbar_wait(bar, phase)) atomicExch(&fail_s, 1);
    phase ^= 1u;
    bar_group(g);
    ptx::fence_after_sync();
    return *(volatile int*)&fail_s == 0;
  };
  auto handoff = [&]() {
    ptx::fence_proxy_async();
    ptx::fence_before_sync();
    bar_group(g);
  };

  const int64_t ntiles = (A.n + 127) / 128;
  for (int64_t t = (int64_t)blockIdx.x * kGroups + g; t < ntiles; t += (int64_t)gridDim.x * kGroups) {
    const int64_t i = t * 128 + row;
    bool valid = i < A.n;
    // ---------------------------------------------------------------- features -> X
    {
      uint32_t w[Kp / 4];
      if (valid) {
        float u, v;
        int lod;
        if (A.screen_w > 0) {
          valid = screen_sample(A, i, u, v, lod);
        } else {
          const float2 uv = reinterpret_cast<const float2*>(A.uv)[i];
          u = uv.x;
          v = uv.y;
          lod = A.lod[i];
        }
        features<SH>(A, u, v, lod, w, tables_s);
        if (A.feat_out) {
          uint4* fo = reinterpret_cast<uint4*>(A.feat_out + i * 24);
#pragma unroll
          for (int j = 0; j < Kp / 16; j++) fo[j] = make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
        }
      } else {
#pragma unroll
        for (int j = 0; j < Kp / 4; j++) w[j] = 0u;
      }
#pragma unroll
      for (int c = 0; c < Kp; c += 16) st16(X, row, c, Kp, w[c / 4], w[c / 4 + 1], w[c / 4 + 2], w[c / 4 + 3]);
    }
    // layer 0 accumulates from the bias (the previous tile's outputs were read before the last barrier)
#pragma unroll
    for (int c = 0; c < kHid; c += 16) tmem_st_bias16(lwin + c);
    tmem_st_wait();
    handoff();
    if (issuer) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < Kp / 32; k++)
        ptx::mma_s8_warp(win, ptx::desc(aX + k * 256, 128, SX), ptx::desc(aW0 + k * 256, 128, SX), I_L01, 1);
      ptx::commit_warp(bar);
    }
    if (!wait_mma()) break;
    // ---------------------------------------------------------------- a0 -> A (over X)
    requant_row(lwin, s0, rcp1, fast1, X, row, kHid);
    handoff();
    if (issuer) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < kHid / 32; k++)
        ptx::mma_s8_warp(win, ptx::desc(aX + k * 256, 128, S64), ptx::desc(aW1 + k * 256, 128, S64), I_L01, 1);
      ptx::commit_warp(bar);
    }
    if (!wait_mma()) break;
    // ---------------------------------------------------------------- a1 -> A
    requant_row(lwin, s1, rcp2, fast2, X, row, kOutRows);
    handoff();
    if (issuer) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < kHid / 32; k++)
        ptx::mma_s8_warp(win, ptx::desc(aX + k * 256, 128, S64), ptx::desc(aWo + k * 256, 128, S64), I_L2, 1);
      ptx::commit_warp(bar);
    }
    if (!wait_mma()) break;
    // ---------------------------------------------------------------- outputs
    {
      float acc[16];
      ptx::ld16(lwin, acc);
      ptx::ld_wait();
      if (valid) {
        // (float)sum * scale, saturated by the multiply; groups of four rows past the channel
        // count (the same for every thread) are skipped
#pragma unroll
        for (int c0 = 0; c0 < kOutRows; c0 += 4)
          if (c0 < C) {
#pragma unroll
            for (int c = c0; c < c0 + 4; c++) acc[c] = __saturatef(__fmul_rn(__fsub_rn(acc[c], 12582912.0f), so[c]));
          }
        if (A.material) {
          store_material(A.out + i * 18, acc, C, A);
        } else {
          float* o = A.out + i * C;
#pragma unroll
          for (int c = 0; c < kOutRows; c++)
            if (c < C) o[c] = acc[c];
        }
      }
    }
    // the next tile's features overwrite X only after every thread has read its outputs
    ptx::fence_before_sync();
    bar_group(g);
  }
  if (*(volatile int*)&fail_s != 0 && tid == 0) atomicExch(A.err, 1);
  ptx::fence_before_sync();
  __syncthreads();
  if (warp == 0) ptx::tmem_dealloc(tbase, 64 * kGroups);
}

template <class SH>
cudaError_t launch_decode_shape(const DecodeArgs& A, int grid, cudaStream_t stream)
{
  constexpr size_t smem = kGroups * DecodeSmem::kTile + kHid * SH::Kp + kHid * kHid + kOutRows * kHid + 1024;
  static_assert(smem <= 227 * 1024, "shared memory budget");
  cudaError_t e = cudaFuncSetAttribute(decode_kernel<SH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  decode_kernel<SH><<<grid, kThreads, smem, stream>>>(A);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_decode(int profile, const DecodeArgs& A, cudaStream_t stream)
{
  if (A.n <= 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long tiles = (A.n + 127) / 128;
  const int grid = (int)std::min<long long>(sms, (tiles + kGroups - 1) / kGroups);
  switch (profile) {  // ntc_decode.hlsli:60-86
    case 0: return launch_decode_shape<DShape<8, 12, 2, 4, 4>>(A, grid, stream);
    case 1: return launch_decode_shape<DShape<12, 20, 4, 4, 4>>(A, grid, stream);
    case 2: return launch_decode_shape<DShape<12, 10, 2, 4, 3>>(A, grid, stream);
    case 3: return launch_decode_shape<DShape<16, 12, 4, 4, 3>>(A, grid, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ontc
