// Float-model decoders: SampleMaterial's sampling (ntc_decode.hlsli:196-342, 605-623) with the
// trained fp32 decoder weights in place of the int8 blob, in FP32, BF16 or FP8 (e4m3 with
// per-layer scales).  The features are the float values the int8 decoder quantises: the g0
// codes dequantised ((code - 2^(b-1)) * 2 / 2^b, the latents training ended with), the bilinear
// blend of the dequantised g1 codes, the 12 triangle waves of the texel coordinate and the
// normalised lod, i.e. the training model's draw_features (ntc_kernel.cu:75-177) at uv; the
// MLP is forward_hardgelu between three layers (libopenntc.cpp:1034-1038); outputs saturate as
// DecodeMaterial does (ntc_decode.hlsli:570).
//
//  * decode_f32_kernel: fp32 on the CUDA cores, one sample per thread, weights transposed in
//    shared memory so each vector load feeds four FMAs.
//  * decode_tc_kernel<FP8>: the int8 decoder's structure (8 groups of 128 samples, one CTA per
//    SM) with three tcgen05 layers, kind::f16 (bf16) or kind::f8f6f4 (e4m3), fp32 accumulators
//    in TMEM; the epilogues apply the layer scales and hardgelu in fp32 and requantise to the
//    next layer's type.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "decode_cells.cuh"
#include "kernels.h"
#include "tc_ptx.cuh"

namespace ontc {

namespace {

template <int C0_, int C1_, int B0_, int B1_, int L0MIPS_>
struct FShape {
  static constexpr int C0 = C0_, C1 = C1_, B0 = B0_, B1 = B1_, L0MIPS = L0MIPS_;
  static constexpr int F = ((4 * C0 + C1 + 13 + 3) / 4) * 4;  // the training feature width
  static constexpr int Kp = ((F + 31) / 32) * 32;             // K of the tensor-core layer 0
};

// The float features of one sample, emitted in order through put(value), then zeros up to Kp.
template <class SH, class Put>
__device__ __forceinline__ void features_f32(const FloatDecodeArgs& A, float u, float v, int lod, Put&& put)
{
  constexpr int C0 = SH::C0, C1 = SH::C1, B0 = SH::B0, B1 = SH::B1;
  const ontc_constants& k = A.k;
  lod = clampi(lod, 0, k.mip_count - 1);
  const int lvl = lod < SH::L0MIPS ? 0 : 1 + (lod - SH::L0MIPS) / 2;
  const int d0 = k.g0_grid_dim[lvl], d1 = k.g1_grid_dim[lvl];
  const uint32_t o0 = k.g0_offset[lvl] >> 2, o1 = k.g1_offset[lvl] >> 2;
  constexpr float q0 = 2.0f / (float)(1 << B0), q1 = 2.0f / (float)(1 << B1);
  constexpr float h0 = (float)(1 << (B0 - 1)), h1 = (float)(1 << (B1 - 1));
  {  // g0: the 4 nearest cells (GetFeaturesPacked's cell choice)
    const int gx = (int)floorf(__fsub_rn(__fmul_rn(u, (float)d0), 0.5f));
    const int gy = (int)floorf(__fsub_rn(__fmul_rn(v, (float)d0), 0.5f));
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int cx = clampi(gx + (q & 1), 0, d0 - 1), cy = clampi(gy + (q >> 1), 0, d0 - 1);
      uint32_t st[(C0 * B0 + 31) / 32];
      cell_stream<C0 * B0>(A.g0, A.g0_words, o0, (uint32_t)(cy * d0 + cx), st);
#pragma unroll
      for (int c = 0; c < C0; c++) put(__fmul_rn((float)code_of<B0>(st, c) - h0, q0));
    }
  }
  {  // g1: bilinear blend of the dequantised codes
    const float g1x = __fsub_rn(__fmul_rn(u, (float)d1), 0.5f);
    const float g1y = __fsub_rn(__fmul_rn(v, (float)d1), 0.5f);
    const float flx = floorf(g1x), fly = floorf(g1y);
    const int hx = (int)flx, hy = (int)fly;
    const float fx = __fsub_rn(g1x, flx), fy = __fsub_rn(g1y, fly);
    const float ofx = __fsub_rn(1.0f, fx), ofy = __fsub_rn(1.0f, fy);
    const float mult[4] = {__fmul_rn(ofx, ofy), __fmul_rn(fx, ofy), __fmul_rn(ofx, fy), __fmul_rn(fx, fy)};
    float acc[C1];
#pragma unroll
    for (int c = 0; c < C1; c++) acc[c] = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int cx = clampi(hx + (q & 1), 0, d1 - 1), cy = clampi(hy + (q >> 1), 0, d1 - 1);
      uint32_t st[(C1 * B1 + 31) / 32];
      cell_stream<C1 * B1>(A.g1, A.g1_words, o1, (uint32_t)(cy * d1 + cx), st);
#pragma unroll
      for (int c = 0; c < C1; c++) acc[c] = __fmaf_rn(mult[q], __fmul_rn((float)code_of<B1>(st, c) - h1, q1), acc[c]);
    }
#pragma unroll
    for (int c = 0; c < C1; c++) put(acc[c]);
  }
  {  // 12 triangle waves of the texel coordinate at this lod, then the normalised lod
    const float cdim = (float)(k.dim >> lod);
    const float tcx = floorf(__fmul_rn(u, cdim)), tcy = floorf(__fmul_rn(v, cdim));
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int a = 0; a < 2; a++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const float P = (float)(8 >> p), rP = 1.0f / P;  // P = 8, 4, 2: dividing = exact scaling
          const float c = a == 0 ? tcx : tcy;
          const float ph = h == 0 ? 0.0f : __fmul_rn(0.25f, P);
          const float t = __fmul_rn(__fadd_rn(__fadd_rn(c, 0.5f), ph), rP);
          put(__fsub_rn(1.0f, __fmul_rn(4.0f, fabsf(__fsub_rn(__fsub_rn(t, floorf(t)), 0.5f)))));
        }
    put(__fdiv_rn((float)lod, (float)(k.mip_count - 1)));
  }
#pragma unroll
  for (int i = 4 * C0 + C1 + 13; i < SH::Kp; i++) put(0.0f);
}

// hardgelu with x / 3 as a product with 1/3 (within an ulp of the division): the correctly
// rounded division costs several XU-pipe instructions and changes nothing measurable here (the
// tensor-core variants round the result to bf16 or e4m3 next).
__device__ __forceinline__ float hardgelu_mul(float x)
{
  return x < -1.5f ? 0.0f : (x < 1.5f ? x * (1.0f / 3.0f) * (x + 1.5f) : x);
}

// ---------------------------------------------------------------------------------- FP32
constexpr int kF32Threads = 128;

template <class SH>
__global__ void __launch_bounds__(kF32Threads) decode_f32_kernel(const __grid_constant__ FloatDecodeArgs A)
{
  constexpr int F = SH::F, XS = F + 1;  // odd row stride: each thread's feature row in its own banks
  extern __shared__ __align__(16) float fsm[];
  float* W0t = fsm;            // [F][64]   W0 transposed
  float* W1t = W0t + F * 64;   // [64][64]  W1 transposed ([j][o])
  float* Wot = W1t + 64 * 64;  // [64][16]  Wout transposed ([o][c])
  float* X = Wot + 64 * 16;    // [128][F + 1]
  const int tid = threadIdx.x;
  for (int i = tid; i < 64 * F; i += kF32Threads) {
    const int h = i / F, f = i - h * F;
    W0t[f * 64 + h] = A.W[i];
  }
  for (int i = tid; i < 64 * 64; i += kF32Threads) W1t[(i & 63) * 64 + (i >> 6)] = A.W[w1_off(F) + i];
  for (int i = tid; i < 16 * 64; i += kF32Threads) Wot[(i & 63) * 16 + (i >> 6)] = A.W[wo_off(F) + i];
  __syncthreads();
  const int C = A.k.channel_count;
  float* xr = X + tid * XS;
  for (int64_t t = blockIdx.x; t * kF32Threads < A.n; t += gridDim.x) {
    const int64_t i = t * kF32Threads + tid;
    if (i >= A.n) continue;
    const float2 uv = reinterpret_cast<const float2*>(A.uv)[i];
    int nf = 0;
    features_f32<SH>(A, uv.x, uv.y, A.lod[i], [&](float x) {
      if (nf < F) xr[nf] = x;
      nf++;
    });
    float h[64];
#pragma unroll
    for (int j = 0; j < 64; j++) h[j] = 0.0f;
    for (int f = 0; f < F; f++) {  // kept rolled: one feature, 64 FMAs per iteration
      const float x = xr[f];
      const float4* w = reinterpret_cast<const float4*>(W0t + f * 64);
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const float4 q = w[j];
        h[4 * j] = __fmaf_rn(q.x, x, h[4 * j]);
        h[4 * j + 1] = __fmaf_rn(q.y, x, h[4 * j + 1]);
        h[4 * j + 2] = __fmaf_rn(q.z, x, h[4 * j + 2]);
        h[4 * j + 3] = __fmaf_rn(q.w, x, h[4 * j + 3]);
      }
    }
    float g[64];
#pragma unroll
    for (int j = 0; j < 64; j++) {
      h[j] = hardgelu_mul(h[j]);
      g[j] = 0.0f;
    }
#pragma unroll
    for (int j = 0; j < 64; j++) {
      const float4* w = reinterpret_cast<const float4*>(W1t + j * 64);
#pragma unroll
      for (int o = 0; o < 16; o++) {
        const float4 q = w[o];
        g[4 * o] = __fmaf_rn(q.x, h[j], g[4 * o]);
        g[4 * o + 1] = __fmaf_rn(q.y, h[j], g[4 * o + 1]);
        g[4 * o + 2] = __fmaf_rn(q.z, h[j], g[4 * o + 2]);
        g[4 * o + 3] = __fmaf_rn(q.w, h[j], g[4 * o + 3]);
      }
    }
    float y[16];
#pragma unroll
    for (int c = 0; c < 16; c++) y[c] = 0.0f;
#pragma unroll
    for (int o = 0; o < 64; o++) {
      const float a = hardgelu_mul(g[o]);
      const float4* w = reinterpret_cast<const float4*>(Wot + o * 16);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const float4 q = w[c];
        y[4 * c] = __fmaf_rn(q.x, a, y[4 * c]);
        y[4 * c + 1] = __fmaf_rn(q.y, a, y[4 * c + 1]);
        y[4 * c + 2] = __fmaf_rn(q.z, a, y[4 * c + 2]);
        y[4 * c + 3] = __fmaf_rn(q.w, a, y[4 * c + 3]);
      }
    }
    float* o = A.out + i * C;
#pragma unroll
    for (int c = 0; c < 16; c++)
      if (c < C) o[c] = fminf(1.0f, fmaxf(0.0f, y[c]));
  }
}

// --------------------------------------------------------------------------- BF16 / FP8
constexpr int kTGroups = 8;  // 1024 threads, 64 TMEM columns per group
constexpr int kTGroupThreads = 128;
constexpr int kTThreads = kTGroups * kTGroupThreads;

__device__ __forceinline__ void bar_tgroup(int g)
{
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kTGroupThreads) : "memory");
}

// Instruction descriptor, kind::f8f6f4 with e4m3 A/B (format 0) and fp32 D, K-major operands.
__host__ __device__ constexpr uint32_t idesc_e4m3(int M, int N)
{
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// issued by the lane elect.sync picks in a converged warp, as ptx::mma_bf16_warp
__device__ __forceinline__ void mma_e4m3(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p, e;\n\telect.sync _|e, 0xffffffff;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "@e tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// One 16-byte row chunk of a K-major operand tile: 8 bf16 (columns c0..c0+7) or 16 e4m3
// (columns c0..c0+15) values, each scaled by `mul` first (e4m3: saturating conversion).
template <bool FP8>
__device__ __forceinline__ void st_chunk_f(uint8_t* base, int r, int c0, int cols, const float* v, float mul)
{
  if constexpr (FP8) {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const uint32_t lo = __nv_cvt_float2_to_fp8x2(make_float2(v[4 * i] * mul, v[4 * i + 1] * mul), __NV_SATFINITE,
                                                   __NV_E4M3);
      const uint32_t hi = __nv_cvt_float2_to_fp8x2(make_float2(v[4 * i + 2] * mul, v[4 * i + 3] * mul),
                                                   __NV_SATFINITE, __NV_E4M3);
      w[i] = lo | (hi << 16);
    }
    *reinterpret_cast<uint4*>(base + ptx::cm_off8(r, c0, cols)) = make_uint4(w[0], w[1], w[2], w[3]);
  } else {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const __nv_bfloat162 b = __floats2bfloat162_rn(v[2 * i] * mul, v[2 * i + 1] * mul);
      w[i] = *reinterpret_cast<const uint32_t*>(&b);
    }
    *reinterpret_cast<uint4*>(base + ptx::cm_off16(r, c0, cols)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// 16 accumulator columns of this thread's row -> scale, hardgelu, rescale -> next layer's tile.
template <bool FP8>
__device__ __forceinline__ void act16(uint32_t taddr, uint8_t* X, int row, int c0, float pre, float post)
{
  float acc[16];
  ptx::ld16(taddr, acc);
  ptx::ld_wait();
#pragma unroll
  for (int j = 0; j < 16; j++) acc[j] = hardgelu_mul(acc[j] * pre);
  if constexpr (FP8) {
    st_chunk_f<true>(X, row, c0, 64, acc, post);
  } else {
    st_chunk_f<false>(X, row, c0, 64, acc, post);
    st_chunk_f<false>(X, row, c0 + 8, 64, acc + 8, post);
  }
}

template <class SH, bool FP8>
__global__ void __launch_bounds__(kTThreads, 1) decode_tc_kernel(const __grid_constant__ FloatDecodeArgs A)
{
  constexpr int Kp = SH::Kp, EB = FP8 ? 1 : 2;
  constexpr int KSTEP = FP8 ? 32 : 16;  // K per MMA: one 32-byte row slice, two core matrices
  constexpr int CHUNK = 16 / EB;        // values per 16-byte row chunk
  constexpr uint32_t SX = (uint32_t)(Kp * EB / 16) * 128, S64 = (uint32_t)(64 * EB / 16) * 128;
  constexpr uint32_t kTile = 128 * Kp * EB;  // per group: X, then a0, then a1 (over X)
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bars[kTGroups];
  __shared__ uint32_t tmem_base_s;
  __shared__ int fail_s;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int g = tid >> 7;
  const int row = tid & 127;
  const int quad = warp & 3;
  uint8_t* X = smem_raw + (size_t)g * kTile;
  uint8_t* sW0 = smem_raw + (size_t)kTGroups * kTile;
  uint8_t* sW1 = sW0 + 64 * Kp * EB;
  uint8_t* sWo = sW1 + 64 * 64 * EB;

  if (tid == 0) {
    for (int i = 0; i < kTGroups; i++) ptx::mbar_init(&bars[i], 1);
    ptx::fence_mbar_init();
    fail_s = 0;
  }
  if (warp == 0) ptx::tmem_alloc(&tmem_base_s, 64 * kTGroups);
  {  // row-major weights -> K-major canonical tiles
    const uint8_t* src = static_cast<const uint8_t*>(A.Wq);
    auto place = [&](uint8_t* dst, const uint8_t* s, int rows, int cols) {
      for (int i = tid; i < rows * cols; i += kTThreads) {
        const int r = i / cols, c = i - r * cols;
        if constexpr (FP8)
          dst[ptx::cm_off8(r, c, cols)] = s[i];
        else
          *reinterpret_cast<uint16_t*>(dst + ptx::cm_off16(r, c, cols)) = reinterpret_cast<const uint16_t*>(s)[i];
      }
    };
    place(sW0, src, 64, Kp);
    place(sW1, src + 64 * Kp * EB, 64, 64);
    place(sWo, src + (64 * Kp + 64 * 64) * EB, 16, 64);
  }
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
  const float inv_sx = 1.0f / A.sx, pre0 = A.sx * A.sw0, post0 = 1.0f / A.sa1;
  const float pre1 = A.sa1 * A.sw1, post1 = 1.0f / A.sa2, outs = A.sa2 * A.swo;

  constexpr uint32_t I_L01 = FP8 ? idesc_e4m3(128, 64) : ptx::idesc_bf16(128, 64, false, false);
  constexpr uint32_t I_L2 = FP8 ? idesc_e4m3(128, 16) : ptx::idesc_bf16(128, 16, false, false);
  const uint32_t aX = ptx::smem_addr(X), aW0 = ptx::smem_addr(sW0), aW1 = ptx::smem_addr(sW1),
                 aWo = ptx::smem_addr(sWo);
  auto mma = [&](uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    if constexpr (FP8)
      mma_e4m3(d, a, b, id, acc);
    else
      ptx::mma_bf16_warp(d, a, b, id, acc);
  };
  auto wait_mma = [&]() -> bool {
    if (poller && !ptx::mbar_wait(bar, phase)) atomicExch(&fail_s, 1);
    phase ^= 1u;
    bar_tgroup(g);
    ptx::fence_after_sync();
    return *(volatile int*)&fail_s == 0;
  };
  auto handoff = [&]() {
    ptx::fence_proxy_async();
    ptx::fence_before_sync();
    bar_tgroup(g);
  };

  const int64_t ntiles = (A.n + 127) / 128;
  for (int64_t t = (int64_t)blockIdx.x * kTGroups + g; t < ntiles; t += (int64_t)gridDim.x * kTGroups) {
    const int64_t i = t * 128 + row;
    const bool valid = i < A.n;
    // ---------------------------------------------------------------- features -> X
    {
      float buf[CHUNK];
      int nf = 0;
      auto put = [&](float x) {
        buf[nf % CHUNK] = x;
        nf++;
        if (nf % CHUNK == 0) st_chunk_f<FP8>(X, row, nf - CHUNK, Kp, buf, inv_sx);
      };
      if (valid) {
        const float2 uv = reinterpret_cast<const float2*>(A.uv)[i];
        features_f32<SH>(A, uv.x, uv.y, A.lod[i], put);
      } else {
#pragma unroll
        for (int c = 0; c < Kp; c++) put(0.0f);
      }
    }
    handoff();
    if (issuer) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < Kp / KSTEP; k++)
        mma(win, ptx::desc(aX + k * 256, 128, SX), ptx::desc(aW0 + k * 256, 128, SX), I_L01, k > 0);
      ptx::commit_warp(bar);
    }
    if (!wait_mma()) break;
    // ---------------------------------------------------------------- a0 -> X
#pragma unroll
    for (int c = 0; c < 64; c += 16) act16<FP8>(lwin + c, X, row, c, pre0, post0);
    handoff();
    if (issuer) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < 64 / KSTEP; k++)
        mma(win, ptx::desc(aX + k * 256, 128, S64), ptx::desc(aW1 + k * 256, 128, S64), I_L01, k > 0);
      ptx::commit_warp(bar);
    }
    if (!wait_mma()) break;
    // ---------------------------------------------------------------- a1 -> X
#pragma unroll
    for (int c = 0; c < 64; c += 16) act16<FP8>(lwin + c, X, row, c, pre1, post1);
    handoff();
    if (issuer) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < 64 / KSTEP; k++)
        mma(win, ptx::desc(aX + k * 256, 128, S64), ptx::desc(aWo + k * 256, 128, S64), I_L2, k > 0);
      ptx::commit_warp(bar);
    }
    if (!wait_mma()) break;
    // ---------------------------------------------------------------- outputs
    {
      float acc[16];
      ptx::ld16(lwin, acc);
      ptx::ld_wait();
      if (valid) {
        float* o = A.out + i * C;
#pragma unroll
        for (int c = 0; c < 16; c++)
          if (c < C) o[c] = fminf(1.0f, fmaxf(0.0f, acc[c] * outs));
      }
    }
    // the next tile's features overwrite X only after every thread has read its outputs
    ptx::fence_before_sync();
    bar_tgroup(g);
  }
  if (*(volatile int*)&fail_s != 0 && tid == 0) atomicExch(A.err, 1);
  ptx::fence_before_sync();
  __syncthreads();
  if (warp == 0) ptx::tmem_dealloc(tbase, 64 * kTGroups);
}

template <class SH>
cudaError_t launch_shape(int mode, const FloatDecodeArgs& A, int sms, cudaStream_t stream)
{
  if (mode == ONTC_DECODE_FP32) {
    constexpr size_t smem = (size_t)(SH::F * 64 + 64 * 64 + 64 * 16 + kF32Threads * (SH::F + 1)) * sizeof(float);
    static_assert(smem <= 227 * 1024, "shared memory budget");
    cudaError_t e =
        cudaFuncSetAttribute(decode_f32_kernel<SH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const long long blocks = (A.n + kF32Threads - 1) / kF32Threads;
    const int grid = (int)std::min<long long>(blocks, (long long)sms * 2);
    decode_f32_kernel<SH><<<grid, kF32Threads, smem, stream>>>(A);
    return cudaGetLastError();
  }
  const long long tiles = (A.n + 127) / 128;
  const int grid = (int)std::min<long long>(sms, (tiles + kTGroups - 1) / kTGroups);
  auto go = [&](auto kernel, int EB) -> cudaError_t {
    const size_t smem = (size_t)kTGroups * 128 * SH::Kp * EB + (size_t)(64 * SH::Kp + 64 * 64 + 16 * 64) * EB + 1024;
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kernel<<<grid, kTThreads, smem, stream>>>(A);
    return cudaGetLastError();
  };
  if (mode == ONTC_DECODE_BF16) return go(decode_tc_kernel<SH, false>, 2);
  if (mode == ONTC_DECODE_FP8) return go(decode_tc_kernel<SH, true>, 1);
  return cudaErrorInvalidValue;
}

}  // namespace

int float_decode_kp(int profile)
{
  switch (profile) {  // ntc_decode.hlsli:60-86
    case 0: return FShape<8, 12, 2, 4, 4>::Kp;
    case 1: return FShape<12, 20, 4, 4, 4>::Kp;
    case 2: return FShape<12, 10, 2, 4, 3>::Kp;
    case 3: return FShape<16, 12, 4, 4, 3>::Kp;
    default: return 0;
  }
}

cudaError_t launch_decode_float(int profile, int mode, const FloatDecodeArgs& A, cudaStream_t stream)
{
  if (A.n <= 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  switch (profile) {
    case 0: return launch_shape<FShape<8, 12, 2, 4, 4>>(mode, A, sms, stream);
    case 1: return launch_shape<FShape<12, 20, 4, 4, 4>>(mode, A, sms, stream);
    case 2: return launch_shape<FShape<12, 10, 2, 4, 3>>(mode, A, sms, stream);
    case 3: return launch_shape<FShape<16, 12, 4, 4, 3>>(mode, A, sms, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ontc
