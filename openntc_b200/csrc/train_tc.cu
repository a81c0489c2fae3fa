// BF16 tensor-core tile kernel for one training step (sm_100a, tcgen05 + TMEM).
//
// Each CTA owns 128-texel work units in turn (persistent grid).  Per unit, the whole
// per-texel pipeline of upstream's step runs on chip:
//
//   gather (ntc_kernel.cu:75-177)             -> sX   [128 x Kp]  bf16, shared memory
//   H0 = X  W0^T          (M128 N64  K=Kp)    -> TMEM, epilogue: A0 = hg(H0) -> sA0
//   H1 = A0 W1^T          (M128 N64  K=64)    -> TMEM, epilogue: A1 = hg(H1) -> sA1
//   Y  = A1 Wout^T        (M128 N16  K=64)    -> TMEM, epilogue: dY = -2(t-y)/(C B) -> sdY
//   dA1 = dY Wout         (M128 N64  K=16)    -> TMEM, epilogue: dH1 = dA1 hg'(H1) -> sdH1
//   dA0 = dH1 W1          (M128 N64  K=64)    -> TMEM, epilogue: dH0 = dA0 hg'(H0) -> sdH0
//   dX  = dH0 W0          (M128 N=Kp K=64)    -> TMEM, epilogue: scatter-add into the latent
//                                                gradients (ntc_kernel.cu:280-341)
// and the weight gradients accumulate in TMEM across all of the CTA's units:
//   dWout^T += A1^T dY (M64 N16), dW1 += dH1^T A0 (M64 N64), dW0 += dH0^T X (M64 N=Kp),
// K = 128 texels each, written once per CTA to its partial-sum slot.
//
// Every operand lives in shared memory in the no-swizzle canonical layout; an activation
// tile [128 texels][n] serves as the K-major A operand of the next layer and, unchanged, as
// the MN-major operand of the weight-gradient products.  Hidden pre-activations stay in
// registers for the backward (no recompute pass, nothing stored to HBM).  One thread issues
// the MMAs and commits them to an mbarrier; every wait is bounded and reports a timeout
// through the error word instead of spinning forever.
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"
#include "tc_ptx.cuh"

namespace ontc {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kTmemCols = 512;
// TMEM column map
constexpr uint32_t kColH = 0;      // H0 / H1 / dA1 / dA0   (64)
constexpr uint32_t kColY = 64;     // Y                      (16)
constexpr uint32_t kColDX = 128;   // dX                     (<= 96)
constexpr uint32_t kColW0 = 256;   // dW0 accumulator, M=64  (<= 96)
constexpr uint32_t kColW1 = 384;   // dW1 accumulator, M=64  (64)
constexpr uint32_t kColWo = 448;   // dWout^T accumulator    (16)

struct TcSmem {
  uint8_t* X;    // [128][Kp]
  uint8_t* A0;   // [128][64]
  uint8_t* A1;   // [128][64]
  uint8_t* dY;   // [128][16]
  uint8_t* dH1;  // [128][64]
  uint8_t* dH0;  // [128][64]
  uint8_t* W0;   // [64][Kp]
  uint8_t* W1;   // [64][64]
  uint8_t* Wo;   // [16][64]
};

__host__ __device__ inline size_t tc_smem_bytes(int Kp)
{
  return (size_t)128 * Kp * 2 + 4 * 128 * 64 * 2 + 128 * 16 * 2 + 64 * Kp * 2 + 64 * 64 * 2 + 16 * 64 * 2 + 1024;
}

__device__ __forceinline__ TcSmem tc_carve(uint8_t* base, int Kp)
{
  TcSmem s;
  s.X = base;
  s.A0 = s.X + 128 * Kp * 2;
  s.A1 = s.A0 + 128 * 64 * 2;
  s.dY = s.A1 + 128 * 64 * 2;
  s.dH1 = s.dY + 128 * 16 * 2;
  s.dH0 = s.dH1 + 128 * 64 * 2;
  s.W0 = s.dH0 + 128 * 64 * 2;
  s.W1 = s.W0 + 64 * Kp * 2;
  s.Wo = s.W1 + 64 * 64 * 2;
  return s;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// Stores 8 consecutive values (columns c0..c0+7, c0 % 8 == 0) of row r as one 16-byte chunk.
__device__ __forceinline__ void st_chunk(uint8_t* base, int r, int c0, int cols, const float* v)
{
  uint4 q;
  q.x = pack_bf16(v[0], v[1]);
  q.y = pack_bf16(v[2], v[3]);
  q.z = pack_bf16(v[4], v[5]);
  q.w = pack_bf16(v[6], v[7]);
  *reinterpret_cast<uint4*>(base + ptx::cm_off16(r, c0, cols)) = q;
}

struct Unit {
  int x, y;
  bool valid;
};

// Gathers one texel's features into row `row` of sX.  half 0 writes the 4*C0 g0 corner
// features; half 1 the C1 bilinear g1 features, positional encodings, lod and zero pad.
__device__ __forceinline__ void gather_row(const Model& M, const StepRec& s, const Unit& u, int row, int half, int Kp,
                                           uint8_t* sX)
{
  const int lvl = s.level;
  const int C0 = M.C0, C1 = M.C1;
  if (!u.valid) {
    const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int lo = half == 0 ? 0 : 4 * C0, hi = half == 0 ? 4 * C0 : Kp;
    for (int c = lo; c < hi; c += 8) st_chunk(sX, row, c, Kp, z);
    return;
  }
  Gather G;
  gather_geometry(u.x, u.y, s.mip_dim, M.g0.dim[lvl], M.g1.dim[lvl], G);
  float buf[8];
  if (half == 0) {
    const float* p0 = M.g0.p[lvl];
    int f = 0;
    for (int k = 0; k < 4; k++) {
      const int base = G.c0[k] * C0;
      for (int c = 0; c < C0; c += 4) {
        const float4 q = *reinterpret_cast<const float4*>(p0 + base + c);
        float v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
          float val = v[i];
          if (s.noise) val = val + latent_noise(M, s, 0u, (uint32_t)(base + c + i));
          buf[f & 7] = val;
          f++;
        }
        if ((f & 7) == 0) st_chunk(sX, row, f - 8, Kp, buf);
      }
    }
  } else {
    const float* p1 = M.g1.p[lvl];
    float acc[32];
    for (int c = 0; c < C1; c++) acc[c] = 0.0f;
    for (int k = 0; k < 4; k++) {
      const int base = G.c1[k] * C1;
      for (int c = 0; c < C1; c += 2) {
        const float2 q = *reinterpret_cast<const float2*>(p1 + base + c);
        float a = q.x, b = q.y;
        if (s.noise) {
          a = a + latent_noise(M, s, 1u, (uint32_t)(base + c));
          b = b + latent_noise(M, s, 1u, (uint32_t)(base + c + 1));
        }
        acc[c] = __fmaf_rn(G.w1[k], a, acc[c]);
        acc[c + 1] = __fmaf_rn(G.w1[k], b, acc[c + 1]);
      }
    }
    int f = 4 * C0;
    int n = 0;
    auto put = [&](float v) {
      buf[n++] = v;
      if (n == 8) {
        st_chunk(sX, row, f, Kp, buf);
        f += 8;
        n = 0;
      }
    };
    for (int c = 0; c < C1; c++) put(acc[c]);
    for (int i = 0; i < 12; i++) put(pos_enc(u.x, u.y, i));
    put(s.norm_lod);
    while (f < Kp) put(0.0f);
  }
}

// Loads the fp32 master weights into the bf16 canonical tiles (zero padding past F / C).
__device__ void load_weights(const Model& M, const TcSmem& sm, int Kp)
{
  const int F = M.F, C = M.C;
  for (int i = threadIdx.x; i < 64 * (Kp / 8); i += kThreads) {
    const int r = i / (Kp / 8), c0 = (i % (Kp / 8)) * 8;
    float v[8];
    for (int j = 0; j < 8; j++) v[j] = (c0 + j) < F ? M.W[w0_off() + r * F + c0 + j] : 0.0f;
    st_chunk(sm.W0, r, c0, Kp, v);
  }
  for (int i = threadIdx.x; i < 64 * 8; i += kThreads) {
    const int r = i / 8, c0 = (i % 8) * 8;
    float v[8];
    for (int j = 0; j < 8; j++) v[j] = M.W[w1_off(F) + r * 64 + c0 + j];
    st_chunk(sm.W1, r, c0, 64, v);
  }
  for (int i = threadIdx.x; i < 16 * 8; i += kThreads) {
    const int r = i / 8, c0 = (i % 8) * 8;
    float v[8];
    for (int j = 0; j < 8; j++) v[j] = r < C ? M.W[wo_off(F) + r * 64 + c0 + j] : 0.0f;
    st_chunk(sm.Wo, r, c0, 64, v);
  }
}

__device__ __forceinline__ double block_sum_d(double v, double* red)
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

template <int KP>
__global__ void __launch_bounds__(kThreads, 1)
tc_unit_kernel(Model M, const StepRec* __restrict__ steps, int step_idx, TileOut out, int* __restrict__ err)
{
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int fail_s;
  __shared__ double red[kThreads / 32];

  constexpr int Kp = KP;
  const StepRec s = steps[step_idx];
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int row = tid & 127;       // texel row == TMEM lane
  const int half = tid >> 7;       // column half of the epilogues
  const int quad = warp & 3;       // TMEM lane quadrant this warp may access
  const TcSmem sm = tc_carve(smem_raw, Kp);
  const int C = M.C;
  const int F = M.F;

  if (tid == 0) {
    ptx::mbar_init(&bar, 1);
    ptx::fence_mbar_init();
    fail_s = 0;
  }
  if (warp == 0) ptx::tmem_alloc(&tmem_base_s, kTmemCols);
  load_weights(M, sm, Kp);
  ptx::fence_proxy_async();
  ptx::fence_before_sync();
  __syncthreads();
  ptx::fence_after_sync();
  const uint32_t tbase = tmem_base_s;
  const uint32_t lane_addr = tbase + ((uint32_t)(quad * 32) << 16);

  const int ntiles = (s.texels + kTile - 1) / kTile;
  const float inv = -2.0f / ((float)C * (float)s.texels);  // libopenntc.cpp:666
  const uint8_t* target = M.package[s.lod];
  uint32_t phase = 0;
  double loss = 0.0;
  bool first = true;

  // one commit -> bounded wait, uniform across the CTA
  auto wait_mma = [&]() -> bool {
    if (!ptx::mbar_wait(&bar, phase)) atomicExch(&fail_s, 1);
    phase ^= 1u;
    ptx::fence_after_sync();
    __syncthreads();
    return fail_s == 0;
  };
  // every thread's shared-memory stores and TMEM reads done -> one thread may issue MMAs
  auto handoff = [&]() {
    ptx::fence_proxy_async();
    ptx::fence_before_sync();
    __syncthreads();
  };

  constexpr uint32_t I_M128_N64_K = ptx::idesc_bf16(128, 64, false, false);
  constexpr uint32_t I_M128_N16_K = ptx::idesc_bf16(128, 16, false, false);
  constexpr uint32_t I_M128_N64_BMN = ptx::idesc_bf16(128, 64, false, true);
  constexpr uint32_t I_M128_NKP_BMN = ptx::idesc_bf16(128, Kp, false, true);
  constexpr uint32_t I_M64_N16_MN = ptx::idesc_bf16(64, 16, true, true);
  constexpr uint32_t I_M64_N64_MN = ptx::idesc_bf16(64, 64, true, true);
  constexpr uint32_t I_M64_NKP_MN = ptx::idesc_bf16(64, Kp, true, true);
  const uint32_t aX = ptx::smem_addr(sm.X), aA0 = ptx::smem_addr(sm.A0), aA1 = ptx::smem_addr(sm.A1);
  const uint32_t adY = ptx::smem_addr(sm.dY), adH1 = ptx::smem_addr(sm.dH1), adH0 = ptx::smem_addr(sm.dH0);
  const uint32_t aW0 = ptx::smem_addr(sm.W0), aW1 = ptx::smem_addr(sm.W1), aWo = ptx::smem_addr(sm.Wo);
  constexpr uint32_t SX = (Kp / 8) * 128;  // 8-row group stride of a [*][Kp] tile
  constexpr uint32_t S64 = 8 * 128;        // ... of a [*][64] tile
  constexpr uint32_t S16 = 2 * 128;        // ... of a [*][16] tile

  for (int unit = blockIdx.x; unit < ntiles; unit += gridDim.x) {
    // ---------------------------------------------------------------- gather
    Unit u;
    {
      const int b = unit * kTile + row;
      u.valid = b < s.texels;
      u.x = u.y = 0;
      if (u.valid) texel_xy(s, b, u.x, u.y);
    }
    gather_row(M, s, u, row, half, Kp, sm.X);
    handoff();
    if (tid == 0) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < Kp / 16; k++)
        ptx::mma_bf16(tbase + kColH, ptx::desc(aX + k * 256, 128, SX), ptx::desc(aW0 + k * 256, 128, SX), I_M128_N64_K,
                      k > 0);
      ptx::commit(&bar);
    }
    if (!wait_mma()) break;

    // ---------------------------------------------------------------- layer 0 epilogue
    float h0[32], h1[32];
    {
      ptx::ld16(lane_addr + kColH + half * 32, h0);
      ptx::ld16(lane_addr + kColH + half * 32 + 16, h0 + 16);
      ptx::ld_wait();
      float a[8];
#pragma unroll
      for (int c = 0; c < 32; c += 8) {
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = hardgelu(h0[c + j]);
        st_chunk(sm.A0, row, half * 32 + c, 64, a);
      }
    }
    handoff();
    if (tid == 0) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < 4; k++)
        ptx::mma_bf16(tbase + kColH, ptx::desc(aA0 + k * 256, 128, S64), ptx::desc(aW1 + k * 256, 128, S64),
                      I_M128_N64_K, k > 0);
      ptx::commit(&bar);
    }
    if (!wait_mma()) break;

    // ---------------------------------------------------------------- layer 1 epilogue
    {
      ptx::ld16(lane_addr + kColH + half * 32, h1);
      ptx::ld16(lane_addr + kColH + half * 32 + 16, h1 + 16);
      ptx::ld_wait();
      float a[8];
#pragma unroll
      for (int c = 0; c < 32; c += 8) {
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = hardgelu(h1[c + j]);
        st_chunk(sm.A1, row, half * 32 + c, 64, a);
      }
    }
    handoff();
    if (tid == 0) {
      ptx::fence_after_sync();
#pragma unroll
      for (int k = 0; k < 4; k++)
        ptx::mma_bf16(tbase + kColY, ptx::desc(aA1 + k * 256, 128, S64), ptx::desc(aWo + k * 256, 128, S64),
                      I_M128_N16_K, k > 0);
      ptx::commit(&bar);
    }
    if (!wait_mma()) break;

    // ---------------------------------------------------------------- output, residual, dY
    {
      float yv[8], d[8];
      ptx::ld8(lane_addr + kColY + half * 8, yv);
      ptx::ld_wait();
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int c = half * 8 + j;
        d[j] = 0.0f;
        if (u.valid && c < C) {
          const float tgt = (float)target[((size_t)u.y * s.mip_dim + u.x) * C + c] / 255.0f;
          const float r = tgt - yv[j];
          loss += (double)r * (double)r;
          d[j] = inv * r;
        }
      }
      st_chunk(sm.dY, row, half * 8, 16, d);
    }
    handoff();
    if (tid == 0) {
      ptx::fence_after_sync();
      // dA1 = dY Wout: B = Wout viewed [c][h] as MN-major (N = h)
      ptx::mma_bf16(tbase + kColH, ptx::desc(adY, 128, S16), ptx::desc(aWo, S64, 128), I_M128_N64_BMN, 0);
      // dWout^T += A1^T dY : A = A1 (M = h), B = dY (N = c), K = texels
#pragma unroll
      for (int k = 0; k < 8; k++)
        ptx::mma_bf16(tbase + kColWo, ptx::desc(aA1 + k * 2 * S64, S64, 128), ptx::desc(adY + k * 2 * S16, S16, 128),
                      I_M64_N16_MN, (first && k == 0) ? 0u : 1u);
      ptx::commit(&bar);
    }
    if (!wait_mma()) break;

    // ---------------------------------------------------------------- dH1
    {
      float da[32];
      ptx::ld16(lane_addr + kColH + half * 32, da);
      ptx::ld16(lane_addr + kColH + half * 32 + 16, da + 16);
      ptx::ld_wait();
      float g[8];
#pragma unroll
      for (int c = 0; c < 32; c += 8) {
#pragma unroll
        for (int j = 0; j < 8; j++) g[j] = da[c + j] * hardgelu_grad(h1[c + j]);
        st_chunk(sm.dH1, row, half * 32 + c, 64, g);
      }
    }
    handoff();
    if (tid == 0) {
      ptx::fence_after_sync();
      // dA0 = dH1 W1 : B = W1 viewed [i][h] as MN-major (N = h), K = i
#pragma unroll
      for (int k = 0; k < 4; k++)
        ptx::mma_bf16(tbase + kColH, ptx::desc(adH1 + k * 256, 128, S64), ptx::desc(aW1 + k * 2 * S64, S64, 128),
                      I_M128_N64_BMN, k > 0);
      // dW1 += dH1^T A0
#pragma unroll
      for (int k = 0; k < 8; k++)
        ptx::mma_bf16(tbase + kColW1, ptx::desc(adH1 + k * 2 * S64, S64, 128), ptx::desc(aA0 + k * 2 * S64, S64, 128),
                      I_M64_N64_MN, (first && k == 0) ? 0u : 1u);
      ptx::commit(&bar);
    }
    if (!wait_mma()) break;

    // ---------------------------------------------------------------- dH0
    {
      float da[32];
      ptx::ld16(lane_addr + kColH + half * 32, da);
      ptx::ld16(lane_addr + kColH + half * 32 + 16, da + 16);
      ptx::ld_wait();
      float g[8];
#pragma unroll
      for (int c = 0; c < 32; c += 8) {
#pragma unroll
        for (int j = 0; j < 8; j++) g[j] = da[c + j] * hardgelu_grad(h0[c + j]);
        st_chunk(sm.dH0, row, half * 32 + c, 64, g);
      }
    }
    handoff();
    if (tid == 0) {
      ptx::fence_after_sync();
      // dX = dH0 W0 : B = W0 viewed [h][f] as MN-major (N = f), K = h
#pragma unroll
      for (int k = 0; k < 4; k++)
        ptx::mma_bf16(tbase + kColDX, ptx::desc(adH0 + k * 256, 128, S64), ptx::desc(aW0 + k * 2 * SX, SX, 128),
                      I_M128_NKP_BMN, k > 0);
      // dW0 += dH0^T X
#pragma unroll
      for (int k = 0; k < 8; k++)
        ptx::mma_bf16(tbase + kColW0, ptx::desc(adH0 + k * 2 * S64, S64, 128), ptx::desc(aX + k * 2 * SX, SX, 128),
                      I_M64_NKP_MN, (first && k == 0) ? 0u : 1u);
      ptx::commit(&bar);
    }
    if (!wait_mma()) break;
    first = false;

    // ---------------------------------------------------------------- scatter dX
    // TMEM loads are warp-collective, so every lane loads; only valid texels scatter.
    {
      const bool scatter = s.grid_update && u.valid;
      const int lvl = s.level;
      Gather G;
      if (scatter) gather_geometry(u.x, u.y, s.mip_dim, M.g0.dim[lvl], M.g1.dim[lvl], G);
      if (half == 0) {
        const int C0 = M.C0;
        float* g0 = M.g0.g[lvl];
        for (int c = 0; c < 4 * C0; c += 16) {
          float dx[16];
          ptx::ld16(lane_addr + kColDX + c, dx);
          ptx::ld_wait();
          if (scatter) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
              const int f = c + j, k = f / C0, ch = f - k * C0;
              atomicAdd(&g0[G.c0[k] * C0 + ch], dx[j]);
            }
          }
        }
      } else {
        const int C0 = M.C0, C1 = M.C1;
        float* g1 = M.g1.g[lvl];
        float dx[32];
        ptx::ld16(lane_addr + kColDX + 4 * C0, dx);
        ptx::ld16(lane_addr + kColDX + 4 * C0 + 16, dx + 16);
        ptx::ld_wait();
        if (scatter)
          for (int k = 0; k < 4; k++)
            for (int c = 0; c < C1; c++) atomicAdd(&g1[G.c1[k] * C1 + c], G.w1[k] * dx[c]);
      }
    }
    ptx::fence_before_sync();
    __syncthreads();
  }

  // ------------------------------------------------------------------ weight gradients out
  const double ls = block_sum_d(loss, red);
  if (tid == 0) out.loss_partial[blockIdx.x] = ls;
  if (fail_s == 0 && !first) {
    ptx::fence_after_sync();
    float* dst = out.dW_partial + (size_t)blockIdx.x * M.nW;
    const int lane = tid & 31;
    const int h = quad * 16 + lane;  // M=64 accumulators: row = lane of the quadrant's first 16
    // dW0 [64][F]: columns split between the two halves in 8-column steps
    for (int c = half * 8; c < Kp; c += 16) {
      float v[8];
      ptx::ld8(lane_addr + kColW0 + c, v);
      ptx::ld_wait();
      if (lane < 16)
        for (int j = 0; j < 8; j++)
          if (c + j < F) dst[w0_off() + h * F + c + j] = v[j];
    }
    {
      float v[32];
      ptx::ld16(lane_addr + kColW1 + half * 32, v);
      ptx::ld16(lane_addr + kColW1 + half * 32 + 16, v + 16);
      ptx::ld_wait();
      // accumulator row = i (dH1 column), column = h (A0 column): dW1[i][h]
      if (lane < 16)
        for (int j = 0; j < 32; j++) dst[w1_off(F) + h * 64 + half * 32 + j] = v[j];
    }
    {
      float v[8];
      ptx::ld8(lane_addr + kColWo + half * 8, v);
      ptx::ld_wait();
      // accumulator row = h, column = c: dWout[c][h]
      if (lane < 16)
        for (int j = 0; j < 8; j++) dst[wo_off(F) + (half * 8 + j) * 64 + h] = v[j];
    }
  }
  if (fail_s != 0 && tid == 0) atomicExch(err, 1);
  ptx::fence_before_sync();
  __syncthreads();
  if (warp == 0) ptx::tmem_dealloc(tbase, kTmemCols);
}

template <int KP>
cudaError_t launch_kp(const Model& M, const StepRec* d_steps, int step_idx, int grid, TileOut out, int* d_error,
                      cudaStream_t stream)
{
  const size_t smem = tc_smem_bytes(KP);
  // at least 150 KB so one CTA owns an SM (and its 512 TMEM columns)
  const size_t smem_req = smem < 150 * 1024 ? 150 * 1024 : smem;
  cudaError_t e = cudaFuncSetAttribute(tc_unit_kernel<KP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_req);
  if (e != cudaSuccess) return e;
  tc_unit_kernel<KP><<<grid, kThreads, smem_req, stream>>>(M, d_steps, step_idx, out, d_error);
  return cudaGetLastError();
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
                            cudaStream_t stream)
{
  switch (M.Fp) {
    case 64: return launch_kp<64>(M, d_steps, step_idx, grid, out, d_error, stream);
    case 80: return launch_kp<80>(M, d_steps, step_idx, grid, out, d_error, stream);
    case 96: return launch_kp<96>(M, d_steps, step_idx, grid, out, d_error, stream);
    default: return cudaErrorNotSupported;
  }
}

}  // namespace ontc
