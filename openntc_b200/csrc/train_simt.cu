// FP32 SIMT tile kernel: one CTA owns a 128-texel work unit at a time and runs the whole
// per-texel pipeline of upstream's training step in shared memory:
//
//   gather (draw_features, ntc_kernel.cu:75-177) -> 3-layer MLP forward
//   (libopenntc.cpp:651-655) -> residual and loss (:659-668) -> backward with the
//   hidden activations kept in shared memory (:672-693) -> scatter-add of the feature
//   gradient into the latent gradient buffers (ntc_kernel.cu:280-341).
//
// It is the plain-FP32 comparator of the BF16 tcgen05 path (all GEMMs are fp32 FMA on
// the CUDA cores) and the forward used by Eval and Calibrate (modes below).
// The grid is persistent (<= one CTA per SM); decoder-weight gradients are accumulated in
// registers across a CTA's units and written once per CTA to a partial-sum slot, so their
// reduction order is fixed and the result is run-to-run deterministic.
#include "common.cuh"
#include "kernels.h"

namespace ontc {

namespace {

constexpr int kThreads = 256;
constexpr int S = kTile + 1;  // row stride of the [rows][texel] buffers (bank-conflict padding)

struct Smem {
  float* W0;  // [64][F]
  float* W1;  // [64][64]
  float* Wo;  // [16][64]
  float* X;   // [F][128]   features, later the feature gradient
  float* H0;  // [64][128]  layer-0 pre-activation
  float* H1;  // [64][128]  layer-1 pre-activation, later dL/dH0
  float* D;   // [16][128]  dL/dY
  float* G;   // [64][128]  dL/dH1
  int* tex;   // [128]      x | y << 16, -1 for padding texels
};

__device__ __forceinline__ Smem carve(float* base, int F)
{
  Smem s;
  s.W0 = base;
  s.W1 = s.W0 + kHidden * F;
  s.Wo = s.W1 + kHidden * kHidden;
  s.X = s.Wo + kOutPad * kHidden;
  s.H0 = s.X + F * S;
  s.H1 = s.H0 + kHidden * S;
  s.D = s.H1 + kHidden * S;
  s.G = s.D + kOutPad * S;
  s.tex = (int*)(s.G + kHidden * S);
  return s;
}

// Writes the feature vectors of the unit's 128 texels into X[f][t].
// Threads 0..127 write the 4*C0 g0 corner features of texel t, threads 128..255 the C1
// bilinear g1 features, the 12 positional features, the lod feature and the zero pad.
__device__ void gather_unit(const Model& M, const StepRec& s, const Smem& sm, bool with_noise)
{
  const int tid = threadIdx.x;
  const int t = tid & (kTile - 1);
  const int code = sm.tex[t];
  const int F = M.F;
  if (code < 0) {
    for (int f = (tid >> 7); f < F; f += 2) sm.X[f * S + t] = 0.0f;
    return;
  }
  const int x = code & 0xFFFF, y = code >> 16;
  const int lvl = s.level;
  const int d0 = M.g0.dim[lvl], d1 = M.g1.dim[lvl];
  Gather G;
  gather_geometry(x, y, s.mip_dim, d0, d1, G);
  if (tid < kTile) {
    const int C0 = M.C0;
    const float* p0 = M.g0.p[lvl];
    for (int k = 0; k < 4; k++) {
      const int base = G.c0[k] * C0;
      for (int c = 0; c < C0; c++) {
        float v = p0[base + c];
        if (with_noise) v = v + latent_noise(M, s, 0u, (uint32_t)(base + c));
        sm.X[(k * C0 + c) * S + t] = v;
      }
    }
  } else {
    const int C0 = M.C0, C1 = M.C1;
    const float* p1 = M.g1.p[lvl];
    for (int c = 0; c < C1; c++) {
      float acc = 0.0f;
      for (int k = 0; k < 4; k++) {
        const int e = G.c1[k] * C1 + c;
        float v = p1[e];
        if (with_noise) v = v + latent_noise(M, s, 1u, (uint32_t)e);
        acc = __fmaf_rn(G.w1[k], v, acc);
      }
      sm.X[(4 * C0 + c) * S + t] = acc;
    }
    int f = 4 * C0 + C1;
    for (int i = 0; i < 12; i++, f++) sm.X[f * S + t] = pos_enc(x, y, i);
    sm.X[f * S + t] = s.norm_lod;
    for (f++; f < F; f++) sm.X[f * S + t] = 0.0f;
  }
}

// acc[i][j] += sum_k A(m0+i, k) * B(k, n0+j)
template <int TM, int TN, class FA, class FB>
__device__ __forceinline__ void mma_loop(float (&acc)[TM][TN], int K, FA a, FB b)
{
  for (int k = 0; k < K; k++) {
    float av[TM], bv[TN];
#pragma unroll
    for (int i = 0; i < TM; i++) av[i] = a(i, k);
#pragma unroll
    for (int j = 0; j < TN; j++) bv[j] = b(k, j);
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
      for (int j = 0; j < TN; j++) acc[i][j] = __fmaf_rn(av[i], bv[j], acc[i][j]);
  }
}

template <int TM, int TN>
__device__ __forceinline__ void zero(float (&acc)[TM][TN])
{
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++) acc[i][j] = 0.0f;
}

__device__ __forceinline__ float block_max(float v, float* red)
{
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = 0.0f;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (kThreads / 32) ? red[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) r = fmaxf(r, __shfl_xor_sync(0xffffffffu, r, o));
  }
  __syncthreads();
  return r;
}

__device__ __forceinline__ double block_sum(double v, double* red)
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

// MODE: kTrain (forward + backward + scatter), kEval (forward + squared error),
// kCalib (forward to layer 1, running max |activation| of layers 0 and 1).
//
// Thread (ty, tx) = (tid / 16, tid % 16).  Texel columns are interleaved (t = tx + 16*j) and
// row-major buffers are padded to stride S, so every shared-memory operand read below is
// either a broadcast or hits 16 distinct banks.
template <int MODE>
__global__ void __launch_bounds__(kThreads, 1)
simt_unit_kernel(Model M, const StepRec* __restrict__ steps, int step_idx, TileOut out)
{
  extern __shared__ __align__(16) float smem_f[];
  __shared__ double red_d[kThreads / 32];
  __shared__ float red_f[kThreads / 32];
  const StepRec s = steps[step_idx];
  const int F = M.F, C = M.C;
  const Smem sm = carve(smem_f, F);
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;

  for (int i = tid; i < kHidden * F; i += kThreads) sm.W0[i] = M.W[w0_off() + i];
  for (int i = tid; i < kHidden * kHidden; i += kThreads) sm.W1[i] = M.W[w1_off(F) + i];
  for (int i = tid; i < kOutPad * kHidden; i += kThreads) sm.Wo[i] = (i / kHidden) < C ? M.W[wo_off(F) + i] : 0.0f;

  // persistent per-thread decoder-gradient accumulators
  float gWo[1][4];  // dWout[ty][tx + 16*j]
  float gW1[4][4];  // dW1[ty*4 + i][tx + 16*j]
  float gW0[4][6];  // dW0[ty*4 + i][tx + 16*j]
  zero(gWo);
  zero(gW1);
  zero(gW0);
  double loss = 0.0;
  float mx0 = 0.0f, mx1 = 0.0f;

  const int ntiles = (s.texels + kTile - 1) / kTile;
  const float inv = -2.0f / ((float)C * (float)s.texels);  // libopenntc.cpp:666
  const uint8_t* target = M.package[s.lod];

  for (int unit = blockIdx.x; unit < ntiles; unit += gridDim.x) {
    __syncthreads();
    if (tid < kTile) {
      const int b = unit * kTile + tid;
      int code = -1;
      if (b < s.texels) {
        int x, y;
        texel_xy(s, b, x, y);
        code = x | (y << 16);
      }
      sm.tex[tid] = code;
    }
    __syncthreads();
    gather_unit(M, s, sm, s.noise != 0);
    __syncthreads();

    // ---- layer 0: H0[h][t] = sum_f W0[h][f] X[f][t]
    {
      float acc[4][8];
      zero(acc);
      mma_loop<4, 8>(acc, F, [&](int i, int k) { return sm.W0[(ty * 4 + i) * F + k]; },
                     [&](int k, int j) { return sm.X[k * S + tx + 16 * j]; });
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
          sm.H0[(ty * 4 + i) * S + tx + 16 * j] = acc[i][j];
          if (MODE == kCalib && sm.tex[tx + 16 * j] >= 0) mx0 = fmaxf(mx0, fabsf(hardgelu(acc[i][j])));
        }
    }
    __syncthreads();
    // ---- layer 1: H1[i][t] = sum_h W1[i][h] hg(H0[h][t])
    {
      float acc[4][8];
      zero(acc);
      mma_loop<4, 8>(acc, kHidden, [&](int i, int k) { return sm.W1[(ty * 4 + i) * kHidden + k]; },
                     [&](int k, int j) { return hardgelu(sm.H0[k * S + tx + 16 * j]); });
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
          sm.H1[(ty * 4 + i) * S + tx + 16 * j] = acc[i][j];
          if (MODE == kCalib && sm.tex[tx + 16 * j] >= 0) mx1 = fmaxf(mx1, fabsf(hardgelu(acc[i][j])));
        }
    }
    __syncthreads();
    if (MODE == kCalib) continue;

    // ---- output layer + residual: row c = ty, texels tx + 16*j
    {
      float acc[1][8];
      zero(acc);
      mma_loop<1, 8>(acc, kHidden, [&](int, int k) { return sm.Wo[ty * kHidden + k]; },
                     [&](int k, int j) { return hardgelu(sm.H1[k * S + tx + 16 * j]); });
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int t = tx + 16 * j;
        const int code = sm.tex[t];
        float d = 0.0f;
        if (ty < C && code >= 0) {
          const int x = code & 0xFFFF, y = code >> 16;
          const float tgt = (float)target[((size_t)y * s.mip_dim + x) * C + ty] / 255.0f;
          const float r = tgt - acc[0][j];
          loss += (double)r * (double)r;
          d = inv * r;
        }
        sm.D[ty * S + t] = d;
      }
    }
    if (MODE == kEval) continue;
    __syncthreads();

    // ---- dWout[c][h] += sum_t D[c][t] hg(H1[h][t]);  dH1 = (Wout^T D) * hg'(H1) -> G
    {
      mma_loop<1, 4>(gWo, kTile, [&](int, int k) { return sm.D[ty * S + k]; },
                     [&](int k, int j) { return hardgelu(sm.H1[(tx + 16 * j) * S + k]); });
      float acc[4][8];
      zero(acc);
      mma_loop<4, 8>(acc, kOutPad, [&](int i, int k) { return sm.Wo[k * kHidden + ty * 4 + i]; },
                     [&](int k, int j) { return sm.D[k * S + tx + 16 * j]; });
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int h = ty * 4 + i, t = tx + 16 * j;
          sm.G[h * S + t] = acc[i][j] * hardgelu_grad(sm.H1[h * S + t]);
        }
    }
    __syncthreads();
    // ---- dW1[i][j] += sum_t dH1[i][t] hg(H0[j][t]);  dH0 = (W1^T dH1) * hg'(H0) -> H1 buffer
    {
      mma_loop<4, 4>(gW1, kTile, [&](int i, int k) { return sm.G[(ty * 4 + i) * S + k]; },
                     [&](int k, int j) { return hardgelu(sm.H0[(tx + 16 * j) * S + k]); });
      float acc[4][8];
      zero(acc);
      mma_loop<4, 8>(acc, kHidden, [&](int i, int k) { return sm.W1[k * kHidden + ty * 4 + i]; },
                     [&](int k, int j) { return sm.G[k * S + tx + 16 * j]; });
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int h = ty * 4 + i, t = tx + 16 * j;
          sm.H1[h * S + t] = acc[i][j] * hardgelu_grad(sm.H0[h * S + t]);
        }
    }
    __syncthreads();
    // ---- dW0[h][f] += sum_t dH0[h][t] X[f][t]
    mma_loop<4, 6>(gW0, kTile, [&](int i, int k) { return sm.H1[(ty * 4 + i) * S + k]; },
                   [&](int k, int j) {
                     const int f = tx + 16 * j;
                     return f < F ? sm.X[f * S + k] : 0.0f;
                   });
    // ---- dX[f][t] = sum_h W0[h][f] dH0[h][t]   (rows f = ty + 16*i, texels tx + 16*j)
    {
      float acc[6][8];
      zero(acc);
      mma_loop<6, 8>(acc, kHidden,
                     [&](int i, int k) {
                       const int f = ty + 16 * i;
                       return f < F ? sm.W0[k * F + f] : 0.0f;
                     },
                     [&](int k, int j) { return sm.H1[k * S + tx + 16 * j]; });
      __syncthreads();  // every thread is done reading X
#pragma unroll
      for (int i = 0; i < 6; i++) {
        const int f = ty + 16 * i;
        if (f < F)
#pragma unroll
          for (int j = 0; j < 8; j++) sm.X[f * S + tx + 16 * j] = acc[i][j];
      }
    }
    __syncthreads();
    // ---- scatter dX into the latent gradients (adjoint of the gather)
    if (s.grid_update) {
      const int t = tid & (kTile - 1);
      const int code = sm.tex[t];
      if (code >= 0) {
        const int x = code & 0xFFFF, y = code >> 16;
        const int lvl = s.level;
        Gather G;
        gather_geometry(x, y, s.mip_dim, M.g0.dim[lvl], M.g1.dim[lvl], G);
        if (tid < kTile) {
          float* g0 = M.g0.g[lvl];
          for (int k = 0; k < 4; k++)
            for (int c = 0; c < M.C0; c++) atomicAdd(&g0[G.c0[k] * M.C0 + c], sm.X[(k * M.C0 + c) * S + t]);
        } else {
          float* g1 = M.g1.g[lvl];
          for (int k = 0; k < 4; k++)
            for (int c = 0; c < M.C1; c++)
              atomicAdd(&g1[G.c1[k] * M.C1 + c], G.w1[k] * sm.X[(4 * M.C0 + c) * S + t]);
        }
      }
    }
  }

  if (MODE == kCalib) {
    const float m0 = block_max(mx0, red_f);
    const float m1 = block_max(mx1, red_f);
    if (tid == 0) {
      atomicMax((int*)&out.calib_max[0], __float_as_int(m0));
      atomicMax((int*)&out.calib_max[1], __float_as_int(m1));
    }
    return;
  }
  const double ls = block_sum(loss, red_d);
  if (tid == 0) out.loss_partial[blockIdx.x] = ls;
  if (MODE == kEval) return;
  float* dst = out.dW_partial + (size_t)blockIdx.x * M.nW;
#pragma unroll
  for (int j = 0; j < 4; j++) dst[wo_off(F) + ty * kHidden + tx + 16 * j] = gWo[0][j];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) dst[w1_off(F) + (ty * 4 + i) * kHidden + tx + 16 * j] = gW1[i][j];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 6; j++) {
      const int f = tx + 16 * j;
      if (f < F) dst[w0_off() + (ty * 4 + i) * F + f] = gW0[i][j];
    }
}

}  // namespace

size_t simt_smem_bytes(int F)
{
  return sizeof(float) * ((size_t)kHidden * F + kHidden * kHidden + kOutPad * kHidden + (size_t)F * S +
                          3 * kHidden * S + kOutPad * S) +
         sizeof(int) * kTile;
}

cudaError_t launch_simt_units(int mode, const Model& M, const StepRec* d_steps, int step_idx, int grid, TileOut out,
                              cudaStream_t stream)
{
  const size_t smem = simt_smem_bytes(M.F);
  cudaError_t e = cudaSuccess;
  switch (mode) {
    case kTrain:
      e = cudaFuncSetAttribute(simt_unit_kernel<kTrain>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) simt_unit_kernel<kTrain><<<grid, kThreads, smem, stream>>>(M, d_steps, step_idx, out);
      break;
    case kEval:
      e = cudaFuncSetAttribute(simt_unit_kernel<kEval>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) simt_unit_kernel<kEval><<<grid, kThreads, smem, stream>>>(M, d_steps, step_idx, out);
      break;
    default:
      e = cudaFuncSetAttribute(simt_unit_kernel<kCalib>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) simt_unit_kernel<kCalib><<<grid, kThreads, smem, stream>>>(M, d_steps, step_idx, out);
      break;
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

}  // namespace ontc
