// Scoring the shipping int8 decode against the training targets: the texel centres of the
// mip chain as decode samples, and the squared error of the decoded channels.  Used by
// ontc_eval_decoded (every texel) and by the calibration search (a fixed subsample).
//
// The mip chain is addressed as one sequence of texels (mip 0 first, row-major inside a mip);
// sample j is texel (j * stride + offset) mod total, with stride coprime to total, so a
// subsample visits distinct texels spread over every mip in proportion to its size, the same
// weighting as upstream's Eval (libopenntc.cpp:972-1053).
#include <algorithm>
#include <cstdint>

#include "kernels.h"

namespace ontc {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void locate(const TexelMap& m, int64_t j, int& mip, int& x, int& y)
{
  const int64_t total = m.start[m.mips];
  const int64_t t = (int64_t)(((uint64_t)j * (uint64_t)m.stride + (uint64_t)m.offset) % (uint64_t)total);
  mip = 0;
#pragma unroll 1
  while (mip + 1 < m.mips && t >= m.start[mip + 1]) mip++;
  const int64_t r = t - m.start[mip];
  y = (int)(r / m.dim[mip]);
  x = (int)(r - (int64_t)y * m.dim[mip]);
}

__global__ void texel_samples_kernel(const __grid_constant__ TexelMap m, int64_t j0, int64_t n, float2* uv,
                                     int32_t* lod)
{
  for (int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x; j < n; j += (int64_t)gridDim.x * kThreads) {
    int mip, x, y;
    locate(m, j0 + j, mip, x, y);
    const float d = (float)m.dim[mip];
    uv[j] = make_float2(__fdiv_rn(__fadd_rn((float)x, 0.5f), d), __fdiv_rn(__fadd_rn((float)y, 0.5f), d));
    lod[j] = mip;
  }
}

// Per block: sum over its samples and channels of (target / 255 - decoded)^2, the residual in
// fp32 and the sum in fp64 as the eval kernel forms them; block sums in a fixed order.
__global__ void decoded_sq_err_kernel(const __grid_constant__ TexelMap m, int64_t j0, int64_t n,
                                      const float* __restrict__ out, double* partial)
{
  __shared__ double red[kThreads / 32];
  double acc = 0.0;
  for (int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x; j < n; j += (int64_t)gridDim.x * kThreads) {
    int mip, x, y;
    locate(m, j0 + j, mip, x, y);
    const uint8_t* t = m.target[mip] + ((int64_t)y * m.dim[mip] + x) * m.C;
    const float* o = out + j * m.C;
    for (int c = 0; c < m.C; c++) {
      const float r = __fsub_rn(__fdiv_rn((float)t[c], 255.0f), o[c]);
      acc += (double)r * (double)r;
    }
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; w++) s += red[w];
    partial[blockIdx.x] = s;
  }
}

}  // namespace

cudaError_t launch_texel_samples(const TexelMap& m, int64_t j0, int64_t n, float* uv, int32_t* lod,
                                 cudaStream_t stream)
{
  if (n <= 0) return cudaSuccess;
  const int blocks = (int)std::min<int64_t>((n + kThreads - 1) / kThreads, 4096);
  texel_samples_kernel<<<blocks, kThreads, 0, stream>>>(m, j0, n, reinterpret_cast<float2*>(uv), lod);
  return cudaGetLastError();
}

cudaError_t launch_decoded_sq_err(const TexelMap& m, int64_t j0, int64_t n, const float* out, double* partial,
                                  int blocks, cudaStream_t stream)
{
  if (n <= 0 || blocks <= 0) return cudaSuccess;
  decoded_sq_err_kernel<<<blocks, kThreads, 0, stream>>>(m, j0, n, out, partial);
  return cudaGetLastError();
}

}  // namespace ontc
