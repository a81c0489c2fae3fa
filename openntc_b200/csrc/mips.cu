// Manifest ingest kernels: channel selection, the separable Lanczos-3 2x mip reduction and
// the interleaved target package (upstream ntc_kernel.cu:533-686, libopenntc.cpp:1296-1362).
//
// The reduction must reproduce upstream's u8 mips exactly (the training targets and the
// .ntc size/PSNR depend on them), so its arithmetic follows filter_lanczos op for op:
// 12 taps at texel_center + i, i in [-6, 6), weight lanczos((0.5 + i) / 2, 3); taps
// outside the image are skipped and the weight sum renormalises; the x pass reads u8/255
// and writes fp32, the y pass reads fp32 and truncates clamp(255 * v) to u8.
// The tap weights are evaluated once per launch on the device, with upstream's expression
// (a double-precision pi product narrowed to float, then CUDA's sinf), into shared memory.
#include "common.cuh"
#include "kernels.h"

namespace ontc {

namespace {

constexpr double kPi = 3.14159265359;  // the constant upstream's filter uses (ntc_kernel.cu:11)

__device__ float sinc_f(float x)
{
  if (fabsf(x) < 1e-8f) return 1.0f;
  return __fdiv_rn(sinf(x), x);
}

__device__ float lanczos_tap(int i)
{
  const float x = (0.5f + (float)i) * 0.5f;
  const float a = 3.0f;
  const float s0 = sinc_f((float)(kPi * (double)x));
  const float s1 = sinc_f((float)(kPi * (double)x / (double)a));
  return __fmul_rn(s0, s1);
}

__global__ void prepare_kernel(const uint8_t* __restrict__ rgba, int dim, int4 cmap, int count, uint8_t* __restrict__ out)
{
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dim || y >= dim) return;
  const size_t t = (size_t)y * dim + x;
  const int c[4] = {cmap.x, cmap.y, cmap.z, cmap.w};
  for (int i = 0; i < count; i++) out[t * count + i] = rgba[t * 4 + c[i]];
}

// x pass: src u8 [dim][dim][c] -> tmp f32 [dim][dim/2][c]
template <int CH>
__global__ void lanczos_x_kernel(const uint8_t* __restrict__ src, int dim, int c, float* __restrict__ tmp)
{
  __shared__ float w[12];
  if (threadIdx.y == 0 && threadIdx.x < 12) w[threadIdx.x] = lanczos_tap((int)threadIdx.x - 6);
  __syncthreads();
  const int ox = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int odim = dim >> 1;
  if (ox >= odim || y >= dim) return;
  const int center = 2 * ox + 1;
  float total[CH];
  for (int j = 0; j < CH; j++) total[j] = 0.0f;
  float tw = 0.0f;
  const uint8_t* row = src + (size_t)y * dim * c;
  for (int i = -6; i < 6; i++) {
    const int sx = center + i;
    if (sx < 0 || sx >= dim) continue;
    const float wt = w[i + 6];
    for (int j = 0; j < c && j < CH; j++) total[j] = __fmaf_rn(__fdiv_rn((float)row[sx * c + j], 255.0f), wt, total[j]);
    tw = __fadd_rn(tw, wt);
  }
  float* o = tmp + ((size_t)y * odim + ox) * c;
  for (int j = 0; j < c && j < CH; j++) o[j] = __fdiv_rn(total[j], tw);
}

// y pass: tmp f32 [dim][dim/2][c] -> dst u8 [dim/2][dim/2][c]
template <int CH>
__global__ void lanczos_y_kernel(const float* __restrict__ tmp, int dim, int c, uint8_t* __restrict__ dst)
{
  __shared__ float w[12];
  if (threadIdx.y == 0 && threadIdx.x < 12) w[threadIdx.x] = lanczos_tap((int)threadIdx.x - 6);
  __syncthreads();
  const int odim = dim >> 1;
  const int ox = blockIdx.x * blockDim.x + threadIdx.x;
  const int oy = blockIdx.y * blockDim.y + threadIdx.y;
  if (ox >= odim || oy >= odim) return;
  const int center = 2 * oy + 1;
  float total[CH];
  for (int j = 0; j < CH; j++) total[j] = 0.0f;
  float tw = 0.0f;
  for (int i = -6; i < 6; i++) {
    const int sy = center + i;
    if (sy < 0 || sy >= dim) continue;
    const float wt = w[i + 6];
    const float* t = tmp + ((size_t)sy * odim + ox) * c;
    for (int j = 0; j < c && j < CH; j++) total[j] = __fmaf_rn(t[j], wt, total[j]);
    tw = __fadd_rn(tw, wt);
  }
  uint8_t* o = dst + ((size_t)oy * odim + ox) * c;
  for (int j = 0; j < c && j < CH; j++) {
    const float v = __fdiv_rn(total[j], tw);
    const float u = fminf(255.0f, fmaxf(0.0f, __fmul_rn(v, 255.0f)));
    o[j] = (uint8_t)u;
  }
}

__global__ void package_kernel(PackageSpec spec, int dim, int C, uint8_t* __restrict__ out)
{
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dim || y >= dim) return;
  const size_t t = (size_t)y * dim + x;
  for (int i = 0; i < C; i++) {
    const int s = spec.feat_src[i];
    out[t * C + i] = spec.src[s][t * spec.src_channels[s] + spec.feat_chan[i]];
  }
}

__global__ void weights_kernel(float* out)
{
  if (threadIdx.x < 12) out[threadIdx.x] = lanczos_tap((int)threadIdx.x - 6);
}

}  // namespace

cudaError_t launch_prepare(const uint8_t* rgba, int dim, const int* cmap, int count, uint8_t* out, cudaStream_t stream)
{
  dim3 b(32, 8), g((dim + 31) / 32, (dim + 7) / 8);
  prepare_kernel<<<g, b, 0, stream>>>(rgba, dim, make_int4(cmap[0], cmap[1], cmap[2], cmap[3]), count, out);
  return cudaGetLastError();
}

cudaError_t launch_lanczos_down(const uint8_t* src, int dim, int c, float* tmp, uint8_t* dst, cudaStream_t stream)
{
  if (c < 1 || c > 4 || dim < 2) return cudaErrorInvalidValue;
  const int odim = dim / 2;
  dim3 b(32, 8);
  dim3 gx((odim + 31) / 32, (dim + 7) / 8);
  dim3 gy((odim + 31) / 32, (odim + 7) / 8);
  lanczos_x_kernel<4><<<gx, b, 0, stream>>>(src, dim, c, tmp);
  lanczos_y_kernel<4><<<gy, b, 0, stream>>>(tmp, dim, c, dst);
  return cudaGetLastError();
}

cudaError_t launch_package(const PackageSpec& spec, int dim, int C, uint8_t* out, cudaStream_t stream)
{
  dim3 b(32, 8), g((dim + 31) / 32, (dim + 7) / 8);
  package_kernel<<<g, b, 0, stream>>>(spec, dim, C, out);
  return cudaGetLastError();
}

cudaError_t lanczos_weights(float* host12)
{
  float* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 12 * sizeof(float));
  if (e != cudaSuccess) return e;
  weights_kernel<<<1, 32>>>(d);
  e = cudaMemcpy(host12, d, 12 * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e;
}

}  // namespace ontc
