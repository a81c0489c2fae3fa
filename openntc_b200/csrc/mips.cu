// Manifest ingest kernels (upstream ntc_kernel.cu:533-686, libopenntc.cpp:1296-1362): the mip
// chain fused with packaging -- mip 0's channel selection and every separable Lanczos-3 2x
// reduction (both passes in one kernel through a shared-memory tile) write a source's mip and
// its channels of that mip's interleaved target package -- and the two-kernel reduction through
// an fp32 intermediate that the caller-buffer entry points use.
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

// ---- the ingest chain fused with packaging -------------------------------------------------
// Mip 0 of one source: its channels picked from the RGBA image (prepare) into the source's mip
// and, at channels [pkg_off, pkg_off + count) of every texel, into the target package.
__global__ void prepare_package_kernel(const uint8_t* __restrict__ rgba, int dim, int4 cmap, int count,
                                       uint8_t* __restrict__ out, uint8_t* __restrict__ pkg, int C, int pkg_off)
{
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dim || y >= dim) return;
  const size_t t = (size_t)y * dim + x;
  const int c[4] = {cmap.x, cmap.y, cmap.z, cmap.w};
  for (int i = 0; i < count; i++) {
    const uint8_t v = rgba[t * 4 + c[i]];
    out[t * count + i] = v;
    pkg[t * C + pkg_off + i] = v;
  }
}

// One 2x Lanczos-3 reduction of a source mip, both passes in one kernel: a CTA owns a
// kTileO x kTileO block of output texels; the x pass fills shared memory with the fp32 rows
// the block's y taps reach (2 kTileO + 10 of them), the y pass reads them back.  Each value is
// formed by exactly the operations of lanczos_x_kernel / lanczos_y_kernel, in their order, so
// the mip is bit-identical to the two-kernel reduction.  The output is written to the source's
// next mip and, at channels [pkg_off, pkg_off + c), into that mip's target package.
constexpr int kTileO = 32;
constexpr int kTileRows = 2 * kTileO + 10;

template <int CH>
__global__ void __launch_bounds__(256) lanczos_down_package_kernel(const uint8_t* __restrict__ src, int dim, int c,
                                                                   uint8_t* __restrict__ dst, uint8_t* __restrict__ pkg,
                                                                   int C, int pkg_off)
{
  __shared__ float w[12];
  __shared__ float unit[256];  // v / 255 for every byte v, divided once (correctly rounded, as per tap)
  __shared__ float xs[kTileRows][kTileO][CH];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;  // 32 x 8 threads
  if (tid < 12) w[tid] = lanczos_tap(tid - 6);
  unit[tid] = __fdiv_rn((float)tid, 255.0f);
  __syncthreads();
  const int odim = dim >> 1;
  const int ox0 = blockIdx.x * kTileO, oy0 = blockIdx.y * kTileO;
  const int r0 = 2 * oy0 - 5;  // input row of xs[0]: the first y tap of output row oy0
  // x pass: rows r0 .. r0 + kTileRows - 1 (those inside the image), output columns of the block
  for (int k = tid; k < kTileRows * kTileO; k += 256) {
    const int r = k / kTileO, ox = ox0 + k % kTileO, y = r0 + r;
    if (y < 0 || y >= dim || ox >= odim) continue;
    const int center = 2 * ox + 1;
    float total[CH];
    for (int j = 0; j < CH; j++) total[j] = 0.0f;
    float tw = 0.0f;
    const uint8_t* row = src + (size_t)y * dim * c;
    for (int i = -6; i < 6; i++) {
      const int sx = center + i;
      if (sx < 0 || sx >= dim) continue;
      const float wt = w[i + 6];
      for (int j = 0; j < c && j < CH; j++) total[j] = __fmaf_rn(unit[row[sx * c + j]], wt, total[j]);
      tw = __fadd_rn(tw, wt);
    }
    for (int j = 0; j < c && j < CH; j++) xs[r][k % kTileO][j] = __fdiv_rn(total[j], tw);
  }
  __syncthreads();
  // y pass: each thread takes every 8th output row of its column
  const int ox = ox0 + (int)threadIdx.x;
  if (ox >= odim) return;
  for (int oy = oy0 + (int)threadIdx.y; oy < oy0 + kTileO && oy < odim; oy += 8) {
    const int center = 2 * oy + 1;
    float total[CH];
    for (int j = 0; j < CH; j++) total[j] = 0.0f;
    float tw = 0.0f;
    for (int i = -6; i < 6; i++) {
      const int sy = center + i;
      if (sy < 0 || sy >= dim) continue;
      const float wt = w[i + 6];
      const float* t = xs[sy - r0][threadIdx.x];
      for (int j = 0; j < c && j < CH; j++) total[j] = __fmaf_rn(t[j], wt, total[j]);
      tw = __fadd_rn(tw, wt);
    }
    const size_t o = (size_t)oy * odim + ox;
    for (int j = 0; j < c && j < CH; j++) {
      const float v = __fdiv_rn(total[j], tw);
      const uint8_t u = (uint8_t)fminf(255.0f, fmaxf(0.0f, __fmul_rn(v, 255.0f)));
      dst[o * c + j] = u;
      pkg[o * C + pkg_off + j] = u;
    }
  }
}

__global__ void weights_kernel(float* out)
{
  if (threadIdx.x < 12) out[threadIdx.x] = lanczos_tap((int)threadIdx.x - 6);
}

}  // namespace

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

cudaError_t launch_prepare_package(const uint8_t* rgba, int dim, const int* cmap, int count, uint8_t* out, uint8_t* pkg,
                                   int C, int pkg_off, cudaStream_t stream)
{
  dim3 b(32, 8), g((dim + 31) / 32, (dim + 7) / 8);
  prepare_package_kernel<<<g, b, 0, stream>>>(rgba, dim, make_int4(cmap[0], cmap[1], cmap[2], cmap[3]), count, out, pkg,
                                              C, pkg_off);
  return cudaGetLastError();
}

cudaError_t launch_lanczos_down_package(const uint8_t* src, int dim, int c, uint8_t* dst, uint8_t* pkg, int C,
                                        int pkg_off, cudaStream_t stream)
{
  if (c < 1 || c > 4 || dim < 2 || pkg_off < 0 || pkg_off + c > C) return cudaErrorInvalidValue;
  const int odim = dim / 2;
  dim3 b(32, 8), g((odim + kTileO - 1) / kTileO, (odim + kTileO - 1) / kTileO);
  lanczos_down_package_kernel<4><<<g, b, 0, stream>>>(src, dim, c, dst, pkg, C, pkg_off);
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
