// Optimiser and latent-quantisation kernels.
//
//  * adam_step_kernel: one launch per training step.  CTAs [0, nDec) reduce the per-CTA
//    decoder-gradient partials in a fixed order and apply Adam to W0/W1/Wout
//    (libopenntc.cpp:722-754); the remaining CTAs stream the step's latent level once,
//    applying Adam + clamp to [-1, 1-delta] and zeroing the gradient in the same pass
//    (libopenntc.cpp:755-790 runs these as three kernels plus a memset, :695-696).
//    HBM-bound: 16 B read + 16 B written per latent.
//  * quantize_grid / quantize_pack: upstream's lock-step snap and final code packing
//    (ntc_kernel.cu:448-507), integer-exact.
#include "common.cuh"
#include "kernels.h"

namespace ontc {

namespace {

constexpr float kBeta1 = 0.9f;
constexpr float kBeta2 = 0.999f;

// Adam for one parameter, the arithmetic of ntc_kernel.cu:389-393 with the rounding of
// every operation pinned (so the CPU restatement can reproduce it bit for bit).
__device__ __forceinline__ void adam1(float& p, float& m, float& v, float g, float lr, float b1, float b2)
{
  const float omb1 = 1.0f - kBeta1, omb2 = 1.0f - kBeta2;
  m = __fmaf_rn(kBeta1, m, __fmul_rn(omb1, g));
  v = __fmaf_rn(kBeta2, v, __fmul_rn(__fmul_rn(omb2, g), g));
  const float mb = __fmul_rn(m, b1);
  const float vb = __fmul_rn(v, b2);
  p = __fsub_rn(p, __fdiv_rn(__fmul_rn(lr, mb), __fadd_rn(__fsqrt_rn(vb), 1e-8f)));
}

__device__ __forceinline__ float clamp_latent(float p, float delta)
{
  return fmaxf(-1.0f, fminf(1.0f - delta, p));  // ntc_kernel.cu:475
}

__device__ __forceinline__ void adam_latent4(float* __restrict__ P, float* __restrict__ Mo, float* __restrict__ V,
                                             float* __restrict__ G, long long i, float lr, float b1, float b2,
                                             float delta)
{
  float4 p = *reinterpret_cast<float4*>(P + i);
  float4 m = *reinterpret_cast<float4*>(Mo + i);
  float4 v = *reinterpret_cast<float4*>(V + i);
  const float4 g = *reinterpret_cast<float4*>(G + i);
  adam1(p.x, m.x, v.x, g.x, lr, b1, b2);
  adam1(p.y, m.y, v.y, g.y, lr, b1, b2);
  adam1(p.z, m.z, v.z, g.z, lr, b1, b2);
  adam1(p.w, m.w, v.w, g.w, lr, b1, b2);
  p.x = clamp_latent(p.x, delta);
  p.y = clamp_latent(p.y, delta);
  p.z = clamp_latent(p.z, delta);
  p.w = clamp_latent(p.w, delta);
  *reinterpret_cast<float4*>(P + i) = p;
  *reinterpret_cast<float4*>(Mo + i) = m;
  *reinterpret_cast<float4*>(V + i) = v;
  *reinterpret_cast<float4*>(G + i) = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void __launch_bounds__(256) adam_step_kernel(Model M, const StepRec* __restrict__ steps, int step_idx,
                                                        const float* __restrict__ dW_partial,
                                                        const double* __restrict__ loss_partial, int grid,
                                                        double* __restrict__ loss_out, int n_dec_blocks)
{
  const StepRec& s = steps[step_idx];
  if ((int)blockIdx.x < n_dec_blocks) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w == 0 && loss_out) {
      double l = 0.0;
      for (int i = 0; i < grid; i++) l += loss_partial[i];
      loss_out[s.step] = l / ((double)M.C * (double)s.texels);
    }
    // upstream updates all of W0, W1 and the first C rows of Wout (libopenntc.cpp:722-754)
    if (w >= M.nW || w >= wo_off(M.F) + M.C * kHidden) return;
    float g = 0.0f;
    for (int i = 0; i < grid; i++) g += dW_partial[(size_t)i * M.nW + w];
    float p = M.W[w], m = M.Wm[w], v = M.Wv[w];
    adam1(p, m, v, g, s.lr_dec, s.b1, s.b2);
    M.W[w] = p;
    M.Wm[w] = m;
    M.Wv[w] = v;
    return;
  }
  if (!s.grid_update) return;
  const int lvl = s.level;
  const long long n0 = (long long)M.g0.dim[lvl] * M.g0.dim[lvl] * M.g0.channels;
  const long long n1 = (long long)M.g1.dim[lvl] * M.g1.dim[lvl] * M.g1.channels;
  const long long q0 = n0 >> 2, q = q0 + (n1 >> 2);
  const long long stride = (long long)(gridDim.x - n_dec_blocks) * blockDim.x;
  for (long long i = (long long)(blockIdx.x - n_dec_blocks) * blockDim.x + threadIdx.x; i < q; i += stride) {
    if (i < q0)
      adam_latent4(M.g0.p[lvl], M.g0.m[lvl], M.g0.v[lvl], M.g0.g[lvl], i << 2, s.lr_grid, s.gb1, s.gb2, M.g0.delta);
    else
      adam_latent4(M.g1.p[lvl], M.g1.m[lvl], M.g1.v[lvl], M.g1.g[lvl], (i - q0) << 2, s.lr_grid, s.gb1, s.gb2,
                   M.g1.delta);
  }
}

__global__ void quantize_grid_kernel(float* g, long long n, int bits, float delta)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float k = rintf(__fdiv_rn(g[i], delta));
  const float kmin = -(float)(1 << (bits - 1));
  const float kmax = (float)(1 << (bits - 1)) - 1.0f;
  g[i] = __fmul_rn(fminf(fmaxf(k, kmin), kmax), delta);
}

// One thread per output word: 32/bits codes, LSB first, code = clamp(round(v*2^(b-1))) + 2^(b-1).
__global__ void quantize_pack_kernel(const float* __restrict__ in, long long n_words, int bits, uint32_t* __restrict__ out)
{
  const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_words) return;
  const int per = 32 / bits;
  const int half = 1 << (bits - 1);
  const float scale = (float)half;
  uint32_t word = 0;
  const float* src = in + w * per;
  for (int s = 0; s < per; s++) {
    int x = (int)roundf(__fmul_rn(src[s], scale));
    x = clampi(x, -half, half - 1);
    word |= (uint32_t)(x + half) << (s * bits);
  }
  out[w] = word;
}

__global__ void fill_kernel(float* p, long long n, float v)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

__global__ void sum_doubles_kernel(const double* in, int n, double* out)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += in[i];
    *out = s;
  }
}

}  // namespace

cudaError_t launch_adam_step(const Model& M, const StepRec* d_steps, int step_idx, const float* dW_partial,
                             const double* loss_partial, int grid, double* loss_out, cudaStream_t stream)
{
  // Sized for the largest level so one launch shape serves every step; CTAs beyond the
  // step level's work exit at once.
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int n_dec = (M.nW + 255) / 256;
  const long long n0 = (long long)M.g0.dim[0] * M.g0.dim[0] * M.g0.channels;
  const long long n1 = (long long)M.g1.dim[0] * M.g1.dim[0] * M.g1.channels;
  long long quads = (n0 + n1) / 4;
  long long lat_blocks = (quads + 255) / 256;
  if (lat_blocks > (long long)sms * 8) lat_blocks = (long long)sms * 8;
  adam_step_kernel<<<(unsigned)(n_dec + lat_blocks), 256, 0, stream>>>(M, d_steps, step_idx, dW_partial, loss_partial,
                                                                        grid, loss_out, n_dec);
  return cudaGetLastError();
}

cudaError_t launch_quantize_grid(float* g, long long n, int bits, float delta, cudaStream_t stream)
{
  if (n <= 0) return cudaSuccess;
  quantize_grid_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(g, n, bits, delta);
  return cudaGetLastError();
}

cudaError_t launch_quantize_pack(const float* in, long long n, int bits, uint32_t* out, cudaStream_t stream)
{
  const long long words = n * bits / 32;
  if (words <= 0) return cudaSuccess;
  quantize_pack_kernel<<<(unsigned)((words + 255) / 256), 256, 0, stream>>>(in, words, bits, out);
  return cudaGetLastError();
}

cudaError_t launch_fill(float* p, long long n, float v, cudaStream_t stream)
{
  if (n <= 0) return cudaSuccess;
  fill_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(p, n, v);
  return cudaGetLastError();
}

cudaError_t launch_sum_doubles(const double* in, int n, double* out, cudaStream_t stream)
{
  sum_doubles_kernel<<<1, 32, 0, stream>>>(in, n, out);
  return cudaGetLastError();
}

}  // namespace ontc
