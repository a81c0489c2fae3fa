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
#include <algorithm>

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

constexpr int kDecWarps = 8;  // warps of a decoder CTA, each summing every 8th partial

// Decoder Adam for 32 weights (CTA `blk` of the decoder part, 256 threads).  The gradient is
// either the `grid` per-CTA partials of a tile kernel, split over 8 warps and combined in a
// fixed order, or (dw_acc) the one row the tcgen05 tile kernel's CTAs add into, which is read
// and then zeroed for the next step.  CTA 0 also reduces the `grid` loss partials into
// loss_out[step].
__device__ __forceinline__ void decoder_block(const Model& M, const StepRec& s, int blk,
                                              float* __restrict__ dW_partial, bool dw_acc,
                                              const double* __restrict__ loss_partial, int grid,
                                              double* __restrict__ loss_out)
{
  __shared__ float red[kDecWarps][32];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  if (blk == 0 && wp == 0) {
    double l = 0.0;
    for (int i = lane; i < grid; i += 32) l += loss_partial[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if (lane == 0 && loss_out) loss_out[s.step] = l / ((double)M.C * (double)s.texels);
  }
  // upstream updates all of W0, W1 and the first C rows of Wout (libopenntc.cpp:722-754)
  const int nupd = min(M.nW, wo_off(M.F) + M.C * kHidden);
  const int w = blk * 32 + lane;
  const int rows = dw_acc ? 1 : grid;
  float g = 0.0f;
  if (w < nupd) {
#pragma unroll 4
    for (int i = wp; i < rows; i += kDecWarps) g += dW_partial[(size_t)i * M.nW + w];
  }
  red[wp][lane] = g;
  __syncthreads();
  // row 0 is zero whenever a tile kernel starts: the accumulating one adds into it, the others
  // overwrite it; every warp has read it by now
  if (wp == 0 && w < M.nW) dW_partial[w] = 0.0f;
  if (wp != 0 || w >= nupd) return;
  g = red[0][lane];
#pragma unroll
  for (int k = 1; k < kDecWarps; k++) g += red[k][lane];
  float p = M.W[w], m = M.Wm[w], v = M.Wv[w];
  adam1(p, m, v, g, s.lr_dec, s.b1, s.b2);
  M.W[w] = p;
  M.Wm[w] = m;
  M.Wv[w] = v;
}

// Decoder Adam when the gradient is the one row the tcgen05 tile kernels add into: one thread per
// weight (CTA `blk` of the decoder part takes weights [256 blk, 256 blk + 256)), the row read and
// zeroed for the next step; CTA 0's first warp also reduces the `grid` loss partials.
constexpr int kDecRowWeights = 256;
__device__ __forceinline__ void decoder_row_block(const Model& M, const StepRec& s, int blk, float* __restrict__ dW,
                                                  const double* __restrict__ loss_partial, int grid,
                                                  double* __restrict__ loss_out)
{
  const int lane = threadIdx.x & 31;
  if (blk == 0 && threadIdx.x < 32) {
    double l = 0.0;
    for (int i = lane; i < grid; i += 32) l += loss_partial[i];
#pragma unroll
    for (int o = 16; o; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if (lane == 0 && loss_out) loss_out[s.step] = l / ((double)M.C * (double)s.texels);
  }
  // upstream updates all of W0, W1 and the first C rows of Wout (libopenntc.cpp:722-754)
  const int nupd = min(M.nW, wo_off(M.F) + M.C * kHidden);
  const int w = blk * kDecRowWeights + (int)threadIdx.x;
  if (w >= M.nW) return;
  const float g = dW[w];
  dW[w] = 0.0f;  // the row is zero whenever a tile kernel starts
  if (w >= nupd) return;
  float p = M.W[w], m = M.Wm[w], v = M.Wv[w];
  adam1(p, m, v, g, s.lr_dec, s.b1, s.b2);
  M.W[w] = p;
  M.Wm[w] = m;
  M.Wv[w] = v;
}

// ---- deferred latent optimiser ------------------------------------------------------------
// Dense Adam touches every latent of the level every step.  Here a latent cell remembers how
// many level steps it has received: max(applied[cell], floor), where the floor is the level
// step up to which the whole level was last swept.  The steps a cell missed carry zero
// gradient, so they are replayed from the ring of per-step (lr, bias1, bias2) exactly as the
// dense update would have applied them (same adam1 arithmetic, same clamp), only later: right
// before the cell is read again (catch-up over the step's footprint) or in a level sweep.

// Each cell's C channels are split into groups of W = 4 (float4) or, when C is not a multiple
// of 4, W = 2 (float2); one thread takes one (cell, group), so a footprint of n cells runs
// n * C / W threads.
template <int C>
struct Groups {
  static constexpr int W = (C % 4 == 0) ? 4 : 2;
  static constexpr int Q = C / W;
};

template <int W>
__device__ __forceinline__ void load_grp(const float* __restrict__ src, int64_t e, float (&x)[W])
{
  if constexpr (W == 4) {
    const float4 t = *reinterpret_cast<const float4*>(src + e);
    x[0] = t.x, x[1] = t.y, x[2] = t.z, x[3] = t.w;
  } else {
    const float2 t = *reinterpret_cast<const float2*>(src + e);
    x[0] = t.x, x[1] = t.y;
  }
}

template <int W>
__device__ __forceinline__ void store_grp(float* __restrict__ dst, int64_t e, const float (&x)[W])
{
  if constexpr (W == 4)
    *reinterpret_cast<float4*>(dst + e) = make_float4(x[0], x[1], x[2], x[3]);
  else
    *reinterpret_cast<float2*>(dst + e) = make_float2(x[0], x[1]);
}

// Replays level steps [a, J) with zero gradient on the W latents at offset e.
template <int W>
__device__ __forceinline__ void replay_grp(const Pyramid& P, int lvl, int64_t e, int a, int J,
                                           const float4* __restrict__ hist)
{
  float p[W], m[W], v[W];
  load_grp<W>(P.p[lvl], e, p);
  load_grp<W>(P.m[lvl], e, m);
  load_grp<W>(P.v[lvl], e, v);
  for (int t = a; t < J; t++) {
    const float4 h = hist[t & (kHistRing - 1)];
#pragma unroll
    for (int c = 0; c < W; c++) {
      adam1(p[c], m[c], v[c], 0.0f, h.x, h.y, h.z);
      p[c] = clamp_latent(p[c], P.delta);
    }
  }
  store_grp<W>(P.p[lvl], e, p);
  store_grp<W>(P.m[lvl], e, m);
  store_grp<W>(P.v[lvl], e, v);
}

// Applies the step's gradient to the W latents at offset e and clears it.
template <int W>
__device__ __forceinline__ void update_grp(const Pyramid& P, int lvl, int64_t e, float lr, float b1, float b2)
{
  float p[W], m[W], v[W], g[W];
  load_grp<W>(P.p[lvl], e, p);
  load_grp<W>(P.m[lvl], e, m);
  load_grp<W>(P.v[lvl], e, v);
  load_grp<W>(P.g[lvl], e, g);
#pragma unroll
  for (int c = 0; c < W; c++) {
    adam1(p[c], m[c], v[c], g[c], lr, b1, b2);
    p[c] = clamp_latent(p[c], P.delta);
    g[c] = 0.0f;
  }
  store_grp<W>(P.p[lvl], e, p);
  store_grp<W>(P.m[lvl], e, m);
  store_grp<W>(P.v[lvl], e, v);
  store_grp<W>(P.g[lvl], e, g);
}

// Footprint work item i of F -> pyramid g, cell index in the level and channel group q.
template <int C0, int C1>
__device__ __forceinline__ bool foot_item(const FootRec& F, int i, const Model& M, int lvl, int& g, int& cell,
                                          int& q)
{
  constexpr int Q0 = Groups<C0>::Q, Q1 = Groups<C1>::Q;
  const int n0 = F.cells[0] * Q0;
  g = i < n0 ? 0 : 1;
  int local;
  if (g == 0) {
    local = i / Q0;
    q = i - local * Q0;
  } else {
    const int j = i - n0;
    if (j >= F.cells[1] * Q1) return false;
    local = j / Q1;
    q = j - local * Q1;
  }
  int r = 0;
  for (int k = 1; k < F.n[g]; k++) r = F.start[g][k] <= local ? k : r;
  const int w = F.r[g][r][2];
  const int off = local - F.start[g][r];
  const int row = off / w;
  const int dim = g == 0 ? M.g0.dim[lvl] : M.g1.dim[lvl];
  cell = (F.r[g][r][1] + row) * dim + F.r[g][r][0] + (off - row * w);
  return true;
}

// kSide: the instance launched on the side stream, in 64-thread CTAs that fill SMs as tile
// CTAs retire and between launches.  (A tile CTA leaves 1,024 registers free in each of the
// SM's four sub-partitions, so only <= 32-register warps could sit beside it; capped at 32 the
// side kernels did, but slowed the tile kernel by more than they saved: 0.157 vs 0.155 ms per
// 2048^2 step.)
constexpr int kSideThreads = 64;

template <int C0, int C1, bool kSide>
__global__ void __launch_bounds__(kSide ? kSideThreads : 256)
    catchup_kernel(Model M, const StepRec* __restrict__ steps, int idx, const __grid_constant__ FootRec F)
{
  const StepRec& s = steps[idx];
  const int lvl = s.level, j = s.gstep, fl = s.gfloor;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int g, cell, q;
  if (!foot_item<C0, C1>(F, i, M, lvl, g, cell, q)) return;
  const int a = max(M.applied[g][lvl][cell], fl);
  if (a >= j) return;
  if (g == 0)
    replay_grp<Groups<C0>::W>(M.g0, lvl, (int64_t)cell * C0 + q * Groups<C0>::W, a, j, M.hist[lvl]);
  else
    replay_grp<Groups<C1>::W>(M.g1, lvl, (int64_t)cell * C1 + q * Groups<C1>::W, a, j, M.hist[lvl]);
}

// Brings every latent of level `lvl` from max(applied, fl) up to J.  Writes no counter: the
// caller raises the level's floor to J.
template <int C0, int C1>
__global__ void __launch_bounds__(256) sweep_kernel(Model M, int lvl, int fl, int J)
{
  constexpr int Q0 = Groups<C0>::Q, Q1 = Groups<C1>::Q;
  const int n0 = M.g0.dim[lvl] * M.g0.dim[lvl] * Q0;
  const int n1 = M.g1.dim[lvl] * M.g1.dim[lvl] * Q1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n0 + n1; i += gridDim.x * blockDim.x) {
    if (i < n0) {
      const int cell = i / Q0, q = i - cell * Q0;
      const int a = max(M.applied[0][lvl][cell], fl);
      if (a < J) replay_grp<Groups<C0>::W>(M.g0, lvl, (int64_t)cell * C0 + q * Groups<C0>::W, a, J, M.hist[lvl]);
    } else {
      const int k = i - n0;
      const int cell = k / Q1, q = k - cell * Q1;
      const int a = max(M.applied[1][lvl][cell], fl);
      if (a < J) replay_grp<Groups<C1>::W>(M.g1, lvl, (int64_t)cell * C1 + q * Groups<C1>::W, a, J, M.hist[lvl]);
    }
  }
}

// Decoder Adam (CTAs [0, n_dec)) and the step's gradient on its footprint, every latent of
// which is at level step gstep (the other CTAs).
template <int C0, int C1>
__global__ void __launch_bounds__(256)
    footprint_update_kernel(Model M, const StepRec* __restrict__ steps, int idx, const __grid_constant__ FootRec F,
                            float* __restrict__ dW_partial, bool dw_acc, const double* __restrict__ loss_partial,
                            int grid, double* __restrict__ loss_out, int n_dec)
{
  const StepRec& s = steps[idx];
  if ((int)blockIdx.x < n_dec) {
    if (dw_acc)
      decoder_row_block(M, s, blockIdx.x, dW_partial, loss_partial, grid, loss_out);
    else
      decoder_block(M, s, blockIdx.x, dW_partial, dw_acc, loss_partial, grid, loss_out);
    return;
  }
  const int lvl = s.level, j = s.gstep;
  const int i = (blockIdx.x - n_dec) * blockDim.x + threadIdx.x;
  int g, cell, q;
  if (!foot_item<C0, C1>(F, i, M, lvl, g, cell, q)) return;
  if (g == 0)
    update_grp<Groups<C0>::W>(M.g0, lvl, (int64_t)cell * C0 + q * Groups<C0>::W, s.lr_grid, s.gb1, s.gb2);
  else
    update_grp<Groups<C1>::W>(M.g1, lvl, (int64_t)cell * C1 + q * Groups<C1>::W, s.lr_grid, s.gb1, s.gb2);
  if (q == 0) M.applied[g][lvl][cell] = j + 1;  // no thread of this kernel reads the counters
}

// The (lr, bias1, bias2) of every latent-updating step of [k0, k1) into its level's ring, at
// its level step (what the deferred replays read).
__global__ void hist_write_kernel(Model M, const StepRec* __restrict__ steps, int k0, int k1)
{
  const int k = k0 + (int)threadIdx.x;
  if (k >= k1) return;
  const StepRec& s = steps[k];
  if (s.grid_update) M.hist[s.level][s.gstep & (kHistRing - 1)] = make_float4(s.lr_grid, s.gb1, s.gb2, 0.0f);
}

__global__ void __launch_bounds__(256) adam_step_kernel(Model M, const StepRec* __restrict__ steps, int step_idx,
                                                        float* __restrict__ dW_partial, bool dw_acc,
                                                        const double* __restrict__ loss_partial, int grid,
                                                        double* __restrict__ loss_out, int n_dec_blocks)
{
  const StepRec& s = steps[step_idx];
  if ((int)blockIdx.x < n_dec_blocks) {
    if (dw_acc)
      decoder_row_block(M, s, blockIdx.x, dW_partial, loss_partial, grid, loss_out);
    else
      decoder_block(M, s, blockIdx.x, dW_partial, dw_acc, loss_partial, grid, loss_out);
    return;
  }
  if (!s.grid_update) return;
  const int lvl = s.level;
  const int b = blockIdx.x - n_dec_blocks;
  const int nb = gridDim.x - n_dec_blocks;
  const long long n0 = (long long)M.g0.dim[lvl] * M.g0.dim[lvl] * M.g0.channels;
  const long long n1 = (long long)M.g1.dim[lvl] * M.g1.dim[lvl] * M.g1.channels;
  const long long q0 = n0 >> 2, q = q0 + (n1 >> 2);
  const long long stride = (long long)nb * blockDim.x;
  for (long long i = (long long)b * blockDim.x + threadIdx.x; i < q; i += stride) {
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

static int sm_count()
{
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

static int dec_blocks(const Model& M) { return (M.nW + 31) / 32; }

// Profile channel pairs (C0, C1) with compiled deferred-optimiser kernels.
#define ONTC_FOR_CHANNEL_PAIRS(X) X(8, 12) X(12, 20) X(12, 10) X(16, 12)

cudaError_t launch_catchup(const Model& M, const StepRec* d_steps, int step_idx, const FootRec& F, bool side,
                           cudaStream_t stream)
{
#define X(a, b)                                                                                          \
  if (M.g0.channels == a && M.g1.channels == b) {                                                        \
    const int total = F.cells[0] * Groups<a>::Q + F.cells[1] * Groups<b>::Q;                             \
    if (total <= 0) return cudaSuccess;                                                                  \
    if (side)                                                                                            \
      catchup_kernel<a, b, true><<<(total + kSideThreads - 1) / kSideThreads, kSideThreads, 0, stream>>>(  \
          M, d_steps, step_idx, F);                                                                      \
    else                                                                                                 \
      catchup_kernel<a, b, false><<<(total + 255) / 256, 256, 0, stream>>>(M, d_steps, step_idx, F);      \
    return cudaGetLastError();                                                                           \
  }
  ONTC_FOR_CHANNEL_PAIRS(X)
#undef X
  return cudaErrorNotSupported;
}

cudaError_t launch_footprint_update(const Model& M, const StepRec* d_steps, int step_idx, const FootRec& F,
                                    bool decoder, float* dW_partial, bool dw_acc, const double* loss_partial, int grid,
                                    double* loss_out, cudaStream_t stream)
{
  // the row gradient of the tcgen05 tile kernels: one thread per weight; per-CTA partials: 32
  // weights per CTA, summed by its eight warps
  const int n_dec = !decoder ? 0 : dw_acc ? (M.nW + kDecRowWeights - 1) / kDecRowWeights : dec_blocks(M);
#define X(a, b)                                                                                          \
  if (M.g0.channels == a && M.g1.channels == b) {                                                        \
    const int total = F.cells[0] * Groups<a>::Q + F.cells[1] * Groups<b>::Q;                             \
    const unsigned blocks = (unsigned)(n_dec + (total + 255) / 256);                                     \
    if (blocks == 0) return cudaSuccess;                                                                 \
    footprint_update_kernel<a, b><<<blocks, 256, 0, stream>>>(M, d_steps, step_idx, F, dW_partial, dw_acc,   \
                                                              loss_partial, grid, loss_out, n_dec);      \
    return cudaGetLastError();                                                                           \
  }
  ONTC_FOR_CHANNEL_PAIRS(X)
#undef X
  return cudaErrorNotSupported;
}

cudaError_t launch_hist_write(const Model& M, const StepRec* d_steps, int k0, int k1, cudaStream_t stream)
{
  if (k1 <= k0) return cudaSuccess;
  if (k1 - k0 > 1024) return cudaErrorInvalidValue;
  hist_write_kernel<<<1, k1 - k0, 0, stream>>>(M, d_steps, k0, k1);
  return cudaGetLastError();
}

cudaError_t launch_sweep(const Model& M, int level, int from, int J, cudaStream_t stream)
{
#define X(a, b)                                                                                          \
  if (M.g0.channels == a && M.g1.channels == b) {                                                        \
    const long long n = (long long)M.g0.dim[level] * M.g0.dim[level] * Groups<a>::Q +                    \
                        (long long)M.g1.dim[level] * M.g1.dim[level] * Groups<b>::Q;                     \
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)sm_count() * 16);           \
    sweep_kernel<a, b><<<(unsigned)blocks, 256, 0, stream>>>(M, level, from, J);                         \
    return cudaGetLastError();                                                                           \
  }
  ONTC_FOR_CHANNEL_PAIRS(X)
#undef X
  return cudaErrorNotSupported;
}

bool deferred_supported(int c0, int c1)
{
#define X(a, b) \
  if (c0 == a && c1 == b) return true;
  ONTC_FOR_CHANNEL_PAIRS(X)
#undef X
  return false;
}

cudaError_t launch_adam_step(const Model& M, const StepRec* d_steps, int step_idx, float* dW_partial, bool dw_acc,
                             const double* loss_partial, int grid, double* loss_out, cudaStream_t stream)
{
  // Sized for the largest level so one launch shape serves every step; CTAs beyond the
  // step level's work exit at once.
  const int n_dec = dw_acc ? (M.nW + kDecRowWeights - 1) / kDecRowWeights : dec_blocks(M);
  const long long n0 = (long long)M.g0.dim[0] * M.g0.dim[0] * M.g0.channels;
  const long long n1 = (long long)M.g1.dim[0] * M.g1.dim[0] * M.g1.channels;
  long long quads = (n0 + n1) / 4;
  long long lat_blocks = (quads + 255) / 256;
  if (lat_blocks > (long long)sm_count() * 8) lat_blocks = (long long)sm_count() * 8;
  adam_step_kernel<<<(unsigned)(n_dec + lat_blocks), 256, 0, stream>>>(M, d_steps, step_idx, dW_partial, dw_acc,
                                                                        loss_partial, grid, loss_out, n_dec);
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
