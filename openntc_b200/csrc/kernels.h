// Host-side launchers of libontc's kernels (all on the caller's stream, all unchecked
// for work errors but checked for launch errors).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"

#include "ontc.h"

namespace ontc {

enum { kTrain = 0, kEval = 1, kCalib = 2 };

// ---- decode (SampleMaterial over a batch of samples, decode.cu)
struct DecodeArgs {
  const uint32_t* g0;   // packed g0 pyramid, every level at its constants offset
  const uint32_t* g1;
  uint32_t g0_words, g1_words;
  const uint8_t* blob;  // int8 decoder blob (W0 | W1 | Wout | scales)
  ontc_constants k;     // the material's NTCConstants
  const float* uv;      // [n][2]
  const int32_t* lod;   // [n]
  int64_t n;
  float* out;           // [n][k.channel_count], or ontc_material_params [n] when `material`
  int* err;             // set to 1 when a bounded wait gave up
  // screen-space sampling (screen_w > 0): uv is a [screen_h][screen_w][2] image, lod unused,
  // n = screen_w * screen_h, and each pixel's (uv, lod) comes from the stochastic filter
  int32_t screen_w = 0, screen_h = 0;
  float noise_frame = 0.0f;
  bool discard_outside = false;
  // DecodeMaterial output: material_dst[c] = float index in ontc_material_params written by
  // channel c (-1: none); material_present = the `present` bits
  bool material = false;
  int8_t material_dst[16] = {};
  uint32_t material_present = 0;
  // test hook (ontc_debug_decode_features): each sample's Kp feature bytes also go to
  // feat_out[i * 24 ..] (rows of 96 bytes)
  uint32_t* feat_out = nullptr;
};
cudaError_t launch_decode(int profile, const DecodeArgs& args, cudaStream_t stream);
// The float-model decoders (decode_float.cu): the trained fp32 decoder weights evaluated on the
// dequantised latent codes.  mode: ONTC_DECODE_FP32 (fp32 CUDA-core arithmetic), BF16
// (tcgen05 bf16, fp32 accumulate), FP8 (tcgen05 e4m3 with per-layer scales, fp32 accumulate).
struct FloatDecodeArgs {
  const uint32_t* g0;
  const uint32_t* g1;
  uint32_t g0_words, g1_words;
  ontc_constants k;
  const float* W;    // FP32: W0 [64][F] | W1 [64][64] | Wout [16][64] (the training layout)
  const void* Wq;    // BF16 / FP8: W0 [64][Kp] | W1 [64][64] | Wout [16][64] elements, row-major
  float sx = 1.0f;   // FP8: feature, weight and activation scales (value = code x scale)
  float sw0 = 1.0f, sw1 = 1.0f, swo = 1.0f, sa1 = 1.0f, sa2 = 1.0f;
  const float* uv;
  const int32_t* lod;
  int64_t n;
  float* out;        // [n][k.channel_count], saturated
  int* err;          // set to 1 when a bounded wait gave up
};
cudaError_t launch_decode_float(int profile, int mode, const FloatDecodeArgs& args, cudaStream_t stream);
// Kp of a profile's float decoder (the training feature width rounded up to 32)
int float_decode_kp(int profile);

// Turns a decoder into a float-model one (mode ONTC_DECODE_FP32 / BF16 / FP8) with the fp32
// weights W (training layout, feature width F), C output channels and the calibration maxima
// (FP8 activation scales).  ONTC_* status.
int decoder_set_float(ontc_decoder* dec, int mode, const float* W, int F, int C, const ontc_calibration& cal);
// Replaces a decoder's int8 blob and activation scales (same layout and shapes); waits for its
// stream first.  ONTC_* status.
int decoder_set_weights(ontc_decoder* dec, const uint8_t* blob, size_t size, float s_a1, float s_a2);

// The mip chain's texels as one sequence (mip 0 first, row-major); sample j is texel
// (j * stride + offset) mod start[mips], stride coprime with the total and j * stride < 2^63.
struct TexelMap {
  int mips = 0, C = 0;
  int dim[ONTC_MAX_MIPS] = {};
  int64_t start[ONTC_MAX_MIPS + 1] = {};
  const uint8_t* target[ONTC_MAX_MIPS] = {};  // [dim][dim][C] u8 training targets
  int64_t stride = 1, offset = 0;
};
// uv (texel centre) and lod (its mip) of samples j0 .. j0 + n - 1
cudaError_t launch_texel_samples(const TexelMap& m, int64_t j0, int64_t n, float* uv, int32_t* lod,
                                 cudaStream_t stream);
// partial[b] = sum over block b's samples of (target / 255 - out)^2, fp32 residuals, fp64 sums
cudaError_t launch_decoded_sq_err(const TexelMap& m, int64_t j0, int64_t n, const float* out, double* partial,
                                  int blocks, cudaStream_t stream);
// one thread waits `polls` suspended polls on a barrier nothing arrives at; *d_out = 1 when it gave up
cudaError_t launch_wait_check(uint32_t polls, int* d_out, cudaStream_t stream);

struct TileOut {
  float* dW_partial;     // kTrain: [grid][nW] per-CTA decoder gradient partials (SIMT kernel); the
                         // tcgen05 tile kernel instead adds every CTA's gradient into row 0
  double* loss_partial;  // [grid] per-CTA sum of squared residuals (kTrain, kEval)
  float* calib_max;      // [2] running max |a0|, |a1| as ordered ints (kCalib)
};

// TMA staging of a 16 x 8 texel unit's latent boxes at one lod (tile kernel): tensor maps of
// the lod's level and the fixed box sizes that cover every unit footprint at that lod.
struct LatentBoxes {
  CUtensorMap g0;          // 3-D {C0, d0, d0} view of the level's g0 latents, box {C0, w0, h0}
  CUtensorMap g1;          // 2-D {d1 * C1, d1} view of g1, box {w1 * C1, h1}
  int32_t w0, h0, w1, h1;  // box sizes in cells; w0 == 0: units at this lod are not staged
  int32_t g1_shift;        // 1: the g1 box starts at the even cell at or below the footprint's first
  uint32_t bytes;          // bytes the two loads deliver
  uint32_t g1_off;         // float offset of the g1 box in a staging buffer (128-byte aligned)
};
// Builds the boxes of lod `lod` for latents p0 / p1 of grid sizes d0 / d1 (staging buffer of
// `cap_floats`); w0 = 0 when the footprint does not fit.  cudaSuccess or the driver's error.
cudaError_t make_latent_boxes(const float* p0, const float* p1, int d0, int d1, int C0, int C1, int mip_dim,
                              int cap_floats, LatentBoxes& out);

// ---- training / eval units
size_t simt_smem_bytes(int F);
cudaError_t launch_simt_units(int mode, const Model& M, const StepRec* d_steps, int step_idx, int grid, TileOut out,
                              cudaStream_t stream);
// tcgen05 tile kernel, bf16 operands or (split) fp32 operands as bf16 high + low parts; returns
// cudaErrorNotSupported when the profile has no tcgen05 variant
cudaError_t launch_tc_units(const Model& M, const StepRec* d_steps, int step_idx, int grid, TileOut out,
                            int* d_error, const LatentBoxes& boxes, bool split, cudaStream_t stream);
// Many materials in one tcgen05 tile launch (bf16 operands): material i runs its step on CTAs
// [cta_begin, cta_begin + cta_count), which follow one another from 0 in material order; every
// material has the same profile shape.  Each material's loss partials are indexed by its own
// CTAs, and its decoder gradient is added into row 0 of its dW buffer as in launch_tc_units.
constexpr int kMaxTileMats = 16;
struct alignas(64) TileMat {
  LatentBoxes boxes;   // the tensor maps of the step's lod (first: 64-byte aligned)
  Model M;
  const StepRec* step;  // the material's step record on the device
  TileOut out;
  int* err;             // the material's tile error flag
  int32_t cta_begin, cta_count;
};
cudaError_t launch_tc_multi(const TileMat* mats, int n, cudaStream_t stream);
// 128-texel units a tile CTA works on at once (its grid: units / this, at most one CTA per SM)
int tc_groups_per_cta(bool split);
// the staging buffer the tile kernel gives a unit's latent boxes, in floats
int tc_box_capacity();
int tc_max_grid();

// ---- optimiser: decoder Adam (reducing `grid` partials, or with dw_acc reading and zeroing the
// one row a tcgen05 tile kernel accumulates into) + dense latent Adam/clamp/zero of the step's
// level, one launch.  Also reduces the `grid` loss partials into loss_out[step].
cudaError_t launch_adam_step(const Model& M, const StepRec* d_steps, int step_idx, float* dW_partial, bool dw_acc,
                             const double* loss_partial, int grid, double* loss_out, cudaStream_t stream);
// deferred latent optimiser (see optim.cu): catch the step's footprint up to its level step,
// apply the step's gradient to the footprint (plus the decoder Adam), sweep a whole level
// `side`: the side-stream instance (64-thread CTAs, which fill SMs as tile CTAs retire);
// otherwise 256-thread CTAs
cudaError_t launch_catchup(const Model& M, const StepRec* d_steps, int step_idx, const FootRec& F, bool side,
                           cudaStream_t stream);
// the step's gradient on the footprint F and, with `decoder`, the decoder Adam + loss
// reduction; one launch
cudaError_t launch_footprint_update(const Model& M, const StepRec* d_steps, int step_idx, const FootRec& F,
                                    bool decoder, float* dW_partial, bool dw_acc, const double* loss_partial, int grid,
                                    double* loss_out, cudaStream_t stream);
// the hist-ring entries of steps [k0, k1) that update latents, from their step records
cudaError_t launch_hist_write(const Model& M, const StepRec* d_steps, int k0, int k1, cudaStream_t stream);
// every latent of `level` from level step max(applied, from) to J
cudaError_t launch_sweep(const Model& M, int level, int from, int J, cudaStream_t stream);
// whether the deferred kernels are compiled for this (C0, C1) pair
bool deferred_supported(int c0, int c1);
// upstream quantize_grid over one latent tensor (ntc_kernel.cu:448-460)
cudaError_t launch_quantize_grid(float* g, long long n, int bits, float delta, cudaStream_t stream);
// upstream quantize_pack (ntc_kernel.cu:486-499), n*bits must be a multiple of 32
cudaError_t launch_quantize_pack(const float* in, long long n, int bits, uint32_t* out, cudaStream_t stream);
// fills n floats with v
cudaError_t launch_fill(float* p, long long n, float v, cudaStream_t stream);
// out = sum over the first n doubles (single CTA, deterministic order)
cudaError_t launch_sum_doubles(const double* in, int n, double* out, cudaStream_t stream);

// ---- upstream-compatible noise (parity mode)
size_t noise_state_bytes(int n_states);
cudaError_t launch_noise_init(void* states, int n_states, cudaStream_t stream);
cudaError_t launch_noise_fill(void* states, int n_states, long long n, float delta, float* out, cudaStream_t stream);

// ---- mip chain (LoadManifest)
// one separable Lanczos-3 2x reduction [dim][dim][c] -> [dim/2][dim/2][c] in two kernels; tmp
// holds dim*dim/2*c floats (the caller-buffer entry points; LoadManifest uses the fused chain)
cudaError_t launch_lanczos_down(const uint8_t* src, int dim, int c, float* tmp, uint8_t* dst, cudaStream_t stream);
// The ingest chain fused with packaging: mip 0 of a source (channel selection) and each 2x
// reduction (both Lanczos passes in one kernel) also write the source's channels
// [pkg_off, pkg_off + count) of that mip's target package [dim][dim][C].
cudaError_t launch_prepare_package(const uint8_t* rgba, int dim, const int* cmap, int count, uint8_t* out, uint8_t* pkg,
                                   int C, int pkg_off, cudaStream_t stream);
cudaError_t launch_lanczos_down_package(const uint8_t* src, int dim, int c, uint8_t* dst, uint8_t* pkg, int C,
                                        int pkg_off, cudaStream_t stream);
// the 12 Lanczos-3 tap weights as the filter computes them (test hook)
cudaError_t lanczos_weights(float* host12);

}  // namespace ontc
