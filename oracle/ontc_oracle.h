/*
 * ontc_oracle.h -- CPU restatement of openntc's training/decoding arithmetic.
 *
 * TEST INFRASTRUCTURE.  Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg call this library, and only to check or time libontc; the product never links it.
 *
 * Every function cites the upstream source lines it restates.  Floating-point steps that
 * upstream performs in fp32 (feature construction, Adam, quantisation, the Lanczos filter)
 * are restated in fp32 with the same rounding sequence (compiled with -ffp-contract=off and
 * explicit fmaf where upstream's nvcc build fuses); the MLP forward/backward, losses and
 * PSNR are evaluated in fp64 as the reference answer for both fp32 and bf16 device paths.
 *
 * Pinning: upstream ships no tests or golden vectors.  The restatement is pinned against
 * upstream compiled from source (oracle/_ref): container bytes on the CPU (tests/golden),
 * and packing, mip reduction and step gradients on the GPU (tests marked gpu).
 */
#ifndef ONTC_ORACLE_H_
#define ONTC_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_model {
  int32_t C0, C1, F, C;        /* g0/g1 channels, feature dim, output channels */
  int32_t g0_dim, g1_dim;      /* latent grid dims of the step's level */
  int32_t mip_dim;             /* texture dim of the step's lod */
  float d0, d1;                /* quantisation steps 2/2^bits */
  const float* g0;             /* [g0_dim][g0_dim][C0] */
  const float* g1;             /* [g1_dim][g1_dim][C1] */
  const float* W;              /* W0 [64][F] | W1 [64][64] | Wout [16][64] */
  const uint8_t* target;       /* [mip_dim][mip_dim][C] */
} orc_model;

typedef struct orc_step {
  int32_t tile_dim, n_grids;
  int32_t ox[8], oy[8];
  int32_t noise;
  uint32_t seed;
  float norm_lod;
} orc_step;

/* libontc's texel enumeration of a step (the texel set equals upstream's wrapped tiles,
 * ntc_kernel.cu:94-99). */
void orc_texel_xy(const orc_step* s, int32_t mip_dim, int32_t b, int32_t* x, int32_t* y);

/* libontc's quantisation-noise value for latent element e of pyramid `which`. */
float orc_noise(uint32_t seed, uint32_t which, uint32_t e, float delta);

/* draw_features (ntc_kernel.cu:75-177) for one texel: F fp32 values. */
void orc_features(const orc_model* m, const orc_step* s, int32_t x, int32_t y, float* out);

/* One step's loss and gradients in fp64 (libopenntc.cpp:651-709 in exact arithmetic):
 * returns mean squared residual; adds dL/dW into dW[n_weights] and dL/dlatent into
 * dG0/dG1 (full-level arrays, may be NULL).  Uses up to `threads` OpenMP threads. */
double orc_step_gradients(const orc_model* m, const orc_step* s, double* dW, double* dG0, double* dG1,
                          int32_t threads);

/* Sum of squared residuals over a full mip (Eval forward, libopenntc.cpp:1007-1045) in fp64,
 * and the max |hardgelu| of layers 0/1 (Calibrate, :951-956). */
double orc_mip_sq_error(const orc_model* m, float norm_lod, int32_t noise, uint32_t seed, float* max_a0,
                        float* max_a1, int32_t threads);

/* Adam + optional clamp as libontc applies it (ntc_kernel.cu:389-393, 475). */
void orc_adam(float* p, float* m, float* v, const float* g, int64_t n, float lr, float b1, float b2, int32_t clamp,
              float delta);

/* quantize_grid (ntc_kernel.cu:448-460) and quantize_pack (ntc_kernel.cu:486-499). */
void orc_quantize_grid(float* g, int64_t n, int32_t bits, float delta);
void orc_quantize_pack(const float* in, int64_t n, int32_t bits, uint32_t* out);

/* Lanczos-3 taps (ntc_kernel.cu:569-579) with the host libm, and one 2x reduction of a
 * [dim][dim][c] u8 image with the given taps (ntc_kernel.cu:581-663). */
void orc_lanczos_weights(float* w12);
void orc_lanczos_down(const uint8_t* src, int32_t dim, int32_t c, const float* w12, uint8_t* dst);

/* QuantizeWeights (libopenntc.cpp:445-469). */
void orc_quantize_weights(const float* Wf, int32_t rows, int32_t cols, float prescale, uint32_t* Wq, float* Ws);

/* SampleMaterial (ntc_decode.hlsli:605-623) with the DP4A inference path (:410-502):
 * decodes n samples (uv pairs, integer lods) into out[n][channel_count] (saturated).
 * g0/g1 are the contiguous packed pyramids, decoder the int8 blob, constants the
 * 240-byte NTCConstants; profile selects the compile-time shape. */
void orc_sample_material(int32_t profile, const uint32_t* g0, const uint32_t* g1, const uint8_t* decoder,
                         const void* constants, const float* uv, const int32_t* lod, int64_t n, float* out,
                         int32_t threads);

/* The NTC pixel shaders' stochastic filter (flat_ntc.hlsl:74-84; ComputeLod,
 * StochasticFilterLod, StochasticFilterUv, InterleavedGradientNoise at ntc_decode.hlsli:143-185)
 * over a uv image img [h][w][2], with HLSL's coarse quad derivatives (backward difference where
 * the image cuts a quad, 0 in a one-pixel dimension): per pixel the jittered uv, the chosen lod,
 * whether it is kept (discard_outside: uv inside [0, 1]), the clamped float lod and the noise
 * value the lod choice compared against. */
void orc_screen_filter(const float* img, int32_t w, int32_t h, int32_t dim, int32_t mip_count, float noise_frame,
                       int32_t discard_outside, float* uv_out, int32_t* lod_out, uint8_t* keep, float* lod_ab,
                       float* noise);

/* DecodeMaterial (ntc_decode.hlsli:524-603): saturated outputs [n][channel_count] and the
 * per-channel semantics -> MaterialParams [n] as 17 floats + the `present` word. */
void orc_decode_material(const float* channels, int64_t n, int32_t channel_count, const uint32_t* semantics,
                         float* params);

/* The float model decode (features from the packed latents dequantised, fp64 MLP with the
 * given fp32 weights), used as the FP64 decode reference. */
void orc_decode_float(int32_t profile, const uint32_t* g0, const uint32_t* g1, const void* constants,
                      const float* W, int32_t C, const float* uv, const int32_t* lod, int64_t n, double* out,
                      int32_t threads);

/* Exhaustive check of the decoder's division by 3 (see ontc_oracle.c); returns mismatches. */
int64_t orc_check_div3(int32_t threads);

#ifdef __cplusplus
}
#endif
#endif
