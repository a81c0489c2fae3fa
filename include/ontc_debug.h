/*
 * ontc_debug.h -- introspection entry points of libontc.so for tests and tools.
 *
 * No upstream counterpart: upstream keeps these tensors private (libopenntc.h:256-322).
 * They let a checker read or overwrite the training state, replay one step's gradient
 * computation for a chosen draw without the optimiser update, and run the bit-exact
 * kernels (latent packing, mip reduction) on arbitrary inputs.
 */
#ifndef ONTC_DEBUG_H_
#define ONTC_DEBUG_H_

#include "ontc.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Tensor selectors for ontc_debug_tensor. */
enum {
  ONTC_DBG_G0 = 0,      /* latents g0[level], fp32 [dim][dim][C0] */
  ONTC_DBG_G1 = 1,      /* latents g1[level] */
  ONTC_DBG_G0_M = 2,    /* Adam first moment of g0[level] */
  ONTC_DBG_G0_V = 3,
  ONTC_DBG_G1_M = 4,
  ONTC_DBG_G1_V = 5,
  ONTC_DBG_G0_GRAD = 6, /* latent gradient buffers (zero between steps) */
  ONTC_DBG_G1_GRAD = 7,
  ONTC_DBG_NOISE0 = 8,  /* upstream-mode noise buffers (level-0 sized; level argument ignored) */
  ONTC_DBG_NOISE1 = 9,
  ONTC_DBG_W = 10,      /* decoder, fp32: W0 [64][F] | W1 [64][64] | Wout [16][64] */
  ONTC_DBG_W_M = 11,
  ONTC_DBG_W_V = 12,
  ONTC_DBG_W_GRAD = 13  /* read-only: decoder gradient of the last ontc_debug_gradients call */
};

/* One step's draw (upstream's lod and tile origins, libopenntc.cpp:564-583). */
typedef struct ontc_debug_step {
  int32_t lod;
  int32_t n_grids;
  int32_t ox[8];
  int32_t oy[8];
  int32_t noise;  /* nonzero: add the quantisation-noise surrogate with stream `seed` */
  uint32_t seed;
  int32_t step;   /* global step index the draw belongs to */
  int32_t level;  /* feature level (filled in by the library) */
  /* schedule of that step (libopenntc.cpp:711-720), reported by ontc_debug_last_step */
  float lr_grid, lr_dec, b1, b2, gb1, gb2;
  int32_t grid_update;
  int32_t pad;
} ontc_debug_step;

/* Copies between a state tensor and host memory (to_device = 0: device -> host).
 * n <= 0 returns the element count without copying.  Returns the count or -1. */
int64_t ontc_debug_tensor(ontc_context* ctx, int32_t which, int32_t level, float* host, int64_t n, int32_t to_device);

/* The draw of the most recent training step. */
int ontc_debug_last_step(ontc_context* ctx, ontc_debug_step* out);

/* Gradient of the step loss for `step` at the current state: zeroes the step level's
 * latent gradients, runs the training tile kernel of the context's precision and leaves
 * the latent gradients in ONTC_DBG_G*_GRAD and the decoder gradient in ONTC_DBG_W_GRAD.
 * Writes the mean squared residual to *loss.  Parameters are not updated. */
int ontc_debug_gradients(ontc_context* ctx, ontc_debug_step* step, double* loss);

/* The tile autotuner's cost of one unit round of the bf16 tcgen05 tile kernel at each lod, in
 * microseconds (out_us[0 .. n), n >= the mip count): timed trials on scratch gradient buffers
 * the first time (the training state is not touched), then the context's or the cache file's
 * values.  ontc_train_batch splits the SMs of its shared tile launches by these costs.  No
 * upstream counterpart. */
int ontc_debug_tile_costs(ontc_context* ctx, float* out_us, int32_t n);

/* Upstream quantize_pack on host floats through libontc's kernel (n * bits % 32 == 0). */
int ontc_debug_quantize_pack(const float* host_in, int64_t n, int32_t bits, uint32_t* host_out);

/* One Lanczos-3 2x reduction of a host [dim][dim][c] u8 image through libontc's kernels. */
int ontc_debug_lanczos_down(const uint8_t* src, int32_t dim, int32_t c, uint8_t* dst);

/* The 12 tap weights the reduction uses, as evaluated on the device. */
int ontc_debug_lanczos_weights(float* out12);

/* The interleaved u8 target package of one mip, [dim][dim][C]. */
int ontc_debug_package(ontc_context* ctx, int32_t mip, uint8_t* out);

/* Geometry: [F, Fp, C, mips, levels, nW, g0_dim[6], g1_dim[6], mip_dim[12], batch_i, lock_i, batch_count] */
int ontc_debug_shape(ontc_context* ctx, int32_t* out32);

/* The deferred optimiser's footprint cover (host code, no device): n half-open rectangles
 * in[k] = {x0, y0, x1, y1} -> disjoint rectangles with the same union in out (4 ints each).
 * Returns their count, or -1 when more than cap are needed. */
int ontc_debug_disjoint_cover(const int32_t* in, int32_t n, int32_t* out, int32_t cap);
/* The same cover of the cells of a[0..na) that lie (op 1) or do not lie (op 2) in some
 * rectangle of b[0..nb): how consecutive steps' footprints are split between the main and the
 * side stream. */
int ontc_debug_cover_op(const int32_t* a, int32_t na, const int32_t* b, int32_t nb, int32_t op, int32_t* out,
                        int32_t cap);

/* Test mode of the BF16 (tcgen05) training tile kernel: each feature gradient is replaced by
 * n * 2^-24, n = clamp(rint(g * 2^24), -15, 15), before it is scattered into the latent
 * gradients.  Every latent gradient is then an exactly representable sum, so the float atomics
 * give the same bits in any order.  The decoder is held fixed in this mode (its learning rate
 * is zero): the two tile groups of a CTA add their weight-gradient products to shared TMEM
 * accumulators in arrival order, so the decoder gradient is not bit-reproducible.  Two runs
 * from the same state then leave bit-identical latents, latent moments and decoder weights
 * (used to compare the deferred latent optimiser with the dense one bit for bit).  Takes
 * effect for steps drawn after the call. */
int ontc_debug_exact_gradients(ontc_context* ctx, int32_t enable);

/* Training completion (upstream libopenntc.cpp:799-876: pack the latents, Calibrate,
 * QuantizeWeights into the decoder blob) on the context's current state, without a training
 * step: lets a test load a state (ontc_debug_tensor) and compare the artefacts with another
 * implementation's.  s_a: NULL, or {s_a1, s_a2} to build the blob with these activation scales
 * instead of the calibrated ones (the calibration maxima are still computed and reported).
 * The context is complete afterwards. */
int ontc_debug_complete(ontc_context* ctx, const float* s_a);

/* The int8 decoder's feature bytes (GetFeaturesPacked, ntc_decode.hlsli:196-342) for n samples
 * on the device: out[n][96] int8, the first Kp (64 or 96) bytes of each row written by the
 * decode kernel itself, the rest zero.  Int8 decoders only. */
int ontc_debug_decode_features(ontc_decoder* dec, const float* d_uv, const int32_t* d_lod, int64_t n, int8_t* d_out);

/* Failure injection on the host: the n-th device allocation the library's contexts make from
 * now on (n >= 1) fails as an out-of-memory cudaMalloc would, without calling it; n = 0 disarms.
 * Returns how many such allocations were made before the call, so a test can count the
 * allocation points of a sequence of calls and fail each one in turn.  Process-wide. */
int64_t ontc_debug_fail_device_alloc(int64_t n);

/* The manifest image loader on its own (host code, no device): the file at `path` as RGBA8,
 * the expansion upstream's stbi_load(path, .., 4) gives (libopenntc.cpp:1302).  Writes the
 * size; rgba (NULL: size only) receives width * height * 4 bytes.  ONTC_FILE_NOT_FOUND when the
 * file cannot be read or decoded (upstream's LoadManifest result for such a file). */
int ontc_debug_load_image(const char* path, int32_t* width, int32_t* height, uint8_t* rgba);

/* The bounded wait of the tcgen05 kernels, exercised: one GPU thread waits `polls` (1..1000)
 * suspended polls of up to ~100 us on a barrier nothing arrives at.  Returns ONTC_CUDA_FAILURE
 * when the wait gave up and reported it (the expected outcome), ONTC_INVALID_STATE otherwise. */
int ontc_debug_wait_timeout(int32_t polls);

#ifdef __cplusplus
}
#endif
#endif /* ONTC_DEBUG_H_ */
