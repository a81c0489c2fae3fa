/*
 * ontc.h -- C ABI of the B200 neural-texture-compression library (libontc.so).
 *
 * This is the drop-in boundary for openntc's libopenntc: every entry point below
 * replaces one member of upstream's openntc::Context (libopenntc/libopenntc.h:168-197)
 * or one free function of its CUDA-free runtime (libopenntc/openntc_runtime.h:55-150).
 * The structs are byte-compatible with upstream's (same field order, same sizes), so a
 * CompressedData produced by either side can be handed to the other.  The header-only
 * C++ wrapper in include/libopenntc/ puts upstream's class and function names on top.
 *
 * Conventions
 *  - Status returns are upstream's openntc::Result values (openntc_runtime.h:18-30).
 *  - One context = one GPU = one CUDA stream (the caller's, or the library's own at the
 *    highest priority).  Training also uses a private lowest-priority stream for deferred
 *    optimiser work that overlaps the tile kernels; it is joined back into the context's
 *    stream (by an event wait) before every training call returns.  Not thread-safe; callers
 *    serialise, as upstream's GUI does (openntc-gui/thread.h:15-28).
 *  - All compute runs on hand-written sm_100a kernels inside libontc.so.  There is no
 *    CPU fallback: with no usable GPU, ontc_init returns ONTC_CUDA_FAILURE.
 */
#ifndef ONTC_H_
#define ONTC_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ONTC_MAX_MIPS 12     /* openntc_runtime.h:51 kMaxMips */
#define ONTC_MAX_CHANNELS 16 /* openntc_runtime.h:52 kMaxChannels */
#define ONTC_MAX_LEVELS 6    /* openntc_runtime.h:53 kMaxLevels */
#define ONTC_MAX_SOURCES 16  /* libopenntc.h:138 kMaxSources */
#define ONTC_MIN_DIMENSION 1024 /* libopenntc.h:171 kMinDimension (see ontc_set_min_dimension) */
#define ONTC_MAX_DIMENSION 8192 /* libopenntc.h:172 kMaxDimension */

/* openntc::Result, openntc_runtime.h:18-30 */
enum {
  ONTC_SUCCESS = 0,
  ONTC_INVALID_DIMENSION = 1,
  ONTC_ALLOCATION_FAILURE = 2,
  ONTC_INVALID_MANIFEST = 3,
  ONTC_FILE_NOT_FOUND = 4,
  ONTC_INVALID_FILE = 5,
  ONTC_FILE_WRITE_FAILURE = 6,
  ONTC_INVALID_STATE = 7,
  ONTC_CUDA_FAILURE = 8
};

/* openntc::Profile, openntc_runtime.h:8-16 */
enum { ONTC_BPP_0_2 = 0, ONTC_BPP_0_5 = 1, ONTC_BPP_1_0 = 2, ONTC_BPP_2_25 = 3 };

/* openntc::Quality, libopenntc.h:147-155 */
enum { ONTC_QUALITY_LOW = 0, ONTC_QUALITY_MEDIUM = 1, ONTC_QUALITY_HIGH = 2, ONTC_QUALITY_ULTRA = 3 };

/* openntc::TrainPhase, libopenntc.h:99-106 */
enum { ONTC_MANIFEST_LOADED = 0, ONTC_TRAIN_IN_PROGRESS = 1, ONTC_TRAIN_COMPLETE = 2, ONTC_TRAIN_ERROR = -1 };

/* MLP arithmetic of the training step (no upstream counterpart: upstream always runs
 * cuBLAS TF32, libopenntc.cpp:374).
 *   BF16 (default): tcgen05/TMEM bf16 operands, fp32 accumulate, fp32 master weights and
 *                   fp32 Adam moments.
 *   FP32:           SIMT fp32 tile kernel (exact fp32 products).
 *   BF16X3:         tcgen05 products of fp32 operands split into bf16 high and low parts
 *                   (h.h + h.l + l.h, three bf16 MMAs, fp32 accumulate), fp32 activations:
 *                   about 16 mantissa bits per product, more than upstream's tf32 products. */
enum { ONTC_PRECISION_BF16 = 0, ONTC_PRECISION_FP32 = 1, ONTC_PRECISION_BF16X3 = 2 };

/* Decoder arithmetic for ontc_decode (upstream: HLSL only, ntc_decode.hlsli:605-623). */
enum {
  ONTC_DECODE_INT8 = 0, /* SampleMaterial semantics, integer-exact with the DP4A path */
  /* The trained float model instead of the int8 blob (ontc_decoder_create_float): features from
   * the dequantised latent codes in fp32, the fp32 decoder weights, saturated outputs. */
  ONTC_DECODE_FP32 = 1, /* fp32 arithmetic throughout (CUDA cores) */
  ONTC_DECODE_BF16 = 2, /* bf16 features, weights and activations; fp32 accumulation (tcgen05) */
  ONTC_DECODE_FP8 = 3   /* e4m3 with per-layer scales: features x 256, weights at max|W| / 448,
                           activations at Calibrate's max |activation| / 448; fp32 accumulation */
};

/* openntc::CalibrationData, openntc_runtime.h:61-67 */
typedef struct ontc_calibration {
  float max_abs_a1;
  float max_abs_a2;
  float s_a1;
  float s_a2;
} ontc_calibration;

/* openntc::NTCConstants, openntc_runtime.h:69-89 (240 bytes; HLSL cbuffer NTC) */
typedef struct ontc_constants {
  int32_t g0_grid_dim[8];
  int32_t g1_grid_dim[8];
  uint32_t g0_offset[8];
  uint32_t g1_offset[8];
  int32_t g0_bits_per_channel;
  int32_t g1_bits_per_channel;
  int32_t g0_channels;
  int32_t g1_channels;
  int32_t dim;
  int32_t mip_count;
  float rcp_s_a1;
  float rcp_s_a2;
  int32_t channel_count;
  int32_t pad0[3];
  uint32_t channel_semantics[16];
} ontc_constants;

/* openntc::CompressedData, openntc_runtime.h:91-121.  Pointers are borrowed (owned by a
 * context or by an ontc_file). */
typedef struct ontc_compressed_data {
  uint32_t* g0[ONTC_MAX_LEVELS];
  uint32_t* g1[ONTC_MAX_LEVELS];
  void* decoder;
  size_t g0_size[ONTC_MAX_LEVELS];
  size_t g1_size[ONTC_MAX_LEVELS];
  size_t g0_offset[ONTC_MAX_LEVELS];
  size_t g1_offset[ONTC_MAX_LEVELS];
  size_t g0_total_size;
  size_t g1_total_size;
  size_t decoder_size;
  int32_t g0_grid_dim[ONTC_MAX_LEVELS];
  int32_t g1_grid_dim[ONTC_MAX_LEVELS];
  int32_t g0_bits_per_channel;
  int32_t g1_bits_per_channel;
  int32_t g0_channels;
  int32_t g1_channels;
  int32_t dim;
  int32_t mip_count;
  int32_t level_count;
  int32_t channel_count;
  int32_t channel_semantics[ONTC_MAX_CHANNELS];
  int32_t profile;
  ontc_calibration caldata;
} ontc_compressed_data;

/* openntc::TrainProgress, libopenntc.h:108-114 */
typedef struct ontc_train_progress {
  int32_t phase;
  int32_t result;
  int32_t batches_complete;
  int32_t total_batches;
} ontc_train_progress;

/* openntc::EvalResults, libopenntc.h:93-97 */
typedef struct ontc_eval_results {
  double mse;
  double psnr;
} ontc_eval_results;

/* openntc::TextureData, libopenntc.h:325-332 */
typedef struct ontc_texture_data {
  int32_t tex_count;
  int32_t mip_count;
  int32_t channels[ONTC_MAX_SOURCES];
  int32_t semantics[ONTC_MAX_SOURCES];
  uint8_t* mips[ONTC_MAX_SOURCES][ONTC_MAX_MIPS];
} ontc_texture_data;

/* Options with no upstream counterpart; zero-initialise and set what you need, then pass
 * to ontc_set_train_options after ontc_begin_training and before the first ontc_train.
 * An all-zero struct keeps upstream's schedule and the default (BF16) arithmetic. */
typedef struct ontc_train_options {
  int32_t steps_override; /* >0: total steps instead of the quality preset; lock moves to 95 % of it */
  int32_t has_lock_step;  /* !=0: use lock_step as the latent lock/snap step */
  int32_t lock_step;
  int32_t precision;      /* ONTC_PRECISION_* */
  int32_t noise_mode;     /* ONTC_NOISE_* */
  int32_t latent_adam;    /* ONTC_LATENT_ADAM_* */
  int32_t calibration;    /* ONTC_CALIBRATION_* */
  int32_t reserved;
} ontc_train_options;

/* How training completion chooses the int8 decoder's scales (same blob layout and .ntc format
 * either way).
 *   UPSTREAM (default): Calibrate's activation scales s_a = 1.1 max|activation| / 127 and
 *                       per-row max weight scales (libopenntc.cpp:445-469, 898-970).
 *   SEARCH:             the activation scales (multiples 0.8^k, k = 0..10, of upstream's) and
 *                       per-row weight scales (max, or squared-error-optimal) that minimise the
 *                       int8 decode's squared error against the training targets on a fixed
 *                       sample of up to 2^21 texels over every mip; upstream's choice is one of
 *                       the candidates.  The chosen s_a1 / s_a2 are the file's calibration. */
enum { ONTC_CALIBRATION_UPSTREAM = 0, ONTC_CALIBRATION_SEARCH = 1 };

/* How the latent Adam update of upstream (libopenntc.cpp:755-790: every latent of the step's
 * level, every step) is carried out.  Both give the same values.
 *   DEFERRED (default): only the latents a step touches are updated in the step; the
 *                       zero-gradient steps the others miss are replayed (same arithmetic)
 *                       before they are next read, in level sweeps, at the lock and before
 *                       ontc_train returns.  The next step's replays outside this step's
 *                       footprint, and this step's updates outside the next one's, run on the
 *                       private stream beside the tile kernels.
 *   DENSE:              one pass over the whole level every step. */
enum { ONTC_LATENT_ADAM_DEFERRED = 0, ONTC_LATENT_ADAM_DENSE = 1 };

/* Quantisation-noise surrogate used before the latent lock.
 *   COUNTER (default): U(-delta/2, delta/2) from a counter-based hash of (step, element),
 *                      generated only at the latents a step touches; nothing stored.
 *   UPSTREAM:          upstream's cuRAND XORWOW stream and level-wide noise buffers
 *                      (ntc_kernel.cu:412-446), for trajectory parity with upstream. */
enum { ONTC_NOISE_COUNTER = 0, ONTC_NOISE_UPSTREAM = 1 };

typedef struct ontc_context ontc_context;
typedef struct ontc_file ontc_file;
typedef struct ontc_decoder ontc_decoder;

/* ---- Context lifecycle (libopenntc.h:177-197) ---------------------------------------- */

/* Context::Context (libopenntc.cpp:271): host RNG std::mt19937(123). */
ontc_context* ontc_create(void);
/* Context::~Context + Destroy (libopenntc.cpp:1443) */
void ontc_destroy(ontc_context* ctx);
/* Context::Init (libopenntc.cpp:280).  `stream` is a cudaStream_t (NULL: a private stream). */
int ontc_init(ontc_context* ctx, int32_t profile, void* stream);
/* No upstream counterpart: lowers the manifest's minimum texture size (upstream fixes it
 * at 1024, libopenntc.h:171) to any power of two >= 16.  Call before ontc_load_manifest. */
int ontc_set_min_dimension(ontc_context* ctx, int32_t dim);
/* Context::LoadManifest (libopenntc.cpp:1125) */
int ontc_load_manifest(ontc_context* ctx, const char* path);
/* Context::UnloadManifest (libopenntc.cpp:1369) */
void ontc_unload_manifest(ontc_context* ctx);
/* Context::BeginTraining (libopenntc.cpp:471) */
void ontc_begin_training(ontc_context* ctx, int32_t quality, int32_t grids_per_batch);
/* No upstream counterpart (upstream sets these only through Quality). */
int ontc_set_train_options(ontc_context* ctx, const ontc_train_options* opts);
/* Context::Train (libopenntc.cpp:536) */
void ontc_train(ontc_context* ctx, int32_t num_batches, ontc_train_progress* out);
/* Context::TrainUntilComplete (libopenntc.cpp:529) */
void ontc_train_until_complete(ontc_context* ctx, ontc_train_progress* out);
/* No upstream counterpart (the batch entry point for many materials; it generalises upstream's
 * grids_per_batch_, libopenntc.h:162): advances each of the n contexts by up to num_batches
 * steps as n ontc_train calls would.  BF16 contexts (at most 16 of each profile) run in lock
 * step and share one tile-kernel launch per profile and step, its SMs split among them by
 * per-lod costs that a first autotuning pass measures and caches (ontc_debug_tile_costs);
 * otherwise the contexts' step chunks are enqueued in turn so that their kernels overlap on
 * the GPU (give each context its own stream).  out[i] receives context i's progress; returns
 * ONTC_SUCCESS or the first failing context's result.  A context may appear only once. */
int ontc_train_batch(ontc_context* const* ctxs, int32_t n, int32_t num_batches, ontc_train_progress* out);

/* Context::Eval (libopenntc.cpp:972).  FP64 reduction. */
void ontc_eval(ontc_context* ctx, ontc_eval_results* out);
/* No upstream counterpart: the PSNR of the shipping int8 decode (ontc_decode at every texel
 * centre of every mip, lod = the mip) against the training targets, with Eval's weighting and
 * arithmetic (fp32 residual of target / 255, fp64 sums).  Only after training completes;
 * failures set the sticky error (ontc_get_last_error) and return zeros, as ontc_eval does. */
void ontc_eval_decoded(ontc_context* ctx, ontc_eval_results* out);
/* Context::Calibrate (libopenntc.cpp:898) */
void ontc_calibrate(ontc_context* ctx, float headroom, ontc_calibration* out);
/* Context::GetCompressedData (libopenntc.cpp:1055) */
void ontc_get_compressed_data(ontc_context* ctx, ontc_compressed_data* out);
/* Context::GetTextureData (libopenntc.cpp:1425) */
void ontc_get_texture_data(ontc_context* ctx, ontc_texture_data* out);
/* Context::GetMipDim (libopenntc.cpp:1495) */
int32_t ontc_get_mip_dim(ontc_context* ctx, int32_t mip);
/* Context::FeatureLevelForLod (libopenntc.cpp:881) */
int32_t ontc_feature_level_for_lod(ontc_context* ctx, int32_t lod);
/* Context::GetLastError (libopenntc.cpp:893) */
int ontc_get_last_error(ontc_context* ctx);
/* GetStepsForQuality (libopenntc.cpp:428) */
int32_t ontc_steps_for_quality(int32_t quality);
/* Mean loss (sum of squared residuals / (C*B)) of the last `n` completed steps, FP64;
 * upstream computes this per step and discards it (libopenntc.cpp:662-663). */
int ontc_get_step_losses(ontc_context* ctx, double* out, int32_t n);

/* ---- Runtime (openntc_runtime.h:55-150) ---------------------------------------------- */

/* FillNTCConstants (openntc_runtime.cpp:156) */
void ontc_fill_constants(const ontc_compressed_data* data, ontc_constants* out);
/* Dump (openntc_runtime.cpp:179): writes the ONTC container. */
int ontc_dump(const char* path, const ontc_compressed_data* data);
/* Load (openntc_runtime.cpp:307) + FileData (openntc_runtime.h:131-150).  On success *file
 * owns the bytes `out` points into; release with ontc_file_free even on failure. */
int ontc_load(const char* path, ontc_file** file, ontc_compressed_data* out);
void ontc_file_free(ontc_file* file);
/* ProfileToString / ProfileFromString / SemanticToString / SemanticFromName /
 * GetChannelCountForSemantic (openntc_runtime.cpp:20-154) */
const char* ontc_profile_to_string(int32_t profile);
int ontc_profile_from_string(const char* s, int32_t* out_profile);
const char* ontc_semantic_to_string(int32_t semantic);
int32_t ontc_semantic_from_name(const char* name);
int32_t ontc_channel_count_for_semantic(int32_t semantic);

/* ---- Decode: SampleMaterial over a batch (ntc_decode.hlsli:605-623) --------------------
 * Upstream decodes in HLSL only (one sample per shader invocation, DP4A or cooperative
 * vectors).  Here a decoder holds one compressed material on the device and evaluates batches
 * of samples with upstream's integer arithmetic: packed latents -> int8 features -> int8 MLP
 * with per-row weight scales and per-layer activation scales -> saturate to [0, 1]. */

/* Uploads `data` (per-level packed pyramids, int8 decoder blob, NTCConstants from
 * ontc_fill_constants) to the current device.  mode: ONTC_DECODE_INT8.  stream: the
 * cudaStream_t decodes run on (NULL = legacy default stream).  The data may be freed after
 * the call.  Returns ONTC_INVALID_FILE when the data does not match its profile's shapes. */
int ontc_decoder_create(const ontc_compressed_data* data, int32_t mode, void* stream, ontc_decoder** out);
void ontc_decoder_destroy(ontc_decoder* dec);
/* Decodes n samples from DEVICE buffers: d_uv [n][2] f32, d_lod [n] i32 (clamped to the mip
 * range as upstream does), into d_out [n][channel_count] f32.  Enqueued on the decoder's
 * stream; returns once enqueued. */
int ontc_decode(ontc_decoder* dec, const float* d_uv, const int32_t* d_lod, int64_t n, float* d_out);
/* The same from HOST buffers: copies in, decodes, copies out, and returns when done.  Works in
 * chunks of 2^20 samples over three internal streams, so one chunk's copy in, another's decode
 * and a third's copy out overlap (with pinned host buffers; pageable ones work, without the
 * overlap); the decoder keeps 3 x 2^20 samples of device staging from the first call on. */
int ontc_decode_host(ontc_decoder* dec, const float* uv, const int32_t* lod, int64_t n, float* out);
/* Waits for the decoder's stream; ONTC_CUDA_FAILURE if a decode failed or timed out. */
int ontc_decoder_status(ontc_decoder* dec);

/* No upstream counterpart: a decoder of a trained context's float model (mode ONTC_DECODE_FP32,
 * BF16 or FP8): the packed latents of ontc_get_compressed_data with the context's fp32 decoder
 * weights in place of the int8 blob (FP8: the calibration maxima give the activation scales).
 * The context must have completed training; the decoder does not keep a reference to it.
 * ontc_decode and ontc_decode_host work as for the int8 decoder (outputs saturated);
 * ontc_decode_material and ontc_sample_screen return ONTC_INVALID_STATE for it. */
int ontc_decoder_create_float(ontc_context* ctx, int32_t mode, void* stream, ontc_decoder** out);

/* MaterialParams (ntc_decode.hlsli:507-522), 72 bytes, filled as DecodeMaterial (:544-603)
 * does: every field starts at DefaultMaterialParams (:524-540) (albedo 0.5, alpha 1,
 * displacement 0.5, emissive 0, gloss 0, metallic 0, normal (0.5, 0.5, 1), ao 1, roughness 1,
 * specular 0.5, transmission 0); channel i < channel_count writes its saturated output into
 * the field of its semantic (the k-th channel of a run of equal semantics into component k of
 * a vector field; components past the third, undefined in the HLSL, are dropped, as are
 * channels of semantic None), and `present`
 * gets bit (1 << semantic) for every such channel. */
typedef struct ontc_material_params {
  float albedo[3];
  float alpha;
  float displacement;
  float emissive;
  float gloss;
  float metallic;
  float normal[3];
  float ao;
  float roughness;
  float specular[3];
  float transmission;
  uint32_t present;
} ontc_material_params;

/* SampleMaterial with its DecodeMaterial step (ntc_decode.hlsli:605-623): n samples from DEVICE
 * buffers d_uv [n][2], d_lod [n] into d_params [n].  Enqueued on the decoder's stream. */
int ontc_decode_material(ontc_decoder* dec, const float* d_uv, const int32_t* d_lod, int64_t n,
                         ontc_material_params* d_params);

/* Flags of ontc_sample_screen. */
enum {
  ONTC_SCREEN_DISCARD_OUTSIDE = 1, /* pixels whose uv has a component outside [0, 1] are left
                                      unwritten (flat_ntc.hlsl:76-77) */
  ONTC_SCREEN_MATERIAL = 2         /* d_out is ontc_material_params [height][width] instead of
                                      f32 [height][width][channel_count] */
};

/* Screen-space sampling, the NTC pixel shaders' sampling (flat_ntc.hlsl:78-84,
 * pbr_ntc.hlsl:96-104) over a uv image: d_uv [height][width][2] f32 holds each pixel's
 * interpolated uv (unjittered, row 0 at the top).  Per pixel:
 *   - ComputeLod (ntc_decode.hlsli:152-168): ddx/ddy of uv as HLSL's ddx/ddy (coarse
 *     derivatives): over the pixel's 2x2 quad, ddx = uv(x0+1, y0) - uv(x0, y0) and
 *     ddy = uv(x0, y0+1) - uv(x0, y0) with (x0, y0) the quad's top-left pixel; where the quad
 *     is cut by an odd width or height the missing neighbour is replaced by the backward
 *     difference (uv(x0, y0) - uv(x0-1, y0)), and by 0 in a 1-pixel dimension;
 *   - noise position = pixel centre (x + 0.5, y + 0.5) + 5.588238 * noise_frame
 *     (flat_ntc.hlsl:82);
 *   - StochasticFilterLod and StochasticFilterUv (:172-185) with InterleavedGradientNoise
 *     (:143-146), then SampleMaterial at the jittered uv and the chosen lod.
 * Every float step is one IEEE round-to-nearest operation in the order written in the HLSL
 * (no fused multiply-add); log2 is CUDA's log2f (within 1 ulp), so the lod of a pixel whose
 * noise value lies within a few ulps of the lod's fraction may differ from an exactly rounded
 * log2 by one.  flags: ONTC_SCREEN_*.  Enqueued on the decoder's stream. */
int ontc_sample_screen(ontc_decoder* dec, const float* d_uv, int32_t width, int32_t height, float noise_frame,
                       int32_t flags, void* d_out);

/* ---- Library facts and kernel timing (no upstream counterpart) ------------------------- */

/* Number of kernel launches this context issued so far (all of them are libontc's own). */
int64_t ontc_kernel_launch_count(ontc_context* ctx);
/* Texels trained so far by this context: the sum over launched steps of grids x min(mip, 256)^2
 * for the step's drawn lod (a step whose mip is smaller than 256^2 trains fewer texels). */
int64_t ontc_texels_trained(ontc_context* ctx);

/* Kernel classes timed by ontc_profile_kernels. */
enum {
  ONTC_KCLASS_UNITS_FP32 = 0, /* fused gather/MLP/backward/scatter tile kernel, fp32 SIMT */
  ONTC_KCLASS_UNITS_BF16 = 1, /* the same, tcgen05 bf16 */
  ONTC_KCLASS_ADAM = 2,       /* fused decoder + latent Adam / clamp / gradient-zero pass */
  ONTC_KCLASS_CATCHUP = 3,    /* deferred optimiser: footprint catch-up and level sweeps */
  ONTC_KCLASS_SIDE_CATCHUP = 4, /* the next step's catch-up, on the side stream beside a tile kernel */
  ONTC_KCLASS_SIDE_UPDATE = 5,  /* kept for the numbering: the whole footprint update now runs in
                                  ONTC_KCLASS_ADAM, so no launch falls in this class */
  ONTC_KCLASS_UNITS_BF16X3 = 6, /* the tile kernel, tcgen05 split-bf16 (BF16X3) */
  ONTC_KCLASS_COUNT = 7
};
typedef struct ontc_kernel_time {
  int64_t launches;
  double total_ms; /* sum of CUDA-event durations on the stream the launches ran on (side-stream
                      spans overlap the tile kernels they run beside) */
  double bytes;    /* algorithmic DRAM bytes of those launches */
  double flops;    /* algorithmic flops of those launches */
} ontc_kernel_time;
/* Enables (1) or disables (0) event timing of every training-step launch and clears the record. */
int ontc_profile_kernels(ontc_context* ctx, int32_t enable);
/* Totals per class since the last ontc_profile_kernels; returns the number of classes written. */
int ontc_kernel_times(ontc_context* ctx, ontc_kernel_time* out, int32_t max_classes);
/* Version string of the build ("ontc <git-describe> sm_100a"). */
const char* ontc_version(void);

/* ---- Mip reduction without device allocation (no upstream counterpart) -------------------
 * One Lanczos-3 2x reduction (the arithmetic of ontc_debug_lanczos_down, upstream's
 * filter_lanczos) of a DEVICE image d_src [dim][dim][ch] u8 into d_dst [dim/2][dim/2][ch],
 * enqueued on `stream` (a cudaStream_t; NULL = legacy default stream) without allocating
 * device memory: for callers whose device memory belongs to their own pool, or that must not
 * stall other streams (cudaFree synchronises the device).  The fp32 intermediate,
 * dim * (dim/2) * ch floats, lives in one fixed device array per device; larger images
 * return ONTC_INVALID_DIMENSION without touching the device (limit: 1024^2 x 4 channels,
 * 2048^2 x 1).  ch 1..4.  Calls whose executions overlap (different streams, or host threads
 * without ordering) race on that array: issue them on one stream or order them.  The first
 * call on each device looks the array up (cudaGetSymbolAddress); make it before any stream
 * capture on that device.  The array is part of the library's device code, so loading
 * libontc reserves its 8 MiB on every device the library runs on, whether or not this entry
 * point is called.  Returns when the work is enqueued; ONTC_CUDA_FAILURE reports a launch
 * error of this call or a sticky error of an earlier fault on the device. */
#define ONTC_NOALLOC_SCRATCH_FLOATS 2097152
int ontc_lanczos_down_noalloc(const uint8_t* d_src, int32_t dim, int32_t ch, uint8_t* d_dst, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ONTC_H_ */
