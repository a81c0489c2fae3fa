// C ABI of the batch decoder (include/ontc.h, "Decode"): one compressed material held on the
// device, decoded with upstream's SampleMaterial arithmetic (ntc_decode.hlsli:605-623) by
// launch_decode (decode.cu).  Upstream has no batch decode API: its decode is HLSL only.
#include <algorithm>
#include <cmath>
#include <cstring>

#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <vector>

#include "kernels.h"
#include "ontc.h"
#include "ontc_debug.h"

struct ontc_decoder {
  int profile = 0;
  int mode = ONTC_DECODE_INT8;
  // float-model decoders: the fp32 weights (FP32) or the row-major bf16 / e4m3 tiles (BF16,
  // FP8) and the FP8 scales
  float* W32 = nullptr;
  void* Wq = nullptr;
  float sx = 1.0f, sw0 = 1.0f, sw1 = 1.0f, swo = 1.0f, sa1 = 1.0f, sa2 = 1.0f;
  cudaStream_t stream = nullptr;
  ontc_constants k = {};
  uint32_t* g0 = nullptr;
  uint32_t* g1 = nullptr;
  uint32_t g0_words = 0, g1_words = 0;
  uint8_t* blob = nullptr;
  int* err = nullptr;
  // ontc_decode_host's pipeline: kPipe streams, each with its own chunk of staging, so one
  // chunk's copy in, another's decode and a third's copy out run at the same time
  static constexpr int kPipe = 3;
  static constexpr int64_t kChunk = 1 << 20;  // samples per chunk
  cudaStream_t pipe[kPipe] = {};
  cudaEvent_t ev_start = nullptr;
  float* uv[kPipe] = {};
  int32_t* lod[kPipe] = {};
  float* out[kPipe] = {};
  bool staged = false;
};

namespace {

// Per-profile packing (ntc_decode.hlsli:60-86): channels, bits and the decoder blob size
// (W0 [64][Fp] | W1 [64][64] | Wout [16][64] int8, then 64 + 64 + 16 float scales).
struct ProfileShape {
  int c0, c1, b0, b1, level0_mips;
};
bool profile_shape(int p, ProfileShape& s)
{
  switch (p) {
    case ONTC_BPP_0_2: s = {8, 12, 2, 4, 4}; return true;
    case ONTC_BPP_0_5: s = {12, 20, 4, 4, 4}; return true;
    case ONTC_BPP_1_0: s = {12, 10, 2, 4, 3}; return true;
    case ONTC_BPP_2_25: s = {16, 12, 4, 4, 3}; return true;
    default: return false;
  }
}
size_t blob_bytes(const ProfileShape& s)
{
  const size_t Fp = ((4 * s.c0 + s.c1 + 13 + 15) / 16) * 16;
  return 64 * Fp + 64 * 64 + 16 * 64 + 4 * (64 + 64 + 16);
}

void release(ontc_decoder* d)
{
  cudaFree(d->g0);
  cudaFree(d->g1);
  cudaFree(d->blob);
  cudaFree(d->err);
  cudaFree(d->W32);
  cudaFree(d->Wq);
  for (int i = 0; i < ontc_decoder::kPipe; i++) {
    cudaFree(d->uv[i]);
    cudaFree(d->lod[i]);
    cudaFree(d->out[i]);
    if (d->pipe[i]) cudaStreamDestroy(d->pipe[i]);
  }
  if (d->ev_start) cudaEventDestroy(d->ev_start);
}

// The pipeline's streams and chunk buffers (kChunk samples of uv, lod and C outputs each).
int ensure_pipeline(ontc_decoder* d)
{
  if (d->staged) return ONTC_SUCCESS;
  const size_t n = ontc_decoder::kChunk, C = (size_t)d->k.channel_count;
  if (cudaEventCreateWithFlags(&d->ev_start, cudaEventDisableTiming) != cudaSuccess) return ONTC_CUDA_FAILURE;
  for (int i = 0; i < ontc_decoder::kPipe; i++) {
    if (cudaStreamCreateWithFlags(&d->pipe[i], cudaStreamNonBlocking) != cudaSuccess) return ONTC_CUDA_FAILURE;
    if (cudaMalloc(&d->uv[i], n * 2 * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d->lod[i], n * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&d->out[i], n * C * sizeof(float)) != cudaSuccess)
      return ONTC_ALLOCATION_FAILURE;
  }
  d->staged = true;
  return ONTC_SUCCESS;
}

// One pyramid, its levels at their byte offsets, into a fresh device buffer.
int upload_pyramid(uint32_t* const* levels, const size_t* sizes, const size_t* offsets, int count, size_t total,
                   uint32_t** dst, uint32_t* words)
{
  if (total == 0 || total % 4 != 0 || total / 4 > 0xFFFFFFFFull) return ONTC_INVALID_FILE;
  for (int l = 0; l < count; l++)
    if (!levels[l] || offsets[l] % 4 != 0 || offsets[l] + sizes[l] > total) return ONTC_INVALID_FILE;
  if (cudaMalloc(dst, total) != cudaSuccess) return ONTC_ALLOCATION_FAILURE;
  if (cudaMemset(*dst, 0, total) != cudaSuccess) return ONTC_CUDA_FAILURE;
  for (int l = 0; l < count; l++)
    if (cudaMemcpy(reinterpret_cast<uint8_t*>(*dst) + offsets[l], levels[l], sizes[l], cudaMemcpyHostToDevice) !=
        cudaSuccess)
      return ONTC_CUDA_FAILURE;
  *words = (uint32_t)(total / 4);
  return ONTC_SUCCESS;
}

ontc::DecodeArgs base_args(const ontc_decoder* d)
{
  ontc::DecodeArgs a;
  a.g0 = d->g0;
  a.g1 = d->g1;
  a.g0_words = d->g0_words;
  a.g1_words = d->g1_words;
  a.blob = d->blob;
  a.k = d->k;
  a.err = d->err;
  return a;
}

// DecodeMaterial (ntc_decode.hlsli:544-603) as a table: the ontc_material_params float each
// channel writes (-1: none) and the `present` bits.  Field offsets: albedo 0-2, alpha 3,
// displacement 4, emissive 5, gloss 6, metallic 7, normal 8-10, ao 11, roughness 12,
// specular 13-15, transmission 16.
void material_table(const ontc_constants& k, ontc::DecodeArgs& a)
{
  static_assert(sizeof(ontc_material_params) == 18 * 4, "MaterialParams is 18 words");
  a.material = true;
  a.material_present = 0;
  uint32_t prev = 0;  // Semantic::None
  int comp = 0;
  for (int i = 0; i < 16; i++) {
    a.material_dst[i] = -1;
    if (i >= k.channel_count) continue;
    const uint32_t sem = k.channel_semantics[i];
    comp = sem == prev ? comp + 1 : 0;
    prev = sem;
    a.material_present |= 1u << (sem & 31u);  // HLSL shifts by the low 5 bits
    const auto vec = [&](int base) { return comp < 3 ? base + comp : -1; };
    switch (sem) {
      case 1: a.material_dst[i] = (int8_t)vec(0); break;  // Albedo
      case 2: a.material_dst[i] = 3; break;               // Alpha
      case 3: a.material_dst[i] = 4; break;               // Displacement
      case 4: a.material_dst[i] = 5; break;               // Emissive
      case 5: a.material_dst[i] = 6; break;               // Gloss
      case 6: a.material_dst[i] = 7; break;               // Metallic
      case 7: a.material_dst[i] = (int8_t)vec(8); break;  // Normal
      case 8: a.material_dst[i] = 11; break;              // AO
      case 9: a.material_dst[i] = 12; break;              // Roughness
      case 10: a.material_dst[i] = (int8_t)vec(13); break;  // Specular
      case 11: a.material_dst[i] = 16; break;             // Transmission
      default: break;
    }
  }
}

int launch(const ontc_decoder* d, const ontc::DecodeArgs& a)
{
  return ontc::launch_decode(d->profile, a, d->stream) == cudaSuccess ? ONTC_SUCCESS : ONTC_CUDA_FAILURE;
}

// A list decode on `stream` in the decoder's mode (int8 blob or float model).
cudaError_t launch_list(const ontc_decoder* d, const float* uv, const int32_t* lod, int64_t n, float* out,
                        cudaStream_t stream)
{
  if (d->mode == ONTC_DECODE_INT8) {
    ontc::DecodeArgs a = base_args(d);
    a.uv = uv;
    a.lod = lod;
    a.n = n;
    a.out = out;
    return ontc::launch_decode(d->profile, a, stream);
  }
  ontc::FloatDecodeArgs a;
  a.g0 = d->g0;
  a.g1 = d->g1;
  a.g0_words = d->g0_words;
  a.g1_words = d->g1_words;
  a.k = d->k;
  a.W = d->W32;
  a.Wq = d->Wq;
  a.sx = d->sx;
  a.sw0 = d->sw0;
  a.sw1 = d->sw1;
  a.swo = d->swo;
  a.sa1 = d->sa1;
  a.sa2 = d->sa2;
  a.uv = uv;
  a.lod = lod;
  a.n = n;
  a.out = out;
  a.err = d->err;
  return ontc::launch_decode_float(d->profile, d->mode, a, stream);
}

float max_abs(const float* w, int n)
{
  float m = 0.0f;
  for (int i = 0; i < n; i++) m = std::max(m, std::fabs(w[i]));
  return m;
}

}  // namespace

namespace ontc {

int decoder_set_float(ontc_decoder* d, int mode, const float* W, int F, int C, const ontc_calibration& cal)
{
  if (!d || !W || (mode != ONTC_DECODE_FP32 && mode != ONTC_DECODE_BF16 && mode != ONTC_DECODE_FP8))
    return ONTC_INVALID_STATE;
  const int H = 64, nW = H * F + H * H + 16 * H;
  // Wout rows past the channel count are not trained (libopenntc.cpp:722-754): zero them
  std::vector<float> w(W, W + nW);
  for (int i = wo_off(F) + C * H; i < nW; i++) w[i] = 0.0f;
  d->mode = mode;
  if (mode == ONTC_DECODE_FP32) {
    if (cudaMalloc(&d->W32, nW * sizeof(float)) != cudaSuccess) return ONTC_ALLOCATION_FAILURE;
    return cudaMemcpy(d->W32, w.data(), nW * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess
               ? ONTC_SUCCESS
               : ONTC_CUDA_FAILURE;
  }
  // row-major W0 [64][Kp] (zero past F) | W1 [64][64] | Wout [16][64]
  const int Kp = float_decode_kp(d->profile);
  if (Kp < F) return ONTC_INVALID_STATE;
  std::vector<float> rows((size_t)H * Kp + H * H + 16 * H, 0.0f);
  for (int r = 0; r < H; r++)
    for (int c = 0; c < F; c++) rows[(size_t)r * Kp + c] = w[(size_t)r * F + c];
  std::copy(w.begin() + w1_off(F), w.end(), rows.begin() + (size_t)H * Kp);
  const float* W0 = rows.data();
  const float* W1 = W0 + H * Kp;
  const float* Wo = W1 + H * H;
  std::vector<uint8_t> bytes;
  if (mode == ONTC_DECODE_BF16) {
    bytes.resize(rows.size() * 2);
    for (size_t i = 0; i < rows.size(); i++) {
      const __nv_bfloat16 b = __float2bfloat16_rn(rows[i]);
      memcpy(&bytes[2 * i], &b, 2);
    }
  } else {
    // per-layer scales: weights at max|W| / 448 (e4m3's largest finite value), features x 256
    // (they lie in [-1, 1]), activations at Calibrate's max |hardgelu| / 448
    auto scale = [](float m) { return m > 0.0f ? m / 448.0f : 1.0f; };
    d->sw0 = scale(max_abs(W0, H * Kp));
    d->sw1 = scale(max_abs(W1, H * H));
    d->swo = scale(max_abs(Wo, 16 * H));
    d->sx = 1.0f / 256.0f;
    d->sa1 = scale(cal.max_abs_a1);
    d->sa2 = scale(cal.max_abs_a2);
    bytes.resize(rows.size());
    for (size_t i = 0; i < rows.size(); i++) {
      const float s = i < (size_t)H * Kp ? d->sw0 : (i < (size_t)H * Kp + H * H ? d->sw1 : d->swo);
      bytes[i] = (uint8_t)__nv_cvt_float_to_fp8(rows[i] / s, __NV_SATFINITE, __NV_E4M3);
    }
  }
  if (cudaMalloc(&d->Wq, bytes.size()) != cudaSuccess) return ONTC_ALLOCATION_FAILURE;
  return cudaMemcpy(d->Wq, bytes.data(), bytes.size(), cudaMemcpyHostToDevice) == cudaSuccess ? ONTC_SUCCESS
                                                                                             : ONTC_CUDA_FAILURE;
}

int decoder_set_weights(ontc_decoder* d, const uint8_t* blob, size_t size, float s_a1, float s_a2)
{
  ProfileShape ps;
  if (!d || !blob || !profile_shape(d->profile, ps) || size != blob_bytes(ps)) return ONTC_INVALID_STATE;
  if (cudaStreamSynchronize(d->stream) != cudaSuccess ||
      cudaMemcpy(d->blob, blob, size, cudaMemcpyHostToDevice) != cudaSuccess)
    return ONTC_CUDA_FAILURE;
  d->k.rcp_s_a1 = 1.0f / s_a1;  // as FillNTCConstants forms them (openntc_runtime.cpp)
  d->k.rcp_s_a2 = 1.0f / s_a2;
  return ONTC_SUCCESS;
}

}  // namespace ontc

extern "C" {

int ontc_decoder_create(const ontc_compressed_data* data, int32_t mode, void* stream, ontc_decoder** out)
{
  if (!out) return ONTC_INVALID_STATE;
  *out = nullptr;
  if (!data || mode != ONTC_DECODE_INT8) return ONTC_INVALID_STATE;
  ProfileShape ps;
  if (!profile_shape(data->profile, ps)) return ONTC_INVALID_FILE;
  if (data->g0_channels != ps.c0 || data->g1_channels != ps.c1 || data->g0_bits_per_channel != ps.b0 ||
      data->g1_bits_per_channel != ps.b1 || data->level_count < 1 || data->level_count > ONTC_MAX_LEVELS ||
      data->channel_count < 1 || data->channel_count > ONTC_MAX_CHANNELS || data->mip_count < 1 ||
      data->mip_count > ONTC_MAX_MIPS || !data->decoder || data->decoder_size < blob_bytes(ps))
    return ONTC_INVALID_FILE;
  // every lod the decoder can be asked for (clamped to the mip range) must have its feature
  // level, with non-empty power-of-two grids (FeatureLevelForLod, ntc_decode.hlsli:127-133)
  const int last = data->mip_count - 1;
  const int top = last < ps.level0_mips ? 0 : 1 + (last - ps.level0_mips) / 2;
  if (top >= data->level_count) return ONTC_INVALID_FILE;
  for (int l = 0; l <= top; l++) {
    const int a = data->g0_grid_dim[l], b = data->g1_grid_dim[l];
    if (a < 1 || b < 1 || (a & (a - 1)) || (b & (b - 1))) return ONTC_INVALID_FILE;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ONTC_CUDA_FAILURE;
  ontc_decoder* d = new ontc_decoder();
  d->profile = data->profile;
  d->stream = static_cast<cudaStream_t>(stream);
  ontc_fill_constants(data, &d->k);
  int r = upload_pyramid(data->g0, data->g0_size, data->g0_offset, data->level_count, data->g0_total_size, &d->g0,
                         &d->g0_words);
  if (r == ONTC_SUCCESS)
    r = upload_pyramid(data->g1, data->g1_size, data->g1_offset, data->level_count, data->g1_total_size, &d->g1,
                       &d->g1_words);
  if (r == ONTC_SUCCESS) {
    if (cudaMalloc(&d->blob, data->decoder_size) != cudaSuccess || cudaMalloc(&d->err, sizeof(int)) != cudaSuccess)
      r = ONTC_ALLOCATION_FAILURE;
    else if (cudaMemcpy(d->blob, data->decoder, data->decoder_size, cudaMemcpyHostToDevice) != cudaSuccess ||
             cudaMemset(d->err, 0, sizeof(int)) != cudaSuccess)
      r = ONTC_CUDA_FAILURE;
  }
  if (r != ONTC_SUCCESS) {
    release(d);
    delete d;
    return r;
  }
  *out = d;
  return ONTC_SUCCESS;
}

void ontc_decoder_destroy(ontc_decoder* d)
{
  if (!d) return;
  cudaStreamSynchronize(d->stream);
  release(d);
  delete d;
}

int ontc_debug_decode_features(ontc_decoder* d, const float* d_uv, const int32_t* d_lod, int64_t n, int8_t* d_out)
{
  if (!d || d->mode != ONTC_DECODE_INT8 || n < 0 || (n > 0 && (!d_uv || !d_lod || !d_out))) return ONTC_INVALID_STATE;
  if (n == 0) return ONTC_SUCCESS;
  float* outs = nullptr;  // the decoded channels, discarded
  if (cudaMalloc(&outs, (size_t)n * d->k.channel_count * sizeof(float)) != cudaSuccess) return ONTC_ALLOCATION_FAILURE;
  cudaError_t e = cudaMemsetAsync(d_out, 0, (size_t)n * 96, d->stream);
  if (!e) {
    ontc::DecodeArgs a = base_args(d);
    a.uv = d_uv;
    a.lod = d_lod;
    a.n = n;
    a.out = outs;
    a.feat_out = reinterpret_cast<uint32_t*>(d_out);
    e = ontc::launch_decode(d->profile, a, d->stream);
  }
  if (!e) e = cudaStreamSynchronize(d->stream);
  cudaFree(outs);
  return e == cudaSuccess ? ONTC_SUCCESS : ONTC_CUDA_FAILURE;
}

int ontc_decode(ontc_decoder* d, const float* d_uv, const int32_t* d_lod, int64_t n, float* d_out)
{
  if (!d || n < 0 || (n > 0 && (!d_uv || !d_lod || !d_out))) return ONTC_INVALID_STATE;
  return launch_list(d, d_uv, d_lod, n, d_out, d->stream) == cudaSuccess ? ONTC_SUCCESS : ONTC_CUDA_FAILURE;
}

int ontc_decode_material(ontc_decoder* d, const float* d_uv, const int32_t* d_lod, int64_t n,
                         ontc_material_params* d_params)
{
  if (!d || n < 0 || (n > 0 && (!d_uv || !d_lod || !d_params))) return ONTC_INVALID_STATE;
  if (d->mode != ONTC_DECODE_INT8 || reinterpret_cast<uintptr_t>(d_params) % 8 != 0) return ONTC_INVALID_STATE;
  ontc::DecodeArgs a = base_args(d);
  a.uv = d_uv;
  a.lod = d_lod;
  a.n = n;
  a.out = reinterpret_cast<float*>(d_params);
  material_table(d->k, a);
  return launch(d, a);
}

int ontc_sample_screen(ontc_decoder* d, const float* d_uv, int32_t width, int32_t height, float noise_frame,
                       int32_t flags, void* d_out)
{
  if (!d || d->mode != ONTC_DECODE_INT8 || width < 0 || height < 0 ||
      (flags & ~(ONTC_SCREEN_DISCARD_OUTSIDE | ONTC_SCREEN_MATERIAL)))
    return ONTC_INVALID_STATE;
  if (width == 0 || height == 0) return ONTC_SUCCESS;
  if (!d_uv || !d_out || reinterpret_cast<uintptr_t>(d_uv) % 8 != 0 ||
      ((flags & ONTC_SCREEN_MATERIAL) && reinterpret_cast<uintptr_t>(d_out) % 8 != 0))
    return ONTC_INVALID_STATE;
  ontc::DecodeArgs a = base_args(d);
  a.uv = d_uv;
  a.lod = nullptr;
  a.n = (int64_t)width * height;
  a.out = static_cast<float*>(d_out);
  a.screen_w = width;
  a.screen_h = height;
  a.noise_frame = noise_frame;
  a.discard_outside = (flags & ONTC_SCREEN_DISCARD_OUTSIDE) != 0;
  if (flags & ONTC_SCREEN_MATERIAL) material_table(d->k, a);
  return launch(d, a);
}

int ontc_decoder_status(ontc_decoder* d)
{
  if (!d) return ONTC_INVALID_STATE;
  int err = 0;
  if (cudaStreamSynchronize(d->stream) != cudaSuccess ||
      cudaMemcpy(&err, d->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return ONTC_CUDA_FAILURE;
  return err ? ONTC_CUDA_FAILURE : ONTC_SUCCESS;
}

int ontc_decode_host(ontc_decoder* d, const float* uv, const int32_t* lod, int64_t n, float* out)
{
  if (!d || n < 0 || (n > 0 && (!uv || !lod || !out))) return ONTC_INVALID_STATE;
  if (n == 0) return ONTC_SUCCESS;
  int r = ensure_pipeline(d);
  if (r != ONTC_SUCCESS) return r;
  const int C = d->k.channel_count;
  // the chunks start after whatever the caller enqueued on the decoder's stream before
  cudaError_t e = cudaEventRecord(d->ev_start, d->stream);
  for (int i = 0; i < ontc_decoder::kPipe && !e; i++) e = cudaStreamWaitEvent(d->pipe[i], d->ev_start, 0);
  // chunk j on stream j % kPipe: in, decode, out; a stream reuses its buffers only after its
  // previous chunk's copy out (stream order).  Host buffers in pinned memory let the copies
  // of different chunks overlap each other and the decodes.
  for (int64_t j0 = 0, j = 0; j0 < n && !e; j0 += ontc_decoder::kChunk, j++) {
    const int p = (int)(j % ontc_decoder::kPipe);
    const int64_t m = std::min<int64_t>(ontc_decoder::kChunk, n - j0);
    e = cudaMemcpyAsync(d->uv[p], uv + 2 * j0, (size_t)m * 2 * sizeof(float), cudaMemcpyHostToDevice, d->pipe[p]);
    if (!e) e = cudaMemcpyAsync(d->lod[p], lod + j0, (size_t)m * sizeof(int32_t), cudaMemcpyHostToDevice, d->pipe[p]);
    if (!e) e = launch_list(d, d->uv[p], d->lod[p], m, d->out[p], d->pipe[p]);
    if (!e)
      e = cudaMemcpyAsync(out + j0 * C, d->out[p], (size_t)m * C * sizeof(float), cudaMemcpyDeviceToHost, d->pipe[p]);
  }
  for (int i = 0; i < ontc_decoder::kPipe; i++)
    if (cudaStreamSynchronize(d->pipe[i]) != cudaSuccess) e = cudaErrorUnknown;
  if (e) return ONTC_CUDA_FAILURE;
  return ontc_decoder_status(d);
}

}  // extern "C"
