// Drop-in replacement for openntc's libopenntc/libopenntc.h, header-only over the C ABI of
// libontc.so (include/ontc.h).  The public surface of upstream's openntc::Context
// (libopenntc.h:168-210) is kept: the same methods, argument meanings, result codes and
// public host outputs (g0_host_, g1_host_, decoder_host_, decoder_size_, caldata_,
// mips_host_).  Upstream's private device tensors (Tensor2d/Tensor3d) have no counterpart:
// the device state lives inside libontc.
#pragma once

#include <cstdint>
#include <string>

#include "../ontc.h"
#include "openntc_runtime.h"

namespace openntc
{
struct ContextInitInfo
{
  Profile profile_;
};

struct EvalResults
{
  double mse_;
  double psnr_;
};

enum TrainPhase : int32_t
{
  ManifestLoaded = 0,
  TrainInProgress = 1,
  TrainComplete = 2,

  TrainError = -1,
};

struct TrainProgress
{
  TrainPhase phase_;
  Result result_;
  int batches_complete_;
  int total_batches_;
};

enum class Channel : int32_t
{
  R = 0,
  G = 1,
  B = 2,
  A = 3,

  Count,
  Invalid = -1
};

constexpr int32_t kMaxSources = ONTC_MAX_SOURCES;

enum class Quality
{
  Low,
  Medium,
  High,
  Ultra,

  Count
};

inline int GetStepsForQuality(Quality quality) { return ontc_steps_for_quality((int32_t)quality); }

struct TrainInfo
{
  Quality quality_;
  int grids_per_batch_;
};

struct TextureData;

class Context
{
 public:
  static const int kMinDimension = ONTC_MIN_DIMENSION;
  static const int kMaxDimension = ONTC_MAX_DIMENSION;
  static const int kMaxMips = openntc::kMaxMips;
  static const int kMaxChannels = openntc::kMaxChannels;
  static const int kMaxLevels = openntc::kMaxLevels;

  Context() : ctx_(ontc_create()) { Refresh(); }
  ~Context() { ontc_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;

  Result Init(const ContextInitInfo& init_info) { return (Result)ontc_init(ctx_, (int32_t)init_info.profile_, nullptr); }
  void Destroy()
  {
    ontc_destroy(ctx_);
    ctx_ = ontc_create();
    Refresh();
  }
  void BeginTraining(const TrainInfo& train_info)
  {
    ontc_begin_training(ctx_, (int32_t)train_info.quality_, train_info.grids_per_batch_);
  }
  TrainProgress Train(int32_t num_batches)
  {
    ontc_train_progress p;
    ontc_train(ctx_, num_batches, &p);
    Refresh();
    return TrainProgress{(TrainPhase)p.phase, (Result)p.result, p.batches_complete, p.total_batches};
  }
  TrainProgress TrainUntilComplete()
  {
    ontc_train_progress p;
    ontc_train_until_complete(ctx_, &p);
    Refresh();
    return TrainProgress{(TrainPhase)p.phase, (Result)p.result, p.batches_complete, p.total_batches};
  }
  EvalResults Eval()
  {
    ontc_eval_results r;
    ontc_eval(ctx_, &r);
    return EvalResults{r.mse, r.psnr};
  }
  Result GetLastError() const { return (Result)ontc_get_last_error(ctx_); }
  CalibrationData Calibrate(float headroom = 1.1f)
  {
    ontc_calibration c;
    ontc_calibrate(ctx_, headroom, &c);
    return CalibrationData{c.max_abs_a1, c.max_abs_a2, c.s_a1, c.s_a2};
  }
  CompressedData GetCompressedData()
  {
    CompressedData d;
    ontc_get_compressed_data(ctx_, reinterpret_cast<ontc_compressed_data*>(&d));
    return d;
  }
  Result LoadManifest(const std::string& filepath)
  {
    Result r = (Result)ontc_load_manifest(ctx_, filepath.c_str());
    Refresh();
    return r;
  }
  void UnloadManifest()
  {
    ontc_unload_manifest(ctx_);
    Refresh();
  }
  inline TextureData GetTextureData();
  int32_t GetMipDim(int mip) const { return ontc_get_mip_dim(ctx_, mip); }
  int32_t FeatureLevelForLod(int32_t mip) const { return ontc_feature_level_for_lod(ctx_, mip); }

  // Host-side outputs after training (borrowed from libontc, valid until the next
  // LoadManifest / UnloadManifest / Destroy), as upstream's public members.
  uint32_t* g0_host_[kMaxLevels];
  uint32_t* g1_host_[kMaxLevels];
  uint32_t* g0_host_packed_ = nullptr;
  uint32_t* g1_host_packed_ = nullptr;
  uint8_t* decoder_host_ = nullptr;
  size_t decoder_size_ = 0;
  CalibrationData caldata_ = {};
  uint8_t* mips_host_[kMaxSources][kMaxMips];

  // The underlying C handle (for the extensions in include/ontc.h).
  ontc_context* Handle() { return ctx_; }

 private:
  ontc_context* ctx_;

  void Refresh()
  {
    ontc_compressed_data d;
    ontc_get_compressed_data(ctx_, &d);
    for (int i = 0; i < kMaxLevels; i++) {
      g0_host_[i] = d.g0[i];
      g1_host_[i] = d.g1[i];
    }
    g0_host_packed_ = d.g0[0];
    g1_host_packed_ = d.g1[0];
    decoder_host_ = (uint8_t*)d.decoder;
    decoder_size_ = d.decoder_size;
    caldata_ = CalibrationData{d.caldata.max_abs_a1, d.caldata.max_abs_a2, d.caldata.s_a1, d.caldata.s_a2};
    ontc_texture_data t;
    ontc_get_texture_data(ctx_, &t);
    for (int s = 0; s < kMaxSources; s++)
      for (int m = 0; m < kMaxMips; m++) mips_host_[s][m] = t.mips[s][m];
  }
};

struct TextureData
{
  int32_t tex_count_;
  int32_t mip_count_;
  int32_t channels_[kMaxSources];
  Semantic semantics_[kMaxSources];
  uint8_t* mips_[kMaxSources][Context::kMaxMips];
};
static_assert(sizeof(TextureData) == sizeof(ontc_texture_data), "C ABI layout");

inline TextureData Context::GetTextureData()
{
  TextureData t;
  ontc_get_texture_data(ctx_, reinterpret_cast<ontc_texture_data*>(&t));
  return t;
}

}  // namespace openntc
