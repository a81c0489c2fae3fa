// Drop-in replacement for openntc's libopenntc/openntc_runtime.h, header-only over the C ABI
// of libontc.so (include/ontc.h).  Same namespace, type names, enum values and struct
// layouts as upstream (openntc_runtime.h:8-150), so code written against upstream's runtime
// compiles unchanged and CompressedData / NTCConstants pass to the C ABI by reference.
#pragma once

#include <cstdint>
#include <string>

#include "../ontc.h"

namespace openntc
{
enum class Profile
{
  Bpp_0_2,
  Bpp_0_5,
  Bpp_1_0,
  Bpp_2_25,

  Count
};

enum class Result
{
  Success,

  InvalidDimension,
  AllocationFailure,
  InvalidManifest,
  FileNotFound,
  InvalidFile,
  FileWriteFailure,
  InvalidState,
  CudaFailure,
};

enum class Semantic : int32_t
{
  None = 0,

  Albedo = 1,
  Alpha = 2,
  Displacement = 3,
  Emissive = 4,
  Gloss = 5,
  Metallic = 6,
  Normal = 7,
  AO = 8,
  Roughness = 9,
  Specular = 10,
  Transmission = 11,

  Count = 12,
};

constexpr int32_t kMaxMips = ONTC_MAX_MIPS;
constexpr int32_t kMaxChannels = ONTC_MAX_CHANNELS;
constexpr int32_t kMaxLevels = ONTC_MAX_LEVELS;

struct CalibrationData
{
  float max_abs_a1_;
  float max_abs_a2_;
  float s_a1_;
  float s_a2_;
};

struct NTCConstants
{
  int32_t g0_grid_dim_[8];
  int32_t g1_grid_dim_[8];
  uint32_t g0_offset_[8];
  uint32_t g1_offset_[8];
  int32_t g0_bits_per_channel_;
  int32_t g1_bits_per_channel_;
  int32_t g0_channels_;
  int32_t g1_channels_;
  int32_t dim_;
  int32_t mip_count_;
  float rcp_s_a1_;
  float rcp_s_a2_;
  int32_t channel_count_;
  int32_t pad0_[3];
  uint32_t channel_semantics_[16];
};
static_assert(sizeof(NTCConstants) == 240, "HLSL cbuffer NTC layout");
static_assert(sizeof(NTCConstants) == sizeof(ontc_constants), "C ABI layout");

struct CompressedData
{
  uint32_t* g0_[kMaxLevels];
  uint32_t* g1_[kMaxLevels];
  void* decoder_;

  size_t g0_size_[kMaxLevels];
  size_t g1_size_[kMaxLevels];
  size_t g0_offset_[kMaxLevels];
  size_t g1_offset_[kMaxLevels];
  size_t g0_total_size_;
  size_t g1_total_size_;
  size_t decoder_size_;

  int g0_grid_dim_[kMaxLevels];
  int g1_grid_dim_[kMaxLevels];
  int g0_bits_per_channel_;
  int g1_bits_per_channel_;
  int g0_channels_;
  int g1_channels_;
  int dim_;
  int mip_count_;
  int level_count_;
  int channel_count_;
  Semantic channel_semantics_[kMaxChannels];

  Profile profile_;

  CalibrationData caldata_;
};
static_assert(sizeof(CompressedData) == sizeof(ontc_compressed_data), "C ABI layout");

inline const ontc_compressed_data* ToC(const CompressedData& d) { return reinterpret_cast<const ontc_compressed_data*>(&d); }

inline const char* ProfileToString(Profile p) { return ontc_profile_to_string((int32_t)p); }
inline bool ProfileFromString(const std::string& s, Profile& o_profile)
{
  int32_t p = 0;
  if (!ontc_profile_from_string(s.c_str(), &p)) return false;
  o_profile = (Profile)p;
  return true;
}
inline const char* SemanticToString(Semantic sem) { return ontc_semantic_to_string((int32_t)sem); }
inline Semantic SemanticFromName(const std::string& s) { return (Semantic)ontc_semantic_from_name(s.c_str()); }
inline int GetChannelCountForSemantic(const Semantic sem) { return ontc_channel_count_for_semantic((int32_t)sem); }

inline void FillNTCConstants(const CompressedData& data, NTCConstants& o_constants)
{
  ontc_fill_constants(ToC(data), reinterpret_cast<ontc_constants*>(&o_constants));
}

class FileData;
inline Result Dump(const std::string& path, const CompressedData& data) { return (Result)ontc_dump(path.c_str(), ToC(data)); }
inline Result Load(const std::string& path, FileData& o_data);

class FileData
{
  friend Result Load(const std::string& path, FileData& o_data);

 public:
  FileData() : data_(), file_(nullptr) {}
  ~FileData() { ontc_file_free(file_); }
  FileData(const FileData&) = delete;
  FileData& operator=(const FileData&) = delete;
  const CompressedData& Data() { return data_; }

 private:
  CompressedData data_;
  ontc_file* file_;
};

inline Result Load(const std::string& path, FileData& o_data)
{
  ontc_file_free(o_data.file_);
  o_data.file_ = nullptr;
  return (Result)ontc_load(path.c_str(), &o_data.file_, reinterpret_cast<ontc_compressed_data*>(&o_data.data_));
}

}  // namespace openntc
