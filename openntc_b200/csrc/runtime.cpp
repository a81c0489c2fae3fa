// CUDA-free runtime half of libontc: semantic/profile tables, the HLSL constant buffer,
// and the ONTC container writer/reader.
//
// The container is a byte-level interface shared with upstream (libopenntc/
// openntc_runtime.cpp:179-456), so its layout is kept exactly:
//   u32 magic 0x43544E4F ("ONTC"), u32 version 4, u32 json_bytes, u32 blob_bytes,
//   json_bytes of compact JSON (keys sorted), then the blobs g0_0..g0_{L-1},
//   g1_0..g1_{L-1}, decoder, each starting at a 256-byte-aligned offset relative to
//   the first blob byte, zero padding in between.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/ontc.h"
#include "json.h"

namespace ontc {

static const char* kSemanticNames[12] = {"None",   "Albedo",   "Alpha",  "Displacement",
                                         "Emissive", "Gloss",  "Metallic", "Normal",
                                         "AO",     "Roughness", "Specular", "Transmission"};

// Accepted manifest / container names and the semantic they select
// (openntc_runtime.cpp:53-75).
static const struct {
  const char* name;
  int32_t sem;
} kSemanticAliases[] = {
    {"Albedo", 1},     {"Diffuse", 1},   {"Alpha", 2},           {"Mask", 2},           {"AlphaMask", 2},
    {"Displ", 3},      {"Displacement", 3}, {"Emissive", 4},     {"Emission", 4},       {"Glossiness", 5},
    {"Gloss", 5},      {"Metalness", 6}, {"Metallic", 6},        {"Normal", 7},         {"Occlusion", 8},
    {"AO", 8},         {"AmbientOcclusion", 8}, {"Roughness", 9}, {"SpecularColor", 10}, {"Specular", 10},
    {"Transmission", 11},
};

// Channel count per semantic; -1 means "any" (None) or invalid (openntc_runtime.cpp:88-102).
static const int32_t kSemanticChannels[13] = {-1, 3, 1, 1, 1, 1, 1, 3, 1, 1, 3, 1, -1};

static const char* kProfileNames[4] = {"bpp_0_2", "bpp_0_5", "bpp_1_0", "bpp_2_25"};

}  // namespace ontc

using namespace ontc;

struct ontc_file {
  std::vector<uint8_t> raw;
  std::vector<uint8_t> g0_packed;
  std::vector<uint8_t> g1_packed;
};

extern "C" {

const char* ontc_semantic_to_string(int32_t sem)
{
  if (sem >= 1 && sem <= 11) return kSemanticNames[sem];
  return "None";
}

int32_t ontc_semantic_from_name(const char* name)
{
  if (!name) return 0;
  for (const auto& a : kSemanticAliases)
    if (strcmp(a.name, name) == 0) return a.sem;
  return 0;
}

int32_t ontc_channel_count_for_semantic(int32_t sem)
{
  if (sem < 0 || sem > 12) return -1;
  return kSemanticChannels[sem];
}

const char* ontc_profile_to_string(int32_t p)
{
  if (p >= 0 && p < 4) return kProfileNames[p];
  return "unknown";
}

int ontc_profile_from_string(const char* s, int32_t* out)
{
  if (!s) return 0;
  for (int i = 0; i < 4; i++)
    if (strcmp(s, kProfileNames[i]) == 0) {
      *out = i;
      return 1;
    }
  return 0;
}

void ontc_fill_constants(const ontc_compressed_data* d, ontc_constants* c)
{
  memset(c, 0, sizeof(*c));
  for (int i = 0; i < d->level_count && i < ONTC_MAX_LEVELS; i++) {
    c->g0_grid_dim[i] = d->g0_grid_dim[i];
    c->g1_grid_dim[i] = d->g1_grid_dim[i];
    c->g0_offset[i] = (uint32_t)d->g0_offset[i];
    c->g1_offset[i] = (uint32_t)d->g1_offset[i];
  }
  c->g0_bits_per_channel = d->g0_bits_per_channel;
  c->g1_bits_per_channel = d->g1_bits_per_channel;
  c->g0_channels = d->g0_channels;
  c->g1_channels = d->g1_channels;
  c->dim = d->dim;
  c->mip_count = d->mip_count;
  c->rcp_s_a1 = 1.0f / d->caldata.s_a1;
  c->rcp_s_a2 = 1.0f / d->caldata.s_a2;
  c->channel_count = d->channel_count;
  for (int i = 0; i < d->channel_count && i < ONTC_MAX_CHANNELS; i++)
    c->channel_semantics[i] = (uint32_t)d->channel_semantics[i];
}

static uint64_t round_up(uint64_t n, uint64_t k) { return ((n + k - 1) / k) * k; }

int ontc_dump(const char* path, const ontc_compressed_data* d)
{
  struct Blob {
    std::string name;
    uint64_t size;
    const void* data;
  };
  std::vector<Blob> blobs;
  int levels = d->level_count;
  if (levels < 0) levels = 0;
  if (levels > ONTC_MAX_LEVELS) levels = ONTC_MAX_LEVELS;
  for (int i = 0; i < levels; i++) blobs.push_back({"g0_" + std::to_string(i), d->g0_size[i], d->g0[i]});
  for (int i = 0; i < levels; i++) blobs.push_back({"g1_" + std::to_string(i), d->g1_size[i], d->g1[i]});
  blobs.push_back({"decoder", d->decoder_size, d->decoder});

  Json j = Json::make_object();
  Json src = Json::make_object();
  src.set("generator", Json::make_string("openntc"));
  src.set("version", Json::make_int(5));
  j.set("source", src);
  j.set("profile", Json::make_string(ontc_profile_to_string(d->profile)));
  Json sems = Json::make_array();
  for (int i = 0; i < d->channel_count; i++) sems.push_back(Json::make_string(ontc_semantic_to_string(d->channel_semantics[i])));
  j.set("channel_semantics", sems);
  j.set("dim", Json::make_int(d->dim));
  j.set("mip_count", Json::make_int(d->mip_count));
  j.set("level_count", Json::make_int(d->level_count));
  for (int g = 0; g < 2; g++) {
    Json jg = Json::make_object();
    Json dims = Json::make_array();
    const int32_t* gd = g == 0 ? d->g0_grid_dim : d->g1_grid_dim;
    for (int i = 0; i < ONTC_MAX_LEVELS; i++) dims.push_back(Json::make_int(gd[i]));
    jg.set("grid_dims", dims);
    jg.set("bits", Json::make_int(g == 0 ? d->g0_bits_per_channel : d->g1_bits_per_channel));
    jg.set("channels", Json::make_int(g == 0 ? d->g0_channels : d->g1_channels));
    j.set(g == 0 ? "g0" : "g1", jg);
  }
  Json cal = Json::make_object();
  cal.set("max_abs_a1", Json::make_float((double)d->caldata.max_abs_a1));
  cal.set("max_abs_a2", Json::make_float((double)d->caldata.max_abs_a2));
  cal.set("s_a1", Json::make_float((double)d->caldata.s_a1));
  cal.set("s_a2", Json::make_float((double)d->caldata.s_a2));
  j.set("calibration", cal);

  uint64_t off = 0;
  Json jb = Json::make_array();
  for (const Blob& b : blobs) {
    off = round_up(off, 256);
    Json e = Json::make_object();
    e.set("name", Json::make_string(b.name));
    e.set("size", Json::make_uint(b.size));
    e.set("offset", Json::make_uint(off));
    jb.push_back(e);
    off += b.size;
  }
  j.set("blobs", jb);

  std::string js = j.dump();
  uint32_t header[4] = {0x43544E4Fu, 4u, (uint32_t)js.size(), (uint32_t)off};

  std::ofstream f(path, std::ios::binary);
  if (!f) return ONTC_FILE_WRITE_FAILURE;
  f.write((const char*)header, sizeof(header));
  f.write(js.data(), (std::streamsize)js.size());
  uint64_t pos = 0;
  static const char zeros[256] = {0};
  for (const Blob& b : blobs) {
    uint64_t aligned = round_up(pos, 256);
    if (aligned > pos) f.write(zeros, (std::streamsize)(aligned - pos));
    pos = aligned;
    if (b.size) f.write((const char*)b.data, (std::streamsize)b.size);
    pos += b.size;
  }
  int res = f.good() ? ONTC_SUCCESS : ONTC_FILE_WRITE_FAILURE;
  f.close();
  return res;
}

}  // extern "C"

template <typename T>
static bool get_int(const Json& j, const char* key, T& out)
{
  const Json* v = j.find(key);
  if (!v || !v->is_integer()) return false;
  out = (T)v->as_int();
  return true;
}

static bool get_u64(const Json& j, const char* key, uint64_t& out)
{
  const Json* v = j.find(key);
  if (!v || !v->is_integer()) return false;
  out = v->as_uint();
  return true;
}

static bool get_float(const Json& j, const char* key, float& out)
{
  const Json* v = j.find(key);
  if (!v || !v->is_number()) return false;
  out = (float)v->as_double();
  return true;
}

static bool get_dims(const Json& j, const char* key, int32_t* out)
{
  const Json* v = j.find(key);
  if (!v || !v->is_array() || v->size() != ONTC_MAX_LEVELS) return false;
  for (int i = 0; i < ONTC_MAX_LEVELS; i++) {
    if (!v->at(i).is_integer()) return false;
    out[i] = (int32_t)v->at(i).as_int();
  }
  return true;
}

extern "C" {

int ontc_load(const char* path, ontc_file** file, ontc_compressed_data* out)
{
  *file = nullptr;
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return ONTC_FILE_NOT_FOUND;
  ontc_file* fd = new ontc_file();
  *file = fd;
  std::streamoff sz = f.tellg();
  if (sz < 0) return ONTC_INVALID_FILE;
  fd->raw.resize((size_t)sz);
  f.seekg(0);
  if (sz > 0) f.read((char*)fd->raw.data(), sz);
  memset(out, 0, sizeof(*out));

  const uint64_t raw_size = fd->raw.size();
  if (raw_size < 16) return ONTC_INVALID_FILE;
  uint32_t header[4];
  memcpy(header, fd->raw.data(), 16);
  if (header[0] != 0x43544E4Fu || header[1] != 4u) return ONTC_INVALID_FILE;
  const uint64_t json_size = header[2];
  const uint64_t blob_size = header[3];
  const uint64_t file_size = 16 + json_size + blob_size;
  const uint64_t blob_off = 16 + json_size;
  // Upstream trusts the header's sizes; a reader must not step past the bytes it has.
  if (blob_off > raw_size) return ONTC_INVALID_FILE;
  Json j;
  if (!Json::parse((const char*)fd->raw.data() + 16, (const char*)fd->raw.data() + blob_off, j)) return ONTC_INVALID_FILE;

  const Json* jg0 = j.find("g0");
  const Json* jg1 = j.find("g1");
  const Json* jcal = j.find("calibration");
  if (!jg0 || !jg1 || !jcal || !jg0->is_object() || !jg1->is_object() || !jcal->is_object()) return ONTC_INVALID_FILE;
  bool ok = true;
  ok &= get_dims(*jg0, "grid_dims", out->g0_grid_dim);
  ok &= get_int(*jg0, "bits", out->g0_bits_per_channel);
  ok &= get_int(*jg0, "channels", out->g0_channels);
  ok &= get_dims(*jg1, "grid_dims", out->g1_grid_dim);
  ok &= get_int(*jg1, "bits", out->g1_bits_per_channel);
  ok &= get_int(*jg1, "channels", out->g1_channels);
  ok &= get_int(j, "dim", out->dim);
  ok &= get_int(j, "mip_count", out->mip_count);
  ok &= get_int(j, "level_count", out->level_count);
  ok &= get_float(*jcal, "max_abs_a1", out->caldata.max_abs_a1);
  ok &= get_float(*jcal, "s_a1", out->caldata.s_a1);
  ok &= get_float(*jcal, "max_abs_a2", out->caldata.max_abs_a2);
  ok &= get_float(*jcal, "s_a2", out->caldata.s_a2);
  if (!ok) return ONTC_INVALID_FILE;

  const Json* jp = j.find("profile");
  if (!jp || !jp->is_string() || !ontc_profile_from_string(jp->as_string().c_str(), &out->profile)) return ONTC_INVALID_FILE;

  const Json* js = j.find("channel_semantics");
  if (!js || !js->is_array() || js->size() > ONTC_MAX_CHANNELS) return ONTC_INVALID_FILE;
  out->channel_count = (int32_t)js->size();
  for (int i = 0; i < out->channel_count; i++) {
    if (!js->at(i).is_string()) return ONTC_INVALID_FILE;
    int32_t sem = ontc_semantic_from_name(js->at(i).as_string().c_str());
    if (sem == 0) return ONTC_INVALID_FILE;
    out->channel_semantics[i] = sem;
  }

  if (out->level_count < 1 || out->level_count > ONTC_MAX_LEVELS || out->mip_count < 1 || out->mip_count > ONTC_MAX_MIPS)
    return ONTC_INVALID_FILE;

  struct Slot {
    std::string name;
    void** dst;
    size_t* size;
    bool found;
  };
  std::vector<Slot> slots;
  for (int i = 0; i < out->level_count; i++) slots.push_back({"g0_" + std::to_string(i), (void**)&out->g0[i], &out->g0_size[i], false});
  for (int i = 0; i < out->level_count; i++) slots.push_back({"g1_" + std::to_string(i), (void**)&out->g1[i], &out->g1_size[i], false});
  slots.push_back({"decoder", &out->decoder, &out->decoder_size, false});

  const Json* jb = j.find("blobs");
  if (!jb || !jb->is_array()) return ONTC_INVALID_FILE;
  for (const Json& b : jb->items()) {
    const Json* jn = b.find("name");
    uint64_t off = 0, size = 0;
    if (!jn || !jn->is_string() || !get_u64(b, "offset", off) || !get_u64(b, "size", size)) return ONTC_INVALID_FILE;
    if (blob_off + off + size > file_size || blob_off + off + size > raw_size || off > raw_size || size > raw_size)
      return ONTC_INVALID_FILE;
    for (Slot& s : slots) {
      if (jn->as_string() == s.name) {
        *s.dst = fd->raw.data() + blob_off + off;
        *s.size = (size_t)size;
        s.found = true;
      }
    }
  }
  for (const Slot& s : slots)
    if (!s.found) return ONTC_INVALID_FILE;

  out->g0_offset[0] = 0;
  out->g1_offset[0] = 0;
  for (int i = 1; i < out->level_count; i++) {
    out->g0_offset[i] = out->g0_offset[i - 1] + out->g0_size[i - 1];
    out->g1_offset[i] = out->g1_offset[i - 1] + out->g1_size[i - 1];
  }
  const int last = out->level_count - 1;
  out->g0_total_size = out->g0_offset[last] + out->g0_size[last];
  out->g1_total_size = out->g1_offset[last] + out->g1_size[last];
  // Re-pack the feature pyramids contiguously (HLSL binds one buffer per pyramid).
  fd->g0_packed.assign(out->g0_total_size + 16, 0);
  fd->g1_packed.assign(out->g1_total_size + 16, 0);
  for (int i = 0; i < out->level_count; i++) {
    if (out->g0_size[i]) memcpy(fd->g0_packed.data() + out->g0_offset[i], out->g0[i], out->g0_size[i]);
    if (out->g1_size[i]) memcpy(fd->g1_packed.data() + out->g1_offset[i], out->g1[i], out->g1_size[i]);
    out->g0[i] = (uint32_t*)(fd->g0_packed.data() + out->g0_offset[i]);
    out->g1[i] = (uint32_t*)(fd->g1_packed.data() + out->g1_offset[i]);
  }
  return ONTC_SUCCESS;
}

void ontc_file_free(ontc_file* f) { delete f; }

}  // extern "C"
