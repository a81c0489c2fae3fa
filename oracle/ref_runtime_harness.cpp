// C entry points around the upstream CUDA-free runtime (libopenntc/openntc_runtime.cpp),
// compiled from the upstream sources into oracle/_ref/libontc_ref_rt.so by oracle/Makefile.
//
// Test infrastructure only: the tests load this library to check the product's
// .ntc writer/reader and constant-buffer fill byte-for-byte against upstream.
// The struct layouts passed through void* are upstream's openntc::CompressedData
// and openntc::NTCConstants (openntc_runtime.h:69-121).
#include <cstdint>
#include <cstring>
#include <string>

#include <libopenntc/openntc_runtime.h>

using namespace openntc;

extern "C" {

int ref_rt_sizeof_compressed(void) { return (int)sizeof(CompressedData); }
int ref_rt_sizeof_constants(void) { return (int)sizeof(NTCConstants); }

// openntc_runtime.cpp:179 Dump
int ref_rt_dump(const char* path, const void* cd)
{
  return (int)Dump(std::string(path), *(const CompressedData*)cd);
}

// openntc_runtime.cpp:307 Load.  Returns an owning handle in *o_handle (free with
// ref_rt_free) and copies the loaded CompressedData into out_cd.
int ref_rt_load(const char* path, void** o_handle, void* out_cd)
{
  FileData* fd = new FileData();
  Result r = Load(std::string(path), *fd);
  *o_handle = fd;
  if (r == Result::Success)
    memcpy(out_cd, &fd->Data(), sizeof(CompressedData));
  return (int)r;
}

void ref_rt_free(void* handle) { delete (FileData*)handle; }

// openntc_runtime.cpp:156 FillNTCConstants
void ref_rt_fill_constants(const void* cd, void* out)
{
  FillNTCConstants(*(const CompressedData*)cd, *(NTCConstants*)out);
}

int ref_rt_semantic_from_name(const char* name) { return (int)SemanticFromName(std::string(name)); }
const char* ref_rt_semantic_to_string(int sem) { return SemanticToString((Semantic)sem); }
int ref_rt_channel_count(int sem) { return GetChannelCountForSemantic((Semantic)sem); }
const char* ref_rt_profile_to_string(int p) { return ProfileToString((Profile)p); }
int ref_rt_profile_from_string(const char* s, int* o)
{
  Profile p;
  bool ok = ProfileFromString(std::string(s), p);
  if (ok) *o = (int)p;
  return ok ? 1 : 0;
}

}  // extern "C"
