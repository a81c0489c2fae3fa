// C entry points around the upstream training library (libopenntc/libopenntc.cpp +
// ntc_kernel.cu, cuBLAS TF32, cuRAND), compiled from the upstream sources into
// oracle/_ref/libontc_ref.so by oracle/Makefile.  Runs only where a GPU exists.
//
// Test and baseline infrastructure only:
//   * parity tests read upstream's internal device tensors (latents, weights,
//     gradients, mip chain) after identical steps;
//   * bench.py's reference arm times upstream's own Context::Train.
//
// Access to upstream's private members goes through `#define private public`
// after every standard header is already included, so no layout changes.
// Upstream's Context constructor leaves manifest_loaded_/train_phase_
// uninitialised (libopenntc.cpp:271); contexts are therefore constructed in
// zero-filled storage.
#include <algorithm>
#include <atomic>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#define private public
#include <libopenntc/libopenntc.h>
#undef private
#include <libopenntc/ntc_kernel.cuh>

using namespace openntc;

extern "C" {

void* ref_create(int profile, int* o_result)
{
  void* mem = calloc(1, sizeof(Context));
  Context* ctx = new (mem) Context();
  ContextInitInfo info = {};
  info.profile_ = (Profile)profile;
  Result r = ctx->Init(info);
  if (o_result) *o_result = (int)r;
  return ctx;
}

void ref_destroy(void* p)
{
  Context* ctx = (Context*)p;
  ctx->~Context();
  free(ctx);
}

int ref_load_manifest(void* p, const char* path) { return (int)((Context*)p)->LoadManifest(std::string(path)); }

// BeginTraining (libopenntc.cpp:471).  steps_override > 0 replaces the quality's
// step count (and lock_i_ = 95 % of it, libopenntc.cpp:475); lock_override >= 0
// then replaces lock_i_.
void ref_begin_training(void* p, int quality, int grids_per_batch, int steps_override, int lock_override)
{
  Context* ctx = (Context*)p;
  TrainInfo ti = {};
  ti.quality_ = (Quality)quality;
  ti.grids_per_batch_ = grids_per_batch;
  ctx->BeginTraining(ti);
  if (steps_override > 0)
  {
    ctx->batch_count_ = steps_override;
    ctx->lock_i_ = (95 * steps_override) / 100;
  }
  if (lock_override >= 0) ctx->lock_i_ = lock_override;
}

void ref_train(void* p, int n, int32_t* o_progress)
{
  TrainProgress tp = ((Context*)p)->Train(n);
  o_progress[0] = (int32_t)tp.phase_;
  o_progress[1] = (int32_t)tp.result_;
  o_progress[2] = tp.batches_complete_;
  o_progress[3] = tp.total_batches_;
}

// Train(n) timed with CUDA events on the legacy default stream, which is where
// every upstream launch and cuBLAS call goes.
int ref_time_train(void* p, int n, float* o_ms, int32_t* o_progress)
{
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0, 0);
  TrainProgress tp = ((Context*)p)->Train(n);
  cudaEventRecord(e1, 0);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(o_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  o_progress[0] = (int32_t)tp.phase_;
  o_progress[1] = (int32_t)tp.result_;
  o_progress[2] = tp.batches_complete_;
  o_progress[3] = tp.total_batches_;
  return (int)cudaGetLastError();
}

void ref_eval(void* p, double* o)
{
  EvalResults e = ((Context*)p)->Eval();
  o[0] = e.mse_;
  o[1] = e.psnr_;
}

void ref_calibrate(void* p, float* o)
{
  CalibrationData c = ((Context*)p)->Calibrate();
  o[0] = c.max_abs_a1_;
  o[1] = c.max_abs_a2_;
  o[2] = c.s_a1_;
  o[3] = c.s_a2_;
}

void ref_get_compressed(void* p, void* out_cd)
{
  CompressedData cd = ((Context*)p)->GetCompressedData();
  memcpy(out_cd, &cd, sizeof(cd));
}

// Shape facts: [level_count, mip_count, feature_dim, feature_dim_padded, out_dim,
//               g0_dims[6], g1_dims[6], mip_dims[12], batch_i, lock_i, batch_count]
void ref_shape(void* p, int32_t* o)
{
  Context* c = (Context*)p;
  o[0] = c->level_count_;
  o[1] = c->mip_count_;
  o[2] = c->feature_dim_;
  o[3] = c->feature_dim_padded_;
  o[4] = c->out_dim_;
  for (int i = 0; i < 6; i++) o[5 + i] = i < c->level_count_ ? c->g0_grid_dim_[i] : 0;
  for (int i = 0; i < 6; i++) o[11 + i] = i < c->level_count_ ? c->g1_grid_dim_[i] : 0;
  for (int i = 0; i < 12; i++) o[17 + i] = i < c->mip_count_ ? c->mip_dim_[i] : 0;
  o[29] = c->batch_i_;
  o[30] = c->lock_i_;
  o[31] = c->batch_count_;
}

static float* tensor_ptr(Context* c, int which, int level, size_t* n)
{
  switch (which)
  {
    case 0: *n = c->g0_[level].NumElems(); return c->g0_[level].DevicePtr();
    case 1: *n = c->g1_[level].NumElems(); return c->g1_[level].DevicePtr();
    case 2: *n = c->dLdG0_[level].NumElems(); return c->dLdG0_[level].DevicePtr();
    case 3: *n = c->dLdG1_[level].NumElems(); return c->dLdG1_[level].DevicePtr();
    case 4: *n = c->mG0_[level].NumElems(); return c->mG0_[level].DevicePtr();
    case 5: *n = c->vG0_[level].NumElems(); return c->vG0_[level].DevicePtr();
    case 6: *n = c->mG1_[level].NumElems(); return c->mG1_[level].DevicePtr();
    case 7: *n = c->vG1_[level].NumElems(); return c->vG1_[level].DevicePtr();
    case 10: *n = c->W0_.NumElems(); return c->W0_.DevicePtr();
    case 11: *n = c->W1_.NumElems(); return c->W1_.DevicePtr();
    case 12: *n = c->Wout_.NumElems(); return c->Wout_.DevicePtr();
    case 13: *n = c->dLdW0_.NumElems(); return c->dLdW0_.DevicePtr();
    case 14: *n = c->dLdW1_.NumElems(); return c->dLdW1_.DevicePtr();
    case 15: *n = c->dLdWout_.NumElems(); return c->dLdWout_.DevicePtr();
    case 16: *n = c->mW0_.NumElems(); return c->mW0_.DevicePtr();
    case 17: *n = c->vW0_.NumElems(); return c->vW0_.DevicePtr();
    case 18: *n = c->g0_noise_.NumElems(); return c->g0_noise_.DevicePtr();
    case 19: *n = c->g1_noise_.NumElems(); return c->g1_noise_.DevicePtr();
    case 20: *n = c->x_.NumElems(); return c->x_.DevicePtr();      // features [F][max_batch]
    case 21: *n = c->dLdx_.NumElems(); return c->dLdx_.DevicePtr();  // feature gradient [F][max_batch]
    case 22: *n = c->Woutx_.NumElems(); return c->Woutx_.DevicePtr();  // predictions [16][max_batch]
    default: *n = 0; return nullptr;
  }
}

// Copies one internal fp32 tensor to (to_device == 0) or from (to_device == 1) host memory.
// Returns the element count, or -1 on a CUDA error / size mismatch.
long long ref_tensor(void* p, int which, int level, float* host, long long n, int to_device)
{
  size_t tn = 0;
  float* dev = tensor_ptr((Context*)p, which, level, &tn);
  if (!dev) return -1;
  if (n <= 0) return (long long)tn;
  if ((size_t)n > tn) return -1;
  cudaError_t e = to_device ? cudaMemcpy(dev, host, n * sizeof(float), cudaMemcpyHostToDevice)
                            : cudaMemcpy(host, dev, n * sizeof(float), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? (long long)n : -1;
}

// package_[mip] u8 [dim][dim][C] (libopenntc.cpp:1275, filled at :1357-1362)
int ref_package(void* p, int mip, uint8_t* host)
{
  Context* c = (Context*)p;
  size_t n = c->package_[mip].NumElems();
  return (int)cudaMemcpy(host, c->package_[mip].DevicePtr(), n, cudaMemcpyDeviceToHost);
}

// mips_host_[source][mip] (libopenntc.cpp:1331-1335)
const uint8_t* ref_mip_host(void* p, int source, int mip) { return ((Context*)p)->mips_host_[source][mip]; }

const uint8_t* ref_decoder_host(void* p, long long* size)
{
  *size = (long long)((Context*)p)->decoder_size_;
  return ((Context*)p)->decoder_host_;
}

// ntc_kernel.cu:486 quantize_pack on an arbitrary host float array.
int ref_quantize_pack(const float* host_in, long long n, int bits, uint32_t* host_out)
{
  float* din = nullptr;
  uint32_t* dout = nullptr;
  long long n_packs = (n * bits) / 32;
  if (cudaMalloc(&din, n * sizeof(float)) != cudaSuccess) return -1;
  if (cudaMalloc(&dout, n_packs * sizeof(uint32_t)) != cudaSuccess) return -1;
  cudaMemcpy(din, host_in, n * sizeof(float), cudaMemcpyHostToDevice);
  launch_quantize_pack((int)n, (int)n_packs, bits, din, dout);
  cudaError_t e = cudaMemcpy(host_out, dout, n_packs * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(din);
  cudaFree(dout);
  return (int)e;
}

// ntc_kernel.cu:638 launch_filter_lanczos (a = 3): one 2x downsample of a
// [dim][dim][c] u8 image into [dim/2][dim/2][c].
int ref_filter_lanczos(const uint8_t* src, int dim_src, int c, uint8_t* dst)
{
  uint8_t *dsrc = nullptr, *ddst = nullptr;
  float* tmp = nullptr;
  size_t ns = (size_t)dim_src * dim_src * c;
  size_t nd = ns / 4;
  cudaMalloc(&dsrc, ns);
  cudaMalloc(&ddst, nd);
  cudaMalloc(&tmp, ns / 2 * sizeof(float));
  cudaMemcpy(dsrc, src, ns, cudaMemcpyHostToDevice);
  launch_filter_lanczos(dim_src, c, 3, dsrc, tmp, ddst);
  cudaError_t e = cudaMemcpy(dst, ddst, nd, cudaMemcpyDeviceToHost);
  cudaFree(dsrc);
  cudaFree(ddst);
  cudaFree(tmp);
  return (int)e;
}

}  // extern "C"
