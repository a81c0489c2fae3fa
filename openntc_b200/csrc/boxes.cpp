// TMA staging boxes of the tile kernel (train_tc.cu): for one lod, the box sizes that cover the
// g0 / g1 latent footprint of every 16 x 8 texel unit at that lod, and the tensor maps that
// load them.  The maps are encoded through the driver's cuTensorMapEncodeTiled, obtained from
// the runtime (no link against the driver library).
#include <math.h>

#include <algorithm>
#include <cstring>

#include <cudaTypedefs.h>

#include "kernels.h"

namespace ontc {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Largest span (cells) along one axis of `len` consecutive texels starting anywhere in a mip of
// size `mip`, in a grid of size gd; with `even`, counting from the even cell at or below the
// first one.
int max_span(int len, int mip, int gd, bool even)
{
  int best = 0;
  for (int a = 0; a + len <= mip; a++) {
    int lo = 0, n = 0;
    foot_span(a, a + len - 1, mip, gd, lo, n);
    best = std::max(best, n + (even ? (lo & 1) : 0));
  }
  return best;
}

}  // namespace

cudaError_t make_latent_boxes(const float* p0, const float* p1, int d0, int d1, int C0, int C1, int mip_dim,
                              int cap_floats, LatentBoxes& out)
{
  memset(&out, 0, sizeof(out));
  // units are 16 x 8 texel blocks of tiles of min(mip, 256)^2 texels (smaller tiles: no staging)
  if (std::min(mip_dim, 256) < 16 || C0 % 4 != 0 || C1 % 2 != 0) return cudaSuccess;
  // a g1 cell of C1 floats that is not a multiple of 16 bytes: start its box at an even cell so
  // that the innermost coordinate (cells x C1 floats) stays a multiple of 16 bytes
  const bool shift = (C1 * 4) % 16 != 0;
  int w0 = max_span(16, mip_dim, d0, false), h0 = max_span(8, mip_dim, d0, false);
  int w1 = max_span(16, mip_dim, d1, shift), h1 = max_span(8, mip_dim, d1, false);
  if (shift) w1 += w1 & 1;  // the box's inner extent, w1 x C1 floats, a multiple of 16 bytes
  const int g0_floats = C0 * w0 * h0;
  const int g1_off = (g0_floats + 31) / 32 * 32;  // 128-byte aligned destination
  const int total = g1_off + w1 * C1 * h1;
  // limits: the scatter's corner masks (64 x 32 cells), TMA boxes (256 per dimension), the buffer
  if (w0 > 64 || h0 > 32 || w1 > 64 || h1 > 32 || w1 * C1 > 256 || total > cap_floats) return cudaSuccess;
  if (w0 > d0 || h0 > d0 || w1 > d1 || h1 > d1) return cudaSuccess;  // boxes within the grids
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc) return cudaErrorNotSupported;
  {
    const cuuint64_t dims[3] = {(cuuint64_t)C0, (cuuint64_t)d0, (cuuint64_t)d0};
    const cuuint64_t strides[2] = {(cuuint64_t)C0 * 4, (cuuint64_t)d0 * C0 * 4};
    const cuuint32_t box[3] = {(cuuint32_t)C0, (cuuint32_t)w0, (cuuint32_t)h0};
    const cuuint32_t es[3] = {1, 1, 1};
    if (enc(&out.g0, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(p0), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaSuccess;  // not staged at this lod
  }
  {
    const cuuint64_t dims[2] = {(cuuint64_t)d1 * C1, (cuuint64_t)d1};
    const cuuint64_t strides[1] = {(cuuint64_t)d1 * C1 * 4};
    const cuuint32_t box[2] = {(cuuint32_t)(w1 * C1), (cuuint32_t)h1};
    const cuuint32_t es[2] = {1, 1};
    if (enc(&out.g1, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(p1), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return cudaSuccess;
  }
  out.w0 = w0;
  out.h0 = h0;
  out.w1 = w1;
  out.h1 = h1;
  out.g1_shift = shift ? 1 : 0;
  out.g1_off = (uint32_t)g1_off;
  out.bytes = (uint32_t)(4 * (g0_floats + w1 * C1 * h1));
  return cudaSuccess;
}

}  // namespace ontc
