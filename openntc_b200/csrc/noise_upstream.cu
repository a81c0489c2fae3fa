// Upstream-compatible quantisation noise (parity mode, ONTC_NOISE_UPSTREAM).
//
// Upstream draws its noise surrogate with cuRAND's XORWOW device generator: 2^20 states
// initialised once per context as curand_init(123, 0, tid) (ntc_kernel.cu:412-425; the
// thread index is the *offset* within one sequence), and before every step a grid-stride
// fill of the step level's g0 then g1 noise buffer, U(0,1] * delta - delta / 2
// (ntc_kernel.cu:427-446, libopenntc.cpp:586-600).  Calling the same cuRAND device functions
// with the same state indexing reproduces those buffers exactly, so training trajectories
// can be compared with upstream's at equal steps.  The default mode never writes noise to
// HBM (counter-based, generated at the touched latents inside the gather).
#include <curand_kernel.h>

#include "kernels.h"

namespace ontc {

namespace {

__global__ void noise_init_kernel(int n, curandState* st)
{
  const int tid = blockDim.x * blockIdx.x + threadIdx.x;
  if (tid >= n) return;
  curand_init(123, 0, tid, &st[tid]);
}

__global__ void noise_fill_kernel(long long n, float delta, curandState* st, float* out)
{
  const long long tid = (long long)blockDim.x * blockIdx.x + threadIdx.x;
  if (tid >= n) return;
  const long long stride = (long long)gridDim.x * blockDim.x;
  curandState rs = st[tid];
  for (long long i = tid; i < n; i += stride) out[i] = __fmaf_rn(curand_uniform(&rs), delta, -(delta / 2.0f));
  st[tid] = rs;
}

}  // namespace

size_t noise_state_bytes(int n_states) { return (size_t)n_states * sizeof(curandState); }

cudaError_t launch_noise_init(void* states, int n_states, cudaStream_t stream)
{
  noise_init_kernel<<<(n_states + 1023) / 1024, 1024, 0, stream>>>(n_states, (curandState*)states);
  return cudaGetLastError();
}

cudaError_t launch_noise_fill(void* states, int n_states, long long n, float delta, float* out, cudaStream_t stream)
{
  noise_fill_kernel<<<(n_states + 1023) / 1024, 1024, 0, stream>>>(n, delta, (curandState*)states, out);
  return cudaGetLastError();
}

}  // namespace ontc
