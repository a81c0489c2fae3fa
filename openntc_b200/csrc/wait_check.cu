// Exercise of the bounded mbarrier wait every tcgen05 kernel of libontc uses (tc_ptx.cuh
// mbar_wait): one thread waits on a barrier nothing arrives at, gives up after `polls`
// suspended polls and reports it, the way the tile and decode kernels report a timed-out MMA
// through their error words.  Nothing faults and nothing hangs: the wait just expires.
#include "kernels.h"
#include "tc_ptx.cuh"

namespace ontc {

namespace {

__global__ void wait_check_kernel(uint32_t polls, int* __restrict__ out)
{
  __shared__ __align__(8) uint64_t bar;
  ptx::mbar_init(&bar, 1);  // expects one arrival that never comes
  ptx::fence_mbar_init();
  const bool done = ptx::mbar_wait(&bar, 0, polls);
  out[0] = done ? 0 : 1;
}

}  // namespace

cudaError_t launch_wait_check(uint32_t polls, int* d_out, cudaStream_t stream)
{
  wait_check_kernel<<<1, 1, 0, stream>>>(polls, d_out);
  return cudaGetLastError();
}

}  // namespace ontc
