// BF16 tcgen05/TMEM tile kernel (see launch_tc_units in kernels.h).
#include "common.cuh"
#include "kernels.h"

namespace ontc {

int tc_max_grid() { return 148; }

cudaError_t launch_tc_units(const Model&, const StepRec*, int, int, TileOut, int*, cudaStream_t)
{
  return cudaErrorNotSupported;
}

}  // namespace ontc
