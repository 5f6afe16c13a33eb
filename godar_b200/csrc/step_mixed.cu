// Mixed-precision instantiation of the step kernel: FP32 pair forces,
// sheltering and drag; FP64 geometry, bond strain/damage, ridging bookkeeping
// and integration.
#include "step_kernel.cuh"
#include "kernels.h"

namespace godar {

void launch_step_mixed(const Views &V, int cur, int diag, int sic, int grid, int block, cudaStream_t st)
{
    k_step<float, false><<<grid, block, 0, st>>>(V, cur, diag, sic);
}

}  // namespace godar
