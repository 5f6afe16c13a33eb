// FP64 ("plain") instantiation of the step kernel.  Compiled with
// --fmad=false so that every FP64 operation rounds exactly as written, which
// makes the step bit-identical to the CPU oracle.
#include "step_kernel.cuh"
#include "kernels.h"

namespace godar {

void launch_step_fp64(const Views &V, int cur, int diag, int sic, int grid, int block, cudaStream_t st)
{
    k_step<double, true><<<grid, block, 0, st>>>(V, cur, diag, sic);
}

}  // namespace godar
