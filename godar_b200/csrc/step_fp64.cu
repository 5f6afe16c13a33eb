// FP64 ("plain") step kernels.  Compiled with --fmad=false so that every FP64
// operation rounds exactly as written, which makes the step bit-identical to
// the CPU oracle.
#include <algorithm>
#include "step_kernel.cuh"
#include "kernels.h"

namespace godar {

static_assert(sizeof(PairRec64) == FP64_PAIR_REC_BYTES, "pair record size");
static_assert(FS64_COUNT == FP64_FLOE_SUMS, "floe sums");

static int fp64_grid(long long n, int block)
{
    return (int)std::max(1LL, std::min<long long>((n + block - 1) / block, 148LL * (4096 / block)));
}

void launch_pairs_fp64_screen(const Views &V, int cur, int diag, int E, const unsigned *erow, unsigned char *pfl,
                              FP64Lists L, int block, int variant, cudaStream_t st)
{
    // variant: 0, 1, 2 = 2, 1, 4 entries per lane
    const int u = variant == 1 ? 1 : variant == 2 ? 4 : 2;
    const int grid = fp64_grid((E + u - 1) / u, block);
    if (u == 1) k_pairs_fp64_screen<1><<<grid, block, 0, st>>>(V, cur, diag, E, erow, pfl, L);
    else if (u == 2) k_pairs_fp64_screen<2><<<grid, block, 0, st>>>(V, cur, diag, E, erow, pfl, L);
    else k_pairs_fp64_screen<4><<<grid, block, 0, st>>>(V, cur, diag, E, erow, pfl, L);
}

void launch_pairs_fp64_work(const Views &V, int cur, int diag, int list, int E, const unsigned *erow,
                            unsigned char *pfl, FP64Lists L, void *rec, int block, cudaStream_t st)
{
    // the list's length is known on the device only: at most one wave, grid-stride
    const int grid = (int)std::max(1LL, std::min<long long>((E + block - 1) / block, 148LL * (1024 / block)));
    if (list) k_pairs_fp64<true><<<grid, block, 0, st>>>(V, cur, diag, L, erow, pfl, (PairRec64 *)rec);
    else k_pairs_fp64<false><<<grid, block, 0, st>>>(V, cur, diag, L, erow, pfl, (PairRec64 *)rec);
}

void launch_row_sums_fp64(const Views &V, int cur, int diag, const unsigned char *pfl, const void *rec, double *fs,
                          int block, cudaStream_t st)
{
    if (diag) k_row_sums_fp64<true><<<fp64_grid(V.N, block), block, 0, st>>>(V, cur, pfl, (const PairRec64 *)rec, fs);
    else k_row_sums_fp64<false><<<fp64_grid(V.N, block), block, 0, st>>>(V, cur, pfl, (const PairRec64 *)rec, fs);
}

void launch_floes_fp64(const Views &V, int cur, int diag, int sic, const double *fs, int *nwork, int block,
                       cudaStream_t st)
{
    if (diag) k_floes_fp64<true><<<fp64_grid(V.N, block), block, 0, st>>>(V, cur, sic, fs, nwork);
    else k_floes_fp64<false><<<fp64_grid(V.N, block), block, 0, st>>>(V, cur, sic, fs, nwork);
}

}  // namespace godar
