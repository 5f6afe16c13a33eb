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

template <int U>
static void screen_u(const Views &V, int cur, int diag, int n, const int *plist, const unsigned *erow,
                     unsigned char *pfl, FP64Lists L, PairRec64 *rec, int grid, int block, cudaStream_t st)
{
    if (diag) launch_step(V.pdl != 0, k_pairs_fp64_screen<U, true>, grid, block, st, V, cur, n, plist, erow, pfl, L, rec);
    else launch_step(V.pdl != 0, k_pairs_fp64_screen<U, false>, grid, block, st, V, cur, n, plist, erow, pfl, L, rec);
}

void launch_pairs_fp64_screen(const Views &V, int cur, int diag, int n, const int *plist, const unsigned *erow,
                              unsigned char *pfl, FP64Lists L, void *rec, int block, int variant, cudaStream_t st)
{
    // variant: 0, 1, 2 = 2, 1, 4 entries per lane
    const int u = variant == 1 ? 1 : variant == 2 ? 4 : 2;
    const int grid = fp64_grid((n + u - 1) / u, block);
    PairRec64 *r = (PairRec64 *)rec;
    if (u == 1) screen_u<1>(V, cur, diag, n, plist, erow, pfl, L, r, grid, block, st);
    else if (u == 2) screen_u<2>(V, cur, diag, n, plist, erow, pfl, L, r, grid, block, st);
    else screen_u<4>(V, cur, diag, n, plist, erow, pfl, L, r, grid, block, st);
}

void launch_pairs_fp64_work(const Views &V, int cur, int diag, int list, int E, unsigned char *pfl, FP64Lists L,
                            void *rec, int block, cudaStream_t st)
{
    // the list's length is known on the device only: at most one wave, grid-stride
    const int grid = (int)std::max(1LL, std::min<long long>((E + block - 1) / block, 148LL * (1024 / block)));
    PairRec64 *r = (PairRec64 *)rec;
    if (list && diag) launch_step(V.pdl != 0, k_pairs_fp64<true, true>, grid, block, st, V, cur, L, pfl, r);
    else if (list) launch_step(V.pdl != 0, k_pairs_fp64<true, false>, grid, block, st, V, cur, L, pfl, r);
    else if (diag) launch_step(V.pdl != 0, k_pairs_fp64<false, true>, grid, block, st, V, cur, L, pfl, r);
    else launch_step(V.pdl != 0, k_pairs_fp64<false, false>, grid, block, st, V, cur, L, pfl, r);
}

void launch_row_sums_fp64(const Views &V, int cur, int diag, const unsigned char *pfl, const void *rec,
                          const int *lo_n, const int *up_n, double *fs, int block, cudaStream_t st)
{
    const PairRec64 *r = (const PairRec64 *)rec;
    if (diag) launch_step(V.pdl != 0, k_row_sums_fp64<true>, fp64_grid(V.N, block), block, st, V, cur, pfl, r, lo_n, up_n, fs);
    else launch_step(V.pdl != 0, k_row_sums_fp64<false>, fp64_grid(V.N, block), block, st, V, cur, pfl, r, lo_n, up_n, fs);
}

void launch_floes_fp64(const Views &V, int cur, int diag, int sic, const double *fs, int *nwork, int block,
                       cudaStream_t st)
{
    if (diag) launch_step(V.pdl != 0, k_floes_fp64<true>, fp64_grid(V.N, block), block, st, V, cur, sic, fs, nwork);
    else launch_step(V.pdl != 0, k_floes_fp64<false>, fp64_grid(V.N, block), block, st, V, cur, sic, fs, nwork);
}

// Owner entries [0, E) at a rebuild (floes on side `side`, at the rebuild
// positions): whether a pair can act on a step without diagnostics before
// the next rebuild.  Until then every floe stays within skin/2 of where it
// is now (a step that takes one farther ends the chunk and a rebuild
// follows) and radii only shrink (ridging), so a pair whose gap exceeds the
// skin cannot touch; a pair without contact, bond or history in a field
// without sheltering changes nothing on such a step (pair_compute resets a
// history that is already zero).  Kept: pairs within reach (with a margin
// far above rounding), bonded pairs, pairs with a history, every pair of a
// sheltering field.
__global__ void k_fp64_mark(Views V, int side, int E, const unsigned *erow, unsigned char *listed)
{
    const Hist4<double> *H = (const Hist4<double> *)V.hist[0];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        const int g = (int)erow[e];
        const InstParams &P = V.P[V.inst[g]];
        const int2 en = V.ent_up[e];
        const int t = en.x, p = en.y;
        bool keep = P.shelter != 0 || V.bidx[p] >= 0;
        if (!keep) {
            const Hist4<double> h = H[p];
            keep = (__double_as_longlong(h.deltat) | __double_as_longlong(h.thetarelc)) != 0;
        }
        if (!keep) {
            const bool px = P.boundary & BC_PERIODIC_X, py = P.boundary & BC_PERIODIC_Y;
            const double dx = wrap_d(V.x[side][g] - V.x[side][t], P.nx, px);
            const double dy = wrap_d(V.y[side][g] - V.y[side][t], P.ny, py);
            const double dist = sqrt(dx * dx + dy * dy);
            const double reach = (V.r[side][g] + V.r[side][t]) + P.skin;
            keep = !(dist > reach + 1e-6 * (dist + reach) + 1e-3);
        }
        listed[p] = keep ? 1 : 0;
    }
}

// Every floe's rows reordered (stably) so that the pairs kept by
// k_fp64_mark come first: up_n / lo_n of them in the owner / partner row.
// tmp holds E + L entries.
__global__ void k_fp64_partition(Views V, const unsigned char *listed, int *up_n, int *lo_n, int2 *tmp, int E)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < V.N; g += gridDim.x * blockDim.x) {
        for (int side = 0; side < 2; side++) {
            int2 *ent = side ? V.ent_lo : V.ent_up;
            const int *off = side ? V.lo_off : V.up_off;
            int2 *t = tmp + (side ? E : 0);
            const int a0 = off[g], a1 = off[g + 1];
            int m = a0;
            for (int a = a0; a < a1; a++)
                if (listed[ent[a].y]) t[m++] = ent[a];
            (side ? lo_n : up_n)[g] = m - a0;
            for (int a = a0; a < a1; a++)
                if (!listed[ent[a].y]) t[m++] = ent[a];
            for (int a = a0; a < a1; a++) ent[a] = t[a];
        }
    }
}

// The owner-row positions the plain steps' screen visits: the first up_n[g]
// of every row, at pos[g] in the list.
__global__ void k_fp64_list(const int *up_off, const int *up_n, const int *pos, int N, int *plist)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < N; g += gridDim.x * blockDim.x) {
        const int a0 = up_off[g], q = pos[g];
        for (int k = 0; k < up_n[g]; k++) plist[q + k] = a0 + k;
    }
}

void launch_fp64_rows(const Views &V, int side, int E, const unsigned *erow, unsigned char *listed, int *up_n,
                      int *lo_n, int2 *tmp, int *pos, int *scan_scratch, int *plist, cudaStream_t st)
{
    if (E > 0) k_fp64_mark<<<fp64_grid(E, 256), 256, 0, st>>>(V, side, E, erow, listed);
    k_fp64_partition<<<fp64_grid(V.N, 128), 128, 0, st>>>(V, listed, up_n, lo_n, tmp, E);
    scan_excl(up_n, pos, V.N, scan_scratch, st);
    k_fp64_list<<<fp64_grid(V.N, 128), 128, 0, st>>>(V.up_off, up_n, pos, V.N, plist);
}

}  // namespace godar
