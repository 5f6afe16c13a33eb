// Device-to-host outputs: per-floe fields back in reference index order, and
// the pair lists the reference writes at output steps
// (diagnostics_outputs.f90:157-167, mpi_coms.f90:691-796).
#include "common.cuh"
#include "kernels.h"

namespace godar {

__global__ void k_gather_field(Views V, int cur, int off, int n, int field, double *out)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int s = off + k;
        double val;
        switch (field) {
        case 0: val = V.x[cur][s]; break;
        case 1: val = V.y[cur][s]; break;
        case 2: val = V.u[cur][s]; break;
        case 3: val = V.v[cur][s]; break;
        case 4: val = V.r[cur][s]; break;
        case 5: val = V.h[cur][s]; break;
        case 6: val = V.th[cur][s]; break;
        case 7: val = V.om[cur][s]; break;
        default: val = V.diag[(size_t)(field - 8) * V.N + s]; break;
        }
        out[V.id[cur][s]] = val;
    }
}

// which: 0 candidates, 1 contacts (pdn of the last diagnostic step), 2 bonds
__global__ void k_list_pairs(Views V, int cur, int off, int n, int which, int *pi, int *pj, double *val,
                             int cap, int *count)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int s = off + k;
        const int ids = V.id[cur][s];
        if (which == 2) {
            const int gl = off + ids;
            for (int b = V.bond_off[gl]; b < V.bond_off[gl + 1]; b++) {
                const BondDyn d = V.bdyn[cur][b];
                if (d.flag != 1) continue;
                const int q = atomicAdd(count, 1);
                if (q < cap) { pi[q] = ids; pj[q] = V.bond_hi[b]; val[q] = d.dmg; }
            }
            continue;
        }
        const int e0 = V.row_off[s] + V.nlo[s], e1 = V.row_off[s + 1];
        for (int e = e0; e < e1; e++) {
            const int2 en = V.ent[e];
            const float dn = V.pdn[en.y];
            if (dn != dn) continue;
            if (which == 1 && !(dn > 0.0f)) continue;
            const int q = atomicAdd(count, 1);
            if (q < cap) { pi[q] = ids; pj[q] = V.id[cur][en.x]; val[q] = (double)dn; }
        }
    }
}

void launch_gather_field(const Views &V, int cur, int inst, int off, int n, int field, double *out, cudaStream_t st)
{
    (void)inst;
    const int grid = n > 0 ? (n + 255) / 256 : 1;
    k_gather_field<<<grid < 2048 ? grid : 2048, 256, 0, st>>>(V, cur, off, n, field, out);
}

void launch_list_pairs(const Views &V, int cur, int inst, int off, int n, int which, int *pi, int *pj,
                       double *val, int cap, int *count, cudaStream_t st)
{
    (void)inst;
    const int grid = n > 0 ? (n + 127) / 128 : 1;
    k_list_pairs<<<grid < 2048 ? grid : 2048, 128, 0, st>>>(V, cur, off, n, which, pi, pj, val, cap, count);
}

}  // namespace godar
