// Checkpoint support: the pair state that a restart needs beyond floes and
// bonds.  The reference restarts from positions, velocities and the bond list
// only (ini_get.f90:129-130, 252-311) and loses the contact histories
// (deltat, thetarelc) and the last contact forces (fcn, fct) that its stress
// diagnostic reads; keeping them makes a restarted run continue exactly.
//
// Histories are exported per pair by reference ids (lower id first) and put
// back after the first rebuild of the restored field into the owner entry of
// the same pair.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace godar {

// Pairs of one instance (slots [off, off + n)) with a nonzero history.
// FILL = false counts them; FILL = true writes (id_lo, id_hi) and the four
// values.  fp64: Hist4<double> at the entry's pair index, side hs; else
// Hist4<float> in place at the owner entry.
template <bool FILL>
__global__ void k_hist_list(Views V, int cur, int off, int n, int fp64, int hs, int *count, int *pi, int *pj,
                            double *h4, int cap)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int s = off + k;
        for (int e = V.up_off[s]; e < V.up_off[s + 1]; e++) {
            const int2 en = V.ent_up[e];
            double h[4];
            if (fp64) {
                const Hist4<double> H = ((const Hist4<double> *)V.hist[hs])[en.y];
                h[0] = H.deltat; h[1] = H.thetarelc; h[2] = H.fcn; h[3] = H.fct;
            } else {
                const Hist4<float> H = ((const Hist4<float> *)V.hist[0])[e];
                h[0] = H.deltat; h[1] = H.thetarelc; h[2] = H.fcn; h[3] = H.fct;
            }
            if (h[0] == 0.0 && h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0) continue;
            const int q = atomicAdd(count, 1);
            if (FILL && q < cap) {
                pi[q] = V.id[cur][s];
                pj[q] = V.id[cur][en.x];
                for (int c = 0; c < 4; c++) h4[4 * (size_t)q + c] = h[c];
            }
        }
    }
}

// Slot of every floe by global id (instance offset + reference id).
__global__ void k_slot_of_all(Views V, int side, int *slot_of)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x)
        slot_of[V.P[V.inst[s]].off + V.id[side][s]] = s;
}

// Puts saved histories back: pair (pi, pj) of the instance at offset off
// (reference ids, pi < pj) into its owner entry, when the pair is in the
// rows.  The mixed path also marks the entry as carrying a history.
__global__ void k_hist_inject(Views V, int cur, int off, int nh, const int *pi, const int *pj, const double *h4,
                              const int *slot_of, int fp64, int hs, unsigned char *pfl)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nh; k += gridDim.x * blockDim.x) {
        const int s = slot_of[off + pi[k]];
        const int jd = pj[k];
        for (int e = V.up_off[s]; e < V.up_off[s + 1]; e++) {
            const int2 en = V.ent_up[e];
            if (V.id[cur][en.x] != jd) continue;
            const double *h = h4 + 4 * (size_t)k;
            if (fp64) {
                Hist4<double> H;
                H.deltat = h[0]; H.thetarelc = h[1]; H.fcn = h[2]; H.fct = h[3];
                ((Hist4<double> *)V.hist[hs])[en.y] = H;
            } else {
                Hist4<float> H;
                H.deltat = (float)h[0]; H.thetarelc = (float)h[1]; H.fcn = (float)h[2]; H.fct = (float)h[3];
                ((Hist4<float> *)V.hist[0])[e] = H;
                if (pfl && (H.deltat != 0.f || H.thetarelc != 0.f)) pfl[e] |= 1u;
            }
            break;
        }
    }
}

static int grid_n(long long n, int block)
{
    return (int)std::max(1LL, std::min<long long>((n + block - 1) / block, 148LL * 16));
}

void launch_hist_list(const Views &V, int cur, int off, int n, int fp64, int hs, int *count, int *pi, int *pj,
                      double *h4, int cap, cudaStream_t st)
{
    if (pi) k_hist_list<true><<<grid_n(n, 128), 128, 0, st>>>(V, cur, off, n, fp64, hs, count, pi, pj, h4, cap);
    else k_hist_list<false><<<grid_n(n, 128), 128, 0, st>>>(V, cur, off, n, fp64, hs, count, pi, pj, h4, cap);
}

void launch_hist_inject(const Views &V, int cur, int off, int nh, const int *pi, const int *pj, const double *h4,
                        int *slot_of, int fp64, int hs, unsigned char *pfl, cudaStream_t st)
{
    if (nh <= 0) return;
    k_slot_of_all<<<grid_n(V.N, 256), 256, 0, st>>>(V, cur, slot_of);
    k_hist_inject<<<grid_n(nh, 128), 128, 0, st>>>(V, cur, off, nh, pi, pj, h4, slot_of, fp64, hs, pfl);
}

}  // namespace godar
