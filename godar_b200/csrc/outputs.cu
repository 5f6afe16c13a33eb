// Device-to-host outputs: per-floe fields back in reference index order, and
// the pair lists the reference writes at output steps
// (diagnostics_outputs.f90:157-167, mpi_coms.f90:691-796).
#include "common.cuh"
#include "kernels.h"

namespace godar {

// all = 0: one instance at slots [off, off+n), out in its id order; all = 1:
// every instance, out concatenated by instance (offset P.off) in id order.
__global__ void k_gather_field(Views V, int cur, int off, int n, int field, double *out, int all)
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
        // wall histories, for checkpoints (GATHER_DTB1 ..)
        case GATHER_DTB1: val = V.dtb1[cur][s]; break;
        case GATHER_DTB1 + 1: val = V.dtb2[cur][s]; break;
        case GATHER_DTB1 + 2: val = V.thb1[cur][s]; break;
        case GATHER_DTB1 + 3: val = V.thb2[cur][s]; break;
        default: val = V.diag[(size_t)(field - 8) * V.N + s]; break;
        }
        out[(all ? V.P[V.inst[s]].off : 0) + V.id[cur][s]] = val;
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
        const int e0 = V.up_off[s], e1 = V.up_off[s + 1];
        for (int e = e0; e < e1; e++) {
            const int2 en = V.ent_up[e];
            const float dn = V.pdn[en.y];
            if (dn != dn) continue;
            if (which == 1 && !(dn > 0.0f)) continue;
            const int q = atomicAdd(count, 1);
            if (q < cap) { pi[q] = ids; pj[q] = V.id[cur][en.x]; val[q] = (double)dn; }
        }
    }
}

// Per instance (one block each): total momentum (x, y), kinetic energy of
// translation and rotation, and the largest speed of its floes on side cur
// (mass = rho_ice pi h r^2 and inertia = m r^2 / 2, floe_properties,
// physics.f90:179-198), summed over a block-stride loop and a fixed tree in
// shared memory: deterministic for a given state in a given memory order of
// the floes (their cell order at the last neighbour rebuild).
constexpr int SUM_THREADS = 256;
__global__ void __launch_bounds__(SUM_THREADS) k_instance_summary(Views V, int cur, double4 *out)
{
    __shared__ double4 red[SUM_THREADS];
    const InstParams &P = V.P[blockIdx.x];
    double4 a = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int i = threadIdx.x; i < P.n; i += SUM_THREADS) {
        const int g = P.off + i;
        const double r = V.r[cur][g], h = V.h[cur][g];
        const double u = V.u[cur][g], v = V.v[cur][g], om = V.om[cur][g];
        const double m = ((P.rhoice * P.pi) * h) * (r * r);
        const double in = (0.5 * m) * (r * r);
        const double s2 = u * u + v * v;
        a.x = a.x + m * u;
        a.y = a.y + m * v;
        a.z = a.z + ((0.5 * m) * s2 + (0.5 * in) * (om * om));
        a.w = fmax(a.w, sqrt(s2));
    }
    red[threadIdx.x] = a;
    __syncthreads();
    for (int w = SUM_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            const double4 b = red[threadIdx.x + w];
            double4 c = red[threadIdx.x];
            c.x = c.x + b.x; c.y = c.y + b.y; c.z = c.z + b.z; c.w = fmax(c.w, b.w);
            red[threadIdx.x] = c;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

void launch_instance_summary(const Views &V, int cur, double *out, cudaStream_t st)
{
    if (V.ninst > 0) k_instance_summary<<<V.ninst, SUM_THREADS, 0, st>>>(V, cur, reinterpret_cast<double4 *>(out));
}

void launch_gather_field(const Views &V, int cur, int inst, int off, int n, int field, double *out, cudaStream_t st)
{
    const int grid = n > 0 ? (n + 255) / 256 : 1;
    k_gather_field<<<grid < 2048 ? grid : 2048, 256, 0, st>>>(V, cur, off, n, field, out, inst < 0 ? 1 : 0);
}

void launch_list_pairs(const Views &V, int cur, int inst, int off, int n, int which, int *pi, int *pj,
                       double *val, int cap, int *count, cudaStream_t st)
{
    (void)inst;
    const int grid = n > 0 ? (n + 127) / 128 : 1;
    k_list_pairs<<<grid < 2048 ? grid : 2048, 128, 0, st>>>(V, cur, off, n, which, pi, pj, val, cap, count);
}

}  // namespace godar

// ------------------------------------------------------------ relayout
// Batch membership changes: resident floes move to their new slots
// device-to-device (new slot g takes old slot repack[g]; -1 = a newly admitted
// floe, uploaded from the host instead), and their bond records follow
// (new bond q takes old bond bmap[q]).
namespace godar {

__global__ void k_gather_floes(Views Vo, int so, Views Vn, int sn, const int *repack, int n)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const int o = repack[g];
        if (o < 0) continue;
        Vn.x[sn][g] = Vo.x[so][o]; Vn.y[sn][g] = Vo.y[so][o]; Vn.th[sn][g] = Vo.th[so][o];
        Vn.u[sn][g] = Vo.u[so][o]; Vn.v[sn][g] = Vo.v[so][o]; Vn.om[sn][g] = Vo.om[so][o];
        Vn.r[sn][g] = Vo.r[so][o]; Vn.h[sn][g] = Vo.h[so][o];
        Vn.dtb1[sn][g] = Vo.dtb1[so][o]; Vn.dtb2[sn][g] = Vo.dtb2[so][o];
        Vn.thb1[sn][g] = Vo.thb1[so][o]; Vn.thb2[sn][g] = Vo.thb2[so][o];
        Vn.id[sn][g] = Vo.id[so][o];
    }
}

// bond_off of resident floes, rebased: the floe with reference id k of
// instance b keeps its bonds at new index  old_off[old_base_b + k] -
// old_bbase_b + new_bbase_b.  new_id_base[b] is the instance's first new slot.
__global__ void k_rebase_bond_off(const int *old_bond_off, int *new_bond_off, const int *inst, const int *old_slot_base,
                                  const int *new_slot_base, const int *old_bbase, const int *new_bbase, int n)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const int b = inst[g];
        if (old_slot_base[b] < 0) continue;
        const int k = g - new_slot_base[b];
        new_bond_off[g] = old_bond_off[old_slot_base[b] + k] - old_bbase[b] + new_bbase[b];
    }
}

__global__ void k_gather_bonds(const int *old_hi, const BondStat *old_st, const BondDyn *old_dy, int *new_hi,
                               BondStat *new_st, BondDyn *new_dy, const int *bmap, int nb)
{
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nb; q += gridDim.x * blockDim.x) {
        const int o = bmap[q];
        if (o < 0) continue;
        new_hi[q] = old_hi[o];
        new_st[q] = old_st[o];
        new_dy[q] = old_dy[o];
    }
}

static int rl_grid(int n) { return n > 0 ? ((n + 255) / 256 < 2368 ? (n + 255) / 256 : 2368) : 1; }

void launch_gather_floes(const Views &Vo, int so, const Views &Vn, int sn, const int *repack, int n, cudaStream_t st)
{
    k_gather_floes<<<rl_grid(n), 256, 0, st>>>(Vo, so, Vn, sn, repack, n);
}

void launch_rebase_bond_off(const int *old_bond_off, int *new_bond_off, const int *inst, const int *old_slot_base,
                            const int *new_slot_base, const int *old_bbase, const int *new_bbase, int n,
                            cudaStream_t st)
{
    k_rebase_bond_off<<<rl_grid(n), 256, 0, st>>>(old_bond_off, new_bond_off, inst, old_slot_base, new_slot_base,
                                                  old_bbase, new_bbase, n);
}

void launch_gather_bonds(const int *old_hi, const BondStat *old_st, const BondDyn *old_dy, int *new_hi,
                         BondStat *new_st, BondDyn *new_dy, const int *bmap, int nb, cudaStream_t st)
{
    if (nb > 0) k_gather_bonds<<<rl_grid(nb), 256, 0, st>>>(old_hi, old_st, old_dy, new_hi, new_st, new_dy, bmap, nb);
}

__global__ void k_set_int(int *p, int v) { *p = v; }

// Sets one device int in stream order (the value is the launch's argument,
// so no host buffer has to outlive the call).
void launch_set_int(int *p, int v, cudaStream_t st)
{
    k_set_int<<<1, 1, 0, st>>>(p, v);
}

}  // namespace godar
