// Bond creation on the device: the bonds of time step 1 (stepper.f90:93-101)
// with their geometry (bond_properties, bonds.f90:237-269), for the fields
// admitted to a batch fresh (not a restart) with cohesion on.
//
// Rule: every candidate pair i < j of a field (dist <= r_i + rtree, the
// reference's radius query) with deltan = (r_i + r_j) - dist >=
// -(bond_lim + bond_lim_rel (r_i + r_j)); with 0 < bond_frac < 1, only the
// pairs whose hash pair_hash32(bond_seed, i, j) / 2^32 is below bond_frac.
//
// At admission the fields' floes sit in their slots in reference order (slot
// = instance offset + reference id).  A cell list over the admitted floes
// (cell keys of the instance grids, stable radix sort, cell ranges) gives
// each floe's neighbours without moving any state; one pass counts each
// floe's bonds, a scan places them, a second pass writes them in ascending
// partner id (the reference's j order in its bond loops) into the batch's
// bond table.  Compiled with --fmad=false: distances and geometry round
// exactly as in the step and in the CPU oracle.
#include "common.cuh"
#include "kernels.h"

namespace godar {

// cell of a position on its instance's grid (the rebuild's cell_of)
GD_DEV void bi_cell(const InstParams &P, double x, double y, int &cx, int &cy)
{
    double fx = x / P.cw, fy = y / P.ch;
    if (!(fx >= 0.0)) fx = 0.0;
    if (!(fy >= 0.0)) fy = 0.0;
    if (fx > (double)P.ncx) fx = (double)P.ncx;
    if (fy > (double)P.ncy) fy = (double)P.ncy;
    cx = (int)floor(fx);
    cy = (int)floor(fy);
    cx = cx < 0 ? 0 : (cx >= P.ncx ? P.ncx - 1 : cx);
    cy = cy < 0 ? 0 : (cy >= P.ncy ? P.ncy - 1 : cy);
}

__global__ void k_bi_keys(Views V, int side, int s0, int n, uint32_t *keys, int *vals)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int s = s0 + k;
        const InstParams &P = V.P[V.inst[s]];
        int cx, cy;
        bi_cell(P, V.x[side][s], V.y[side][s], cx, cy);
        keys[k] = (uint32_t)(P.coff + (long long)cy * P.ncx + cx);
        vals[k] = s;
    }
}

// Visits, for floe s (slot = instance offset + reference id), every floe t of
// higher id of its field that the rule bonds to s, with their distance.
// The cell stencil (kx, ky) covers r_max + rtree + skin, beyond the
// candidate radius r_i + rtree.
template <class F>
GD_DEV void bi_partners(const Views &V, int side, const BondRule &R, const int *cstart, const int *cend,
                        const int *vals, int s, F f)
{
    const InstParams &P = V.P[V.inst[s]];
    const double xs = V.x[side][s], ys = V.y[side][s], rs = V.r[side][s];
    const int ids = s - P.off;
    const bool px = P.boundary & BC_PERIODIC_X, py = P.boundary & BC_PERIODIC_Y;
    const double Rc = rs + P.rtree;
    int cx, cy;
    bi_cell(P, xs, ys, cx, cy);
    int x0 = cx - P.kx, x1 = cx + P.kx, y0 = cy - P.ky, y1 = cy + P.ky;
    if (px && x1 - x0 + 1 >= P.ncx) { x0 = 0; x1 = P.ncx - 1; }
    if (py && y1 - y0 + 1 >= P.ncy) { y0 = 0; y1 = P.ncy - 1; }
    for (int yy = y0; yy <= y1; yy++) {
        int wy = yy;
        if (py) wy = (yy % P.ncy + P.ncy) % P.ncy;
        else if (yy < 0 || yy >= P.ncy) continue;
        for (int xx = x0; xx <= x1; xx++) {
            int wx = xx;
            if (px) wx = (xx % P.ncx + P.ncx) % P.ncx;
            else if (xx < 0 || xx >= P.ncx) continue;
            const long long c = P.coff + (long long)wy * P.ncx + wx;
            for (int q = cstart[c]; q < cend[c]; q++) {
                const int t = vals[q];
                const int idt = t - P.off;
                if (idt <= ids) continue;
                const double dx = wrap_d(xs - V.x[side][t], P.nx, px);
                const double dy = wrap_d(ys - V.y[side][t], P.ny, py);
                const double dist = sqrt(dx * dx + dy * dy);
                if (!(dist <= Rc)) continue;
                const double rt = V.r[side][t];
                const double deltan = (rs + rt) - dist;
                const double lim = R.lim + R.lim_rel * (rs + rt);
                bool sel = true;
                if (R.frac > 0.0 && R.frac < 1.0)
                    sel = (double)pair_hash32((uint32_t)R.seed, (uint32_t)ids, (uint32_t)idt) * 0x1.0p-32 < R.frac;
                if (deltan >= -lim && sel) f(idt, dist);
            }
        }
    }
}

// Per admitted floe (sorted position k): the number of bonds it owns (it is
// the lower id), at cnt[s - s0]; zero for fields without fresh bonds.
__global__ void k_bi_count(Views V, int side, int s0, int n, const BondRule *rule, const int *cstart,
                           const int *cend, const int *vals, int *cnt)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int s = vals[k];
        const BondRule R = rule[V.inst[s]];
        int c = 0;
        if (R.fresh) bi_partners(V, side, R, cstart, cend, vals, s, [&](int, double) { c++; });
        cnt[s - s0] = c;
    }
}

// Bonds of each admitted field: the scanned counts at the field's first and
// last floe (first = the instance offset relative to s0).
__global__ void k_bi_totals(const int *scan, const int *first, const int *last, int m, int *tot)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        tot[k] = scan[last[k]] - scan[first[k]];
}

// Writes floe s's bonds: bond_off of its global id, then partner ids and
// geometry in ascending partner id.  The partners are first written with
// their distance (the distance slot lb of the static record), sorted in
// place (a floe has few bonds), then completed.
__global__ void k_bi_fill(Views V, int side, int s0, int n, const BondRule *rule, const int *cstart,
                          const int *cend, const int *vals, const int *scan, int *bond_off, int *bond_hi,
                          BondStat *bstat, BondDyn *bdyn)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int s = vals[k];
        const int ig = V.inst[s];
        const BondRule R = rule[ig];
        if (!R.fresh) continue;
        const InstParams &P = V.P[ig];
        // slot = global id for an admitted field; its bonds start at its
        // table offset plus the bonds of its lower ids
        const int b0 = R.boff + (scan[s - s0] - scan[P.off - s0]);
        bond_off[s] = b0;
        int m = 0;
        bi_partners(V, side, R, cstart, cend, vals, s, [&](int idt, double dist) {
            bond_hi[b0 + m] = idt;
            bstat[b0 + m].lb = dist;
            m++;
        });
        for (int a = 1; a < m; a++) {
            const int ja = bond_hi[b0 + a];
            const double da = bstat[b0 + a].lb;
            int b = a - 1;
            while (b >= 0 && bond_hi[b0 + b] > ja) {
                bond_hi[b0 + b + 1] = bond_hi[b0 + b];
                bstat[b0 + b + 1].lb = bstat[b0 + b].lb;
                b--;
            }
            bond_hi[b0 + b + 1] = ja;
            bstat[b0 + b + 1].lb = da;
        }
        const double ri = V.r[side][s], hi = V.h[side][s];
        for (int a = 0; a < m; a++) {
            const int t = P.off + bond_hi[b0 + a];
            const double rj = V.r[side][t], hj = V.h[side][t];
            const double dist = bstat[b0 + a].lb;
            // bond_properties (bonds.f90:255-262)
            BondStat bs;
            bs.rb = P.lambda_rb * (ri < rj ? ri : rj);
            bs.hb = (hi + hj) / 2.0;
            bs.lb = dist;
            bs.sb = (2.0 * bs.rb) * bs.hb;
            bs.ib = ((2.0 / 3.0) * bs.hb) * ((bs.rb * bs.rb) * bs.rb);
            bs.pad = 0.0;
            // undamaged beam coefficients (bonds.f90:109-117) for the mixed path
            const double EA = P.eb * bs.sb, EI = P.eb * bs.ib, L = bs.lb;
            bs.k_ax = (float)(EA / L);
            bs.k_sh1 = (float)((12.0 * EI) / ((L * L) * L));
            bs.k_sh2 = (float)((6.0 * EI) / (L * L));
            bs.k_r1 = (float)((4.0 * EI) / L);
            bs.k_r2 = (float)((2.0 * EI) / L);
            bs.ei_l = (float)(EI / L);
            bs.ea_l = (float)(EA * L);
            bs.inv_l = (float)(1.0 / L);
            bstat[b0 + a] = bs;
            BondDyn d;
            d.dnb = 0.0; d.dtb = 0.0; d.thji = 0.0; d.thij = 0.0; d.dmg = 0.0;
            d.flag = 1;
            d.pad = 0;
            bdyn[b0 + a] = d;
        }
    }
}

static int bi_grid(long long n, int block)
{
    return (int)std::max(1LL, std::min<long long>((n + block - 1) / block, 148LL * (2048 / block)));
}

void launch_bond_init_count(const Views &V, int side, int s0, int n, const BondRule *rule, uint32_t *keys,
                            int *vals, uint32_t *keys_alt, int *vals_alt, int key_bits, int *rs_counts,
                            int *scan_scratch, int *cstart, int *cend, int *cnt, int *scan, cudaStream_t st)
{
    if (n <= 0) return;
    k_bi_keys<<<bi_grid(n, 256), 256, 0, st>>>(V, side, s0, n, keys, vals);
    radix_sort(keys, vals, keys_alt, vals_alt, n, key_bits, rs_counts, scan_scratch, st);
    launch_cell_ranges(keys, n, cstart, cend, st);
    k_bi_count<<<bi_grid(n, 128), 128, 0, st>>>(V, side, s0, n, rule, cstart, cend, vals, cnt);
    scan_excl(cnt, scan, n, scan_scratch, st);
}

void launch_bond_init_totals(const int *scan, const int *first, const int *last, int m, int *tot, cudaStream_t st)
{
    if (m > 0) k_bi_totals<<<bi_grid(m, 128), 128, 0, st>>>(scan, first, last, m, tot);
}

void launch_bond_init_fill(const Views &V, int side, int s0, int n, const BondRule *rule, const int *cstart,
                           const int *cend, const int *vals, const int *scan, int *bond_off, int *bond_hi,
                           BondStat *bstat, BondDyn *bdyn, cudaStream_t st)
{
    if (n <= 0) return;
    k_bi_fill<<<bi_grid(n, 128), 128, 0, st>>>(V, side, s0, n, rule, cstart, cend, vals, scan, bond_off,
                                               bond_hi, bstat, bdyn);
}

}  // namespace godar
