// Kernel (a): the neighbour search that replaces coretran's kd-tree
// (KdTree build, kdtree_utils.f90:21-24; radius query kNearest,
// stepper.f90:77-78).
//
// Pipeline of one rebuild (all instances of a batch at once):
//   1. cell key of every floe (its instance's first key + row-major cell)
//   2. stable LSD radix sort of (key, slot), 8-bit digits, as many passes as
//      the key range needs
//   3. gather the floe state into cell order (the other ping-pong side)
//   4. first/last slot of every non-empty cell
//   5. count, scan and fill the symmetric neighbour superset: every t with
//      dist(s,t) <= r_lo + rtree + skin, lo = the floe of lower id; rows are
//      sorted (lower-id partners by id, then higher-id partners by distance;
//      by id in the mixed path)
//   6. link every lower entry to the record of its pair (owned by the
//      lower-id floe's upper entry), migrate contact histories from the
//      previous rows by reference ids, and link bonds.
// The step kernel filters the superset with the exact candidate predicate
// every step, so the candidate set is the kd-tree's radius query exactly as
// long as no floe moved more than skin/2 since the rebuild (checked every
// step).  This file is compiled with --fmad=false: distances must round
// exactly as in the step kernel and the CPU oracle.
#include "common.cuh"
#include "kernels.h"

namespace godar {

// ------------------------------------------------------------ cell keys
GD_DEV void cell_of(const InstParams &P, double x, double y, int &cx, int &cy)
{
    // clamp before the integer conversion so that non-finite or far-away
    // positions land in an edge cell
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

__global__ void k_cell_keys(Views V, int cur, uint32_t *keys, int *vals)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < V.N; g += gridDim.x * blockDim.x) {
        const InstParams &P = V.P[V.inst[g]];
        int cx, cy;
        cell_of(P, V.x[cur][g], V.y[cur][g], cx, cy);
        keys[g] = (uint32_t)(P.coff + (long long)cy * P.ncx + cx);
        vals[g] = g;
    }
}

// ------------------------------------------------------------ radix sort
// Tile of RS_THREADS x RS_ITEMS keys per block; item k of the tile is key
// tile_base + round*RS_THREADS + tid, so ranking round by round, warp by warp
// and lane by lane keeps equal digits in input order (stable).
constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARPS = RS_THREADS / 32;

__global__ void __launch_bounds__(RS_THREADS) k_radix_hist(const uint32_t *keys, int n, int shift, int *counts, int ntiles)
{
    __shared__ int hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * RS_TILE;
#pragma unroll
    for (int k = 0; k < RS_ITEMS; k++) {
        const int i = base + k * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 255], 1);
    }
    __syncthreads();
    counts[threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const uint32_t *keys, const int *vals, uint32_t *okeys,
                                                            int *ovals, int n, int shift, const int *offsets, int ntiles)
{
    __shared__ int wcnt[RS_WARPS][256];
    __shared__ int run[256];
    __shared__ int tot[256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    run[tid] = offsets[tid * ntiles + blockIdx.x];
    const int base = blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; k++) {
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) wcnt[w][tid] = 0;
        __syncthreads();
        const int i = base + k * RS_THREADS + tid;
        const bool valid = i < n;
        uint32_t key = 0;
        int val = 0, d = 0;
        if (valid) {
            key = keys[i];
            val = vals[i];
            d = (key >> shift) & 255;
        }
        const unsigned act = __ballot_sync(0xffffffffu, valid);
        unsigned peers = 0;
        int rank = 0;
        if (valid) {
            peers = __match_any_sync(act, d);
            rank = __popc(peers & ((1u << lane) - 1u));
            if (rank == 0) wcnt[warp][d] = __popc(peers);
        }
        __syncthreads();
        {   // exclusive prefix over warps for digit tid
            int acc = 0;
#pragma unroll
            for (int w = 0; w < RS_WARPS; w++) {
                const int c = wcnt[w][tid];
                wcnt[w][tid] = acc;
                acc += c;
            }
            tot[tid] = acc;
        }
        __syncthreads();
        if (valid) {
            const int pos = run[d] + wcnt[warp][d] + rank;
            okeys[pos] = key;
            ovals[pos] = val;
        }
        __syncthreads();
        run[tid] += tot[tid];
        __syncthreads();
    }
}

// ------------------------------------------------------------ exclusive scan
// out[i] = sum_{k<i} in[i]; out[n] = total.  Three phases: per-block scan,
// scan of block sums by one block, add.
constexpr int SC_THREADS = 512;
constexpr int SC_ITEMS = 4;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

GD_DEV int block_excl_scan(int v, int *sh, int &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        int s = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    total = sh[(blockDim.x >> 5) - 1];
    const int pre = warp > 0 ? sh[warp - 1] : 0;
    __syncthreads();
    return pre + x - v;
}

__global__ void __launch_bounds__(SC_THREADS) k_scan_tiles(const int *in, int *out, int n, int *tile_sums)
{
    __shared__ int sh[32];
    const int base = blockIdx.x * SC_TILE + threadIdx.x * SC_ITEMS;
    int v[SC_ITEMS], s = 0;
#pragma unroll
    for (int k = 0; k < SC_ITEMS; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int pre = block_excl_scan(s, sh, total);
#pragma unroll
    for (int k = 0; k < SC_ITEMS; k++) {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_sums(int *tile_sums, int ntiles, int *total_out)
{
    __shared__ int sh[32];
    int carry = 0;
    for (int base = 0; base < ntiles; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < ntiles ? tile_sums[i] : 0;
        int total;
        const int pre = block_excl_scan(v, sh, total);
        if (i < ntiles) tile_sums[i] = carry + pre;
        carry += total;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(int *out, int n, const int *tile_sums, const int *total, int *out_n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] += tile_sums[i / SC_TILE];
    if (blockIdx.x == 0 && threadIdx.x == 0 && out_n) *out_n = *total;
}

void scan_excl(const int *in, int *out, int n, int *scratch, cudaStream_t st)
{
    // scratch: ntiles + 1 ints; out must hold n + 1 ints
    const int ntiles = (n + SC_TILE - 1) / SC_TILE;
    if (n > 0) k_scan_tiles<<<ntiles, SC_THREADS, 0, st>>>(in, out, n, scratch + 1);
    k_scan_sums<<<1, 1024, 0, st>>>(scratch + 1, ntiles, scratch);
    k_scan_add<<<n > 0 ? (n + 255) / 256 : 1, 256, 0, st>>>(out, n, scratch + 1, scratch, out + n);
}

void radix_sort(uint32_t *keys, int *vals, uint32_t *keys_alt, int *vals_alt, int n, int bits,
                int *counts, int *scratch, cudaStream_t st)
{
    const int ntiles = (n + RS_TILE - 1) / RS_TILE;
    const int passes = (bits + 7) / 8;
    uint32_t *ki = keys, *ko = keys_alt;
    int *vi = vals, *vo = vals_alt;
    for (int p = 0; p < passes; p++) {
        const int shift = 8 * p;
        k_radix_hist<<<ntiles, RS_THREADS, 0, st>>>(ki, n, shift, counts, ntiles);
        scan_excl(counts, counts, 256 * ntiles, scratch, st);
        k_radix_scatter<<<ntiles, RS_THREADS, 0, st>>>(ki, vi, ko, vo, n, shift, counts, ntiles);
        uint32_t *tk = ki; ki = ko; ko = tk;
        int *tv = vi; vi = vo; vo = tv;
    }
    if (ki != keys) {
        cudaMemcpyAsync(keys, ki, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals, vi, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, st);
    }
}

// ------------------------------------------------------------ permutation
// new slot s takes the floe at pre-sort slot vals[s]; old_slot[s] is that
// floe's slot in the previous layout (repack[] maps pre-sort slots to the
// previous layout; -1 for floes new to the batch).
__global__ void k_permute(Views V, int cur, const int *vals, const int *repack, int *old_slot)
{
    const int nxt = cur ^ 1;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const int o = vals[s];
        V.x[nxt][s] = V.x[cur][o];
        V.y[nxt][s] = V.y[cur][o];
        V.th[nxt][s] = V.th[cur][o];
        V.u[nxt][s] = V.u[cur][o];
        V.v[nxt][s] = V.v[cur][o];
        V.om[nxt][s] = V.om[cur][o];
        V.r[nxt][s] = V.r[cur][o];
        V.h[nxt][s] = V.h[cur][o];
        V.dtb1[nxt][s] = V.dtb1[cur][o];
        V.dtb2[nxt][s] = V.dtb2[cur][o];
        V.thb1[nxt][s] = V.thb1[cur][o];
        V.thb2[nxt][s] = V.thb2[cur][o];
        V.id[nxt][s] = V.id[cur][o];
        V.x0[nxt][s] = V.x[cur][o];
        V.y0[nxt][s] = V.y[cur][o];
        old_slot[s] = repack ? repack[o] : o;
    }
}

__global__ void k_cell_ranges(const uint32_t *keys, int n, int *cstart, int *cend)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint32_t k = keys[s];
        if (s == 0 || keys[s - 1] != k) cstart[k] = s;
        if (s == n - 1 || keys[s + 1] != k) cend[k] = s + 1;
    }
}

// ------------------------------------------------------------ neighbour rows
// Visits every floe t != s of s's instance within the stencil and calls
// f(t, dist, id of t) when dist <= r_lo + rtree + skin.
template <class F>
GD_DEV void for_superset(const Views &V, int side, const int *cstart, const int *cend, int s, F f)
{
    const InstParams &P = V.P[V.inst[s]];
    const double xs = V.x[side][s], ys = V.y[side][s], rs = V.r[side][s];
    const int ids = V.id[side][s];
    const bool px = P.boundary & BC_PERIODIC_X, py = P.boundary & BC_PERIODIC_Y;
    int cx, cy;
    cell_of(P, xs, ys, cx, cy);
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
            const int t0 = cstart[c], t1 = cend[c];
            for (int t = t0; t < t1; t++) {
                if (t == s) continue;
                const double dx = wrap_d(xs - V.x[side][t], P.nx, px);
                const double dy = wrap_d(ys - V.y[side][t], P.ny, py);
                const double d = sqrt(dx * dx + dy * dy);
                const int idt = V.id[side][t];
                const double rlo = ids < idt ? rs : V.r[side][t];
                if (d <= (rlo + P.rtree) + P.skin) f(t, d, idt);
            }
        }
    }
}

__global__ void k_nbr_count(Views V, int side, const int *cstart, const int *cend, int *cnt)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        int c = 0;
        for_superset(V, side, cstart, cend, s, [&](int, double, int) { c++; });
        cnt[s] = c;
    }
}

// fills the rows of the new generation (ent2/edist2 at row_off2) and sorts
// each row: partners of lower id ascending by id, then partners of higher id
// ascending by (distance, id).
// up_by_id: the partners of higher id by id as well (the mixed path, whose
// per-floe sums follow the row order: the order then depends only on the
// reference ids, not on when the rows were built); otherwise by distance
// (the FP64 path re-sorts them by distance every step, the kd-tree's order).
__global__ void k_nbr_fill(Views V, int side, const int *cstart, const int *cend, const int *row_off2,
                           int2 *ent2, double *dist2, int *nlo2, int up_by_id)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const int e0 = row_off2[s], e1 = row_off2[s + 1];
        int k = e0;
        // .y holds the partner's id while the row is sorted (no gathers in
        // the comparisons); it becomes the pair index afterwards
        for_superset(V, side, cstart, cend, s, [&](int t, double d, int idt) {
            if (k < e1) { ent2[k] = make_int2(t, idt); dist2[k] = d; }
            k++;
        });
        const int ids = V.id[side][s];
        // insertion sort by (upper?, upper && !up_by_id ? dist : 0, id)
        int nlo = 0;
        for (int a = e0; a < e1; a++) {
            const int2 ea = ent2[a];
            const double da = dist2[a];
            const int ida = ea.y;
            const bool ua = ida > ids;
            if (!ua) nlo++;
            int b = a - 1;
            while (b >= e0) {
                const int idb = ent2[b].y;
                const bool ub = idb > ids;
                const double db = dist2[b];
                bool gt;   // entry b sorts after entry a
                if (ub != ua) gt = ub;
                else if (!ua || up_by_id) gt = idb > ida;
                else gt = (db > da) || (db == da && idb > ida);
                if (!gt) break;
                ent2[b + 1] = ent2[b];
                dist2[b + 1] = db;
                b--;
            }
            ent2[b + 1] = ea;
            dist2[b + 1] = da;
        }
        nlo2[s] = nlo;
        for (int a = e0 + nlo; a < e1; a++) ent2[a].y = a;   // pair record = upper entry
    }
}

// pair index of every lower entry: the upper entry of the partner's row that
// points back at s
__global__ void k_nbr_link(Views V, const int *row_off2, const int *nlo2, int2 *ent2)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const int e0 = row_off2[s], el = e0 + nlo2[s];
        for (int e = e0; e < el; e++) {
            const int t = ent2[e].x;
            const int q0 = row_off2[t] + nlo2[t], q1 = row_off2[t + 1];
            int found = -1;
            for (int q = q0; q < q1; q++)
                if (ent2[q].x == s) { found = q; break; }
            ent2[e].y = found;
            if (found < 0) atomicOr(V.status, ST_ROW_OVERFLOW);
        }
    }
}

// Splits the combined rows into the partner CSR (ent_lo: partners of lower
// id, ascending id; .y = the pair's index) and the owner CSR (ent_up:
// partners of higher id, ascending distance - ascending id in the mixed path;
// .y = own index = pair index).
__global__ void k_split_rows(int N, const int *row_off2, const int *nlo2, const int2 *ent2, const int *lo_off,
                             const int *up_off, int2 *ent_lo, int2 *ent_up)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x) {
        const int e0 = row_off2[s], nl = nlo2[s], e1 = row_off2[s + 1];
        const int lo0 = lo_off[s], up0 = up_off[s];
        for (int k = 0; k < nl; k++) {
            const int2 en = ent2[e0 + k];
            const int t = en.x, q = en.y;     // q: combined index of the owner entry in t's row
            const int pidx = q < 0 ? -1 : up_off[t] + (q - row_off2[t] - nlo2[t]);
            ent_lo[lo0 + k] = make_int2(t, pidx);
        }
        for (int k = 0; k < e1 - e0 - nl; k++) {
            const int e = e0 + nl + k;
            ent_up[up0 + k] = make_int2(ent2[e].x, up0 + k);
        }
    }
}

// Contact histories of the new pairs, taken from the previous pairs by
// reference ids; bond index of every pair.
template <typename H4>
__global__ void k_migrate(Views V, int side_new, const int *old_slot, const int *old_up_off, const int2 *old_ent_up,
                          const int *old_id, const H4 *old_hist, const int *up_off2, const int2 *ent_up2, H4 *hist2,
                          int *bidx2)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const InstParams &P = V.P[V.inst[s]];
        const int ids = V.id[side_new][s];
        const int os = old_slot[s];
        const int e0 = up_off2[s], e1 = up_off2[s + 1];
        const int gl = P.off + ids;
        const int b0 = V.bond_off[gl], b1 = V.bond_off[gl + 1];
        for (int e = e0; e < e1; e++) {
            const int idt = V.id[side_new][ent_up2[e].x];
            H4 h;
            h.deltat = 0; h.thetarelc = 0; h.fcn = 0; h.fct = 0;
            if (os >= 0 && old_up_off) {
                const int q0 = old_up_off[os], q1 = old_up_off[os + 1];
                for (int q = q0; q < q1; q++) {
                    const int2 oe = old_ent_up[q];
                    if (old_id[oe.x] == idt) { h = old_hist[oe.y]; break; }
                }
            }
            hist2[e] = h;
            // bonds of this floe are sorted by the partner's id
            int lo = b0, hi = b1 - 1, bi = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) >> 1;
                const int v = V.bond_hi[mid];
                if (v == idt) { bi = mid; break; }
                if (v < idt) lo = mid + 1; else hi = mid - 1;
            }
            bidx2[e] = bi;
        }
    }
}

__global__ void k_copy_ids(Views V, int from)
{
    const int to = from ^ 1;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        V.id[to][s] = V.id[from][s];
        V.x0[to][s] = V.x0[from][s];
        V.y0[to][s] = V.y0[from][s];
    }
}

// ------------------------------------------------------------ host side
static int grid_for(int n, int block) { return n <= 0 ? 1 : (int)std::min<long long>((n + block - 1) / block, 148LL * 16); }

void launch_cell_keys(const Views &V, int cur, uint32_t *keys, int *vals, cudaStream_t st)
{
    k_cell_keys<<<grid_for(V.N, 256), 256, 0, st>>>(V, cur, keys, vals);
}

void launch_permute(const Views &V, int cur, const int *vals, const int *repack, int *old_slot, cudaStream_t st)
{
    k_permute<<<grid_for(V.N, 256), 256, 0, st>>>(V, cur, vals, repack, old_slot);
}

void launch_cell_ranges(const uint32_t *keys, int n, int *cstart, int *cend, cudaStream_t st)
{
    k_cell_ranges<<<grid_for(n, 256), 256, 0, st>>>(keys, n, cstart, cend);
}

void launch_nbr_count(const Views &V, int side, const int *cstart, const int *cend, int *cnt, cudaStream_t st)
{
    k_nbr_count<<<grid_for(V.N, 128), 128, 0, st>>>(V, side, cstart, cend, cnt);
}

void launch_nbr_fill(const Views &V, int side, const int *cstart, const int *cend, const int *row_off2,
                     int2 *ent2, double *dist2, int *nlo2, int up_by_id, cudaStream_t st)
{
    k_nbr_fill<<<grid_for(V.N, 128), 128, 0, st>>>(V, side, cstart, cend, row_off2, ent2, dist2, nlo2, up_by_id);
}

void launch_nbr_link(const Views &V, const int *row_off2, const int *nlo2, int2 *ent2, cudaStream_t st)
{
    k_nbr_link<<<grid_for(V.N, 128), 128, 0, st>>>(V, row_off2, nlo2, ent2);
}

void launch_split_rows(int N, const int *row_off2, const int *nlo2, const int2 *ent2, const int *lo_off,
                       const int *up_off, int2 *ent_lo, int2 *ent_up, cudaStream_t st)
{
    k_split_rows<<<grid_for(N, 128), 128, 0, st>>>(N, row_off2, nlo2, ent2, lo_off, up_off, ent_lo, ent_up);
}

void launch_migrate(const Views &V, int fp64, int side_new, const int *old_slot, const int *old_up_off,
                    const int2 *old_ent_up, const int *old_id, const void *old_hist, const int *up_off2,
                    const int2 *ent_up2, void *hist2, int *bidx2, cudaStream_t st)
{
    if (fp64)
        k_migrate<Hist4<double>><<<grid_for(V.N, 128), 128, 0, st>>>(
            V, side_new, old_slot, old_up_off, old_ent_up, old_id, (const Hist4<double> *)old_hist, up_off2,
            ent_up2, (Hist4<double> *)hist2, bidx2);
    else
        k_migrate<Hist4<float>><<<grid_for(V.N, 128), 128, 0, st>>>(
            V, side_new, old_slot, old_up_off, old_ent_up, old_id, (const Hist4<float> *)old_hist, up_off2,
            ent_up2, (Hist4<float> *)hist2, bidx2);
}

__global__ void k_row_lengths(int N, const int *row_off2, const int *nlo2, int *nup)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x)
        nup[s] = row_off2[s + 1] - row_off2[s] - nlo2[s];
}

void launch_row_lengths(int N, const int *row_off2, const int *nlo2, int *nup, cudaStream_t st)
{
    k_row_lengths<<<grid_for(N, 256), 256, 0, st>>>(N, row_off2, nlo2, nup);
}

void launch_copy_ids(const Views &V, int from, cudaStream_t st)
{
    k_copy_ids<<<grid_for(V.N, 256), 256, 0, st>>>(V, from);
}

}  // namespace godar
