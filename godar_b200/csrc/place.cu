// Initial-condition generator on the GPU: places disks of given radii in a
// rectangular domain without overlap (random sequential addition with
// relaxation), for the dense polydisperse fields the benchmark
// configurations need.  The reference builds its initial fields with
// tools/init/gridded_placement.py:111-313 (a jittered lattice written as
// files/{x,y,r,h}<n>.dat, one value per line); the fields placed here are
// written in that format by generators.Field.write_reference_inputs.
//
// Disks are placed largest first, in radius classes (class c holds radii in
// [rmin 2^c, rmin 2^(c+1))).  For a class, the grid's cells are twice the
// class's largest radius, every disk already placed is entered into each
// cell its bounding box meets, and rounds repeat until the class is placed:
//   1. every unplaced disk of the class draws random positions (a
//      counter-based generator of seed, disk, round and attempt) and relaxes
//      each one by pushing it out of the placed disks it overlaps (the sum of
//      the overlaps, 12 iterations), keeping the first position that is free;
//   2. a free position is kept if no free position of a disk of the class
//      with a lower index overlaps it (the others retry next round).
// Every list is ordered (cells by key, disks by index within a cell), so a
// placement depends only on its inputs and seed.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/godar_gpu.h"
#include "common.cuh"
#include "kernels.h"

namespace godar {
namespace {

struct PGrid {
    int ncx, ncy;
    double cwx, cwy, Lx, Ly;
    int px, py;
};

GD_DEV uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

GD_DEV double uni(uint64_t &s)
{
    s += 0x9e3779b97f4a7c15ULL;
    return (double)(mix64(s) >> 11) * 0x1.0p-53;
}

GD_DEV double pwrap(double d, double L, int per)
{
    if (!per) return d;
    if (d > 0.5 * L) d -= L;
    else if (d < -0.5 * L) d += L;
    return d;
}

// Cell index range [a, b] of the interval [lo, hi] on one axis; a periodic
// range longer than the axis becomes the whole axis.
GD_DEV void cell_span(double lo, double hi, double cw, int nc, int per, int &a, int &b)
{
    a = (int)floor(lo / cw);
    b = (int)floor(hi / cw);
    if (per) {
        if (b - a + 1 >= nc) { a = 0; b = nc - 1; }
    } else {
        a = max(a, 0);
        b = min(b, nc - 1);
    }
}

GD_DEV int wrapc(int c, int nc, int per) { return per ? ((c % nc) + nc) % nc : c; }

// Coverage of the placed disks: one (cell, disk) item per cell that a placed
// disk's bounding box meets.
__global__ void k_cover_count(int n, const double *x, const double *y, const double *r,
                              const unsigned char *placed, PGrid G, int *cnt)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int c = 0;
        if (placed[i]) {
            int ax, bx, ay, by;
            cell_span(x[i] - r[i], x[i] + r[i], G.cwx, G.ncx, G.px, ax, bx);
            cell_span(y[i] - r[i], y[i] + r[i], G.cwy, G.ncy, G.py, ay, by);
            c = max(0, bx - ax + 1) * max(0, by - ay + 1);
        }
        cnt[i] = c;
    }
}

__global__ void k_cover_fill(int n, const double *x, const double *y, const double *r,
                             const unsigned char *placed, PGrid G, const int *off, uint32_t *key, int *val)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!placed[i]) continue;
        int ax, bx, ay, by;
        cell_span(x[i] - r[i], x[i] + r[i], G.cwx, G.ncx, G.px, ax, bx);
        cell_span(y[i] - r[i], y[i] + r[i], G.cwy, G.ncy, G.py, ay, by);
        int q = off[i];
        for (int cy = ay; cy <= by; cy++)
            for (int cx = ax; cx <= bx; cx++) {
                key[q] = (uint32_t)(wrapc(cy, G.ncy, G.py) * G.ncx + wrapc(cx, G.ncx, G.px));
                val[q] = i;
                q++;
            }
    }
}

// Whether wrapped cell coordinate w lies in the span [a, b] of cell_span.
GD_DEV bool in_span(int w, int a, int b, int nc, int per)
{
    if (!per) return w >= a && w <= b;
    if (b - a + 1 >= nc) return true;
    return ((w - a) % nc + nc) % nc <= b - a;
}

// Step 1: free positions of the unplaced disks [c0, c1).  A candidate spans
// at most 2 x 2 cells (cells are at least twice the class's largest
// radius); a placed disk met in several of them is counted in the first.
__global__ void k_trial(int c0, int c1, const double *r, const unsigned char *placed, const double *x,
                        const double *y, PGrid G, const int *cstart, const int *cend, const int *cov,
                        uint64_t seed, int round, int attempts, unsigned char *cand, double *tx, double *ty)
{
    for (int i = c0 + blockIdx.x * blockDim.x + threadIdx.x; i < c1; i += gridDim.x * blockDim.x) {
        cand[i] = 0;
        if (placed[i]) continue;
        const double rad = r[i];
        const double xlo = G.px ? 0.0 : rad, xhi = G.px ? G.Lx : G.Lx - rad;
        const double ylo = G.py ? 0.0 : rad, yhi = G.py ? G.Ly : G.Ly - rad;
        if (!(xhi > xlo && yhi > ylo)) continue;
        uint64_t s = mix64(seed ^ (0x632be59bd9b4e019ULL * (uint64_t)(i + 1))) ^ mix64((uint64_t)round + 1);
        bool found = false;
        for (int a = 0; a < attempts && !found; a++) {
            double cx = xlo + (xhi - xlo) * uni(s);
            double cy = ylo + (yhi - ylo) * uni(s);
            for (int it = 0; it < 12; it++) {
                int ax, bx, ay, by;
                cell_span(cx - rad, cx + rad, G.cwx, G.ncx, G.px, ax, bx);
                cell_span(cy - rad, cy + rad, G.cwy, G.ncy, G.py, ay, by);
                int wxs[2], wys[2];
                const int nxs = min(bx - ax + 1, 2), nys = min(by - ay + 1, 2);
                for (int k = 0; k < nxs; k++) wxs[k] = wrapc(ax + k, G.ncx, G.px);
                for (int k = 0; k < nys; k++) wys[k] = wrapc(ay + k, G.ncy, G.py);
                double mx = 0.0, my = 0.0;
                int hits = 0;
                for (int ci = 0; ci < nxs * nys; ci++) {
                    const int wx = wxs[ci % nxs], wy = wys[ci / nxs];
                    const int cell = wy * G.ncx + wx;
                    for (int q = cstart[cell]; q < cend[cell]; q++) {
                        const int j = cov[q];
                        const double dx = pwrap(cx - x[j], G.Lx, G.px), dy = pwrap(cy - y[j], G.Ly, G.py);
                        const double d = sqrt(dx * dx + dy * dy);
                        const double sep = rad + r[j];
                        if (!(d < sep)) continue;
                        int jax, jbx, jay, jby;
                        cell_span(x[j] - r[j], x[j] + r[j], G.cwx, G.ncx, G.px, jax, jbx);
                        cell_span(y[j] - r[j], y[j] + r[j], G.cwy, G.ncy, G.py, jay, jby);
                        bool seen = false;
                        for (int cj = 0; cj < ci && !seen; cj++)
                            seen = in_span(wxs[cj % nxs], jax, jbx, G.ncx, G.px) &&
                                   in_span(wys[cj / nxs], jay, jby, G.ncy, G.py);
                        if (seen) continue;
                        const double push = (sep - d) * 1.0001 + 1e-9 * sep;
                        if (d > 0) { mx += dx / d * push; my += dy / d * push; }
                        else mx += push;
                        hits++;
                    }
                }
                if (!hits) {
                    cand[i] = 1;
                    tx[i] = cx;
                    ty[i] = cy;
                    found = true;
                    break;
                }
                cx += mx;
                cy += my;
                if (G.px) cx -= G.Lx * floor(cx / G.Lx);
                else cx = fmin(fmax(cx, xlo), xhi);
                if (G.py) cy -= G.Ly * floor(cy / G.Ly);
                else cy = fmin(fmax(cy, ylo), yhi);
            }
        }
    }
}

__global__ void k_cand_keys(int c0, int c1, const unsigned char *cand, const double *tx, const double *ty, PGrid G,
                            uint32_t *key, int *val)
{
    for (int i = c0 + blockIdx.x * blockDim.x + threadIdx.x; i < c1; i += gridDim.x * blockDim.x) {
        const int k = i - c0;
        if (cand[i]) {
            const int cx = min(max((int)floor(tx[i] / G.cwx), 0), G.ncx - 1);
            const int cy = min(max((int)floor(ty[i] / G.cwy), 0), G.ncy - 1);
            key[k] = (uint32_t)(cy * G.ncx + cx);
        } else {
            key[k] = 0xffffffffu;      // sorts last, never looked up
        }
        val[k] = i;
    }
}

// Step 2: a free position is kept unless a free position of a lower-index
// disk of the class overlaps it (class radii are at most half a cell, so
// such a disk's centre lies in one of the 3 x 3 cells around).
__global__ void k_accept(int c0, int c1, const double *r, unsigned char *cand, const double *tx, const double *ty,
                         PGrid G, const int *cstart, const int *cend, const int *vals, unsigned char *placed,
                         double *x, double *y, int *nplaced)
{
    for (int i = c0 + blockIdx.x * blockDim.x + threadIdx.x; i < c1; i += gridDim.x * blockDim.x) {
        if (!cand[i]) continue;
        const int cx = min(max((int)floor(tx[i] / G.cwx), 0), G.ncx - 1);
        const int cy = min(max((int)floor(ty[i] / G.cwy), 0), G.ncy - 1);
        bool ok = true;
        for (int dyc = -1; dyc <= 1 && ok; dyc++)
            for (int dxc = -1; dxc <= 1 && ok; dxc++) {
                int xx = cx + dxc, yy = cy + dyc;
                if (G.px) xx = wrapc(xx, G.ncx, 1); else if (xx < 0 || xx >= G.ncx) continue;
                if (G.py) yy = wrapc(yy, G.ncy, 1); else if (yy < 0 || yy >= G.ncy) continue;
                // small grids: a wrapped neighbour may repeat the own cell or
                // another; repeats only repeat the same tests
                const int cell = yy * G.ncx + xx;
                for (int q = cstart[cell]; q < cend[cell]; q++) {
                    const int j = vals[q];
                    if (j >= i) continue;
                    const double dx = pwrap(tx[i] - tx[j], G.Lx, G.px), dy = pwrap(ty[i] - ty[j], G.Ly, G.py);
                    if (sqrt(dx * dx + dy * dy) < r[i] + r[j]) { ok = false; break; }
                }
            }
        if (ok) {
            placed[i] = 1;
            x[i] = tx[i];
            y[i] = ty[i];
            atomicAdd(nplaced, 1);
        }
    }
}

struct DevMem {
    std::vector<void *> ptrs;
    ~DevMem() { for (void *p : ptrs) cudaFree(p); }
    template <class T> T *get(size_t count) {
        void *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return (T *)p;
    }
};

int grid_n(long long n, int block) { return (int)std::max(1LL, std::min<long long>((n + block - 1) / block, 148LL * 16)); }

}  // namespace

// engine.cu: the thread's last error message
void set_last_error(const std::string &msg);

int place_disks(int n, const double *r_in, double Lx, double Ly, int px, int py, uint64_t seed, int max_rounds,
                double gap, double *x_out, double *y_out, int *placed_out)
{
    // largest first; ties keep input order
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return r_in[a] > r_in[b]; });
    std::vector<double> rs(n);
    for (int k = 0; k < n; k++) rs[k] = r_in[order[k]] + 0.5 * gap;
    const double rmin = std::max(rs[n - 1], 1e-9);
    auto cls = [&](double v) { return (int)std::floor(std::log2(std::max(v / rmin, 1.0))); };

    DevMem M;
    double *r = M.get<double>(n), *x = M.get<double>(n), *y = M.get<double>(n);
    double *tx = M.get<double>(n), *ty = M.get<double>(n);
    unsigned char *placed = M.get<unsigned char>(n), *cand = M.get<unsigned char>(n);
    int *cnt = M.get<int>(n + 1), *off = M.get<int>(n + 1), *counter = M.get<int>(4);
    if (!r || !x || !y || !tx || !ty || !placed || !cand || !cnt || !off || !counter) {
        set_last_error("device allocation failed");
        return GODAR_ERR_NOMEM;
    }
    cudaMemcpy(r, rs.data(), (size_t)n * 8, cudaMemcpyHostToDevice);
    cudaMemset(placed, 0, (size_t)n);
    cudaMemset(counter, 0, 16);
    int total_placed = 0;
    int k0 = 0;
    while (k0 < n) {
        // the class of disk k0: every disk down to half its class's radius
        const int c = cls(rs[k0]);
        int k1 = k0;
        while (k1 < n && cls(rs[k1]) == c) k1++;
        const double R = rs[k0];
        PGrid G;
        G.Lx = Lx; G.Ly = Ly; G.px = px; G.py = py;
        const double cell = std::max(2.0 * R, 1e-9);
        G.ncx = std::max(1, std::min(8192, (int)std::floor(Lx / cell)));
        G.ncy = std::max(1, std::min(8192, (int)std::floor(Ly / cell)));
        G.cwx = Lx / G.ncx;
        G.cwy = Ly / G.ncy;
        const long long ncell = (long long)G.ncx * G.ncy;
        int *cstart = M.get<int>(ncell), *cend = M.get<int>(ncell);
        int *c2s = M.get<int>(ncell), *c2e = M.get<int>(ncell);
        const int m = k1 - k0;
        uint32_t *ck = M.get<uint32_t>(m), *cka = M.get<uint32_t>(m);
        int *cv = M.get<int>(m), *cva = M.get<int>(m);
        const int nt2 = (m + 2047) / 2048;
        int *rsc2 = M.get<int>(256 * (size_t)nt2 + 1), *scr2 = M.get<int>(256 * (size_t)nt2 / 2048 + 64 + m / 2048 + 64);
        if (!cstart || !cend || !c2s || !c2e || !ck || !cka || !cv || !cva || !rsc2 || !scr2) {
            set_last_error("device allocation failed");
            return GODAR_ERR_NOMEM;
        }
        const int bits = std::max(1, (int)std::ceil(std::log2((double)std::max<long long>(ncell + 1, 2))));
        int left = m;
        for (int round = 0; round < max_rounds && left > 0; round++) {
            // coverage of every disk placed so far
            k_cover_count<<<grid_n(n, 256), 256>>>(n, x, y, r, placed, G, cnt);
            int *scr1 = nullptr;
            {
                const int nt = (n + 2047) / 2048;
                scr1 = M.get<int>(256 * (size_t)nt / 2048 + 64 + (size_t)n / 2048 + 64);
            }
            scan_excl(cnt, off, n, scr1, 0);
            int P = 0;
            cudaMemcpy(&P, off + n, sizeof(int), cudaMemcpyDeviceToHost);
            uint32_t *key = M.get<uint32_t>(P), *keya = M.get<uint32_t>(P);
            int *val = M.get<int>(P), *vala = M.get<int>(P);
            const int nt = (P + 2047) / 2048;
            int *rsc = M.get<int>(256 * (size_t)nt + 1), *scr = M.get<int>(256 * (size_t)nt / 2048 + 64 + P / 2048 + 64);
            if (!scr1 || !key || !keya || !val || !vala || !rsc || !scr) {
                set_last_error("device allocation failed");
                return GODAR_ERR_NOMEM;
            }
            cudaMemset(cstart, 0, (size_t)ncell * 4);
            cudaMemset(cend, 0, (size_t)ncell * 4);
            if (P > 0) {
                k_cover_fill<<<grid_n(n, 256), 256>>>(n, x, y, r, placed, G, off, key, val);
                radix_sort(key, val, keya, vala, P, bits, rsc, scr, 0);
                launch_cell_ranges(key, P, cstart, cend, 0);
            }
            // step 1
            k_trial<<<grid_n(m, 128), 128>>>(k0, k1, r, placed, x, y, G, cstart, cend, val, seed, round, 8, cand,
                                              tx, ty);
            // step 2: free positions by cell
            k_cand_keys<<<grid_n(m, 256), 256>>>(k0, k1, cand, tx, ty, G, ck, cv);
            radix_sort(ck, cv, cka, cva, m, 32, rsc2, scr2, 0);
            cudaMemset(c2s, 0, (size_t)ncell * 4);
            cudaMemset(c2e, 0, (size_t)ncell * 4);
            // keys of disks without a free position (0xffffffff) sort last:
            // ranges only for the real cells
            int mc = 0;
            {
                std::vector<uint32_t> hk(m);
                cudaMemcpy(hk.data(), ck, (size_t)m * 4, cudaMemcpyDeviceToHost);
                mc = (int)(std::lower_bound(hk.begin(), hk.end(), 0xffffffffu) - hk.begin());
            }
            if (mc > 0) launch_cell_ranges(ck, mc, c2s, c2e, 0);
            cudaMemset(counter, 0, sizeof(int));
            k_accept<<<grid_n(m, 128), 128>>>(k0, k1, r, cand, tx, ty, G, c2s, c2e, cv, placed, x, y, counter);
            int got = 0;
            if (cudaMemcpy(&got, counter, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
                set_last_error("placement kernels failed");
                return GODAR_ERR_CUDA;
            }
            left -= got;
            total_placed += got;
            // this round's temporaries
            for (int q = 0; q < 7; q++) {
                cudaFree(M.ptrs.back());
                M.ptrs.pop_back();
            }
        }
        if (left > 0) break;     // the caller enlarges the domain
        k0 = k1;
    }
    std::vector<double> hx(n), hy(n);
    std::vector<unsigned char> hp(n);
    cudaMemcpy(hx.data(), x, (size_t)n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(hy.data(), y, (size_t)n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(hp.data(), placed, (size_t)n, cudaMemcpyDeviceToHost);
    if (cudaGetLastError() != cudaSuccess) {
        set_last_error("placement kernels failed");
        return GODAR_ERR_CUDA;
    }
    for (int k = 0; k < n; k++) {
        x_out[order[k]] = hp[k] ? hx[k] : NAN;
        y_out[order[k]] = hp[k] ? hy[k] : NAN;
    }
    if (placed_out) *placed_out = total_placed;
    return GODAR_OK;
}

}  // namespace godar

extern "C" int godar_gpu_place(int n, const double *r, double Lx, double Ly, int periodic_x, int periodic_y,
                               uint64_t seed, int max_rounds, double gap, double *x, double *y, int *placed)
{
    if (n <= 0 || !r || !x || !y || !(Lx > 0) || !(Ly > 0) || !std::isfinite(Lx) || !std::isfinite(Ly) ||
        max_rounds <= 0 || !std::isfinite(gap))
        return GODAR_ERR_BAD_INPUT;
    // a negative gap lets disks overlap by up to -gap, as long as every
    // disk keeps a positive placement radius r + gap / 2
    for (int i = 0; i < n; i++)
        if (!(r[i] > 0) || !std::isfinite(r[i]) || !(r[i] + 0.5 * gap > 0)) return GODAR_ERR_BAD_INPUT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return GODAR_ERR_NO_DEVICE;
    }
    return godar::place_disks(n, r, Lx, Ly, periodic_x != 0, periodic_y != 0, seed, max_rounds, gap, x, y, placed);
}
