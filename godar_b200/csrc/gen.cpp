// Synthetic floe-field placement (host code; input generation, not the step).
//
// GODAR builds initial fields with tools/init/gridded_placement.py:111-313
// (lattice placement with random radii).  The benchmark fields here need
// 70-85% area fraction with polydisperse radii, beyond what plain random
// sequential addition reaches, so disks are placed largest first; a rejected
// trial position is relaxed by pushing it out of the disks it overlaps (a few
// iterations) before a new random trial is drawn.  Overlap queries use one
// uniform grid per radius class (class c holds radii in [rmin 2^c, rmin 2^(c+1)))
// so that small disks do not scan the large cells of big disks.
#include <cmath>
#include <cstdint>
#include <vector>
#include <algorithm>
#include <numeric>

namespace {

struct Rng {  // splitmix64
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    double uni() { return (double)(next() >> 11) * 0x1.0p-53; }
};

struct ClassGrid {
    double rmax = 0, cwx = 1, cwy = 1;   // cells tile the domain exactly
    int ncx = 1, ncy = 1;
    std::vector<std::vector<int>> cells;
};

struct Placer {
    double Lx, Ly;
    bool px, py;
    const double *r;
    std::vector<double> X, Y;
    std::vector<ClassGrid> grids;
    double rmin;

    int cls(double rad) const {
        int c = (int)std::floor(std::log2(std::max(rad / rmin, 1.0)));
        return std::min<int>(c, (int)grids.size() - 1);
    }
    double wrapd(double d, double L, bool per) const {
        if (!per) return d;
        if (d > 0.5 * L) d -= L;
        else if (d < -0.5 * L) d += L;
        return d;
    }
    // Calls f(j, dx, dy, dist, minsep) for every placed disk j within reach.
    template <class F> void near(double x, double y, double rad, F f) const {
        for (const ClassGrid &g : grids) {
            if (g.rmax <= 0) continue;
            double reach = rad + g.rmax;
            int kx = (int)std::ceil(reach / g.cwx), ky = (int)std::ceil(reach / g.cwy);
            int cx = std::min((int)std::floor(x / g.cwx), g.ncx - 1);
            int cy = std::min((int)std::floor(y / g.cwy), g.ncy - 1);
            cx = std::max(cx, 0);
            cy = std::max(cy, 0);
            int x0 = cx - kx, x1 = cx + kx, y0 = cy - ky, y1 = cy + ky;
            if (!px) { x0 = std::max(x0, 0); x1 = std::min(x1, g.ncx - 1); }
            else if (x1 - x0 + 1 > g.ncx) { x0 = 0; x1 = g.ncx - 1; }
            if (!py) { y0 = std::max(y0, 0); y1 = std::min(y1, g.ncy - 1); }
            else if (y1 - y0 + 1 > g.ncy) { y0 = 0; y1 = g.ncy - 1; }
            for (int yy = y0; yy <= y1; yy++) {
                int wy = py ? ((yy % g.ncy) + g.ncy) % g.ncy : yy;
                for (int xx = x0; xx <= x1; xx++) {
                    int wx = px ? ((xx % g.ncx) + g.ncx) % g.ncx : xx;
                    for (int j : g.cells[(size_t)wy * g.ncx + wx]) {
                        double dx = wrapd(x - X[j], Lx, px), dy = wrapd(y - Y[j], Ly, py);
                        double d = std::sqrt(dx * dx + dy * dy);
                        double sep = rad + r[j];
                        if (d < sep) f(j, dx, dy, d, sep);
                    }
                }
            }
        }
    }
    bool fits(double x, double y, double rad) const {
        bool ok = true;
        near(x, y, rad, [&](int, double, double, double, double) { ok = false; });
        return ok;
    }
    void insert(int j) {
        ClassGrid &g = grids[cls(r[j])];
        int cx = (int)std::floor(X[j] / g.cwx), cy = (int)std::floor(Y[j] / g.cwy);
        cx = std::min(std::max(cx, 0), g.ncx - 1);
        cy = std::min(std::max(cy, 0), g.ncy - 1);
        g.cells[(size_t)cy * g.ncx + cx].push_back(j);
    }
};

}  // namespace

extern "C" {

// Places n disks of radii r in [0,Lx] x [0,Ly] (periodic flags per axis; on
// a non-periodic axis disks stay inside the walls).  Writes x, y for every
// disk; placement stops at the first disk that finds no place, and the disks
// not placed get NaN.  Returns the number placed.
int godar_gen_place(int n, const double *r, double Lx, double Ly, int periodic_x,
                    int periodic_y, uint64_t seed, int max_trials, double gap,
                    double *x, double *y)
{
    if (n <= 0) return 0;
    Placer P;
    std::vector<double> rg(r, r + n);
    for (double &v : rg) v += 0.5 * gap;  // keep a minimum gap between disks
    P.Lx = Lx; P.Ly = Ly; P.px = periodic_x != 0; P.py = periodic_y != 0; P.r = rg.data();
    P.X.assign(n, NAN); P.Y.assign(n, NAN);
    double rmin = *std::min_element(rg.begin(), rg.end()), rmax = *std::max_element(rg.begin(), rg.end());
    P.rmin = rmin > 0 ? rmin : 1.0;
    int nclass = 1 + (int)std::floor(std::log2(std::max(rmax / P.rmin, 1.0)));
    P.grids.resize(nclass);
    for (int c = 0; c < nclass; c++) {
        ClassGrid &g = P.grids[c];
        g.rmax = std::min(rmax, P.rmin * std::ldexp(1.0, c + 1));
        const double cell = std::max(2.0 * g.rmax, 1e-9);
        g.ncx = std::max(1, std::min(8192, (int)std::floor(Lx / cell)));
        g.ncy = std::max(1, std::min(8192, (int)std::floor(Ly / cell)));
        g.cwx = Lx / g.ncx;
        g.cwy = Ly / g.ncy;
        g.cells.assign((size_t)g.ncx * g.ncy, {});
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rg[a] > rg[b]; });
    Rng rng(seed * 0x2545F4914F6CDD1DULL + 1);
    int placed = 0;
    for (int idx : order) {
        double rad = rg[idx];
        double xlo = P.px ? 0.0 : rad, xhi = P.px ? Lx : Lx - rad;
        double ylo = P.py ? 0.0 : rad, yhi = P.py ? Ly : Ly - rad;
        if (xhi <= xlo || yhi <= ylo) continue;
        bool ok = false;
        double cx = 0, cy = 0;
        for (int t = 0; t < max_trials && !ok; t++) {
            cx = xlo + (xhi - xlo) * rng.uni();
            cy = ylo + (yhi - ylo) * rng.uni();
            for (int it = 0; it < 12; it++) {
                double mx = 0, my = 0;
                int hits = 0;
                P.near(cx, cy, rad, [&](int, double dx, double dy, double d, double sep) {
                    double push = (sep - d) * 1.0001 + 1e-9 * sep;
                    if (d > 0) { mx += dx / d * push; my += dy / d * push; }
                    else { mx += push; }
                    hits++;
                });
                if (!hits) { ok = true; break; }
                cx += mx; cy += my;
                if (P.px) cx -= Lx * std::floor(cx / Lx);
                else cx = std::min(std::max(cx, xlo), xhi);
                if (P.py) cy -= Ly * std::floor(cy / Ly);
                else cy = std::min(std::max(cy, ylo), yhi);
            }
        }
        if (!ok) break;   // the caller enlarges the domain and starts over
        P.X[idx] = cx; P.Y[idx] = cy;
        P.insert(idx);
        placed++;
    }
    for (int i = 0; i < n; i++) { x[i] = P.X[i]; y[i] = P.Y[i]; }
    return placed;
}

}  // extern "C"
