// Shared device-side definitions: per-instance parameters, the device state
// views, and the small helpers every kernel uses.
//
// Data layout in HBM (structure of arrays, one batch = many floe fields):
//   floes      N slots; instance b owns slots [off_b, off_b + n_b).  Within an
//              instance the slots are kept in cell order (re-sorted at every
//              neighbour-list rebuild) so that neighbours sit close in memory.
//              id[s] is the floe's reference index (0-based) in its instance;
//              all reference semantics (lower index, summation order) use id.
//   state      two sides (ping-pong): a step reads side c and writes side 1-c,
//              because neighbours read a floe's start-of-step state while the
//              floe itself integrates.
//   rows       a neighbour superset (Verlet list): every t with
//              dist(s,t) <= r_lo + rtree + skin at build time (lo = the floe of
//              lower id), split into owner rows (partners of higher id,
//              ascending distance in the FP64 path, ascending id in the
//              mixed path) and partner rows (partners of lower id,
//              ascending id).
//   pairs      one record per unordered pair, indexed by its owner entry:
//              contact history (deltat, thetarelc, last fcn, last fct),
//              updated in place (one thread owns a pair in a step), and a
//              bond index.
//   bonds      one table per batch, keyed by the reference ids, CSR by the
//              lower id; static geometry and strain/damage state (in place).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace godar {

enum : int {
    BC_PERIODIC_X = 1, BC_PERIODIC_Y = 2, BC_OPEN_LEFT = 4,
    BC_OPEN_RIGHT = 8, BC_OPEN_BOTTOM = 16, BC_OPEN_TOP = 32
};

// Whether a field has any solid wall (a side neither periodic nor open).
__host__ __device__ inline bool has_walls(int b)
{
    const bool wy = !(b & BC_PERIODIC_Y) && (!(b & BC_OPEN_BOTTOM) || !(b & BC_OPEN_TOP));
    const bool wx = !(b & BC_PERIODIC_X) && (!(b & BC_OPEN_LEFT) || !(b & BC_OPEN_RIGHT));
    return wx || wy;
}

// status bits written by kernels
enum : int {
    ST_EXPIRED = 1,      // a floe moved more than skin/2 since the last rebuild
    ST_NAN = 2,          // non-finite state produced
    ST_ROW_OVERFLOW = 4, // neighbour rows exceed their capacity
    ST_ORPHAN = 8,       // a live bond left the neighbour superset
    ST_TIMEOUT = 16      // a bounded device wait gave up (the step did not complete)
};
// the states in which the step kernels do nothing until the host has acted
constexpr int ST_ABORT = ST_EXPIRED | ST_NAN | ST_ROW_OVERFLOW | ST_TIMEOUT;

struct InstParams {
    double dt, rtree, skin;
    double rhoair, rhoice, rhowater, Cdair, Csair, Cdwater, Cswater, z0w;
    double ec, gc, beta, pi, sin_lat, mu, sigmanc_crit;
    double eb, lambda_rb, lambda_lb, sigmatb_crit, sigmacb_crit, tau_crit, dmax, dtd, dth;
    double ua, va, uw, vw;
    double nx, ny;
    double cw, ch;          // cell width / height [m]
    double log10z0;         // log(10 / z0w) (forcing.f90:222), precomputed
    float log10z0f;
    long long field_off;    // this instance's forcing grid in the batch field array, -1 = none
    int fnx, fny;
    int slipping, ridging, shelter, cohesion, boundary, bond_seed;
    int n, off;             // slots [off, off + n)
    int ncx, ncy;           // cell grid
    long long coff;         // first global cell key of this instance
    int kx, ky;             // neighbour-build stencil half widths [cells]
    // FP32 constants of the mixed path
    float f_dt, f_piec, f_ktc, f_beta, f_mu, f_sigc, f_llb, f_rhoipi, f_hfa, f_hfw;
    float f_eb, f_inv_tau, f_inv_sigcb, f_inv_sigtb;   // mixed bonds: eb and 1 / the critical stresses
    double dt_dtd, dt_dth;  // dt / dtd, dt / dth (mixed damage update)
    double hfa_fac, hfw_fac;   // (rhowater - rhoice) / rhowater, rhoice / rhowater (mixed shapes)
};

template <typename T> struct Hist4 { T deltat, thetarelc, fcn, fct; };

// Bond records (array of structures: one bond is a few sectors, not eleven
// separate arrays).  Dynamic state has two ping-pong sides.
struct __align__(16) BondDyn {
    double dnb, dtb, thji, thij, dmg;   // deltanb, deltatb, thetarelb(j,i), thetarelb(i,j), damageb
    int flag;                           // bond(j,i)
    int pad;
};
struct __align__(16) BondStat {
    double rb, hb, lb, sb, ib;          // bond_properties (bonds.f90:255-262)
    double pad;
    // FP32 undamaged beam coefficients of bonds.f90:109-117 for the mixed
    // path: EA/L, 12EI/L^3, 6EI/L^2, 4EI/L, 2EI/L, EI/L, EA L, 1/L
    float k_ax, k_sh1, k_sh2, k_r1, k_r2, ei_l, ea_l, inv_l;
};

// The bond rule of one field for bond creation at admission (stepper.f90:93-101
// with the relative limit and hashed fraction extensions): fresh = create
// the field's bonds on the device; boff = its first index in the bond table.
struct BondRule {
    double lim, lim_rel, frac;
    int seed, fresh, boff, pad;
};

// The mixed path's copy of a bond's static record (16 bytes): rb, hb, lb
// (bond_properties, bonds.f90:255-262) and 1/lb in FP32.  sb and ib, the
// beam coefficients of bonds.f90:109-117 and the section factors of
// bond_breaking (bonds.f90:164-212) follow from them in registers
// (BondStat32).
struct __align__(16) BondGeom32 {
    float rb, hb, lb, inv_l;
};

// A bond's coefficients in FP32 as the mixed bond kernel uses them: EA/L,
// EI/L, EA L and 1/L, from which every beam coefficient follows, and the
// section numbers as the factors they are used with: sb, 1/sb, rb/ib and the
// reciprocals of the critical stresses times hb.
struct BondStat32 {
    float k_ax, ei_l, ea_l, inv_l;
    float sb, inv_sb, rb_ib, inv_tau_hb;
    float inv_sigc_hb, inv_sigt_hb;
};

// What a neighbour reads of a floe in the mixed-precision pair kernel, packed
// into one 48-byte record (positions and radius FP64, the rest FP32).
// The first 32-byte sector holds what the candidate screen reads (position,
// radius, instance); the moment of inertia is m r^2 / 2 (physics.f90:191).
struct __align__(16) Snap {
    double x, y, r;
    int inst;
    float h;
    float u, v, om;
    float mass;                         // floe_properties (physics.f90:190)
};

// Device pointers of one batch.  Arrays with [2] are the two ping-pong sides.
struct Views {
    int N;                 // slots
    int ninst;
    const InstParams *P;   // [ninst]
    const int *inst;       // [N] instance of each slot
    // floe state, two sides
    double *x[2], *y[2], *th[2], *u[2], *v[2], *om[2], *r[2], *h[2];
    double *dtb1[2], *dtb2[2], *thb1[2], *thb2[2];   // wall histories (CB_variables.h:55-58)
    int *id[2];
    double *x0[2], *y0[2];                          // positions at the last rebuild
    // neighbour rows, as two CSRs over slots: the owner rows (partners of
    // higher id; entry .y = the pair's index, its position at build time) and
    // the partner rows (partners of lower id, ascending id; .y = the pair's
    // index in the owner rows)
    int *up_off;           // [N+1]
    int *lo_off;           // [N+1]
    int2 *ent_up;          // [P]
    int2 *ent_lo;          // [P]
    int *bidx;             // [P] bond index of the pair, -1 none
    void *hist[2];         // [P] Hist4<double> (FP64) or Hist4<float> (mixed), in place: both sides are one table
    float *pdn;            // [P] deltan of the last diagnostic step (NaN: not a candidate)
    double *edist;         // [P] FP64 path: the step's distance of every owner entry the screen visited (row order)
    // bonds
    int *bond_off;         // [N+1] CSR over global ids (off_b + id), by lower id
    int *bond_hi;          // [NB] higher id of the bond
    BondStat *bstat;       // [NB]
    BondDyn *bdyn[2];      // [NB] in place: both sides are one table
    // mixed path: packed neighbour view of every floe, per side
    Snap *snap[2];
    // forcing grids
    const double *field;
    // outputs
    double *diag;          // [14][N]
    // status
    int *status;
    int *expired_at;       // the global number of the first step that expired
    const int *step_base;  // the global number of the running chunk's first step
    int pdl;               // host side: launch the step kernels with programmatic dependent launch
    unsigned long long *counters;   // [4] candidates, contacts, bonds, plastic events
};

#define GD_DEV __device__ __forceinline__

// the FP64 pair work lists: [0] general, [1] bonded pairs out of contact
// (no sheltering, no diagnostics); n[0], n[1] their lengths
struct __align__(32) FP64Item {
    int p, g, t, bi;     // pair index, owner slot, partner slot, bond index
    double dx, dy;       // the pair's minimum-image offset x_g - x_t, y_g - y_t
};
struct FP64Lists {
    FP64Item *work[2];
    int *n;
};

// The global number of step `sic` of the running chunk: steps are numbered
// from the last neighbour-list rebuild across chunks, so that a chunk queued
// behind one that has not been checked yet knows an expiry from before it.
GD_DEV int global_step(const Views &V, int sic) { return *V.step_base + sic; }

// Whether the floe update of step `sic` of a chunk must stop: an error state,
// or a neighbour list that expired at an EARLIER step.  The floe update is
// the kernel that raises ST_EXPIRED, and the step that raised it is kept, so
// its blocks that start after another block of the same launch raised it
// still run (expired_at is then this step, not below it).  The kernels
// before the floe update in a step stop on any ST_ABORT state: an expiry
// they see was raised by an earlier step.
GD_DEV bool floe_update_stopped(const Views &V, int sic)
{
    const int s = *(volatile const int *)V.status;
    if (s & (ST_ABORT & ~ST_EXPIRED)) return true;
    return (s & ST_EXPIRED) && *(volatile const int *)V.expired_at < global_step(V, sic);
}

// Programmatic dependent launch of the step kernels.  A step kernel launched
// with it may be scheduled while the kernel before it on the stream still
// runs its last blocks; griddepcontrol.wait holds every thread, before it
// touches memory, until that kernel has completed and its writes are
// visible, so the kernel sees memory exactly as in plain stream order (the
// wait returns at once for a kernel launched without it).  The kernel then
// lets the next step kernel be scheduled.
GD_DEV void step_kernel_entry()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

GD_DEV double wrap_d(double d, double L, bool per)
{
    if (!per) return d;
    if (d > 0.5 * L) d = d - L;
    else if (d < -0.5 * L) d = d + L;
    return d;
}

// floe_properties (physics.f90:179-198)
struct Shape { double r, h, mass, inertia, hfa, hfw; };

GD_DEV Shape make_shape(const InstParams &P, double r, double h)
{
    Shape s;
    s.r = r;
    s.h = h;
    s.mass = ((P.rhoice * P.pi) * h) * (r * r);
    s.inertia = (0.5 * s.mass) * (r * r);
    s.hfa = (h * (P.rhowater - P.rhoice)) / P.rhowater;
    s.hfw = (h * P.rhoice) / P.rhowater;
    return s;
}

// seeded pair hash of the bond_frac extension (same on host and device)
__host__ __device__ inline uint32_t pair_hash32(uint32_t seed, uint32_t i, uint32_t j)
{
    uint32_t h = seed * 0x9e3779b9u ^ (i * 0x85ebca6bu) ^ (j * 0xc2b2ae35u + 0x27d4eb2fu);
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    return h;
}

// winds_currents (forcing.f90:1-29): uniform values plus the bilinear
// interpolation of the optional node grid (extension).
GD_DEV void wind_at(const InstParams &P, const double *field, double x, double y,
                    double &ua, double &va, double &uw, double &vw)
{
    if (P.field_off < 0) {
        ua = P.ua; va = P.va; uw = P.uw; vw = P.vw;
        return;
    }
    const int fnx = P.fnx, fny = P.fny;
    const double xc = x < 0.0 ? 0.0 : (x > P.nx ? P.nx : x);
    const double yc = y < 0.0 ? 0.0 : (y > P.ny ? P.ny : y);
    double fx = (xc / P.nx) * (double)(fnx - 1);
    double fy = (yc / P.ny) * (double)(fny - 1);
    // non-finite positions sample the corner node instead of leaving the grid
    if (!(fx >= 0.0)) fx = 0.0;
    if (!(fy >= 0.0)) fy = 0.0;
    if (fx > (double)(fnx - 1)) fx = (double)(fnx - 1);
    if (fy > (double)(fny - 1)) fy = (double)(fny - 1);
    int ix = (int)floor(fx), iy = (int)floor(fy);
    if (ix > fnx - 2) ix = fnx - 2;
    if (iy > fny - 2) iy = fny - 2;
    const double tx = fx - (double)ix, ty = fy - (double)iy;
    const double *F = field + P.field_off;
    double val[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const double *Fc = F + (size_t)c * fnx * fny;
        const double v00 = Fc[iy * fnx + ix], v10 = Fc[iy * fnx + ix + 1];
        const double v01 = Fc[(iy + 1) * fnx + ix], v11 = Fc[(iy + 1) * fnx + ix + 1];
        val[c] = (1.0 - ty) * ((1.0 - tx) * v00 + tx * v10) + ty * ((1.0 - tx) * v01 + tx * v11);
    }
    ua = P.ua + val[0]; va = P.va + val[1]; uw = P.uw + val[2]; vw = P.vw + val[3];
}

}  // namespace godar
