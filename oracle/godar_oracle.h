/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product.
 *
 * A plain-C FP64 restatement of GODAR's per-time-step loop `stepper`
 * (model/src/stepper.f90:1-345) and every routine it calls.  It is the checker
 * for the CUDA path: tests, the smoke check and the bench's CPU-baseline leg
 * call it; nothing in godar_b200/ does.
 *
 * PARITY UNPINNED against the reference binary: the reference is Fortran + MPI
 * + the external coretran kd-tree library, none of which can be built here,
 * and the reference ships no tests, golden vectors or fixtures.  The oracle is
 * pinned instead by analytic known-answer tests (tests/test_oracle_kat.py) and
 * by the committed fixtures under tests/golden/ that it generated.
 *
 * Semantics pinned by this restatement where the reference is silent:
 *   - coretran's radius query is taken as: all j with
 *     sqrt((x_i-x_j)^2 + (y_i-y_j)^2) <= r_i + rtree (FP64, no FMA), returned in
 *     ascending distance, ties by index; element 1 (the query floe itself) is
 *     dropped as at stepper.f90:80-82.
 *   - integer powers x**2, x**3, x**4, x**5 are evaluated as x*x, (x*x)*x,
 *     (x*x)*(x*x), ((x*x)*x)*(x*x); real powers **2d0 and **3d0 likewise.
 *   - Fortran single-precision literals keep their single-precision value:
 *     0.18 in S_shelter (forcing.f90:261) is (double)0.18f.
 *   - sign(1d0, -0d0) = -1 and heaviside(-0d0) = 0 (IEEE copysign).
 *
 * Two ridging orders (see gdo_step):
 *   GDO_RIDGE_REFERENCE  r, h, mass... of a floe change inside the pair loop as
 *                        soon as a plastic contact fires (ridging.f90:71-93),
 *                        exactly the reference's sequential order.
 *   GDO_RIDGE_DEFERRED   every pair computation reads the shapes at the start of
 *                        the step (plus the pair's own update); the shape
 *                        changes are applied to each floe in its own event
 *                        order, before its wall contacts.  This is the order the
 *                        GPU uses.
 */
#ifndef GODAR_ORACLE_H
#define GODAR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same field order and types as godar_params in include/godar_gpu.h. */
typedef struct gdo_params {
    int32_t dynamics, slipping, thermodyn, cohesion, ridging, shelter;
    double rtree, ntree, dt, nt, comp;
    double Cdair, Csair, Cdwater, Cswater, z0w, lat, rhoair, rhoice, rhowater;
    double e_modul, poiss_ratio, friction_coeff, rest_coeff, sigmanc_crit;
    double eb, lambda_rb, lambda_lb, sigmatb_crit, sigmacb_crit, tau_crit,
           bond_lim, dmax, dtd, dth;
    double uw, vw, ua, va;
    double nx, ny;
    double ec, gc, beta, pi, sin_lat;
    int32_t boundary;
    int32_t bond_seed;
    double bond_lim_rel;
    double bond_frac;
    int32_t field_nx, field_ny;
} gdo_params;

enum { GDO_RIDGE_REFERENCE = 0, GDO_RIDGE_DEFERRED = 1 };
enum { GDO_MATH_DET = 0, GDO_MATH_LIBM = 1 };

/* Per-floe output fields, in this order, for gdo_get_floes(). */
enum {
    GDO_F_X, GDO_F_Y, GDO_F_U, GDO_F_V, GDO_F_R, GDO_F_H, GDO_F_THETA,
    GDO_F_OMEGA, GDO_F_TFX, GDO_F_TFY, GDO_F_FCX, GDO_F_FCY, GDO_F_FBX,
    GDO_F_FBY, GDO_F_M, GDO_F_MC, GDO_F_MB, GDO_F_TSIGXX, GDO_F_TSIGYY,
    GDO_F_TSIGXY, GDO_F_TSIGYX, GDO_F_TP, GDO_F_FAX, GDO_F_FAY, GDO_F_FWX,
    GDO_F_FWY, GDO_F_MA, GDO_F_MW, GDO_F_FCORX, GDO_F_FCORY, GDO_F_FXBC,
    GDO_F_FYBC, GDO_F_MBC, GDO_F_HSFA, GDO_F_HSFW, GDO_F_MASS,
    GDO_F_COUNT
};

/* Pair lists for gdo_get_pairs(). */
enum { GDO_P_CANDIDATES = 0, GDO_P_CONTACTS = 1, GDO_P_BONDS = 2 };

typedef struct gdo_state gdo_state;

int gdo_params_size(void);

/* Creates a field of n floes (0-based indices; i < j means "i is the
 * reference's lower index").  u, v may be NULL (zero, ini_get.f90:170-174).
 * nb restart bonds (bi < bj) with damage (may be NULL) as read by
 * read_sparse_restart; their geometry is computed from the given positions.
 * field: NULL or 4*fnx*fny doubles (ua, va, uw, vw planes) sampled bilinearly
 * on the nodes of a fnx x fny grid spanning [0,nx] x [0,ny]. */
gdo_state *gdo_create(const gdo_params *p, int n, const double *x,
                      const double *y, const double *r, const double *h,
                      const double *theta, const double *omega,
                      const double *u, const double *v, int nb,
                      const int32_t *bi, const int32_t *bj,
                      const double *damage, const double *field);
void gdo_set_modes(gdo_state *s, int ridge_mode, int math_mode);
/* One call of `stepper(tstep, restart)`. */
int gdo_step(gdo_state *s, int tstep, int restart);
int gdo_run(gdo_state *s, int tstep0, int nsteps, int restart);
/* out: GDO_F_COUNT * n doubles, field-major. */
void gdo_get_floes(const gdo_state *s, double *out);
/* Fills (i, j, value) for the list; returns the count (may exceed cap). */
int gdo_get_pairs(const gdo_state *s, int which, int32_t *pi, int32_t *pj,
                  double *val, int cap);
/* Pair history (deltat, thetarelc, fcn, fct) of pair (i,j); 0 if absent. */
int gdo_get_pair_hist(const gdo_state *s, int i, int j, double *out4);
void gdo_destroy(gdo_state *s);

/* Deterministic math, exported for the tests. */
double gdo_exp(double x);
double gdo_log(double x);
double gdo_asin(double x);
double gdo_acos(double x);

#ifdef __cplusplus
}
#endif
#endif
