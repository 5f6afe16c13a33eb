/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- a plain-C FP64 restatement of GODAR's
 * time step.  Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline
 * use it; the product never links it.  PARITY UNPINNED against the reference
 * binary (no Fortran/MPI/coretran here, no reference tests or golden vectors);
 * see godar_oracle.h for the pinned semantics and the analytic known-answer
 * tests that check it.
 *
 * Each routine names the reference routine it restates (file:line within the
 * GODAR project).  Expressions keep the reference's operand order so that
 * rounding matches the Fortran evaluation order; build with -ffp-contract=off.
 */
#include "godar_oracle.h"
#include "detmath_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define BC_PERIODIC_X 1
#define BC_PERIODIC_Y 2
#define BC_OPEN_LEFT 4
#define BC_OPEN_RIGHT 8
#define BC_OPEN_BOTTOM 16
#define BC_OPEN_TOP 32

/* ------------------------------------------------------------------ */
/* sparse stand-in for the dense (n,n) pair arrays of CB_variables.h,  */
/* CB_bond.h, CB_forcings.h; an absent key reads as all zero, exactly  */
/* like the zero-initialised COMMON storage (ini_get.f90:206-227).     */
/* ------------------------------------------------------------------ */
typedef struct pairrec {
    uint64_t key;
    double deltat, thetarelc, fcn, fct, fcr, mcc, deltan, delt_ridge, ac;
    int32_t bond;
    double damageb, deltanb, deltatb, thb_ji, thb_ij;
    double rb, hb, lb, sb, ib, fbn, fbt, mbb_ji, mbb_ij;
} pairrec;

#define EMPTY_KEY 0xffffffffffffffffULL

struct gdo_state {
    gdo_params p;
    int n;
    int ridge_mode, math_mode;
    double *x, *y, *r, *h, *hfa, *hfw, *mass, *inertia, *u, *v, *theta, *omega;
    double *r0, *h0, *hfa0, *hfw0, *mass0, *inertia0;
    double *ua_i, *va_i, *uw_i, *vw_i;
    double *fcx, *fcy, *mc, *fbx, *fby, *mb, *tfx, *tfy, *m, *fcorx, *fcory;
    double *fn_bc, *ft_bc, *fr_bc, *fx_bc, *fy_bc, *mc_bc, *m_bc;
    double *deltat_bc1, *deltat_bc2, *theta_bc1, *theta_bc2, *delt_ridge_bc;
    double *sigxx, *sigyy, *sigxy, *sigyx;
    double *sigxx_bc, *sigyy_bc, *sigxy_bc, *sigyx_bc;
    double *sigxx_aw, *sigyy_aw, *sigxy_aw, *sigyx_aw;
    double *tsigxx, *tsigyy, *tsigxy, *tsigyx;
    double *tac, *tab, *pc, *pb, *tp, *ta_bc, *p_bc;
    double *fax, *fay, *fwx, *fwy, *ma, *mw;
    double *hsfa_min, *hsfw_min; /* local_hsfa_min / local_hsfw_min (CB_mpi.h:75-76) */
    double *field;
    /* pair map */
    pairrec *tab_p;
    uint64_t cap, used;
    /* candidates of the last step (for topology checks) */
    int32_t *cand_i, *cand_j;
    int ncand, capcand;
    /* candidate search scratch */
    int *cell_head, *cell_next;
    int ncx, ncy;
    double cwx, cwy;
    int *qbuf; double *qdist; int qcap;
};

/* ------------------------------ math ------------------------------ */
static inline double M_exp(const gdo_state *s, double x) { return s->math_mode == GDO_MATH_LIBM ? exp(x) : odm_exp(x); }
static inline double M_log(const gdo_state *s, double x) { return s->math_mode == GDO_MATH_LIBM ? log(x) : odm_log(x); }
static inline double M_acos(const gdo_state *s, double x) { return s->math_mode == GDO_MATH_LIBM ? acos(x) : odm_acos(x); }
static inline double M_asin(const gdo_state *s, double x) { return s->math_mode == GDO_MATH_LIBM ? asin(x) : odm_asin(x); }

double gdo_exp(double x) { return odm_exp(x); }
double gdo_log(double x) { return odm_log(x); }
double gdo_asin(double x) { return odm_asin(x); }
double gdo_acos(double x) { return odm_acos(x); }

int gdo_params_size(void) { return (int)sizeof(gdo_params); }

static inline double fmaxd(double a, double b) { return a > b ? a : b; }
static inline double fmind(double a, double b) { return a < b ? a : b; }

/* ---------------------------- pair map ---------------------------- */
static uint64_t hash64(uint64_t k)
{
    k ^= k >> 33; k *= 0xff51afd7ed558ccdULL; k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL; k ^= k >> 33;
    return k;
}

static void map_grow(gdo_state *s);

static pairrec *map_find(const gdo_state *s, int i, int j)
{
    uint64_t key = ((uint64_t)(uint32_t)i << 32) | (uint32_t)j;
    uint64_t mask = s->cap - 1, h = hash64(key) & mask;
    for (;;) {
        pairrec *e = &s->tab_p[h];
        if (e->key == key) return e;
        if (e->key == EMPTY_KEY) return NULL;
        h = (h + 1) & mask;
    }
}

static pairrec *map_get(gdo_state *s, int i, int j)
{
    pairrec *e = map_find(s, i, j);
    if (e) return e;
    if ((s->used + 1) * 2 > s->cap) map_grow(s);
    uint64_t key = ((uint64_t)(uint32_t)i << 32) | (uint32_t)j;
    uint64_t mask = s->cap - 1, h = hash64(key) & mask;
    while (s->tab_p[h].key != EMPTY_KEY) h = (h + 1) & mask;
    e = &s->tab_p[h];
    memset(e, 0, sizeof(*e));
    e->key = key;
    s->used++;
    return e;
}

static void map_grow(gdo_state *s)
{
    uint64_t oldcap = s->cap;
    pairrec *old = s->tab_p;
    s->cap = oldcap ? oldcap * 2 : 1024;
    s->tab_p = (pairrec *)malloc(s->cap * sizeof(pairrec));
    for (uint64_t k = 0; k < s->cap; k++) s->tab_p[k].key = EMPTY_KEY;
    s->used = 0;
    for (uint64_t k = 0; k < oldcap; k++) {
        if (old[k].key == EMPTY_KEY) continue;
        uint64_t mask = s->cap - 1, h = hash64(old[k].key) & mask;
        while (s->tab_p[h].key != EMPTY_KEY) h = (h + 1) & mask;
        s->tab_p[h] = old[k];
        s->used++;
    }
    free(old);
}

/* --------------------------- geometry ----------------------------- */
static inline double wrap_dx(const gdo_state *s, double dx, int axis)
{
    int per = axis == 0 ? (s->p.boundary & BC_PERIODIC_X) : (s->p.boundary & BC_PERIODIC_Y);
    if (!per) return dx;
    double L = axis == 0 ? s->p.nx : s->p.ny;
    if (dx > 0.5 * L) dx = dx - L;
    else if (dx < -0.5 * L) dx = dx + L;
    return dx;
}

/* hash used by the bond_frac extension (a seeded selection of pairs) */
static inline uint32_t pair_hash32(uint32_t seed, uint32_t i, uint32_t j)
{
    uint32_t h = seed * 0x9e3779b9u ^ (i * 0x85ebca6bu) ^ (j * 0xc2b2ae35u + 0x27d4eb2fu);
    h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
    return h;
}

/* floe_properties (physics.f90:179-198) */
static void floe_properties(const gdo_params *p, double r, double h, double *mass,
                            double *inertia, double *hfa, double *hfw)
{
    double ms = ((p->rhoice * p->pi) * h) * (r * r);
    *mass = ms;
    *inertia = (0.5 * ms) * (r * r);
    *hfa = (h * (p->rhowater - p->rhoice)) / p->rhowater;
    *hfw = (h * p->rhoice) / p->rhowater;
}

/* fit (contact_forces.f90:247-266) */
static inline double fit(double xi)
{
    const double p1 = 9117e-4, p2 = 2722e-4, p3 = 3324e-6, q1 = 1524e-3, q2 = 3159e-5;
    return ((p1 * (xi * xi) + p2 * xi) + p3) / (((xi * xi) + q1 * xi) + q2);
}

/* heaviside (forcing.f90:226-236): sign(0.5, x) + 0.5, IEEE sign of zero */
static inline double heaviside(double x) { return copysign(0.5, x) + 0.5; }

/* S_shelter (forcing.f90:238-270) */
static double S_shelter(const gdo_state *s, double hfi, double hfj, double deltan,
                        double cosa, double sina, double uf, double vf)
{
    double wnorm = sqrt(uf * uf + vf * vf) + 1e-20;
    double costheta = (uf * cosa + vf * sina) / wnorm;
    const double c018 = (double)0.18f;
    double ex = M_exp(s, -((c018 * fabs(deltan / costheta)) / hfj));
    double D = (1.0 - (1.0 - heaviside(deltan)) * (1.0 - ex))
               - (heaviside(deltan) * heaviside(hfi - hfj)) * (1.0 - hfj / hfi);
    double G = heaviside(costheta) * costheta;
    return 1.0 - D * G;
}

/* winds_currents (forcing.f90:1-29) + the gridded-field extension */
static void winds_currents(gdo_state *s, int i)
{
    const gdo_params *p = &s->p;
    if (!s->field || p->field_nx < 2 || p->field_ny < 2) {
        s->ua_i[i] = p->ua; s->va_i[i] = p->va;
        s->uw_i[i] = p->uw; s->vw_i[i] = p->vw;
        return;
    }
    int fnx = p->field_nx, fny = p->field_ny;
    double xc = s->x[i] < 0.0 ? 0.0 : (s->x[i] > p->nx ? p->nx : s->x[i]);
    double yc = s->y[i] < 0.0 ? 0.0 : (s->y[i] > p->ny ? p->ny : s->y[i]);
    double fx = (xc / p->nx) * (double)(fnx - 1);
    double fy = (yc / p->ny) * (double)(fny - 1);
    if (!(fx >= 0.0)) fx = 0.0;   /* non-finite positions sample the corner */
    if (!(fy >= 0.0)) fy = 0.0;
    if (fx > (double)(fnx - 1)) fx = (double)(fnx - 1);
    if (fy > (double)(fny - 1)) fy = (double)(fny - 1);
    int ix = (int)floor(fx), iy = (int)floor(fy);
    if (ix > fnx - 2) ix = fnx - 2;
    if (iy > fny - 2) iy = fny - 2;
    double tx = fx - (double)ix, ty = fy - (double)iy;
    double val[4];
    for (int c = 0; c < 4; c++) {
        const double *F = s->field + (size_t)c * fnx * fny;
        double v00 = F[iy * fnx + ix], v10 = F[iy * fnx + ix + 1];
        double v01 = F[(iy + 1) * fnx + ix], v11 = F[(iy + 1) * fnx + ix + 1];
        val[c] = (1.0 - ty) * ((1.0 - tx) * v00 + tx * v10) + ty * ((1.0 - tx) * v01 + tx * v11);
    }
    s->ua_i[i] = p->ua + val[0]; s->va_i[i] = p->va + val[1];
    s->uw_i[i] = p->uw + val[2]; s->vw_i[i] = p->vw + val[3];
}

/* ------------------------ creation / reset ------------------------ */
#define ALLOC(f) s->f = (double *)calloc((size_t)n, sizeof(double))

gdo_state *gdo_create(const gdo_params *p, int n, const double *x, const double *y,
                      const double *r, const double *h, const double *theta,
                      const double *omega, const double *u, const double *v, int nb,
                      const int32_t *bi, const int32_t *bj, const double *damage,
                      const double *field)
{
    gdo_state *s = (gdo_state *)calloc(1, sizeof(gdo_state));
    s->p = *p;
    s->n = n;
    s->ridge_mode = GDO_RIDGE_DEFERRED;
    s->math_mode = GDO_MATH_DET;
    ALLOC(x); ALLOC(y); ALLOC(r); ALLOC(h); ALLOC(hfa); ALLOC(hfw); ALLOC(mass);
    ALLOC(inertia); ALLOC(u); ALLOC(v); ALLOC(theta); ALLOC(omega);
    ALLOC(r0); ALLOC(h0); ALLOC(hfa0); ALLOC(hfw0); ALLOC(mass0); ALLOC(inertia0);
    ALLOC(ua_i); ALLOC(va_i); ALLOC(uw_i); ALLOC(vw_i);
    ALLOC(fcx); ALLOC(fcy); ALLOC(mc); ALLOC(fbx); ALLOC(fby); ALLOC(mb);
    ALLOC(tfx); ALLOC(tfy); ALLOC(m); ALLOC(fcorx); ALLOC(fcory);
    ALLOC(fn_bc); ALLOC(ft_bc); ALLOC(fr_bc); ALLOC(fx_bc); ALLOC(fy_bc);
    ALLOC(mc_bc); ALLOC(m_bc);
    ALLOC(deltat_bc1); ALLOC(deltat_bc2); ALLOC(theta_bc1); ALLOC(theta_bc2);
    ALLOC(delt_ridge_bc);
    ALLOC(sigxx); ALLOC(sigyy); ALLOC(sigxy); ALLOC(sigyx);
    ALLOC(sigxx_bc); ALLOC(sigyy_bc); ALLOC(sigxy_bc); ALLOC(sigyx_bc);
    ALLOC(sigxx_aw); ALLOC(sigyy_aw); ALLOC(sigxy_aw); ALLOC(sigyx_aw);
    ALLOC(tsigxx); ALLOC(tsigyy); ALLOC(tsigxy); ALLOC(tsigyx);
    ALLOC(tac); ALLOC(tab); ALLOC(pc); ALLOC(pb); ALLOC(tp); ALLOC(ta_bc); ALLOC(p_bc);
    ALLOC(fax); ALLOC(fay); ALLOC(fwx); ALLOC(fwy); ALLOC(ma); ALLOC(mw);
    ALLOC(hsfa_min); ALLOC(hsfw_min);
    for (int i = 0; i < n; i++) {
        s->x[i] = x[i]; s->y[i] = y[i]; s->r[i] = r[i]; s->h[i] = h[i];
        s->theta[i] = theta ? theta[i] : 0.0;
        s->omega[i] = omega ? omega[i] : 0.0;
        s->u[i] = u ? u[i] : 0.0;
        s->v[i] = v ? v[i] : 0.0;
        floe_properties(p, s->r[i], s->h[i], &s->mass[i], &s->inertia[i], &s->hfa[i], &s->hfw[i]);
    }
    if (field && p->field_nx >= 2 && p->field_ny >= 2) {
        size_t nf = (size_t)4 * p->field_nx * p->field_ny;
        s->field = (double *)malloc(nf * sizeof(double));
        memcpy(s->field, field, nf * sizeof(double));
    }
    s->cap = 0; s->used = 0; s->tab_p = NULL;
    map_grow(s);
    /* restart bonds (read_sparse_restart, ini_get.f90:252-311); geometry from
       the given positions by bond_properties (bonds.f90:237-269) */
    for (int k = 0; k < nb; k++) {
        int i = bi[k], j = bj[k];
        if (i > j) { int t = i; i = j; j = t; }
        pairrec *e = map_get(s, i, j);
        e->bond = 1;
        e->damageb = damage ? damage[k] : 0.0;
        double dx = wrap_dx(s, s->x[i] - s->x[j], 0), dy = wrap_dx(s, s->y[i] - s->y[j], 1);
        double dist = sqrt(dx * dx + dy * dy);
        e->rb = p->lambda_rb * fmind(s->r[i], s->r[j]);
        e->hb = (s->h[i] + s->h[j]) / 2.0;
        e->lb = dist;
        e->sb = (2.0 * e->rb) * e->hb;
        e->ib = ((2.0 / 3.0) * e->hb) * ((e->rb * e->rb) * e->rb);
    }
    return s;
}

void gdo_set_modes(gdo_state *s, int ridge_mode, int math_mode)
{
    s->ridge_mode = ridge_mode;
    s->math_mode = math_mode;
}

/* reset_forces (reset.f90:73-178) */
static void reset_forces(gdo_state *s)
{
    size_t b = (size_t)s->n * sizeof(double);
    double *arr[] = {s->mc, s->mb, s->fcx, s->fcy, s->fbx, s->fby, s->m, s->tfx, s->tfy,
                     s->mc_bc, s->m_bc, s->fn_bc, s->ft_bc, s->fx_bc, s->fy_bc,
                     s->sigxx, s->sigyy, s->sigxy, s->sigyx,
                     s->sigxx_bc, s->sigyy_bc, s->sigxy_bc, s->sigyx_bc,
                     s->tp, s->tac, s->tab, s->pc, s->pb, s->p_bc, s->ta_bc};
    for (size_t k = 0; k < sizeof(arr) / sizeof(arr[0]); k++) memset(arr[k], 0, b);
}

/* ---------------------------- candidates -------------------------- */
static void build_cells(gdo_state *s)
{
    const gdo_params *p = &s->p;
    int n = s->n;
    double rmax = 0.0;
    for (int i = 0; i < n; i++) rmax = fmaxd(rmax, s->r0[i]);
    double cs = rmax + p->rtree;
    if (!(cs > 0.0)) cs = 1.0;
    int ncx = (int)floor(p->nx / cs), ncy = (int)floor(p->ny / cs);
    if (ncx < 1) ncx = 1;
    if (ncy < 1) ncy = 1;
    if (ncx > 2048) ncx = 2048;
    if (ncy > 2048) ncy = 2048;
    if (s->ncx != ncx || s->ncy != ncy || !s->cell_head) {
        free(s->cell_head);
        s->cell_head = (int *)malloc((size_t)ncx * ncy * sizeof(int));
        s->ncx = ncx; s->ncy = ncy;
    }
    if (!s->cell_next) s->cell_next = (int *)malloc((size_t)n * sizeof(int));
    s->cwx = p->nx / ncx; s->cwy = p->ny / ncy;
    for (int c = 0; c < ncx * ncy; c++) s->cell_head[c] = -1;
    for (int i = n - 1; i >= 0; i--) {
        double fx = s->x[i] / s->cwx, fy = s->y[i] / s->cwy;
        if (!(fx >= 0.0)) fx = 0.0;
        if (!(fy >= 0.0)) fy = 0.0;
        if (fx > (double)ncx) fx = (double)ncx;
        if (fy > (double)ncy) fy = (double)ncy;
        int cx = (int)floor(fx), cy = (int)floor(fy);
        if (cx < 0) cx = 0;
        if (cx >= ncx) cx = ncx - 1;
        if (cy < 0) cy = 0;
        if (cy >= ncy) cy = ncy - 1;
        int c = cy * ncx + cx;
        s->cell_next[i] = s->cell_head[c];
        s->cell_head[c] = i;
    }
}


typedef struct { double d; int j; } cand_t;
static int cmp_cand_q(const void *a, const void *b)
{
    const cand_t *x = (const cand_t *)a, *y = (const cand_t *)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->j > y->j) - (x->j < y->j);
}

/* kNearest(radius = r(i) + rtree) restricted to j > i (stepper.f90:77-87):
   all j with distance <= radius, ascending distance, ties by index. */
static int query(gdo_state *s, int i, double radius, cand_t **out)
{
    static __thread cand_t *buf = NULL;
    static __thread int bcap = 0;
    int cnt = 0;
    const gdo_params *p = &s->p;
    int px = p->boundary & BC_PERIODIC_X, py = p->boundary & BC_PERIODIC_Y;
    double qx = s->x[i] / s->cwx, qy = s->y[i] / s->cwy;
    if (!(qx >= 0.0)) qx = 0.0;
    if (!(qy >= 0.0)) qy = 0.0;
    if (qx > (double)s->ncx) qx = (double)s->ncx;
    if (qy > (double)s->ncy) qy = (double)s->ncy;
    int cx = (int)floor(qx), cy = (int)floor(qy);
    if (cx < 0) cx = 0;
    if (cx >= s->ncx) cx = s->ncx - 1;
    if (cy < 0) cy = 0;
    if (cy >= s->ncy) cy = s->ncy - 1;
    int xs[3], ys[3], nxs = 0, nys = 0;
    for (int d = -1; d <= 1; d++) {
        int c = cx + d;
        if (px) c = ((c % s->ncx) + s->ncx) % s->ncx;
        else if (c < 0 || c >= s->ncx) continue;
        int dup = 0;
        for (int k = 0; k < nxs; k++) dup |= xs[k] == c;
        if (!dup) xs[nxs++] = c;
    }
    for (int d = -1; d <= 1; d++) {
        int c = cy + d;
        if (py) c = ((c % s->ncy) + s->ncy) % s->ncy;
        else if (c < 0 || c >= s->ncy) continue;
        int dup = 0;
        for (int k = 0; k < nys; k++) dup |= ys[k] == c;
        if (!dup) ys[nys++] = c;
    }
    for (int a = 0; a < nys; a++)
        for (int b = 0; b < nxs; b++)
            for (int j = s->cell_head[ys[a] * s->ncx + xs[b]]; j >= 0; j = s->cell_next[j]) {
                if (j <= i) continue;
                double dx = wrap_dx(s, s->x[i] - s->x[j], 0);
                double dy = wrap_dx(s, s->y[i] - s->y[j], 1);
                double d = sqrt(dx * dx + dy * dy);
                if (d <= radius) {
                    if (cnt == bcap) {
                        bcap = bcap ? bcap * 2 : 256;
                        buf = (cand_t *)realloc(buf, (size_t)bcap * sizeof(cand_t));
                    }
                    buf[cnt].d = d; buf[cnt].j = j; cnt++;
                }
            }
    qsort(buf, (size_t)cnt, sizeof(cand_t), cmp_cand_q);
    *out = buf;
    return cnt;
}

/* ------------------------- the pair body -------------------------- */
/* Shape view for one floe inside a pair computation. */
typedef struct { double r, h, mass, inertia, hfa, hfw; } shape_t;

/* update_shape's per-floe part (ridging.f90:88-99 / 74-86): returns the
   thickness change applied to the shape. */
static void apply_dh(const gdo_params *p, shape_t *sh, double Vol)
{
    double dh = Vol / (p->pi * (sh->r * sh->r));
    sh->r = sh->r * sqrt(sh->h / (sh->h + dh));
    sh->h = sh->h + dh;
    floe_properties(p, sh->r, sh->h, &sh->mass, &sh->inertia, &sh->hfa, &sh->hfw);
}

static void running_event(gdo_state *s, int k, double Vol)
{
    shape_t sh = {s->r[k], s->h[k], s->mass[k], s->inertia[k], s->hfa[k], s->hfw[k]};
    apply_dh(&s->p, &sh, Vol);
    s->r[k] = sh.r; s->h[k] = sh.h; s->mass[k] = sh.mass; s->inertia[k] = sh.inertia;
    s->hfa[k] = sh.hfa; s->hfw[k] = sh.hfw;
}

static void load_shape(const gdo_state *s, int k, shape_t *sh)
{
    if (s->ridge_mode == GDO_RIDGE_REFERENCE) {
        sh->r = s->r[k]; sh->h = s->h[k]; sh->mass = s->mass[k]; sh->inertia = s->inertia[k];
        sh->hfa = s->hfa[k]; sh->hfw = s->hfw[k];
    } else {
        sh->r = s->r0[k]; sh->h = s->h0[k]; sh->mass = s->mass0[k]; sh->inertia = s->inertia0[k];
        sh->hfa = s->hfa0[k]; sh->hfw = s->hfw0[k];
    }
}

/* stepper.f90:89-271 for one candidate pair (i < j) */
static void pair_body(gdo_state *s, int i, int j, int tstep, int restart)
{
    const gdo_params *p = &s->p;
    const double dt = p->dt;
    pairrec *e = map_get(s, i, j);
    shape_t si, sj;
    load_shape(s, i, &si);
    load_shape(s, j, &sj);

    /* rel_pos_vel (physics.f90:73-114) */
    double dx = wrap_dx(s, s->x[i] - s->x[j], 0);
    double dy = wrap_dx(s, s->y[i] - s->y[j], 1);
    double dist = sqrt(dx * dx + dy * dy);
    double cosa = (-dx) / dist;
    double sina = (-dy) / dist;
    double omegarel = s->omega[j] - s->omega[i];
    double veln = (s->u[j] - s->u[i]) * cosa + (s->v[j] - s->v[i]) * sina;
    double veltb = -((s->u[j] - s->u[i]) * sina) + (s->v[j] - s->v[i]) * cosa;
    double velt = veltb - (s->omega[i] * si.r + s->omega[j] * sj.r);
    double deltan = (si.r + sj.r) - dist;
    e->deltan = deltan;

    /* bond initialisation (stepper.f90:93-101) */
    if (tstep == 1 && restart != 1 && p->cohesion) {
        double lim = p->bond_lim + p->bond_lim_rel * (si.r + sj.r);
        int sel = 1;
        if (p->bond_frac > 0.0 && p->bond_frac < 1.0)
            sel = (double)pair_hash32((uint32_t)p->bond_seed, (uint32_t)i, (uint32_t)j) * 0x1.0p-32 < p->bond_frac;
        if (deltan >= -lim && sel) {
            e->bond = 1;
            e->damageb = 0.0;
            /* bond_properties (bonds.f90:237-269) */
            e->rb = p->lambda_rb * fmind(si.r, sj.r);
            e->hb = (si.h + sj.h) / 2.0;
            e->lb = dist;
            e->sb = (2.0 * e->rb) * e->hb;
            e->ib = ((2.0 / 3.0) * e->hb) * ((e->rb * e->rb) * e->rb);
        }
    }

    if (deltan > 0.0) {
        /* contact_forces (contact_forces.f90:1-87) */
        e->deltat = -(velt * dt) + e->deltat;
        double q = ((dist * dist - sj.r * sj.r) + si.r * si.r) / (2.0 * dist);
        double dr = 2.0 * sqrt(si.r * si.r - q * q);
        e->thetarelc = -(omegarel * dt) + e->thetarelc;
        double m_redu = (si.mass * sj.mass) / (si.mass + sj.mass);
        double r_redu = (si.r * sj.r) / (si.r + sj.r);
        double hmin = fmind(si.h, sj.h);
        double knc = ((p->pi * p->ec) * hmin) * fit((deltan * r_redu) / (2.0 * (hmin * hmin)));
        double ktc = ((6.0 * p->gc) / p->ec) * knc;
        double krc = (knc * (dr * dr)) / 12.0;
        double gamn = -(p->beta * sqrt((4.0 * knc) * m_redu));
        double gamt = -((2.0 * p->beta) * sqrt(((2.0 / 3.0) * ktc) * m_redu));
        double gamr = (gamn * (dr * dr)) / 12.0;
        double fcn = fmaxd(knc * deltan - gamn * veln, 0.0);
        double fct = ktc * e->deltat - gamt * velt;
        if (p->ridging) {
            if (p->sigmanc_crit * hmin <= (fcn / dr) / hmin) {
                /* plastic_contact (ridging.f90:1-33) */
                double knp = ((p->sigmanc_crit * (hmin * hmin)) * dr) / deltan;
                ktc = ((6.0 * p->gc) / p->ec) * knp;
                krc = (knp * (dr * dr)) / 12.0;
                gamn = -(p->beta * sqrt((4.0 * knp) * m_redu));
                gamt = -((2.0 * p->beta) * sqrt(((2.0 / 3.0) * ktc) * m_redu));
                gamr = (gamn * (dr * dr)) / 12.0;
                fcn = fmind(fcn, (p->sigmanc_crit * (hmin * hmin)) * dr);
                fct = ktc * e->deltat - gamt * velt;
                /* update_shape (ridging.f90:36-99) */
                double hm2 = fmind(si.h, sj.h);
                double dij = ((dist * dist - sj.r * sj.r) + si.r * si.r) / (2.0 * dist);
                double dji = ((dist * dist - si.r * si.r) + sj.r * sj.r) / (2.0 * dist);
                double Area = (((si.r * si.r) * M_acos(s, dij / si.r) - (dij * dr) / 2.0)
                               + (sj.r * sj.r) * M_acos(s, dji / sj.r)) - (dji * dr) / 2.0;
                double Vol = fmaxd((Area * hm2) / 2.0, 0.0);
                int who = -1;
                if (hm2 == si.h) who = i;
                else if (hm2 == sj.h) who = j;
                if (who == i) apply_dh(p, &si, Vol);
                else if (who == j) apply_dh(p, &sj, Vol);
                if (who >= 0) {
                    if (s->ridge_mode == GDO_RIDGE_REFERENCE) {
                        shape_t *w = who == i ? &si : &sj;
                        s->r[who] = w->r; s->h[who] = w->h; s->mass[who] = w->mass;
                        s->inertia[who] = w->inertia; s->hfa[who] = w->hfa; s->hfw[who] = w->hfw;
                    } else {
                        running_event(s, who, Vol);
                    }
                }
                double q2 = ((dist * dist - sj.r * sj.r) + si.r * si.r) / (2.0 * dist);
                dr = 2.0 * sqrt(si.r * si.r - q2 * q2);
            }
        }
        /* coulomb (physics.f90:1-33) */
        double fcr;
        if (fabs(fct) > p->friction_coeff * fabs(fcn)) {
            fct = -((p->friction_coeff * fabs(fcn)) * copysign(1.0, velt));
            fcr = fct;
            if (p->slipping) e->deltat = (fct + gamt * velt) / ktc;
        } else {
            fcr = fct;
        }
        if (e->bond == 0) {
            double mrolling = krc * e->thetarelc - gamr * omegarel;
            if (fabs(e->thetarelc) > ((2.0 * fabs(fcn)) / knc) / dr) mrolling = 0.0;
            e->mcc = mrolling;
        }
        e->fcn = fcn; e->fct = fct; e->fcr = fcr; e->delt_ridge = dr;
        /* stepper.f90:113-146 */
        s->fcx[i] = (s->fcx[i] - fcn * cosa) + fcr * sina;
        s->fcy[i] = (s->fcy[i] - fcn * sina) - fcr * cosa;
        s->mc[i] = (s->mc[i] - si.r * fct) - e->mcc;
        s->fcx[j] = (s->fcx[j] + fcn * cosa) - fcr * sina;
        s->fcy[j] = (s->fcy[j] + fcn * sina) + fcr * cosa;
        s->mc[j] = (s->mc[j] - sj.r * fct) + e->mcc;
        e->ac = dr * fmind(si.h, sj.h);
        s->tac[i] = s->tac[i] + e->ac;
        s->pc[i] = s->pc[i] - fcn * e->ac;
        s->tac[j] = s->tac[j] + e->ac;
        s->pc[j] = s->pc[j] - fcn * e->ac;
    } else {
        /* reset_contact (reset.f90:1-15) */
        e->thetarelc = 0.0; e->deltat = 0.0; e->delt_ridge = 0.0;
    }

    if (e->bond == 1) {
        /* bond_forces_euler (bonds.f90:74-161) */
        e->deltanb = veln * dt + e->deltanb;
        e->deltatb = veltb * dt + e->deltatb;
        e->thb_ji = s->omega[i] * dt + e->thb_ji;
        e->thb_ij = s->omega[j] * dt + e->thb_ij;
        double m_redu = (si.mass * sj.mass) / (si.mass + sj.mass);
        double i_redu = (si.inertia * sj.inertia) / (si.inertia + sj.inertia);
        double L = e->lb;
        double EA = ((1.0 - e->damageb) * p->eb) * e->sb;
        double EI = ((1.0 - e->damageb) * p->eb) * e->ib;
        double k_axial = EA / L;
        double k_shear1 = (12.0 * EI) / ((L * L) * L);
        double k_shear2 = (6.0 * EI) / (L * L);
        double k_rot1 = (4.0 * EI) / L;
        double k_rot2 = (2.0 * EI) / L;
        double eta_i = 2.0 * sqrt((EI * i_redu) / L);
        double eta_a = 2.0 * sqrt((EA * m_redu) * L);
        double gam_axial = eta_a / L;
        double gam_shear1 = (12.0 * eta_i) / ((L * L) * L);
        double gam_shear2 = (6.0 * eta_i) / (L * L);
        double gam_rot1 = (4.0 * eta_i) / L;
        double gam_rot2 = (2.0 * eta_i) / L;
        double fbn = k_axial * e->deltanb + gam_axial * veln;
        double fbt = ((k_shear1 * e->deltatb + k_shear2 * (e->thb_ji + e->thb_ij))
                      + gam_shear1 * veltb) + gam_shear2 * (s->omega[i] + s->omega[j]);
        double mji = ((((k_rot1 * e->thb_ji + k_rot2 * e->thb_ij) - k_shear2 * e->deltatb)
                       + gam_rot1 * s->omega[i]) + gam_rot2 * s->omega[j]) - gam_shear2 * veltb;
        double mij = ((((k_rot2 * e->thb_ji + k_rot1 * e->thb_ij) - k_shear2 * e->deltatb)
                       + gam_rot2 * s->omega[i]) + gam_rot1 * s->omega[j]) - gam_shear2 * veltb;
        /* bond_breaking (bonds.f90:164-212) */
        double taub = fabs(fbt) / e->sb;
        double sigmatb = -(fbn / e->sb) + (fabs(mji) * e->rb) / e->ib;
        double sigmacb = fbn / e->sb + (fabs(mji) * e->rb) / e->ib;
        double t1 = taub / (p->tau_crit * e->hb);
        double phi = t1 * t1;
        if (sigmacb > 0.0) { double t2 = sigmacb / (p->sigmacb_crit * e->hb); phi = phi + t2 * t2; }
        if (sigmatb > 0.0) { double t3 = sigmatb / (p->sigmatb_crit * e->hb); phi = phi + t3 * t3; }
        double psi = fmind(1.0, 1.0 / sqrt(phi));
        double D = e->damageb;
        D = (D + (((1.0 - psi) * (1.0 - D)) * dt) / p->dtd) - (D * dt) / p->dth;
        e->damageb = D;
        if (D >= p->dmax) {
            e->bond = 0; fbn = 0.0; fbt = 0.0; mji = 0.0; e->damageb = 1.0;
        }
        e->fbn = fbn; e->fbt = fbt; e->mbb_ji = mji; e->mbb_ij = mij;
        if (e->bond == 1) {
            /* stepper.f90:163-198 */
            s->fbx[i] = (s->fbx[i] + fbn * cosa) - fbt * sina;
            s->fby[i] = (s->fby[i] + fbn * sina) + fbt * cosa;
            s->mb[i] = (s->mb[i] - (p->lambda_lb * si.r) * fbt) - mji;
            s->fbx[j] = (s->fbx[j] - fbn * cosa) + fbt * sina;
            s->fby[j] = (s->fby[j] - fbn * sina) - fbt * cosa;
            s->mb[j] = (s->mb[j] - (p->lambda_lb * sj.r) * fbt) - mij;
            s->tab[i] = s->tab[i] + e->sb;
            s->pb[i] = s->pb[i] - fbn * e->sb;
            s->tab[j] = s->tab[j] + e->sb;
            s->pb[j] = s->pb[j] - fbn * e->sb;
        }
    } else {
        /* reset_bond (reset.f90:18-34) */
        e->thb_ji = 0.0; e->thb_ij = 0.0; e->deltanb = 0.0; e->deltatb = 0.0;
    }

    if (p->shelter) {
        /* sheltering (forcing.f90:162-186) + thread minima (stepper.f90:211-224) */
        double a_ij = S_shelter(s, si.hfa, sj.hfa, deltan, cosa, sina, s->ua_i[i], s->va_i[i]);
        double w_ij = S_shelter(s, si.hfw, sj.hfw, deltan, cosa, sina, s->uw_i[i], s->vw_i[i]);
        double a_ji = S_shelter(s, sj.hfa, si.hfa, deltan, -cosa, -sina, s->ua_i[i], s->va_i[i]);
        double w_ji = S_shelter(s, sj.hfw, si.hfw, deltan, -cosa, -sina, s->uw_i[i], s->vw_i[i]);
        s->hsfa_min[i] = fmind(s->hsfa_min[i], a_ji);
        s->hsfa_min[j] = fmind(s->hsfa_min[j], a_ij);
        s->hsfw_min[i] = fmind(s->hsfw_min[i], w_ji);
        s->hsfw_min[j] = fmind(s->hsfw_min[j], w_ij);
    }

    /* stress diagnostics (stepper.f90:238-271); uses r(i) for both floes */
    double S = sqrt(e->fcn * e->fcn + e->fct * e->fct) + sqrt(e->fbn * e->fbn + e->fbt * e->fbt);
    double sxx = ((S * cosa) * si.r) * cosa, syy = ((S * sina) * si.r) * sina;
    double sxy = ((S * sina) * si.r) * cosa, syx = ((S * cosa) * si.r) * sina;
    s->sigxx[i] = s->sigxx[i] - sxx; s->sigyy[i] = s->sigyy[i] - syy;
    s->sigxy[i] = s->sigxy[i] - sxy; s->sigyx[i] = s->sigyx[i] - syx;
    s->sigxx[j] = s->sigxx[j] - sxx; s->sigyy[j] = s->sigyy[j] - syy;
    s->sigxy[j] = s->sigxy[j] - sxy; s->sigyx[j] = s->sigyx[j] - syx;
}

/* ------------------------------ walls ----------------------------- */
/* coulomb_bc (physics.f90:36-70) */
static void coulomb_bc(gdo_state *s, int i, double velt_bc, double ktc, double gamt, double *deltat_bc)
{
    const gdo_params *p = &s->p;
    if (fabs(s->ft_bc[i]) > p->friction_coeff * fabs(s->fn_bc[i])) {
        s->ft_bc[i] = -((p->friction_coeff * fabs(s->fn_bc[i])) * copysign(1.0, velt_bc));
        s->fr_bc[i] = s->ft_bc[i];
        if (p->slipping) *deltat_bc = (s->ft_bc[i] + gamt * velt_bc) / ktc;
    } else {
        s->fr_bc[i] = s->ft_bc[i];
    }
}

/* contact_bc (contact_forces.f90:90-244) with plastic_contact_bc and
   update_shape_bc (ridging.f90:102-180) */
static void contact_bc(gdo_state *s, int i, int dir1, int dir2, int bd)
{
    const gdo_params *p = &s->p;
    const double dt = p->dt;
    double d1 = (double)dir1, d2 = (double)dir2;
    double cosa_bc = (double)(dir1 * (dir2 - (1 - dir2)));
    double sina_bc = (double)((1 - dir1) * (dir2 - (1 - dir2)));
    double veln_bc = -(s->u[i] * cosa_bc) - s->v[i] * sina_bc;
    double velt_bc = (s->u[i] * sina_bc - s->v[i] * cosa_bc) - s->omega[i] * s->r[i];
    double deltan_bc = ((1.0 - d2) * (s->r[i] - s->x[i]) + d2 * ((s->r[i] + s->x[i]) - p->nx)) * d1
                       + ((1.0 - d2) * (s->r[i] - s->y[i]) + d2 * ((s->r[i] + s->y[i]) - p->ny)) * (1.0 - d1);
    double deltat_bc = 0.0;
    {
        double t = s->r[i] - deltan_bc;
        s->delt_ridge_bc[i] = 2.0 * sqrt(s->r[i] * s->r[i] - t * t);
    }
    if (bd == 1) {
        s->deltat_bc1[i] = -(velt_bc * dt) + s->deltat_bc1[i];
        deltat_bc = s->deltat_bc1[i];
        s->theta_bc1[i] = -(s->omega[i] * dt) + s->theta_bc1[i];
    } else {
        s->deltat_bc2[i] = -(velt_bc * dt) + s->deltat_bc2[i];
        deltat_bc = s->deltat_bc2[i];
        s->theta_bc2[i] = -(s->omega[i] * dt) + s->theta_bc2[i];
    }
    double h = s->h[i], r = s->r[i];
    double knc = ((p->pi * p->ec) * h) * fit((deltan_bc * r) / ((1.0 * 2.0) * (h * h)));
    double ktc = ((6.0 * p->gc) / p->ec) * knc;
    double dr = s->delt_ridge_bc[i];
    double krc = (knc * (dr * dr)) / 12.0;
    double gamn = -(p->beta * sqrt(((4.0 * knc) * s->mass[i]) / 1.0));
    double gamt = -((2.0 * p->beta) * sqrt((((2.0 / 3.0) * ktc) * s->mass[i]) / 1.0));
    double gamr = (gamn * (dr * dr)) / 12.0;
    s->fn_bc[i] = fmaxd(knc * deltan_bc - gamn * veln_bc, 0.0);
    s->ft_bc[i] = ktc * deltat_bc - gamt * velt_bc;
    if (p->ridging) {
        if (p->sigmanc_crit * h <= (s->fn_bc[i] / dr) / h) {
            /* plastic_contact_bc: uses m(i), the total moment, zeroed by
               reset_forces (ridging.f90:127-128; reset.f90:97) */
            double mtot = s->m[i];
            double knp = ((p->sigmanc_crit * (h * h)) * dr) / deltan_bc;
            ktc = ((6.0 * p->gc) / p->ec) * knp;
            krc = (knp * (dr * dr)) / 12.0;
            gamn = -(p->beta * sqrt(((4.0 * knp) * mtot) / 1.0));
            gamt = -((2.0 * p->beta) * sqrt((((2.0 / 3.0) * ktc) * mtot) / 1.0));
            gamr = (gamn * (dr * dr)) / 12.0;
            s->fn_bc[i] = fmind(s->fn_bc[i], (p->sigmanc_crit * (h * h)) * dr);
            s->ft_bc[i] = ktc * deltat_bc - gamt * velt_bc;
            /* update_shape_bc */
            double Area = (r * r) * M_asin(s, (dr / 2.0) / r) - (dr * (r - deltan_bc)) / 2.0;
            double Vol = fmaxd(Area * h, 0.0);
            running_event(s, i, Vol);
            double t = s->r[i] - deltan_bc;
            s->delt_ridge_bc[i] = 2.0 * sqrt(s->r[i] * s->r[i] - t * t);
            dr = s->delt_ridge_bc[i];
        }
    }
    double mrolling_bc;
    if (bd == 1) {
        coulomb_bc(s, i, velt_bc, ktc, gamt, &s->deltat_bc1[i]);
        mrolling_bc = krc * s->theta_bc1[i] - gamr * s->omega[i];
        if (fabs(s->theta_bc1[i]) > ((2.0 * fabs(s->fn_bc[i])) / knc) / dr) mrolling_bc = 0.0;
    } else {
        coulomb_bc(s, i, velt_bc, ktc, gamt, &s->deltat_bc2[i]);
        mrolling_bc = krc * s->theta_bc2[i] - gamr * s->omega[i];
        if (fabs(s->theta_bc2[i]) > ((2.0 * fabs(s->fn_bc[i])) / knc) / dr) mrolling_bc = 0.0;
    }
    s->mc_bc[i] = mrolling_bc;
}

/* check_wall (boundaries.f90:100-146) */
static void check_wall(gdo_state *s, int i, int dir1, int dir2, int bd)
{
    contact_bc(s, i, dir1, dir2, bd);
    double c = (double)(dir1 * (dir2 - (1 - dir2)));
    double sn = (double)((1 - dir1) * (dir2 - (1 - dir2)));
    s->fx_bc[i] = (s->fx_bc[i] - s->fn_bc[i] * c) + s->fr_bc[i] * sn;
    s->fy_bc[i] = (s->fy_bc[i] - s->fn_bc[i] * sn) - s->fr_bc[i] * c;
    s->m_bc[i] = (s->m_bc[i] - s->mc_bc[i]) - s->r[i] * s->ft_bc[i];
    double q = sqrt(s->fn_bc[i] * s->fn_bc[i] + s->ft_bc[i] * s->ft_bc[i]);
    s->sigxx_bc[i] = -((q * s->r[i]) * (c * c));
    s->sigyy_bc[i] = -((q * s->r[i]) * (sn * sn));
    s->sigxy_bc[i] = -(((q * s->r[i]) * c) * sn);
    s->sigyx_bc[i] = -(((q * s->r[i]) * sn) * c);
    s->ta_bc[i] = s->ta_bc[i] + s->delt_ridge_bc[i] * s->h[i];
    s->p_bc[i] = s->p_bc[i] - (s->fn_bc[i] * s->delt_ridge_bc[i]) * s->h[i];
}

/* reset_boundary (reset.f90:37-69) */
static void reset_boundary(gdo_state *s, int i, int bd)
{
    if (bd == 1) { s->theta_bc1[i] = 0.0; s->deltat_bc1[i] = 0.0; }
    else if (bd == 2) { s->theta_bc2[i] = 0.0; s->deltat_bc2[i] = 0.0; }
    else { s->theta_bc1[i] = 0.0; s->theta_bc2[i] = 0.0; s->deltat_bc1[i] = 0.0; s->deltat_bc2[i] = 0.0; }
    s->delt_ridge_bc[i] = 0.0;
}

/* verify_bc (boundaries.f90:1-97); walls on periodic or open sides are
   absent (extension; boundary == 0 is the reference's four walls) */
static void verify_bc(gdo_state *s, int i)
{
    const gdo_params *p = &s->p;
    int b = p->boundary;
    int t1 = 0, t2 = 0;
    int wb = !(b & BC_PERIODIC_Y) && !(b & BC_OPEN_BOTTOM);
    int wt = !(b & BC_PERIODIC_Y) && !(b & BC_OPEN_TOP);
    int wl = !(b & BC_PERIODIC_X) && !(b & BC_OPEN_LEFT);
    int wr = !(b & BC_PERIODIC_X) && !(b & BC_OPEN_RIGHT);
    if (wb && s->y[i] - s->r[i] < 0.0) { t1 = 1; check_wall(s, i, 0, 0, 1); }
    if (wt && s->y[i] + s->r[i] > p->ny) { t1 = 1; check_wall(s, i, 0, 1, 1); }
    if (wl && s->x[i] - s->r[i] < 0.0) { t2 = 1; check_wall(s, i, 1, 0, 2); }
    if (wr && s->x[i] + s->r[i] > p->nx) { t2 = 1; check_wall(s, i, 1, 1, 2); }
    if (t1 + t2 == 0) reset_boundary(s, i, 0);
    if (t2 == 0) reset_boundary(s, i, 2);
    if (t1 == 0) reset_boundary(s, i, 1);
}

/* log_profile (forcing.f90:209-224) */
static inline double log_profile(const gdo_state *s, double hf, double z0)
{
    double a = M_log(s, hf / z0) / M_log(s, 10.0 / z0);
    return a * a;
}

/* forcing (forcing.f90:32-159) */
static void forcing(gdo_state *s, int i)
{
    const gdo_params *p = &s->p;
    double sca = s->hsfa_min[i], scw = s->hsfw_min[i];
    double dua = s->ua_i[i] - s->u[i], dva = s->va_i[i] - s->v[i];
    double duw = s->uw_i[i] - s->u[i], dvw = s->vw_i[i] - s->v[i];
    double an = sqrt(dua * dua + dva * dva);
    double on = sqrt(duw * duw + dvw * dvw);
    double alog = log_profile(s, s->hfa[i], p->z0w);
    double olog = log_profile(s, s->hfw[i], p->z0w);
    double r = s->r[i], om = s->omega[i], aom = fabs(om);
    double r2 = r * r;
    double fdax, fday, fsax, fsay, fdwx, fdwy, fswx, fswy;
    if (an == 0.0) {
        fdax = fday = fsax = fsay = 0.0;
    } else {
        fdax = (((((((p->rhoair * p->Cdair) * s->hfa[i]) * r) * dua) * an) * alog) * sca) * p->pi / 2.0;
        fday = (((((((p->rhoair * p->Cdair) * s->hfa[i]) * r) * dva) * an) * alog) * sca) * p->pi / 2.0;
        double g = an * an + (r2 * (aom * aom)) / 4.0;
        fsax = (((((p->rhoair * p->pi) * r2) * p->Csair) * dua) / an) * g;
        fsay = (((((p->rhoair * p->pi) * r2) * p->Csair) * dva) / an) * g;
    }
    if (on == 0.0) {
        fdwx = fdwy = fswx = fswy = 0.0;
    } else {
        fdwx = (((((((p->rhowater * p->Cdwater) * s->hfw[i]) * r) * duw) * on) * olog) * scw) * p->pi / 2.0;
        fdwy = (((((((p->rhowater * p->Cdwater) * s->hfw[i]) * r) * dvw) * on) * olog) * scw) * p->pi / 2.0;
        double g = on * on + (r2 * (aom * aom)) / 4.0;
        fswx = (((((p->rhowater * p->pi) * r2) * p->Cswater) * duw) / on) * g;
        fswy = (((((p->rhowater * p->pi) * r2) * p->Cswater) * dvw) / on) * g;
    }
    s->fax[i] = fdax + fsax; s->fay[i] = fday + fsay;
    s->fwx[i] = fdwx + fswx; s->fwy[i] = fdwy + fswy;
    double r4 = r2 * r2, r5 = (r2 * r) * r2;
    if (an < 1e-2)
        s->ma[i] = -((((((2.0 * p->pi) / 5.0) * r5) * p->rhoair) * p->Csair) * om * aom);
    else
        s->ma[i] = -(((((((3.0 / 4.0) * p->pi) * p->rhoair) * p->Csair) * an) * om) * r4);
    if (on < 1e-3)
        s->mw[i] = -((((((2.0 * p->pi) / 5.0) * r5) * p->rhowater) * p->Cswater) * om * aom);
    else
        s->mw[i] = -(((((((3.0 / 4.0) * p->pi) * p->rhowater) * p->Cswater) * on) * om) * r4);
    s->sigxx_aw[i] = (s->fax[i] + s->fwx[i]) * r;
    s->sigyy_aw[i] = (s->fay[i] + s->fwy[i]) * r;
    s->sigxy_aw[i] = 0.0;
    s->sigyx_aw[i] = 0.0;
}

/* coriolis (forcing.f90:189-206), sin(lat) precomputed on the host */
static void coriolis(gdo_state *s, int i)
{
    const double oe = 7.2921e-5;
    s->fcorx[i] = (((s->mass[i] * 2.0) * oe) * s->p.sin_lat) * s->v[i];
    s->fcory[i] = -((((s->mass[i] * 2.0) * oe) * s->p.sin_lat) * s->u[i]);
}

/* ----------------------------- stepper ---------------------------- */
int gdo_step(gdo_state *s, int tstep, int restart)
{
    const gdo_params *p = &s->p;
    int n = s->n;
    /* snapshot of the shapes at the start of the step */
    memcpy(s->r0, s->r, n * sizeof(double)); memcpy(s->h0, s->h, n * sizeof(double));
    memcpy(s->mass0, s->mass, n * sizeof(double)); memcpy(s->inertia0, s->inertia, n * sizeof(double));
    memcpy(s->hfa0, s->hfa, n * sizeof(double)); memcpy(s->hfw0, s->hfw, n * sizeof(double));

    reset_forces(s);
    if (p->shelter) {
        /* reset_shelter (reset.f90:181-203) */
        for (int i = 0; i < n; i++) { s->hsfa_min[i] = 1.0; s->hsfw_min[i] = 1.0; }
    }
    build_cells(s);
    s->ncand = 0;
    for (int i = 0; i < n; i++) {
        winds_currents(s, i);
        double rad = (s->ridge_mode == GDO_RIDGE_REFERENCE ? s->r[i] : s->r0[i]) + p->rtree;
        cand_t *c;
        int nc = query(s, i, rad, &c);
        for (int k = 0; k < nc; k++) {
            int j = c[k].j;
            if (s->ncand == s->capcand) {
                s->capcand = s->capcand ? s->capcand * 2 : 4096;
                s->cand_i = (int32_t *)realloc(s->cand_i, s->capcand * sizeof(int32_t));
                s->cand_j = (int32_t *)realloc(s->cand_j, s->capcand * sizeof(int32_t));
            }
            s->cand_i[s->ncand] = i; s->cand_j[s->ncand] = j; s->ncand++;
            pair_body(s, i, j, tstep, restart);
        }
        verify_bc(s, i);
    }
    /* stepper.f90:285-303: min-reduce (already folded), forcing, coriolis */
    for (int i = 0; i < n; i++) { forcing(s, i); coriolis(s, i); }
    /* totals (stepper.f90:312-332) */
    for (int i = 0; i < n; i++) {
        s->tfx[i] = ((((s->fcx[i] + s->fbx[i]) + s->fax[i]) + s->fwx[i]) + s->fcorx[i]) + s->fx_bc[i];
        s->tfy[i] = ((((s->fcy[i] + s->fby[i]) + s->fay[i]) + s->fwy[i]) + s->fcory[i]) + s->fy_bc[i];
        s->m[i] = (((s->mc[i] + s->mb[i]) + s->ma[i]) + s->mw[i]) + s->m_bc[i];
        s->tsigxx[i] = (s->sigxx[i] + s->sigxx_bc[i]) + s->sigxx_aw[i];
        s->tsigyy[i] = (s->sigyy[i] + s->sigyy_bc[i]) + s->sigyy_aw[i];
        s->tsigxy[i] = (s->sigxy[i] + s->sigxy_bc[i]) + s->sigxy_aw[i];
        s->tsigyx[i] = (s->sigyx[i] + s->sigyx_bc[i]) + s->sigyx_aw[i];
        double a = s->tac[i] != 0.0 ? s->pc[i] / s->tac[i] : 0.0;
        double b = s->tab[i] != 0.0 ? s->pb[i] / s->tab[i] : 0.0;
        double c = s->ta_bc[i] != 0.0 ? s->p_bc[i] / s->ta_bc[i] : 0.0;
        s->tp[i] = (a + b) + c;
    }
    /* velocity, position (integration.f90:1-38) + periodic wrap (extension) */
    const double dt = p->dt;
    for (int i = 0; i < n; i++) {
        s->u[i] = s->u[i] + (s->tfx[i] / s->mass[i]) * dt;
        s->v[i] = s->v[i] + (s->tfy[i] / s->mass[i]) * dt;
        s->omega[i] = s->omega[i] + (s->m[i] / s->inertia[i]) * dt;
    }
    for (int i = 0; i < n; i++) {
        s->x[i] = s->x[i] + s->u[i] * dt;
        s->y[i] = s->y[i] + s->v[i] * dt;
        s->theta[i] = s->theta[i] + s->omega[i] * dt;
        if (p->boundary & BC_PERIODIC_X) {
            if (s->x[i] < 0.0) s->x[i] = s->x[i] + p->nx;
            else if (s->x[i] >= p->nx) s->x[i] = s->x[i] - p->nx;
        }
        if (p->boundary & BC_PERIODIC_Y) {
            if (s->y[i] < 0.0) s->y[i] = s->y[i] + p->ny;
            else if (s->y[i] >= p->ny) s->y[i] = s->y[i] - p->ny;
        }
    }
    return 0;
}

int gdo_run(gdo_state *s, int tstep0, int nsteps, int restart)
{
    for (int k = 0; k < nsteps; k++) gdo_step(s, tstep0 + k, restart);
    return 0;
}

void gdo_get_floes(const gdo_state *s, double *out)
{
    int n = s->n;
    const double *src[GDO_F_COUNT] = {
        s->x, s->y, s->u, s->v, s->r, s->h, s->theta, s->omega, s->tfx, s->tfy,
        s->fcx, s->fcy, s->fbx, s->fby, s->m, s->mc, s->mb, s->tsigxx, s->tsigyy,
        s->tsigxy, s->tsigyx, s->tp, s->fax, s->fay, s->fwx, s->fwy, s->ma, s->mw,
        s->fcorx, s->fcory, s->fx_bc, s->fy_bc, s->m_bc, s->hsfa_min, s->hsfw_min, s->mass};
    for (int f = 0; f < GDO_F_COUNT; f++) memcpy(out + (size_t)f * n, src[f], n * sizeof(double));
}

typedef struct { int32_t i, j; double v; } trip_t;
static int cmp_trip(const void *a, const void *b)
{
    const trip_t *x = (const trip_t *)a, *y = (const trip_t *)b;
    if (x->i != y->i) return x->i < y->i ? -1 : 1;
    return (x->j > y->j) - (x->j < y->j);
}

int gdo_get_pairs(const gdo_state *s, int which, int32_t *pi, int32_t *pj, double *val, int cap)
{
    int cnt = 0;
    trip_t *t = NULL;
    int tcap = 0;
    if (which == GDO_P_CANDIDATES) {
        tcap = s->ncand;
        t = (trip_t *)malloc((size_t)(tcap + 1) * sizeof(trip_t));
        for (int k = 0; k < s->ncand; k++) {
            const pairrec *e = map_find(s, s->cand_i[k], s->cand_j[k]);
            t[cnt].i = s->cand_i[k]; t[cnt].j = s->cand_j[k];
            t[cnt].v = e ? e->deltan : 0.0;
            cnt++;
        }
    } else {
        tcap = (int)s->used;
        t = (trip_t *)malloc((size_t)(tcap + 1) * sizeof(trip_t));
        for (uint64_t k = 0; k < s->cap; k++) {
            const pairrec *e = &s->tab_p[k];
            if (e->key == EMPTY_KEY) continue;
            int i = (int)(e->key >> 32), j = (int)(e->key & 0xffffffffu);
            if (which == GDO_P_CONTACTS && e->deltan > 0.0) {
                t[cnt].i = i; t[cnt].j = j; t[cnt].v = e->deltan; cnt++;
            } else if (which == GDO_P_BONDS && e->bond == 1) {
                t[cnt].i = i; t[cnt].j = j; t[cnt].v = e->damageb; cnt++;
            }
        }
    }
    qsort(t, (size_t)cnt, sizeof(trip_t), cmp_trip);
    for (int k = 0; k < cnt && k < cap; k++) {
        if (pi) pi[k] = t[k].i;
        if (pj) pj[k] = t[k].j;
        if (val) val[k] = t[k].v;
    }
    free(t);
    return cnt;
}

int gdo_get_pair_hist(const gdo_state *s, int i, int j, double *out4)
{
    const pairrec *e = map_find(s, i, j);
    if (!e) { out4[0] = out4[1] = out4[2] = out4[3] = 0.0; return 0; }
    out4[0] = e->deltat; out4[1] = e->thetarelc; out4[2] = e->fcn; out4[3] = e->fct;
    return 1;
}

void gdo_destroy(gdo_state *s)
{
    if (!s) return;
    double **arr[] = {&s->x, &s->y, &s->r, &s->h, &s->hfa, &s->hfw, &s->mass, &s->inertia, &s->u, &s->v,
                      &s->theta, &s->omega, &s->r0, &s->h0, &s->hfa0, &s->hfw0, &s->mass0, &s->inertia0,
                      &s->ua_i, &s->va_i, &s->uw_i, &s->vw_i, &s->fcx, &s->fcy, &s->mc, &s->fbx, &s->fby,
                      &s->mb, &s->tfx, &s->tfy, &s->m, &s->fcorx, &s->fcory, &s->fn_bc, &s->ft_bc, &s->fr_bc,
                      &s->fx_bc, &s->fy_bc, &s->mc_bc, &s->m_bc, &s->deltat_bc1, &s->deltat_bc2,
                      &s->theta_bc1, &s->theta_bc2, &s->delt_ridge_bc, &s->sigxx, &s->sigyy, &s->sigxy,
                      &s->sigyx, &s->sigxx_bc, &s->sigyy_bc, &s->sigxy_bc, &s->sigyx_bc, &s->sigxx_aw,
                      &s->sigyy_aw, &s->sigxy_aw, &s->sigyx_aw, &s->tsigxx, &s->tsigyy, &s->tsigxy,
                      &s->tsigyx, &s->tac, &s->tab, &s->pc, &s->pb, &s->tp, &s->ta_bc, &s->p_bc, &s->fax,
                      &s->fay, &s->fwx, &s->fwy, &s->ma, &s->mw, &s->hsfa_min, &s->hsfw_min, &s->field};
    for (size_t k = 0; k < sizeof(arr) / sizeof(arr[0]); k++) free(*arr[k]);
    free(s->tab_p); free(s->cand_i); free(s->cand_j); free(s->cell_head); free(s->cell_next);
    free(s);
}
