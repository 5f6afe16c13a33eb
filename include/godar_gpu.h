/*
 * godar_gpu.h -- C ABI of libgodar_gpu.so, the B200 replacement for GODAR's
 * per-time-step routine.
 *
 * The reference exposes no plugin API; its seam is the Fortran call
 *     call stepper(tstep, restart)                       (model/src/godar.f90:193)
 * declared `subroutine stepper (tstep, restart)`      (model/src/stepper.f90:1,24)
 * with all state in COMMON blocks (model/inc/CB_*.h).  A replacement
 * stepper.f90 of the same name and signature calls these entry points through
 * an ISO_C_BINDING interface module (godar_b200/fortran/).  Every entry point
 * takes plain pointers and sizes; every one returns a GODAR_* status (0 = OK).
 *
 * Indexing: floe k of the arrays below is the reference's floe k+1.  Pair
 * lists use 0-based (i, j) with i < j, i.e. the reference's (j, i) slot with
 * i < j (stepper.f90:84-87).
 *
 * Threading: one context per host thread at a time; the library owns all
 * device memory and its own CUDA stream; no host pointer is retained after a
 * call returns.  Calls that read results synchronise the context's stream.
 */
#ifndef GODAR_GPU_H
#define GODAR_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
    GODAR_OK = 0,
    GODAR_ERR_CUDA = 1,        /* a CUDA call failed (see godar_gpu_last_error) */
    GODAR_ERR_BAD_INPUT = 2,   /* null pointer, n <= 0, non-finite input, bad enum */
    GODAR_ERR_CAPACITY = 3,    /* a fixed-size table is too small (no-alloc entry) */
    GODAR_ERR_NAN = 4,         /* the state became non-finite during a step */
    GODAR_ERR_TIMEOUT = 5,     /* a bounded device wait gave up */
    GODAR_ERR_NOMEM = 6,       /* device allocation failed */
    GODAR_ERR_STATE = 7,       /* call made in the wrong order (e.g. step before upload) */
    GODAR_ERR_BUDGET = 8,      /* batch admission refused: HBM budget exceeded */
    GODAR_ERR_NOT_FOUND = 9,   /* unknown instance id */
    GODAR_ERR_NO_DEVICE = 10,  /* no CUDA device visible */
    GODAR_ERR_IO = 11          /* an output file could not be opened, written or deleted */
};

/* ---------------------------------------------------------------- params */
/* Boundary flags (extensions).  0 = the reference's four solid walls at
 * x = 0, nx and y = 0, ny (boundaries.f90:1-97). */
enum {
    GODAR_BC_PERIODIC_X = 1,
    GODAR_BC_PERIODIC_Y = 2,
    GODAR_BC_OPEN_LEFT = 4,
    GODAR_BC_OPEN_RIGHT = 8,
    GODAR_BC_OPEN_BOTTOM = 16,
    GODAR_BC_OPEN_TOP = 32
};

/*
 * Run parameters: the eight namelist groups read by read_namelist
 * (model/src/par_get.f90:130-155, defaults par_get.f90:16-109), the
 * compile-time domain size (model/inc/parameter.h:5-10), the derived
 * constants of par_get.f90:263-266, and a few extensions whose zero value
 * reproduces the reference.  Logicals are int32 0/1.
 */
typedef struct godar_params {
    /* options_nml */
    int32_t dynamics, slipping, thermodyn, cohesion, ridging, shelter;
    /* numerical_param_nml */
    double rtree, ntree, dt, nt, comp;
    /* physical_param_nml */
    double Cdair, Csair, Cdwater, Cswater, z0w, lat, rhoair, rhoice, rhowater;
    /* disk_param_nml */
    double e_modul, poiss_ratio, friction_coeff, rest_coeff, sigmanc_crit;
    /* bond_param_nml */
    double eb, lambda_rb, lambda_lb, sigmatb_crit, sigmacb_crit, tau_crit,
           bond_lim, dmax, dtd, dth;
    /* forcings_nml: uniform current (uw, vw) and wind (ua, va) */
    double uw, vw, ua, va;
    /* parameter.h: domain size [m] */
    double nx, ny;
    /* derived on the host: ec, gc, beta (par_get.f90:264-266),
       pi = 4 atan(1) (par_get.f90:35), sin(lat) (forcing.f90:202) */
    double ec, gc, beta, pi, sin_lat;
    /* --- extensions (0 = reference behaviour) --- */
    int32_t boundary;      /* GODAR_BC_* flags */
    int32_t bond_seed;     /* seed of the bond_frac selection hash */
    double bond_lim_rel;   /* bond when deltan >= -(bond_lim + bond_lim_rel*(r_i+r_j)) */
    double bond_frac;      /* in (0,1): keep that hashed fraction of qualifying pairs */
    int32_t field_nx, field_ny; /* forcing grid nodes (0 = uniform forcing only) */
} godar_params;

/* Precision modes. */
enum {
    GODAR_PREC_FP64 = 0,   /* plain method: every step in FP64, the reference's
                              summation order; bit-identical to the FP64 oracle */
    GODAR_PREC_MIXED = 1   /* FP32 pair forces, drag and sheltering; FP64
                              integration, bond strain/damage and ridging
                              bookkeeping */
};

/* Per-floe fields readable with godar_gpu_get_floe_field(). */
enum {
    GODAR_F_X = 0, GODAR_F_Y, GODAR_F_U, GODAR_F_V, GODAR_F_R, GODAR_F_H,
    GODAR_F_THETA, GODAR_F_OMEGA,
    /* the following are filled on the last step of each godar_gpu_step call */
    GODAR_F_TFX, GODAR_F_TFY, GODAR_F_FCX, GODAR_F_FCY, GODAR_F_FBX,
    GODAR_F_FBY, GODAR_F_M, GODAR_F_MC, GODAR_F_MB, GODAR_F_TSIGXX,
    GODAR_F_TSIGYY, GODAR_F_TSIGXY, GODAR_F_TSIGYX, GODAR_F_TP,
    GODAR_F_COUNT
};

/* Pair lists readable with godar_gpu_get_pairs(). */
enum {
    GODAR_P_CANDIDATES = 0, /* (i,j) candidate pairs of the last step, value deltan */
    GODAR_P_CONTACTS = 1,   /* pairs with deltan > 0 at the last step, value deltan
                               (diagnostics_outputs.f90:163-165) */
    GODAR_P_BONDS = 2       /* bonded pairs, value damage
                               (diagnostics_outputs.f90:159-161) */
};

typedef struct godar_ctx godar_ctx;

/* Library version string and the last error message of this thread. */
const char *godar_gpu_version(void);
const char *godar_gpu_errstr(int status);
const char *godar_gpu_last_error(void);
int godar_gpu_params_size(void);

/* Fills p with get_default (par_get.f90:1-111) and the derived constants. */
int godar_gpu_default_params(godar_params *p);
/* Recomputes ec, gc, beta, pi, sin_lat from the namelist values
 * (par_get.f90:263-266). */
int godar_gpu_derive_params(godar_params *p);

/*
 * One simulation of n floes.  Replaces the state set up by ini_get
 * (model/src/ini_get.f90:1-249) + broadcasting_ini (mpi_coms.f90:1-218).
 */
int godar_gpu_create(const godar_params *p, int n, int precision, godar_ctx **out);

/*
 * Copies the initial floe state to the device (ini_get.f90:155-176, 245).
 * u, v, theta, omega may be NULL (zero).  nb restart bonds with damage
 * (read_sparse_restart, ini_get.f90:252-311), i < j; their geometry is
 * computed from the given positions (bond_properties, bonds.f90:237-269).
 */
int godar_gpu_upload(godar_ctx *c, const double *x, const double *y,
                     const double *r, const double *h, const double *theta,
                     const double *omega, const double *u, const double *v,
                     int nb, const int32_t *bond_i, const int32_t *bond_j,
                     const double *damage);

/* Optional gridded forcing (extension of winds_currents, forcing.f90:1-29):
 * 4 planes (ua, va, uw, vw) of field_nx*field_ny node values spanning
 * [0,nx] x [0,ny], row-major (y slowest), added to the uniform values. */
int godar_gpu_set_field(godar_ctx *c, const double *field);

/*
 * Advances nsteps time steps starting at time step tstep: the equivalent of
 *     do k = 0, nsteps-1; call stepper(tstep + k, restart); end do
 * (stepper.f90:1-345).  Bonds are created on time step 1 when restart /= 1
 * and cohesion is on (stepper.f90:93-101).  Diagnostics (forces, stresses,
 * pressure) are produced for the last of the nsteps steps.
 */
int godar_gpu_step(godar_ctx *c, int tstep, int restart, int nsteps);

/* godar_gpu_step without waiting: queues the steps behind those of earlier
 * calls and returns; the status of earlier calls' steps is read once these
 * are queued, so the device always has the next step (a driver that advances
 * one step per call, as the reference's time loop does, godar.f90:191-213,
 * no longer waits for each).  An error of a queued step (NaN, capacity,
 * timeout) is returned by the next call on the context.  A step queued behind
 * one whose neighbour list expired does nothing; the engine rebuilds and runs
 * it again with the diagnostics setting it was queued with, so results equal
 * those of godar_gpu_step bit for bit.  Every other context call but
 * godar_gpu_set_diagnostics first waits for all queued steps.  While the
 * autotuner measures it runs the steps as godar_gpu_step does. */
int godar_gpu_step_async(godar_ctx *c, int tstep, int restart, int nsteps);

/* Copies one per-floe field (GODAR_F_*) of n doubles to host memory. */
int godar_gpu_get_floe_field(godar_ctx *c, int field, double *out);

/* Copies a pair list; *count receives the full size, at most cap entries are
 * written.  Any of pi, pj, val may be NULL. */
int godar_gpu_get_pairs(godar_ctx *c, int which, int32_t *pi, int32_t *pj,
                        double *val, int cap, int *count);

/* All per-floe outputs and one pair list in one call: floe_out is an array
 * of GODAR_F_COUNT pointers indexed by GODAR_F_* (NULL entries, or a NULL
 * array, are skipped); which selects GODAR_P_* (negative: no pair list) with
 * the arguments of godar_gpu_get_pairs.  Replaces the copies back into the
 * COMMON arrays on output steps (godar.f90:195 -> sea_ice_post,
 * diagnostics_outputs.f90:149-182). */
int godar_gpu_download(godar_ctx *ctx, double *const *floe_out, int which, int32_t *pair_i, int32_t *pair_j,
                       double *pair_val, int cap, int *count);
/* The output step of the reference's driver (godar.f90:195-203): appends one
 * record to each of the 25 text files that sea_ice_post writes
 * (diagnostics_outputs.f90:1-189), "<dir>/<name>.<expno>" with dir NULL
 * meaning "output": the per-floe fields x y u v r h theta omega tfx tfy fcx
 * fcy fbx fby mom mc mb tsigxx tsigyy tsigxy tsigyx tp (one record of n
 * values each), the bonds "int(tstep/comp), j, i" with i < j (1-based, in the
 * reference's loop order) followed by an empty record, the damage of each
 * bond, and the contact angle atan2(y(j)-y(i), x(j)-x(i)) * 180/pi of every
 * pair with deltan > 0.  The layout is gfortran's list-directed output (a
 * leading blank, one blank between items, INTEGER(4) in 11 columns, REAL(8)
 * as G25.17E3).  Reads the state and diagnostics of the last step, as
 * godar_gpu_download does. */
int godar_gpu_write_posts(godar_ctx *ctx, const char *dir, const char *expno, int tstep, double comp);
/* clear_posts (diagnostics_ini_io.f90:1-100): deletes the output files of
 * experiment expno (and its info file) in dir (NULL: "output"); missing
 * files are not an error. */
int godar_gpu_clear_posts(const char *dir, const char *expno);
/* One list-directed record of n REAL(8) values, as godar_gpu_write_posts
 * writes it, newline included, NUL-terminated; *len receives its length
 * without the NUL (out NULL: only *len).  GODAR_ERR_CAPACITY when cap is too
 * small. */
int godar_posts_format_reals(const double *v, int n, char *out, size_t cap, size_t *len);

/* Initial-condition generator (the role of tools/init/gridded_placement.py:
 * 111-313): places n disks of radii r (> 0) without overlap in
 * [0,Lx] x [0,Ly], periodic per axis or inside the walls, keeping at least
 * `gap` between disks (a finite gap; a negative one lets disks overlap by up
 * to -gap, and every r + gap/2 must stay > 0); largest first, by random
 * sequential addition with relaxation, on the GPU.  x, y receive the
 * centres (NaN for disks that
 * found no place within max_rounds rounds of their radius class; *placed
 * counts the others; the caller then enlarges the domain).  The result
 * depends only on the inputs and seed.  Allocates device memory for the
 * call and frees it before returning. */
int godar_gpu_place(int n, const double *r, double Lx, double Ly, int periodic_x, int periodic_y, uint64_t seed,
                    int max_rounds, double gap, double *x, double *y, int *placed);

/* Checkpoint of a field that has stepped: the floe state with the wall
 * histories, the complete bond table (geometry, strain, rotation, damage,
 * state) and the pair histories (deltat, thetarelc and the last fcn, fct) in
 * a flat buffer.  With buf NULL only *bytes is set; with cap < *bytes,
 * GODAR_ERR_CAPACITY.  The reference restarts from positions and the bond
 * list (ini_get.f90:129-130, 252-311) and recomputes bond geometry and
 * histories; this one continues the run bit for bit on the FP64 path. */
int godar_gpu_checkpoint(godar_ctx *ctx, void *buf, size_t cap, size_t *bytes);
/* Loads a checkpoint into a context created with the same n (replacing any
 * staged upload).  Set the forcing grid again if the field has one, then step
 * on with the time step after the checkpoint and restart = 1. */
int godar_gpu_restore(godar_ctx *ctx, const void *buf, size_t bytes);
/* Chooses GODAR_PREC_FP64 or GODAR_PREC_MIXED for a context that has not
 * stepped yet (the staged upload is kept); GODAR_ERR_STATE afterwards, since
 * the two paths keep different pair-history and bond-state layouts.  No
 * counterpart in the reference (always FP64). */
int godar_gpu_set_precision(godar_ctx *ctx, int mode);
/* Device time of the last godar_gpu_step call [ms] and counters of the last
 * step: candidate pairs, contacts, bonds, plastic events. */
int godar_gpu_stats(godar_ctx *c, double *ms, int64_t *counts4);

void godar_gpu_destroy(godar_ctx *c);

/*
 * ---------------------------------------------------------------- batches
 * Many independent floe fields ("instances") advanced together.  The
 * reference runs one field per MPI job (utils/duplication.sh:551-588); a
 * batch runs many on one GPU, each time step of all instances in one pass
 * over HBM.  Instances are admitted against an HBM budget and keep their
 * state on the device until removed.
 */
typedef struct godar_batch godar_batch;

int godar_batch_create(int precision, size_t hbm_budget_bytes, godar_batch **out);
/* Bytes of device memory an instance of n floes and nb initial bonds uses. */
size_t godar_batch_instance_bytes(int n, int nb);
/* Admits one instance (state as in godar_gpu_upload; field may be NULL).
 * Returns GODAR_ERR_BUDGET when it does not fit.  Fresh instances
 * (restart == 0) get their bonds created on their first step. */
int godar_batch_add(godar_batch *b, const godar_params *p, int n,
                    const double *x, const double *y, const double *r,
                    const double *h, const double *theta, const double *omega,
                    const double *u, const double *v, int nb,
                    const int32_t *bond_i, const int32_t *bond_j,
                    const double *damage, const double *field, int restart,
                    int *instance_id);
int godar_batch_remove(godar_batch *b, int instance_id);
/* Advances every instance by nsteps time steps and returns once they are
 * done, with the first error any of them raised. */
int godar_batch_step(godar_batch *b, int nsteps);
/* Queues nsteps time steps and returns without waiting for them; the steps
 * of earlier calls are checked once these are queued behind them, so the
 * device always has the next step.  An error of a queued step (NaN,
 * capacity, timeout) is returned by the next call on the batch.  A step
 * queued behind one whose neighbour list expired does nothing; the engine
 * then rebuilds and runs it again with the uniform forcing it was queued with
 * (godar_batch_set_uniform_forcing), so results equal those of
 * godar_batch_step bit for bit.  godar_batch_summary_async and
 * godar_batch_get_all_async read the state after the queued steps without
 * waiting when the last call queued one step (they wait otherwise); every
 * other batch call first waits for all queued steps.  While the autotuner
 * measures, while an admission or removal waits, or without CUDA graphs it
 * runs the steps as godar_batch_step does.  No counterpart in the reference
 * (its time loop is synchronous). */
int godar_batch_step_async(godar_batch *b, int nsteps);
/* Waits for the batch's stream; returns the device time of the work since the
 * previous sync [ms]. */
int godar_batch_sync(godar_batch *b, double *ms);
int godar_batch_get_floe_field(godar_batch *b, int instance_id, int field, double *out);
int godar_batch_steps_done(godar_batch *b, int instance_id, int64_t *steps);
int godar_batch_count(godar_batch *b, int *instances, int64_t *floes);
size_t godar_batch_bytes_in_use(godar_batch *b);
/* Replaces the uniform wind and current of every instance (4 doubles per
 * instance: ua, va, uw, vw, in admission order); takes effect from the next
 * step.  The reference reads them from forcings_nml once (par_get.f90:148-149)
 * and applies them every step (winds_currents, forcing.f90:24-27); a driver
 * may change them between steps. */
int godar_batch_set_uniform_forcing(godar_batch *b, const double *uvw);
/* Copies one per-floe field of every instance, concatenated in admission
 * order, each instance in reference index order. */
int godar_batch_get_all(godar_batch *b, int field, double *out);
/* Asynchronous form for state fields (GODAR_F_X .. GODAR_F_OMEGA, at most 4
 * per call): the gathers and the copies to outs (pinned host memory for them
 * to overlap) are queued after the current step; the next godar_batch_step
 * runs meanwhile.  The call returns once the previous call's copies are
 * complete, so that two read-backs are in flight at most and the copies of
 * consecutive steps run back to back: outs are valid after the next call of
 * this function returns, after godar_batch_wait, or after any synchronous
 * read, admission or removal.  No counterpart in the reference. */
int godar_batch_get_all_async(godar_batch *b, int nfields, const int *fields, double *const *outs);
/* A per-field summary of the current state for monitoring a run without
 * reading its floes: for every instance, in admission order, 4 doubles -
 * total momentum x and y [kg m/s], kinetic energy of translation and
 * rotation [J] (masses and inertias as floe_properties, physics.f90:179-198)
 * and the largest floe speed [m/s].  Reduced on the device in a fixed order
 * over the floes' current memory order (deterministic for a given state and
 * neighbour-list history; a rebuild reorders the floes, so a summary read
 * after godar_batch_step_async, before the engine has learnt of an expiry
 * that godar_batch_step would have rebuilt after at once, can differ in the
 * last bits) and copied to out (pinned host memory, 4 x instances doubles) like
 * godar_batch_get_all_async, with which it shares the two read-back slots.
 * No counterpart in the reference (its driver prints no per-step totals). */
int godar_batch_summary_async(godar_batch *b, double *out);
int godar_batch_wait(godar_batch *b);
/* Device time spent inside the step kernels of the timed steps since the
 * batch was created [ms] (from the first to the last kernel of each; see
 * godar_batch_set_phase_timing), the number of time steps launched,
 * neighbour-list rebuilds, and the counters of the last step (candidate
 * pairs, contacts, bonds, plastic). */
int godar_batch_stats(godar_batch *b, double *kernel_ms, int64_t *launches,
                      int64_t *rebuilds, int64_t *counts4);
/* The same device time split by kernel (CUDA events between the kernels of
 * each timed step), up to nphase entries: GODAR_PREC_MIXED [pair screen, pair
 * work list, bonds, floe sums, floe update], GODAR_PREC_FP64 [entry screen,
 * general work list, bond work list, row sums, floe update]; the number of
 * step kernels launched; and the number of steps timed.  No counterpart in
 * the reference (its timers are the wall-clock prints of godar.f90). */
#define GODAR_NPHASES 5
int godar_batch_phase_stats(godar_batch *b, double *phase_ms, int nphase, int64_t *kernel_launches,
                            int64_t *timed_steps);
/* Which steps godar_batch_step times kernel by kernel: every `every`-th step
 * of each chunk of steps (0, the default: none beyond the autotuner's).  A
 * CUDA event recorded between two kernels of a captured graph costs several
 * microseconds of device time, so an interval of 16 or more keeps the cost
 * under 1 % on large batches.  Steps queued by godar_batch_step_async are
 * never timed.  Read when steps are launched. */
int godar_batch_set_phase_timing(godar_batch *b, int every);
/* Launch configuration in use: per step kernel, its block size in the low 16
 * bits of blocks[q] and its variant above them (the pair screen's items per
 * lane: 0 = 8, 1 = 4, 2 = 16; the bonds: 1 = records streamed through shared
 * memory by bulk copies), chosen by the online autotuner over the first steps
 * of a batch (or the block size of GODAR_BLOCK, variant 0); whether chunks of
 * steps run as captured CUDA graphs, and how many graph launches there
 * were.  Environment: GODAR_TUNE=0 disables the tuner, GODAR_TUNE_LOG=1
 * prints its measurements, GODAR_BOND_VARIANT=v fixes the bond kernel's
 * variant, GODAR_GRAPHS=0 disables the graphs; GODAR_OVERLAP_BONDS=1 runs
 * the mixed bond kernel on a second stream beside the pair kernels (batches
 * without ridging only). */
int godar_batch_launch_config(godar_batch *b, int *blocks, int nphase, int *graphs_on, int64_t *graph_launches);
/* Whether the last step of each step call computes the diagnostics
 * (GODAR_F_TFX .. GODAR_F_TP, the contact list, the counters of the stats);
 * on by default.  A caller that reads only the state (positions, velocities)
 * can switch them off: a diagnostic step walks every candidate pair, not
 * only those that can touch.  While off, diagnostic outputs keep the values
 * of the last diagnostic step.  The reference computes them every step and
 * writes them on output steps (godar.f90:195). */
int godar_batch_set_diagnostics(godar_batch *b, int on);
int godar_gpu_set_diagnostics(godar_ctx *ctx, int on);
/* Neighbour-list rebuilds: total host wall time [ms] (each to its end on
 * the device), count, and the current row sizes: pairs in the neighbour
 * superset and owner entries on the mixed path's contact list. */
int godar_batch_rebuild_stats(godar_batch *b, double *rebuild_ms, int64_t *rebuilds, int64_t *pairs,
                              int64_t *contact_list);
/* Captures ahead of time the CUDA graphs that the next
 * godar_batch_step(b, nsteps) will launch (no device work), so that a timed
 * call does not pay for capture.  A no-op while the autotuner is running. */
int godar_batch_prepare(godar_batch *b, int nsteps);
/* Grows the batch's device memory pool to hold at least `bytes` (device
 * memory that the batch's buffers then draw on without the CUDA driver's
 * allocator), so that admissions and relayouts of a serving loop do not
 * allocate.  The pool keeps what it holds until the batch is destroyed and
 * grows past it on demand. */
int godar_batch_reserve(godar_batch *b, size_t bytes);
void godar_batch_destroy(godar_batch *b);

/*
 * ------------------------------------------------------- no-allocation search
 * No counterpart in the reference.  The candidate pairs (i < j,
 * dist(i,j) <= r_i + rtree) of one floe field, computed without allocating
 * any device memory, for callers that cannot call cudaMalloc (a host program
 * whose own allocator already holds the GPU's memory, or a time-critical loop
 * that must avoid cudaMalloc's implicit synchronisation).  x, y, r, pair_i and
 * pair_j are device pointers owned by the caller; *count (host) receives the
 * number of pairs.  Along a periodic axis (boundary flags) positions may lie
 * any number of periods outside [0, L): they are wrapped into the domain.
 *
 * All scratch lives in a fixed device array of about 2.4 MB.  CUDA loads the
 * library's device code lazily, so the driver allocates that array on a
 * device when this entry point is first used there, and it stays until the
 * process exits: a call with n = 0 does only that set-up (it reads no other
 * argument) and should come first, before the caller's allocator reserves the
 * device's memory and before any stream capture on that device.
 *
 * n above GODAR_NOALLOC_MAX_FLOES is rejected with GODAR_ERR_CAPACITY, as is a
 * result larger than cap (pairs beyond cap are not written; *count is the full
 * size).  Calls share the scratch array: calls that overlap on the GPU race,
 * so serialise them.  Runs on the calling thread's per-thread default stream
 * and returns after it completes.
 */
#define GODAR_NOALLOC_MAX_FLOES 65536
int godar_gpu_candidates_noalloc(const double *x, const double *y, const double *r, int n,
                                 double nx, double ny, double rtree, int boundary,
                                 int32_t *pair_i, int32_t *pair_j, int cap, int *count);

#ifdef __cplusplus
}
#endif
#endif
