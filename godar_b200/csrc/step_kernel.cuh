// One time step of every floe of a batch in FP64: the body of `stepper`
// (stepper.f90:44-343) as three kernels, bit-identical to the reference's
// sequential order.
//
//   k_pairs_fp64_screen, one thread per owner entry (pair of candidates
//   i < j by id, stored in the row of the lower-id floe i): the FP64
//   distance of the pair and the candidate test (dist <= r_i + rtree,
//   stepper.f90:89-92); entries that need no pair physics are finished
//   there, the others go on a work list.
//
//   k_pairs_fp64, one thread per work-list entry: (b) contact
//   (contact_forces.f90:1-87), ridging (ridging.f90:1-99), bond forces and
//   damage (bonds.f90:74-212), sheltering (forcing.f90:162-186) and the
//   stress magnitude (stepper.f90:238-271), computed ONCE per pair.  The
//   pair history and bond state are updated in place (one thread owns a
//   pair); what the two floes add to their sums goes to a record of the pair
//   (the operands of every sum term, not partial sums), written only when the
//   pair contributes anything.
//
//   k_row_sums_fp64, one thread per floe: sorts the floe's own row by
//   (distance, id) - the kd-tree's order, nearly sorted from the previous
//   step - then adds its pairs' records in the reference's order (partners
//   of lower id, ascending id, the floe as "j"; then its own row, the floe
//   as "i") with the same expressions as a sequential walk, so every FP64 sum
//   rounds as in the reference, and applies the pairs' ridging events in
//   that order (d).
//
//   k_floes_fp64, one thread per floe: its wall contacts (verify_bc,
//   boundaries.f90:1-97), drag, Coriolis and the shelter minimum (c,
//   forcing.f90:32-206), totals (stepper.f90:312-332) and the symplectic
//   Euler update (e, integration.f90:1-38).
//
// The kernels read the start-of-step floe state (side cur) and write side
// cur ^ 1.  No floe sum uses atomics, and no pair is evaluated twice.
#pragma once
#include "physics.cuh"

namespace godar {

GD_DEV void bond_load(const Views &V, int bi, int side, BondLocal &B)
{
    const BondDyn d = V.bdyn[side][bi];
    const BondStat c = V.bstat[bi];
    B.flag = d.flag;
    B.dmg = d.dmg; B.dnb = d.dnb; B.dtb = d.dtb; B.thji = d.thji; B.thij = d.thij;
    B.rb = c.rb; B.hb = c.hb; B.lb = c.lb; B.sb = c.sb; B.ib = c.ib;
}

GD_DEV void bond_store(const Views &V, int bi, int side, const BondLocal &B)
{
    BondDyn d;
    d.dnb = B.dnb; d.dtb = B.dtb; d.thji = B.thji; d.thij = B.thij; d.dmg = B.dmg;
    d.flag = B.flag;
    d.pad = 0;
    V.bdyn[side][bi] = d;
}

// What one candidate pair adds to the sums of its two floes, in 32-byte
// groups: each group is written and read only when its flag says so (a
// bond on a plain step: the first and the third).
struct __align__(32) PairRec64 {
    double cosa, sina, ri_l, rj_l;     // any term (PR_CONTACT, PR_BOND, PR_SHEL, PR_DIAG)
    double fcn, fcr, fct, mcc;         // PR_CONTACT
    double fbn, fbt, mji, mij;         // PR_BOND
    double ac, vol, sbt, S;            // diagnostic step: ac (contact), sbt (bond), S (PR_DIAG); vol: a ridging event
    double a_ij, a_ji, w_ij, w_ji;     // PR_SHEL
};

// Pair flags (one byte per pair, every owner entry writes its own).
enum : unsigned char {
    PR_CAND = 1,       // a candidate (dist <= r_i + rtree)
    PR_CONTACT = 2,
    PR_BOND = 4,       // a live bond after this step's breaking test
    PR_SHEL = 8,       // a shelter factor other than exactly 1
    PR_DIAG = 16,      // a stress term other than +-0 (diagnostic steps)
    PR_WHO1 = 32,      // ridging of the lower-id floe
    PR_WHO2 = 64,      // ridging of the higher-id floe
};

GD_DEV double stress_term(double S, double c1, double rl, double c2) { return ((S * c1) * rl) * c2; }

// Owner entries, first pass (few registers): the FP64 distance (kept for
// the row sort) and the candidate test, and the entries that need no pair
// physics finished here.  A non-candidate keeps its history and bond state.
// A candidate that is not in contact, has no bond and is in a field without
// sheltering only has its tangential and rolling histories reset
// (reset_contact, reset.f90:1-15) and, on a diagnostic step, its normal,
// the stress magnitude of its history's last contact forces
// (stepper.f90:238-271) and its overlap recorded: all pair_compute gives it.
// The other candidates go on one of two work lists with their slots, bond
// index and offset: bonded pairs out of contact in fields without
// sheltering (work[1], most of them), and all others (work[0]).
// A plain step visits the positions of plist only (n of them: the pairs
// that can act before the next rebuild, see k_fp64_mark); a diagnostic step
// every owner entry (plist null, n = E).
// U entries per lane (a warp takes 32 U consecutive items): every load of
// the U entries is issued before the first store, so that they overlap.
template <int U, bool DIAG>
__global__ void __launch_bounds__(256) k_pairs_fp64_screen(Views V, int cur, int n, const int *plist,
                                                           const unsigned *erow, unsigned char *pfl, FP64Lists L,
                                                           PairRec64 *rec)
{
    step_kernel_entry();
    if (*(volatile int *)V.status & ST_ABORT) return;
    Hist4<double> *Hs = (Hist4<double> *)V.hist[0];   // in place: one thread per pair
    unsigned long long n_cand = 0;
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    // every lane of a warp runs the same iterations (the list append is warp-wide)
    for (int b0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32 * U; b0 < n; b0 += nwarps * 32 * U) {
        int g[U], t[U], p[U], bi[U];
        double xg[U], yg[U], rg[U], xt[U], yt[U], rt[U];
        double2 h01[U];
        const InstParams *Pk[U];
        int ek[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            // lanes past the end read item 0 and store nothing
            const int i = b0 + 32 * k + lane < n ? b0 + 32 * k + lane : 0;
            ek[k] = plist ? plist[i] : i;
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            const int e = ek[k];
            g[k] = (int)erow[e];
            const int2 en = V.ent_up[e];
            t[k] = en.x;
            p[k] = en.y;
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            Pk[k] = &V.P[V.inst[g[k]]];
            xg[k] = V.x[cur][g[k]]; yg[k] = V.y[cur][g[k]]; rg[k] = V.r[cur][g[k]];
            xt[k] = V.x[cur][t[k]]; yt[k] = V.y[cur][t[k]]; rt[k] = V.r[cur][t[k]];
            bi[k] = V.bidx[p[k]];
            h01[k] = *(const double2 *)&Hs[p[k]];
        }
        double dxk[U], dyk[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const int e = ek[k];
            bool heavy = false, bond_only = false;
            dxk[k] = dyk[k] = 0.0;
            if (b0 + 32 * k + lane < n) {
                const InstParams &P = *Pk[k];
                const bool px = P.boundary & BC_PERIODIC_X, py = P.boundary & BC_PERIODIC_Y;
                const double dx = wrap_d(xg[k] - xt[k], P.nx, px);
                const double dy = wrap_d(yg[k] - yt[k], P.ny, py);
                dxk[k] = dx;
                dyk[k] = dy;
                const double dist = sqrt(dx * dx + dy * dy);
                V.edist[e] = dist;
                if (!(dist <= rg[k] + P.rtree)) {
                    // history and bond state stay as they are
                    pfl[p[k]] = 0;
                    if (DIAG) V.pdn[p[k]] = __int_as_float(0x7fc00000);
                } else {
                    const double deltan = (rg[k] + rt[k]) - dist;
                    const bool general = deltan > 0.0 || P.shelter != 0;
                    heavy = general || bi[k] >= 0;
                    bond_only = !general && bi[k] >= 0;
                    if (!heavy) {
                        // reset_contact: deltat and thetarelc to +0 (most already are)
                        if (__double_as_longlong(h01[k].x) | __double_as_longlong(h01[k].y))
                            *(double2 *)&Hs[p[k]] = make_double2(0.0, 0.0);
                        unsigned f = PR_CAND;
                        if (DIAG) {
                            // pair_compute's normal, stress magnitude (no bond
                            // forces) and overlap, by the same expressions
                            const double2 fc = *(const double2 *)&Hs[p[k]].fcn;
                            const double S = sqrt(fc.x * fc.x + fc.y * fc.y) + sqrt(0.0 * 0.0 + 0.0 * 0.0);
                            const double cosa = -dx / dist, sina = -dy / dist;
                            const double ri = rg[k];
                            if (!(stress_term(S, cosa, ri, cosa) == 0.0 && stress_term(S, sina, ri, sina) == 0.0
                                  && stress_term(S, sina, ri, cosa) == 0.0 && stress_term(S, cosa, ri, sina) == 0.0)) {
                                f |= PR_DIAG;
                                PairRec64 &Q = rec[p[k]];
                                Q.cosa = cosa; Q.sina = sina; Q.ri_l = ri; Q.rj_l = rt[k];
                                Q.S = S;
                            }
                            V.pdn[p[k]] = (float)deltan;
                            n_cand++;
                        }
                        pfl[p[k]] = f;
                    }
                }
            }
#pragma unroll
            for (int l = 0; l < 2; l++) {
                const bool mine = l ? bond_only : heavy && !bond_only;
                const unsigned m = __ballot_sync(0xffffffffu, mine);
                if (m) {
                    int base = 0;
                    if (lane == 0) base = atomicAdd(&L.n[l], __popc(m));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (mine) {
                        FP64Item it;
                        it.p = p[k]; it.g = g[k]; it.t = t[k]; it.bi = bi[k];
                        it.dx = dxk[k]; it.dy = dyk[k];
                        L.work[l][base + __popc(m & ((1u << lane) - 1))] = it;
                    }
                }
            }
        }
    }
    if (DIAG) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n_cand += __shfl_down_sync(0xffffffffu, n_cand, o);
        if (lane == 0 && n_cand) atomicAdd(&V.counters[0], n_cand);
    }
}

// A work list: the pair physics of every remaining candidate, once.
// BONDS: list 1 (bonded, no contact, no sheltering), with the contact
// branch compiled out.  DIAG: a diagnostic step (stress records, overlaps,
// counts).
template <bool BONDS, bool DIAG>
__global__ void __launch_bounds__(128) k_pairs_fp64(Views V, int cur, FP64Lists L, unsigned char *pfl,
                                                    PairRec64 *rec)
{
    step_kernel_entry();
    constexpr bool diag = DIAG;
    if (*(volatile int *)V.status & ST_ABORT) return;
    Hist4<double> *Hs = (Hist4<double> *)V.hist[0];   // in place: one thread per pair
    unsigned long long n_cand = 0, n_cont = 0, n_bond = 0, n_plast = 0;
    const int stride = gridDim.x * blockDim.x;
    const int n = *(volatile const int *)&L.n[BONDS];
    const FP64Item *work = L.work[BONDS];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        // the screen passes the pair, both slots, the bond index and the
        // pair's offset along
        const FP64Item w = work[k];
        const int p = w.p, g = w.g, t = w.t, bi = w.bi;
        const InstParams &P = V.P[V.inst[g]];
        const bool shel = !BONDS && P.shelter != 0;
        const double r = V.r[cur][g];
        const double dx = w.dx, dy = w.dy;
        // the screen's distance, by the same expression
        const double dist = sqrt(dx * dx + dy * dy);
        Hist4<double> H = Hs[p];
        BondLocal BL;
        if (bi >= 0) bond_load(V, bi, 0, BL);
        const Shape si = make_shape(P, r, V.h[cur][g]);
        const Shape sj = make_shape(P, V.r[cur][t], V.h[cur][t]);
        double ua = 0.0, va = 0.0, uw = 0.0, vw = 0.0;
        if (shel) wind_at(P, V.field, V.x[cur][g], V.y[cur][g], ua, va, uw, vw);
        const PairRes<double> R = pair_compute<double, !BONDS>(P, dx, dy, dist, V.u[cur][g], V.v[cur][g], V.om[cur][g],
                                                       V.u[cur][t], V.v[cur][t], V.om[cur][t], si, sj,
                                                       ua, va, uw, vw, H, bi >= 0 ? &BL : nullptr, shel);
        Hs[p] = H;
        if (bi >= 0) bond_store(V, bi, 0, BL);

        unsigned f = PR_CAND;
        if (R.contact) f |= PR_CONTACT;
        if (R.bond_on) f |= PR_BOND;
        if (R.who == 1) f |= PR_WHO1;
        else if (R.who == 2) f |= PR_WHO2;
        if (shel && !(R.a_ij == 1.0 && R.a_ji == 1.0 && R.w_ij == 1.0 && R.w_ji == 1.0)) f |= PR_SHEL;
        // a stress term of +-0 leaves a sum unchanged (the sums start at +0
        // and never become -0), so only nonzero ones (NaN included) count
        if (diag && !(stress_term(R.S, R.cosa, R.ri_l, R.cosa) == 0.0 && stress_term(R.S, R.sina, R.ri_l, R.sina) == 0.0
                      && stress_term(R.S, R.sina, R.ri_l, R.cosa) == 0.0
                      && stress_term(R.S, R.cosa, R.ri_l, R.sina) == 0.0))
            f |= PR_DIAG;
        PairRec64 &Q = rec[p];
        if (f & (PR_CONTACT | PR_BOND | PR_SHEL | PR_DIAG)) {
            Q.cosa = R.cosa; Q.sina = R.sina; Q.ri_l = R.ri_l; Q.rj_l = R.rj_l;
        }
        if (f & PR_CONTACT) {
            Q.fcn = R.fcn; Q.fcr = R.fcr; Q.fct = R.fct; Q.mcc = R.mcc;
            if (diag) Q.ac = R.ac;
        }
        if (f & (PR_WHO1 | PR_WHO2)) Q.vol = R.vol;
        if (f & PR_BOND) {
            Q.fbn = R.fbn; Q.fbt = R.fbt; Q.mji = R.mji; Q.mij = R.mij;
            if (diag) Q.sbt = R.sbt;
        }
        if (f & PR_DIAG) Q.S = R.S;
        if (f & PR_SHEL) { Q.a_ij = R.a_ij; Q.a_ji = R.a_ji; Q.w_ij = R.w_ij; Q.w_ji = R.w_ji; }
        pfl[p] = (unsigned char)f;
        if (diag) {
            V.pdn[p] = (float)R.deltan;
            n_cand++;
            n_cont += R.contact;
            n_bond += R.bond_on;
            n_plast += R.who != 0;
        }
    }

    if (diag) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_cand += __shfl_down_sync(0xffffffffu, n_cand, o);
            n_cont += __shfl_down_sync(0xffffffffu, n_cont, o);
            n_bond += __shfl_down_sync(0xffffffffu, n_bond, o);
            n_plast += __shfl_down_sync(0xffffffffu, n_plast, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&V.counters[0], n_cand);
            atomicAdd(&V.counters[1], n_cont);
            atomicAdd(&V.counters[2], n_bond);
            atomicAdd(&V.counters[3], n_plast);
        }
    }
}

// The pair result one floe's sums need, from the pair's record.  A group the
// flags leave out holds values that make its terms no-ops: no contact, no
// bond, shelter factors of exactly 1 (what the pair computed), stress of 0.
GD_DEV PairRes<double> rec_load(const PairRec64 *rec, int p, unsigned f, bool diag)
{
    PairRes<double> R;
    R.contact = (f & PR_CONTACT) != 0;
    R.bond_on = (f & PR_BOND) != 0;
    R.cosa = R.sina = R.ri_l = R.rj_l = 0.0;
    R.fcn = R.fcr = R.fct = R.mcc = R.ac = 0.0;
    R.fbn = R.fbt = R.mji = R.mij = R.sbt = 0.0;
    R.a_ij = R.a_ji = R.w_ij = R.w_ji = 1.0;
    R.S = 0.0;
    R.vol = 0.0;
    R.who = (f & PR_WHO1) ? 1 : (f & PR_WHO2) ? 2 : 0;
    const PairRec64 &Q = rec[p];
    if (f & (PR_CONTACT | PR_BOND | PR_SHEL | PR_DIAG)) {
        R.cosa = Q.cosa; R.sina = Q.sina; R.ri_l = Q.ri_l; R.rj_l = Q.rj_l;
    }
    if (f & PR_CONTACT) {
        R.fcn = Q.fcn; R.fcr = Q.fcr; R.fct = Q.fct; R.mcc = Q.mcc;
        if (diag) R.ac = Q.ac;
    }
    if (R.who) R.vol = Q.vol;
    if (f & PR_BOND) {
        R.fbn = Q.fbn; R.fbt = Q.fbt; R.mji = Q.mji; R.mij = Q.mij;
        if (diag) R.sbt = Q.sbt;
    }
    if (f & PR_DIAG) R.S = Q.S;
    if (f & PR_SHEL) { R.a_ij = Q.a_ij; R.a_ji = Q.a_ji; R.w_ij = Q.w_ij; R.w_ji = Q.w_ji; }
    return R;
}

// Per-floe outputs of the row sums, [FS64_COUNT][N] doubles (the last eight
// on diagnostic steps only).
enum {
    FS64_FCX, FS64_FCY, FS64_MC, FS64_FBX, FS64_FBY, FS64_MB, FS64_HSFA, FS64_HSFW, FS64_R, FS64_H,
    FS64_TAC, FS64_PC, FS64_TAB, FS64_PB, FS64_SXX, FS64_SYY, FS64_SXY, FS64_SYX, FS64_COUNT
};

// Adds one pair's record to the sums of a floe: `LO` - a partner of lower id
// (the floe is "j"), else one of its own partners ("i").
template <bool DIAG, bool LO>
GD_DEV void add_pair(const PairRec64 *rec, int p, unsigned f, const InstParams &P, Acc<double> &A, Shape &run,
                     bool shel)
{
    if (!f) return;
    const PairRes<double> R = rec_load(rec, p, f, DIAG);
    if (LO) {
        acc_side_j(A, R, P.lambda_lb, shel, DIAG);
        if (R.who == 2) apply_dh(P, run, R.vol);
    } else {
        acc_side_i(A, R, P.lambda_lb, shel, DIAG);
        if (R.who == 1) apply_dh(P, run, R.vol);
    }
}

// Adds the pair records of row entries [e0, e1) of a floe in order.  Flags
// and entries are fetched four at a time so that their loads overlap; the
// sums themselves run strictly in row order.
template <bool DIAG, bool LO>
GD_DEV void row_sum(const int2 *ent, int e0, int e1, const unsigned char *pfl, const PairRec64 *rec,
                    const InstParams &P, Acc<double> &A, Shape &run, bool shel)
{
    for (int e = e0; e < e1; e += 4) {
        int pk[4];
        unsigned fk[4];
#pragma unroll
        for (int k = 0; k < 4; k++) pk[k] = e + k < e1 ? ent[e + k].y : -1;
#pragma unroll
        for (int k = 0; k < 4; k++) fk[k] = pk[k] >= 0 ? pfl[pk[k]] : 0u;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (fk[k]) add_pair<DIAG, LO>(rec, pk[k], fk[k], P, A, run, shel);
    }
}

// Sorts owner-row entries [a0, a1) into the kd-tree's order: ascending
// distance, ties by id.  Rows are nearly sorted from the previous step, so
// insertion sort is linear.
GD_DEV void sort_own(const Views &V, int cur, int a0, int a1)
{
    for (int a = a0 + 1; a < a1; a++) {
        const double da = V.edist[a];
        double db = V.edist[a - 1];
        if (db < da) continue;
        const int2 ea = V.ent_up[a];
        const int ida = V.id[cur][ea.x];
        int b = a - 1;
        while (b >= a0) {
            db = V.edist[b];
            if (db < da || (db == da && V.id[cur][V.ent_up[b].x] < ida)) break;
            V.ent_up[b + 1] = V.ent_up[b];
            V.edist[b + 1] = db;
            b--;
        }
        V.ent_up[b + 1] = ea;
        V.edist[b + 1] = da;
    }
}

// Floes [0, N), first part: the ordered sums of the floe's pairs' records
// and its pairs' ridging events, in the reference's order (partners of
// lower id in ascending id, then its own row in the kd-tree's order).  Every
// row holds first the pairs that can act on a step without diagnostics
// before the next rebuild (lo_n / up_n of them), then the others, each part
// in the row's order: a plain step walks the first part only; a diagnostic
// step, on which every candidate adds its stress, walks both parts merged.
template <bool DIAG>
__global__ void __launch_bounds__(128) k_row_sums_fp64(Views V, int cur, const unsigned char *pfl,
                                                       const PairRec64 *rec, const int *lo_n, const int *up_n,
                                                       double *fs)
{
    step_kernel_entry();
    if (*(volatile int *)V.status & ST_ABORT) return;
    const size_t N = (size_t)V.N;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < V.N; g += gridDim.x * blockDim.x) {
        const InstParams &P = V.P[V.inst[g]];
        const bool shel = P.shelter != 0;
        Acc<double> A;
        A.fcx = A.fcy = A.mc = A.fbx = A.fby = A.mb = 0.0;
        A.tac = A.pc = A.tab = A.pb = 0.0;
        A.sxx = A.syy = A.sxy = A.syx = 0.0;
        A.hsfa = A.hsfw = shel ? 1.0 : 0.0;
        Shape run = make_shape(P, V.r[cur][g], V.h[cur][g]);
        const int l0 = V.lo_off[g], l1 = V.lo_off[g + 1], lm = l0 + lo_n[g];
        const int el = V.up_off[g], e1 = V.up_off[g + 1], em = el + up_n[g];

        if (!DIAG) {
            row_sum<false, true>(V.ent_lo, l0, lm, pfl, rec, P, A, run, shel);
            sort_own(V, cur, el, em);
            row_sum<false, false>(V.ent_up, el, em, pfl, rec, P, A, run, shel);
        } else {
            // ---- partners of lower id (the floe is the reference's "j"):
            // the two parts merged by ascending id
            int a = l0, b = lm;
            int ida = a < lm ? V.id[cur][V.ent_lo[a].x] : 0, idb = b < l1 ? V.id[cur][V.ent_lo[b].x] : 0;
            while (a < lm || b < l1) {
                int take;
                if (b >= l1 || (a < lm && ida < idb)) {
                    take = a++;
                    if (a < lm) ida = V.id[cur][V.ent_lo[a].x];
                } else {
                    take = b++;
                    if (b < l1) idb = V.id[cur][V.ent_lo[b].x];
                }
                const int p = V.ent_lo[take].y;
                add_pair<true, true>(rec, p, pfl[p], P, A, run, shel);
            }
            // ---- own row (the floe is "i"): each part sorted, merged by
            // (distance, id)
            sort_own(V, cur, el, em);
            sort_own(V, cur, em, e1);
            a = el;
            b = em;
            while (a < em || b < e1) {
                bool first = b >= e1;
                if (!first && a < em) {
                    const double da = V.edist[a], db = V.edist[b];
                    first = da < db || (da == db && V.id[cur][V.ent_up[a].x] < V.id[cur][V.ent_up[b].x]);
                }
                const int p = V.ent_up[first ? a++ : b++].y;
                add_pair<true, false>(rec, p, pfl[p], P, A, run, shel);
            }
        }

        fs[FS64_FCX * N + g] = A.fcx; fs[FS64_FCY * N + g] = A.fcy; fs[FS64_MC * N + g] = A.mc;
        fs[FS64_FBX * N + g] = A.fbx; fs[FS64_FBY * N + g] = A.fby; fs[FS64_MB * N + g] = A.mb;
        fs[FS64_HSFA * N + g] = A.hsfa; fs[FS64_HSFW * N + g] = A.hsfw;
        fs[FS64_R * N + g] = run.r; fs[FS64_H * N + g] = run.h;
        if (DIAG) {
            fs[FS64_TAC * N + g] = A.tac; fs[FS64_PC * N + g] = A.pc;
            fs[FS64_TAB * N + g] = A.tab; fs[FS64_PB * N + g] = A.pb;
            fs[FS64_SXX * N + g] = A.sxx; fs[FS64_SYY * N + g] = A.syy;
            fs[FS64_SXY * N + g] = A.sxy; fs[FS64_SYX * N + g] = A.syx;
        }
    }
}

// Floes [0, N), second part: walls with the shape after the floe's pair
// events, drag and Coriolis with the final shape, totals and the FP64
// update.  The shape after the events is make_shape of the radius and
// thickness the sums wrote (apply_dh ends with make_shape too).
template <bool DIAG>
__global__ void __launch_bounds__(128) k_floes_fp64(Views V, int cur, int sic, const double *fs, int *nwork)
{
    step_kernel_entry();
    // the work lists were used by the pair kernels before this one
    if (blockIdx.x == 0 && threadIdx.x < 2) nwork[threadIdx.x] = 0;
    if (floe_update_stopped(V, sic)) return;
    const int nxt = cur ^ 1;
    const size_t N = (size_t)V.N;
    unsigned long long n_plast = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < V.N; g += gridDim.x * blockDim.x) {
        const InstParams &P = V.P[V.inst[g]];
        const bool px = P.boundary & BC_PERIODIC_X, py = P.boundary & BC_PERIODIC_Y;
        const double x = V.x[cur][g], y = V.y[cur][g], th = V.th[cur][g];
        const double u = V.u[cur][g], v = V.v[cur][g], om = V.om[cur][g];
        double dtb1 = V.dtb1[cur][g], dtb2 = V.dtb2[cur][g];
        double thb1 = V.thb1[cur][g], thb2 = V.thb2[cur][g];
        double ua, va, uw, vw;
        wind_at(P, V.field, x, y, ua, va, uw, vw);
        Shape run = make_shape(P, fs[FS64_R * N + g], fs[FS64_H * N + g]);

        // ---- walls with the shape after this floe's pair events
        WallOut W;
        int wev = 0;
        verify_bc(P, x, y, u, v, om, run, dtb1, dtb2, thb1, thb2, W, wev);
        n_plast += DIAG ? wev : 0;

        // ---- drag and Coriolis with the final shape
        const Drag<double> D = forcing<double>(P, run, u, v, om, ua, va, uw, vw, fs[FS64_HSFA * N + g],
                                               fs[FS64_HSFW * N + g]);

        // ---- totals and integration (FP64)
        const double fcx = fs[FS64_FCX * N + g], fcy = fs[FS64_FCY * N + g];
        const double fbx = fs[FS64_FBX * N + g], fby = fs[FS64_FBY * N + g];
        const double mc = fs[FS64_MC * N + g], mb = fs[FS64_MB * N + g];
        const double fax = D.fax, fay = D.fay, fwx = D.fwx, fwy = D.fwy;
        const double tfx = ((((fcx + fbx) + fax) + fwx) + D.fcorx) + W.fx_bc;
        const double tfy = ((((fcy + fby) + fay) + fwy) + D.fcory) + W.fy_bc;
        const double mt = (((mc + mb) + D.ma) + D.mw) + W.m_bc;
        const double dt = P.dt;
        const double u1 = u + (tfx / run.mass) * dt;
        const double v1 = v + (tfy / run.mass) * dt;
        const double om1 = om + (mt / run.inertia) * dt;
        double x1 = x + u1 * dt;
        double y1 = y + v1 * dt;
        const double th1 = th + om1 * dt;
        if (px) { if (x1 < 0.0) x1 = x1 + P.nx; else if (x1 >= P.nx) x1 = x1 - P.nx; }
        if (py) { if (y1 < 0.0) y1 = y1 + P.ny; else if (y1 >= P.ny) y1 = y1 - P.ny; }
        V.x[nxt][g] = x1; V.y[nxt][g] = y1; V.th[nxt][g] = th1;
        V.u[nxt][g] = u1; V.v[nxt][g] = v1; V.om[nxt][g] = om1;
        V.r[nxt][g] = run.r; V.h[nxt][g] = run.h;
        V.dtb1[nxt][g] = dtb1; V.dtb2[nxt][g] = dtb2;
        V.thb1[nxt][g] = thb1; V.thb2[nxt][g] = thb2;

        // ---- neighbour-list validity and finiteness
        const double ddx = wrap_d(x1 - V.x0[cur][g], P.nx, px), ddy = wrap_d(y1 - V.y0[cur][g], P.ny, py);
        const double half = 0.5 * P.skin;
        if (ddx * ddx + ddy * ddy > half * half) {
            atomicOr(V.status, ST_EXPIRED);
            atomicMin(V.expired_at, global_step(V, sic));
        }
        if (!(isfinite(x1) && isfinite(y1) && isfinite(u1) && isfinite(v1) && isfinite(om1) && isfinite(th1)))
            atomicOr(V.status, ST_NAN);

        if (DIAG) {
            const double rr = run.r;
            const double sxx = (fs[FS64_SXX * N + g] + W.sxx) + (fax + fwx) * rr;
            const double syy = (fs[FS64_SYY * N + g] + W.syy) + (fay + fwy) * rr;
            const double sxy = (fs[FS64_SXY * N + g] + W.sxy) + 0.0;
            const double syx = (fs[FS64_SYX * N + g] + W.syx) + 0.0;
            const double tac = fs[FS64_TAC * N + g], tab = fs[FS64_TAB * N + g];
            const double pa = tac != 0.0 ? fs[FS64_PC * N + g] / tac : 0.0;
            const double pbv = tab != 0.0 ? fs[FS64_PB * N + g] / tab : 0.0;
            const double pw = W.ta_bc != 0.0 ? W.p_bc / W.ta_bc : 0.0;
            double *D0 = V.diag;
            D0[0 * N + g] = tfx; D0[1 * N + g] = tfy; D0[2 * N + g] = fcx; D0[3 * N + g] = fcy;
            D0[4 * N + g] = fbx; D0[5 * N + g] = fby; D0[6 * N + g] = mt; D0[7 * N + g] = mc;
            D0[8 * N + g] = mb; D0[9 * N + g] = sxx; D0[10 * N + g] = syy; D0[11 * N + g] = sxy;
            D0[12 * N + g] = syx; D0[13 * N + g] = (pa + pbv) + pw;
        }
    }

    if (DIAG) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) n_plast += __shfl_down_sync(0xffffffffu, n_plast, o);
        if ((threadIdx.x & 31) == 0 && n_plast) atomicAdd(&V.counters[3], n_plast);
    }
}

}  // namespace godar
