// The mixed-precision time step as three kernels.
//
// (b) k_pairs_mixed: one lane per owner-row entry (each unordered pair once,
//     stepper.f90:89-271 without the bond terms).  Most candidates are not in
//     contact: a lane that can see from the squared distance that the pair
//     neither touches nor carries a contact history does nothing beyond
//     clearing its flags.  A contact, a pair with history, every candidate of
//     a sheltering field and every candidate on a diagnostic step leaves a
//     32-byte record at its own index (force on the lower-id floe, both
//     moments, shelter factors) and sets a flag byte in both rows; histories
//     are updated in place.  No reductions and no atomics.
// (b') k_bonds_mixed: one lane per bond (bonds.f90:74-212), in bond order, so
//     the bond state is read and written contiguously; it leaves a 16-byte
//     record per bond.
// (c)-(e) k_floes_mixed: one thread per floe; sums the flagged records of its
//     two rows and of its bonds, then walls, ridging, drag, Coriolis and the
//     FP64 update.
// Pair forces, sheltering and drag are FP32; geometry that cancels, bond
// strain/damage, ridging bookkeeping and integration are FP64.
#include <algorithm>
#include <cstdlib>

#include "physics.cuh"
#include "kernels.h"

namespace godar {

// flag bits of a pair (owner entry) and of its mirror partner entry
enum : unsigned {
    PF_HIST = 1,     // owner entry only: deltat or thetarelc nonzero
    PF_REC = 2,      // the pair left a force record this step (contact, or a sheltering field)
    PF_DG = 4,       // the pair left diagnostic sums (a diagnostic step: a candidate with a nonzero term)
    PF_REX = 8       // ... and a ridging event (rx holds the excesses)
};

// Contact part of stepper.f90:89-271 (contact_forces.f90:1-87,
// physics.f90:1-33, ridging.f90:1-99) for one candidate pair, FP32 forces.
struct ContactOut {
    bool contact;
    int who;             // ridging event: 0 none, 1 lower-id floe, 2 higher-id floe
    double vol;
    float fx, fy, mi, mj;   // force on the lower-id floe; moments of both floes
    float fcn, ac;          // diagnostics: normal force, contact area
    float ri_l, rj_l, hi_l, hj_l;   // radii and thicknesses after the pair's own event
};

GD_DEV void contact_mixed(const InstParams &P, double dist, float cosa, float sina, const Snap &I, const Snap &J,
                          Hist4<float> &H, bool bond_active, ContactOut &C)
{
    const float dt = P.f_dt;
    const float omegarel = J.om - I.om;
    const float du = J.u - I.u, dv = J.v - I.v;
    const float veln = du * cosa + dv * sina;
    const float veltb = -(du * sina) + dv * cosa;
    float ri = (float)I.r, rj = (float)J.r;
    const float velt = veltb - (I.om * ri + J.om * rj);
    const double deltan = (I.r + J.r) - dist;
    const float dn = (float)deltan;
    float hi_l = I.h, hj_l = J.h;
    C.who = 0;
    C.vol = 0.0;
    C.contact = deltan > 0.0;
    C.fx = C.fy = C.mi = C.mj = C.fcn = C.ac = 0.f;
    if (C.contact) {
        H.deltat = -(velt * dt) + H.deltat;
        const double q = ((dist * dist - J.r * J.r) + I.r * I.r) / (2.0 * dist);
        double drd = 2.0 * sqrt(I.r * I.r - q * q);
        float dr = (float)drd;
        H.thetarelc = -(omegarel * dt) + H.thetarelc;
        const float m_redu = (I.mass * J.mass) / (I.mass + J.mass);
        const float r_redu = (ri * rj) / (ri + rj);
        const float hmin = fminf(I.h, J.h);
        const float beta = P.f_beta;
        const float knc = (P.f_piec * hmin) * fit<float>((dn * r_redu) / (2.f * (hmin * hmin)));
        float ktc = P.f_ktc * knc;
        float krc = (knc * (dr * dr)) * (1.f / 12.f);
        float gamn = -(beta * sqrtf((4.f * knc) * m_redu));
        float gamt = -((2.f * beta) * sqrtf(((2.f / 3.f) * ktc) * m_redu));
        float gamr = (gamn * (dr * dr)) * (1.f / 12.f);
        float fcn = fmaxf(knc * dn - gamn * veln, 0.f);
        float fct = ktc * H.deltat - gamt * velt;
        if (P.ridging && P.f_sigc * hmin <= (fcn / dr) / hmin) {
            // plastic_contact (ridging.f90:1-33)
            const float knp = ((P.f_sigc * (hmin * hmin)) * dr) / dn;
            ktc = P.f_ktc * knp;
            krc = (knp * (dr * dr)) * (1.f / 12.f);
            gamn = -(beta * sqrtf((4.f * knp) * m_redu));
            gamt = -((2.f * beta) * sqrtf(((2.f / 3.f) * ktc) * m_redu));
            gamr = (gamn * (dr * dr)) * (1.f / 12.f);
            fcn = fminf(fcn, (P.f_sigc * (hmin * hmin)) * dr);
            fct = ktc * H.deltat - gamt * velt;
            // update_shape (ridging.f90:36-99) in FP64
            Shape si = make_shape(P, I.r, (double)I.h), sj = make_shape(P, J.r, (double)J.h);
            const double hm2 = si.h < sj.h ? si.h : sj.h;
            const double dij = ((dist * dist - sj.r * sj.r) + si.r * si.r) / (2.0 * dist);
            const double dji = ((dist * dist - si.r * si.r) + sj.r * sj.r) / (2.0 * dist);
            const double Area = (((si.r * si.r) * dm::acos(dij / si.r) - (dij * drd) / 2.0)
                                 + (sj.r * sj.r) * dm::acos(dji / sj.r)) - (dji * drd) / 2.0;
            const double a2 = (Area * hm2) / 2.0;
            const double Vol = a2 > 0.0 ? a2 : 0.0;
            if (hm2 == si.h) { C.who = 1; apply_dh(P, si, Vol); }
            else if (hm2 == sj.h) { C.who = 2; apply_dh(P, sj, Vol); }
            C.vol = Vol;
            const double q2 = ((dist * dist - sj.r * sj.r) + si.r * si.r) / (2.0 * dist);
            drd = 2.0 * sqrt(si.r * si.r - q2 * q2);
            dr = (float)drd;
            ri = (float)si.r; rj = (float)sj.r;
            hi_l = (float)si.h; hj_l = (float)sj.h;
        }
        float fcr;
        const float mu = P.f_mu;
        if (fabsf(fct) > mu * fabsf(fcn)) {
            fct = -((mu * fabsf(fcn)) * copysignf(1.f, velt));
            fcr = fct;
            if (P.slipping) H.deltat = (fct + gamt * velt) / ktc;
        } else {
            fcr = fct;
        }
        float mcc = 0.f;
        if (!bond_active) {
            float mrolling = krc * H.thetarelc - gamr * omegarel;
            if (fabsf(H.thetarelc) > ((2.f * fabsf(fcn)) / knc) / dr) mrolling = 0.f;
            mcc = mrolling;
        }
        H.fcn = fcn;
        H.fct = fct;
        // the lower-id floe's share (stepper.f90:113-129); the partner's force
        // is its negative, its moment -rj fct + mcc
        C.fx = -(fcn * cosa) + fcr * sina;
        C.fy = -(fcn * sina) - fcr * cosa;
        C.mi = -(ri * fct) - mcc;
        C.mj = -(rj * fct) + mcc;
        C.fcn = fcn;
        C.ac = dr * fminf(hi_l, hj_l);
    } else {
        H.thetarelc = 0.f;
        H.deltat = 0.f;
    }
    C.ri_l = ri; C.rj_l = rj;
    C.hi_l = hi_l; C.hj_l = hj_l;
}

// bond_forces_euler and bond_breaking (bonds.f90:74-212) for one live bond:
// strain and damage in FP64, beam coefficients (1 - D) x the undamaged FP32
// ones.  ri_l, rj_l: radii after the pair's own ridging event.
struct BondOut {
    bool on;
    float fx, fy, mi, mj;   // force on the lower-id floe; moments of both floes
    float fbn, sb, S;       // diagnostics
};

// The FP32 coefficients of a bond from its geometry: sb = 2 rb hb and
// ib = 2/3 hb rb^3 (bonds.f90:260-261), EA = eb sb, EI = eb ib.
GD_DEV BondStat32 bond_coeffs(const InstParams &P, const BondGeom32 &G)
{
    BondStat32 s;
    const float rb = G.rb, hb = G.hb;
    const float sb = (2.f * rb) * hb;
    const float ib = ((2.f / 3.f) * hb) * ((rb * rb) * rb);
    const float ea = P.f_eb * sb, ei = P.f_eb * ib;
    const float inv_hb = __fdividef(1.f, hb);
    s.inv_l = G.inv_l;
    s.k_ax = ea * G.inv_l;
    s.ei_l = ei * G.inv_l;
    s.ea_l = ea * G.lb;
    s.sb = sb;
    s.inv_sb = __fdividef(1.f, sb);
    s.rb_ib = __fdividef(rb, ib);
    s.inv_tau_hb = P.f_inv_tau * inv_hb;
    s.inv_sigc_hb = P.f_inv_sigcb * inv_hb;
    s.inv_sigt_hb = P.f_inv_sigtb * inv_hb;
    return s;
}

GD_DEV void bond_mixed(const InstParams &P, const BondStat32 &BS, BondDyn &B, float cosa, float sina,
                       const Snap &I, const Snap &J, float ri_l, float rj_l, BondOut &O)
{
    const float du = J.u - I.u, dv = J.v - I.v;
    const float veln = du * cosa + dv * sina;
    const float veltb = -(du * sina) + dv * cosa;
    B.dnb = (double)veln * P.dt + B.dnb;
    B.dtb = (double)veltb * P.dt + B.dtb;
    B.thji = (double)I.om * P.dt + B.thji;
    B.thij = (double)J.om * P.dt + B.thij;
    const float omd = (float)(1.0 - B.dmg);
    // FP32 arithmetic with fast divisions and the products of square roots
    // taken as one root (the mixed tolerance allows it)
    const float m_redu = __fdividef(I.mass * J.mass, I.mass + J.mass);
    const float rfi = (float)I.r, rfj = (float)J.r;
    const float Ii = (0.5f * I.mass) * (rfi * rfi), Ij = (0.5f * J.mass) * (rfj * rfj);
    const float i_redu = __fdividef(Ii * Ij, Ii + Ij);
    // EA/L, 12EI/L^3, 6EI/L^2, 4EI/L, 2EI/L and EA L from EA/L, EI/L, 1/L
    const float il = BS.inv_l, eil = BS.ei_l;
    const float k_axial = omd * BS.k_ax;
    const float k_shear1 = omd * ((12.f * eil) * (il * il)), k_shear2 = omd * ((6.f * eil) * il);
    const float k_rot1 = omd * (4.f * eil), k_rot2 = omd * (2.f * eil);
    const float eta_i = 2.f * sqrtf((omd * eil) * i_redu);
    const float eta_a = 2.f * sqrtf((omd * BS.ea_l) * m_redu);
    const float gam_axial = eta_a * il;
    const float gam_shear1 = ((12.f * eta_i) * il) * (il * il);
    const float gam_shear2 = ((6.f * eta_i) * il) * il;
    const float gam_rot1 = (4.f * eta_i) * il, gam_rot2 = (2.f * eta_i) * il;
    const float dnb = (float)B.dnb, dtb = (float)B.dtb, thji = (float)B.thji, thij = (float)B.thij;
    float fbn = k_axial * dnb + gam_axial * veln;
    float fbt = ((k_shear1 * dtb + k_shear2 * (thji + thij)) + gam_shear1 * veltb) + gam_shear2 * (I.om + J.om);
    float mji = ((((k_rot1 * thji + k_rot2 * thij) - k_shear2 * dtb) + gam_rot1 * I.om) + gam_rot2 * J.om)
                - gam_shear2 * veltb;
    float mij = ((((k_rot2 * thji + k_rot1 * thij) - k_shear2 * dtb) + gam_rot2 * I.om) + gam_rot1 * J.om)
                - gam_shear2 * veltb;
    const float sb = BS.sb;
    const float taub = fabsf(fbt) * BS.inv_sb;
    const float bend = fabsf(mji) * BS.rb_ib;
    const float sn = fbn * BS.inv_sb;
    const float sigmatb = -sn + bend;
    const float sigmacb = sn + bend;
    const float t1 = taub * BS.inv_tau_hb;
    float phi = t1 * t1;
    if (sigmacb > 0.f) { const float t2 = sigmacb * BS.inv_sigc_hb; phi = phi + t2 * t2; }
    if (sigmatb > 0.f) { const float t3 = sigmatb * BS.inv_sigt_hb; phi = phi + t3 * t3; }
    const float psi = fminf(1.f, rsqrtf(phi));
    double D = B.dmg;
    D = (D + ((1.0 - (double)psi) * (1.0 - D)) * P.dt_dtd) - D * P.dt_dth;
    B.dmg = D;
    if (D >= P.dmax) {
        B.flag = 0;
        fbn = 0.f; fbt = 0.f; mji = 0.f;
        B.dmg = 1.0;
    }
    O.S = sqrtf(fbn * fbn + fbt * fbt);
    O.on = B.flag == 1;
    if (O.on) {
        const float llb = P.f_llb;
        O.fx = fbn * cosa - fbt * sina;
        O.fy = fbn * sina + fbt * cosa;
        O.mi = -((llb * ri_l) * fbt) - mji;
        O.mj = -((llb * rj_l) * fbt) - mij;
        O.fbn = fbn;
        O.sb = sb;
    } else {
        O.fx = O.fy = O.mi = O.mj = O.fbn = O.sb = 0.f;
    }
}

// Adds a warp's diagnostic count to counters[k] (every lane must call it).
GD_DEV void warp_count(unsigned long long a, unsigned long long *counters, int k)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0 && a) atomicAdd(&counters[k], a);
}

// Screening pass: one lane per owner entry, few registers.  A pair with no
// contact history in a field without sheltering can only matter if it
// touches, and d2 > (ri + rj)^2 (1 + 1e-9) is safely beyond contact in FP64;
// such a lane only clears stale record flags.  Every other pair (and every
// pair on a diagnostic step) is appended to the work list (one atomic per
// warp for the slots; the results do not depend on the list's order).
// The contact list of the current rows is two arrays: {entry, bound bits}
// (eb) and {row slot, partner slot} (st) per item (eb null: every owner
// entry, as on diagnostic steps); the bound test reads only the first.
//
// Conservative advancement.  D_k bounds how far any floe of the batch has
// moved since the rebuild: D grows each step by the largest step of any
// floe (k_floes_mixed reduces it), in FP32 rounded up.  An item holds
// b = g_t + 2 D_t, rounded down, from the last step t at which the pair was
// tested in FP64, where g_t = d_t - (ri + rj)(1 + 1e-9) (at the rebuild,
// D = 0 and b is the gap there).  Between t and now each floe moved at most
// D_k - D_t, so d_k >= d_t - 2 (D_k - D_t) and a pair with b > 2 D_k (plus
// 1e-6 m for the FP64 rounding of d) is beyond the FP64 test without reading
// either floe.  Every FP64 test that finds the pair apart stores a fresh b.
// b = -inf marks pairs that are always tested (sheltering or ridging
// fields, whose radii change).
// The FP64 test of contact-list item k (entry c.x, bound c.y, slots st;
// f0 the entry's flags): whether the pair goes on the work list.  A pair
// found apart drops a stale record flag and stores a fresh bound.
GD_DEV bool screen_test(const Views &V, const Snap *S, int2 *eb, int k, const int2 c, const int2 st, unsigned f0,
                        float Dk, const MixedBufs &B)
{
    const int e = c.x, s = st.x, t = st.y;
    const double xi = S[s].x, yi = S[s].y, ri = S[s].r;
    const double xj = S[t].x, yj = S[t].y, rj = S[t].r;
    const InstParams &Pm = V.P[S[s].inst];
    if (Pm.shelter || (f0 & PF_HIST)) return true;
    const bool px = Pm.boundary & BC_PERIODIC_X, py = Pm.boundary & BC_PERIODIC_Y;
    const double dx = wrap_d(xi - xj, Pm.nx, px), dy = wrap_d(yi - yj, Pm.ny, py);
    const double rs = ri + rj;
    const double d2 = dx * dx + dy * dy;
    if (!(d2 > (rs * rs) * (1.0 + 1e-9))) return true;
    if (f0 & PF_REC) {
        B.pfl[e] = 0;
        B.lfl[B.lo_of[e]] = 0;
    }
    if (__int_as_float(c.y) != -INFINITY) {
        const double b = (sqrt(d2) - rs * (1.0 + 1e-9)) + 2.0 * (double)Dk;
        reinterpret_cast<int *>(eb + k)[1] = __float_as_int(__double2float_rd(b));
    }
    return false;
}

// Appends entry e of every lane with `heavy` to the work list, with its
// slots st where known (st.x >= 0), one atomic per warp; every lane of the
// warp must call it.
GD_DEV void work_append(bool heavy, int e, int2 st, int lane, const MixedBufs &B)
{
    const unsigned m = __ballot_sync(0xffffffffu, heavy);
    if (m) {
        int base = 0;
        if (lane == 0) base = atomicAdd(B.nwork, __popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (heavy) {
            const int q = base + __popc(m & ((1u << lane) - 1u));
            B.work[q] = e;
            if (st.x >= 0) B.work_st[q] = st;
        }
    }
}

// SCREEN_U: contact-list items per lane per round (the screen's tile,
// chosen per batch by the autotuner among 4, 8 and 16)
template <int SCREEN_U>
__global__ void __launch_bounds__(256) k_pairs_screen(Views V, int cur, int diag, int P, int2 *eb,
                                                      const int2 *stl, MixedBufs B)
{
    step_kernel_entry();
    if (*(volatile int *)V.status & ST_ABORT) return;
    // items of a round that need the FP64 test, per warp
    __shared__ int chk[256 / 32][SCREEN_U * 32];
    const Snap *S = V.snap[cur];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int stride = gridDim.x * blockDim.x;
    const int nit = (P + stride - 1) / stride;
    // D of this step: the previous step's D and largest step (side cur ^ 1);
    // one thread publishes it and clears the slot this step's update fills
    const int o = cur ^ 1;
    const float Dk = __fadd_ru(__uint_as_float(__ldcg(B.dsp + 2 + o)),
                               __fmul_ru(__fsqrt_ru(__uint_as_float(__ldcg(B.dsp + o))), 1.00001f));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        B.dsp[2 + cur] = __float_as_uint(Dk);
        B.dsp[cur] = 0u;
    }
    // a diagnostic step computes every owner entry: the pair kernel walks
    // them itself, without a work list
    if (diag || !eb) return;
    const float thr = __fadd_ru(2.f * Dk, 1e-6f);
    const unsigned lt = (1u << lane) - 1u;
    int k0 = blockIdx.x * blockDim.x + threadIdx.x;
    for (int it = 0; it < nit; it += SCREEN_U, k0 += SCREEN_U * stride) {
        // the bound test of SCREEN_U items per lane, their loads issued
        // together; the items that fail it are gathered per warp ...
        //
        // A pair with a contact history, or with a force record from its last
        // computation, is in contact or was at that computation; conservative
        // advancement keeps its bound at or below the threshold from then on
        // (and the contact list is built with a bound of at most -1 for a pair
        // with a history), so an item that passes the bound test carries
        // neither: its flags need not be read.
        int2 c[SCREEN_U];
#pragma unroll
        for (int u = 0; u < SCREEN_U; u++) {
            const int k = k0 + u * stride;
            c[u] = make_int2(-1, 0);
            if (it + u < nit && k < P) c[u] = eb[k];
        }
        int cnt = 0;
#pragma unroll
        for (int u = 0; u < SCREEN_U; u++) {
            const bool need = c[u].x >= 0 && !(__int_as_float(c[u].y) > thr);
            // gathered per warp, then tested together
            const unsigned m = __ballot_sync(0xffffffffu, need);
            if (need) chk[warp][cnt + __popc(m & lt)] = k0 + u * stride;
            cnt += __popc(m);
        }
        __syncwarp();
        // ... one item per lane: a pair with a history goes on the work list
        // at once, the others by the FP64 test
        for (int j0 = 0; j0 < cnt; j0 += 32) {
            bool heavy = false;
            int e = 0;
            int2 st = make_int2(-1, -1);
            if (j0 + lane < cnt) {
                const int k = chk[warp][j0 + lane];
                const int2 ck = eb[k];
                e = ck.x;
                st = stl[k];
                heavy = screen_test(V, S, eb, k, ck, st, (unsigned)B.pfl[e], Dk, B);
            }
            work_append(heavy, e, st, lane, B);
        }
        __syncwarp();
    }
}

// Pairs of the work list: contact forces, ridging events, sheltering,
// history updates and records.
__global__ void __launch_bounds__(256, 3) k_pairs_mixed(Views V, int cur, int diag, int P, const unsigned *erow,
                                                        MixedBufs B)
{
    step_kernel_entry();
    if (*(volatile int *)V.status & ST_ABORT) return;
    Hist4<float> *Hh = (Hist4<float> *)V.hist[0];
    const Snap *S = V.snap[cur];
    unsigned long long n_cand = 0, n_cont = 0, n_plast = 0;
    // the work list of the screen, or on a diagnostic step every owner entry
    const int n = diag ? P : *(volatile const int *)B.nwork;
    const int stride = gridDim.x * blockDim.x;
    // every lane of a warp runs the same number of iterations (the counters
    // are reduced with full-warp shuffles at the end)
    const int nit = (n + stride - 1) / stride;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    for (int it = 0; it < nit; it++, k += stride) {
        if (k >= n) continue;
        const int e = diag ? k : B.work[k];
        // the screen passes the slots along, except on diagnostic steps
        int s, t;
        if (diag) {
            s = (int)erow[e];
            t = V.ent_up[e].x;
        } else {
            const int2 st = B.work_st[k];
            s = st.x;
            t = st.y;
        }
        const unsigned f0 = B.pfl[e];
        // the entry's own records, loaded beside the snapshots rather than
        // after the distance test
        const Hist4<float> Hraw = Hh[e];
        const int bix = V.bidx[e];
        const int wix = bix >= 0 ? B.winv[bix] : -1;
        const Snap Si = S[s], Sj = S[t];      // s has the lower id: the reference's "i"
        const InstParams &Pm = V.P[Si.inst];
        const bool px = Pm.boundary & BC_PERIODIC_X, py = Pm.boundary & BC_PERIODIC_Y;
        const bool shel = Pm.shelter != 0;
        const double dx = wrap_d(Si.x - Sj.x, Pm.nx, px), dy = wrap_d(Si.y - Sj.y, Pm.ny, py);
        const double d2 = dx * dx + dy * dy;
        unsigned f1 = f0 & PF_HIST;
        const double dist = sqrt(d2);
        if (dist <= Si.r + Pm.rtree) {
            Hist4<float> H;
            if ((f0 & PF_HIST) || diag) H = Hraw;
            else { H.deltat = 0.f; H.thetarelc = 0.f; H.fcn = 0.f; H.fct = 0.f; }
            const float fd = (float)dist;
            const float cosa = (float)(-dx) / fd;
            const float sina = (float)(-dy) / fd;
            ContactOut C;
            int bi = -1;
            bool bond_active = false;
            if ((Si.r + Sj.r) - dist > 0.0) {
                // the bond's working index; its state at the start of the
                // step (the bond kernel may be updating it at the same time)
                bi = wix;
                if (bi >= 0) {
                    bond_active = B.bfl_rd[bi] == 1;
                }
            }
            contact_mixed(Pm, dist, cosa, sina, Si, Sj, H, bond_active, C);
            if (C.contact || (f0 & PF_HIST)) {
                Hh[e] = H;
                f1 = (H.deltat != 0.f || H.thetarelc != 0.f) ? PF_HIST : 0u;
            }
            if (C.who != 0 && bi >= 0) {
                // tell the bond kernel the pair's post-event radius
                const float rl = C.who == 1 ? C.ri_l : -C.rj_l;
                B.wdyn[bi].pad = __float_as_int(rl);
            }
            // force records only where a force or shelter factor can be
            // nonzero, so that entries off the contact list never carry one
            if (C.contact || shel) {
                B.rec[2 * (size_t)e] = make_float4(C.fx, C.fy, C.mi, C.mj);
                if (shel) {
                    double a0, a1, a2, a3;
                    wind_at(Pm, V.field, Si.x, Si.y, a0, a1, a2, a3);
                    const float ua = (float)a0, va = (float)a1, uw = (float)a2, vw = (float)a3;
                    const float dn = (float)((Si.r + Sj.r) - dist);
                    const float hfai = Pm.f_hfa * C.hi_l, hfaj = Pm.f_hfa * C.hj_l;
                    const float hfwi = Pm.f_hfw * C.hi_l, hfwj = Pm.f_hfw * C.hj_l;
                    const float a_ij = S_shelter<float>(hfai, hfaj, dn, cosa, sina, ua, va);
                    const float w_ij = S_shelter<float>(hfwi, hfwj, dn, cosa, sina, uw, vw);
                    const float a_ji = S_shelter<float>(hfaj, hfai, dn, -cosa, -sina, ua, va);
                    const float w_ji = S_shelter<float>(hfwj, hfwi, dn, -cosa, -sina, uw, vw);
                    B.rec[2 * (size_t)e + 1] = make_float4(a_ji, w_ji, a_ij, w_ij);
                }
                f1 |= PF_REC;
                if (C.who != 0) {
                    const double rex = C.who == 1 ? C.vol / ((Pm.pi * (Si.r * Si.r)) * (double)Si.h)
                                                  : C.vol / ((Pm.pi * (Sj.r * Sj.r)) * (double)Sj.h);
                    B.rx[e] = C.who == 1 ? make_float2((float)rex, 0.f) : make_float2(0.f, (float)rex);
                    f1 |= PF_REX;
                }
            }
            if (diag) {
                // contact part of the stress sums (stepper.f90:238-271); the
                // reference's S adds the bond force, done per bond.  A pair
                // out of contact whose last normal and tangential forces are
                // zero (it has not touched since it entered the rows) adds
                // only zeros: it leaves no record (a sum that starts at +0
                // never becomes -0, so adding a zero changes no bit)
                const float Sc = sqrtf(H.fcn * H.fcn + H.fct * H.fct);
                if (C.contact || Sc != 0.f) {
                    f1 |= PF_DG;
                    const float rl = C.ri_l;
                    B.pdg[2 * (size_t)e] = make_float4(C.ac, -(C.fcn * C.ac), -(((Sc * cosa) * rl) * cosa),
                                                       -(((Sc * sina) * rl) * sina));
                    B.pdg[2 * (size_t)e + 1] = make_float4(-(((Sc * sina) * rl) * cosa),
                                                           -(((Sc * cosa) * rl) * sina), 0.f, 0.f);
                }
                V.pdn[e] = (float)((Si.r + Sj.r) - dist);
                n_cand++;
                n_cont += C.contact;
                n_plast += C.who != 0;
            }
        } else if (diag) {
            V.pdn[e] = __int_as_float(0x7fc00000);
        }
        if (f1 != f0) {
            B.pfl[e] = (unsigned char)f1;
            B.lfl[B.lo_of[e]] = (unsigned char)(f1 & ~PF_HIST);
        }
    }
    if (diag) {
        warp_count(n_cand, V.counters, 0);
        warp_count(n_cont, V.counters, 1);
        warp_count(n_plast, V.counters, 3);
    }
}

// One lane per bond.  A broken bond is skipped (its record was zeroed when it
// broke); a live bond outside the candidate radius keeps its state and
// contributes nothing this step, as in the reference's neighbour loop.
GD_DEV void bond_diag_zero(float4 *bdg, int2 pos)
{
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    bdg[2 * (size_t)pos.x] = z; bdg[2 * (size_t)pos.x + 1] = z;
    bdg[2 * (size_t)pos.y] = z; bdg[2 * (size_t)pos.y + 1] = z;
}

// One bond of the working order, its records already loaded (q: slots of
// both floes and positions of their records; bd: the dynamic record; G: the
// FP32 geometry).  A broken bond writes only its flag; a live bond outside
// the candidate radius keeps its state and leaves zero records, as in the
// reference's neighbour loop.  Returns whether the bond is live after the
// step (for the diagnostic count).
// A live bond (bd.flag == 1) with both floes' snapshots at hand (Si: the
// lower id).
GD_DEV bool bond_live(const Views &V, const Snap &Si, const Snap &Sj, int diag, int b, const int4 q, BondDyn bd,
                      const BondGeom32 G, float4 *brec, float4 *bdg, unsigned char *bfl_wr, BondDyn *BD)
{
    const int2 pos = make_int2(q.z, q.w);
    const InstParams &Pm = V.P[Si.inst];
    const bool px = Pm.boundary & BC_PERIODIC_X, py = Pm.boundary & BC_PERIODIC_Y;
    const double dx = wrap_d(Si.x - Sj.x, Pm.nx, px), dy = wrap_d(Si.y - Sj.y, Pm.ny, py);
    const double d2 = dx * dx + dy * dy;
    // the candidate test of the reference in FP64; the exact root only near
    // its edge
    const double Rc = Si.r + Pm.rtree;
    const bool cand = d2 <= (Rc * Rc) * (1.0 - 1e-9) ? true
                    : (d2 > (Rc * Rc) * (1.0 + 1e-9) ? false : sqrt(d2) <= Rc);
    BondOut O;
    O.on = false;
    O.fx = O.fy = O.mi = O.mj = O.fbn = O.sb = O.S = 0.f;
    float rl = (float)Si.r;
    if (cand) {
        const float inv = rsqrtf((float)d2);
        const float cosa = (float)(-dx) * inv;
        const float sina = (float)(-dy) * inv;
        float ri_l = (float)Si.r, rj_l = (float)Sj.r;
        const float ev = __int_as_float(bd.pad);
        if (ev > 0.f) ri_l = ev;
        else if (ev < 0.f) rj_l = -ev;
        bd.pad = 0;
        rl = ri_l;
        bond_mixed(Pm, bond_coeffs(Pm, G), bd, cosa, sina, Si, Sj, ri_l, rj_l, O);
        BD[b] = bd;
        if (diag) {
            // the same diagnostic sums for both floes (stepper.f90:215-271)
            const float Sb = O.S;
            const float4 d0 = make_float4(O.sb, -(O.fbn * O.sb), -(((Sb * cosa) * rl) * cosa),
                                          -(((Sb * sina) * rl) * sina));
            const float4 d1 = make_float4(-(((Sb * sina) * rl) * cosa), -(((Sb * cosa) * rl) * sina), 0.f, 0.f);
            bdg[2 * (size_t)pos.x] = d0; bdg[2 * (size_t)pos.x + 1] = d1;
            bdg[2 * (size_t)pos.y] = d0; bdg[2 * (size_t)pos.y + 1] = d1;
        }
    } else if (diag) {
        bond_diag_zero(bdg, pos);
    }
    bfl_wr[b] = (unsigned char)(bd.flag == 1);
    // each floe's bond records are contiguous, in id order
    brec[pos.x] = make_float4(O.fx, O.fy, O.mi, 0.f);
    brec[pos.y] = make_float4(-O.fx, -O.fy, O.mj, 0.f);
    return O.on;
}

// A broken bond: its flag only (its records were zeroed when it broke).
GD_DEV void bond_broken(int diag, int b, const int4 q, float4 *bdg, unsigned char *bfl_wr)
{
    bfl_wr[b] = 0;
    if (diag) bond_diag_zero(bdg, make_int2(q.z, q.w));
}

GD_DEV bool bond_step(const Views &V, const Snap *S, int diag, int b, const int4 q, BondDyn bd, const BondGeom32 G,
                      float4 *brec, float4 *bdg, unsigned char *bfl_wr, BondDyn *BD)
{
    if (bd.flag != 1) {
        bond_broken(diag, b, q, bdg, bfl_wr);
        return false;
    }
    const Snap Si = S[q.x], Sj = S[q.y];   // q.x: the lower id
    return bond_live(V, Si, Sj, diag, b, q, bd, G, brec, bdg, bfl_wr, BD);
}

// Bonds in their working order (by the slot of the lower-id floe), so that
// the lower-id floe's snapshot and record are read and written in sequence.
// One lane per bond; the bond's own records are loaded together, ahead of
// the floes' snapshots that depend on them.
__global__ void __launch_bounds__(256) k_bonds_mixed(Views V, int cur, int diag, int NB, const int4 *bsp,
                                                     const BondGeom32 *bst, float4 *brec,
                                                     float4 *bdg, unsigned char *bfl_wr, BondDyn *BD)
{
    step_kernel_entry();
    if (*(volatile int *)V.status & ST_ABORT) return;
    const Snap *S = V.snap[cur];
    unsigned long long n_bond = 0;
    const int stride = gridDim.x * blockDim.x;
    const int nit = (NB + stride - 1) / stride;
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    for (int it = 0; it < nit; it++, b += stride) {
        if (b >= NB) continue;
        const int4 q = bsp[b];
        const BondDyn bd = BD[b];
        const BondGeom32 G = bst[b];
        const bool on = bond_step(V, S, diag, b, q, bd, G, brec, bdg, bfl_wr, BD);
        if (diag) n_bond += on;
    }
    if (diag) warp_count(n_bond, V.counters, 2);
}

// The same bonds with their records streamed into shared memory by the
// tensor-memory accelerator: a tile of BT bonds' slots, dynamic records and
// geometry (80 bytes a bond, contiguous in working order) is one bulk copy
// per array, two tiles in flight per block, completion on an mbarrier.  The
// only loads left on a lane's dependent chain are the two floes' snapshots.
// Every wait is bounded: a wait that gives up sets ST_TIMEOUT, waits (again
// bounded) for the block's copies still in flight and returns.
constexpr int BT = 128;
struct BondTile {
    int4 sp[BT];
    BondDyn dy[BT];
    BondGeom32 ge[BT];
};
constexpr unsigned MBAR_SPIN_LIMIT = 1u << 26;    // tries of a wait before it gives up

GD_DEV unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

GD_DEV void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait for the phase of the given parity to complete (at most
// `limit` tries).
GD_DEV bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned limit = MBAR_SPIN_LIMIT)
{
    const unsigned a = smem_u32(bar);
    for (unsigned k = 0; k < limit; k++) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Thread 0: the copies of tile t into stage buffer T, completing on bar.
GD_DEV void bond_tile_load(BondTile &T, unsigned long long *bar, int t, int NB, const int4 *bsp, const BondDyn *BD,
                           const BondGeom32 *bst)
{
    const int b0 = t * BT;
    const int nb = min(BT, NB - b0);
    const unsigned bytes = (unsigned)nb * (unsigned)(sizeof(int4) + sizeof(BondDyn) + sizeof(BondGeom32));
    const unsigned a = smem_u32(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(a), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(T.sp)), "l"(bsp + b0), "r"((unsigned)nb * (unsigned)sizeof(int4)), "r"(a)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(T.dy)), "l"(BD + b0), "r"((unsigned)nb * (unsigned)sizeof(BondDyn)), "r"(a)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(T.ge)), "l"(bst + b0), "r"((unsigned)nb * (unsigned)sizeof(BondGeom32)), "r"(a)
                 : "memory");
}

// test_spins > 0 (a test of the timeout path only): before any copy, every
// block waits at most test_spins tries on a barrier that nothing completes,
// and so takes the path of a wait that gives up.
__global__ void __launch_bounds__(BT, 8) k_bonds_tma(Views V, int cur, int diag, int NB, const int4 *bsp,
                                                  const BondGeom32 *bst, float4 *brec, float4 *bdg,
                                                  unsigned char *bfl_wr, BondDyn *BD, unsigned test_spins)
{
    __shared__ __align__(128) BondTile tile[2];
    __shared__ __align__(8) unsigned long long bar[3];
    step_kernel_entry();
    if (*(volatile int *)V.status & ST_ABORT) return;
    const int ntiles = (NB + BT - 1) / BT;
    const int stride = gridDim.x;
    if ((int)blockIdx.x >= ntiles) return;
    const int tid = threadIdx.x;
    const Snap *S = V.snap[cur];
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_init(&bar[2], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (test_spins > 0 && __syncthreads_or(!mbar_wait(&bar[2], 0u, test_spins))) {
        // nothing is in flight yet: report and leave
        if (tid == 0) atomicOr(V.status, ST_TIMEOUT);
        return;
    }
    if (tid == 0) {
        bond_tile_load(tile[0], &bar[0], blockIdx.x, NB, bsp, BD, bst);
        if ((int)blockIdx.x + stride < ntiles) bond_tile_load(tile[1], &bar[1], blockIdx.x + stride, NB, bsp, BD, bst);
    }
    unsigned long long n_bond = 0;
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += stride, it++) {
        const int st = it & 1;
        const bool ok = mbar_wait(&bar[st], (unsigned)(it >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            // give up: the step is reported as not completed; the copies
            // still in flight into this block's shared memory land first
            if (tid == 0) {
                atomicOr(V.status, ST_TIMEOUT);
                mbar_wait(&bar[st], (unsigned)(it >> 1) & 1u);
                if (t + stride < ntiles) mbar_wait(&bar[st ^ 1], (unsigned)((it + 1) >> 1) & 1u);
            }
            __syncthreads();
            return;
        }
        const int b = t * BT + tid;
        if (b < NB) {
            const bool on = bond_step(V, S, diag, b, tile[st].sp[tid], tile[st].dy[tid], tile[st].ge[tid], brec, bdg,
                                      bfl_wr, BD);
            if (diag) n_bond += on;
        }
        // every lane has read this stage: refill it with the tile after next
        __syncthreads();
        if (tid == 0 && t + 2 * stride < ntiles) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bond_tile_load(tile[st], &bar[st], t + 2 * stride, NB, bsp, BD, bst);
        }
    }
    if (diag) warp_count(n_bond, V.counters, 2);
}

// floe_properties (physics.f90:179-198) for the mixed floe update: the
// freeboard factors as products with precomputed density ratios
GD_DEV Shape shape_mixed(const InstParams &P, double r, double h)
{
    Shape s;
    s.r = r;
    s.h = h;
    s.mass = ((P.rhoice * P.pi) * h) * (r * r);
    s.inertia = (0.5 * s.mass) * (r * r);
    s.hfa = h * P.hfa_fac;
    s.hfw = h * P.hfw_fac;
    return s;
}

GD_DEV Snap pack_snap(double x, double y, const Shape &sh, double u, double v, double om, int inst)
{
    Snap s;
    s.x = x; s.y = y; s.r = sh.r;
    s.inst = inst;
    s.h = (float)sh.h; s.u = (float)u; s.v = (float)v; s.om = (float)om;
    s.mass = (float)sh.mass;
    return s;
}

GD_DEV void add4(float4 &a, const float4 &b)
{
    a.x += b.x; a.y += b.y; a.z += b.z; a.w += b.w;
}

// The bits `bits` (repeated in every byte) of the flag bytes [e0, e1) of
// one 8-byte word.
GD_DEV unsigned long long flag_word(const unsigned char *fl, int w, int e0, int e1, unsigned long long bits)
{
    const unsigned long long word = reinterpret_cast<const unsigned long long *>(fl)[w];
    const int lo = max(e0 - (w << 3), 0), hi = min(e1 - (w << 3), 8);
    const unsigned long long mhi = hi >= 8 ? ~0ULL : ((1ULL << (8 * hi)) - 1ULL);
    const unsigned long long mlo = (1ULL << (8 * lo)) - 1ULL;
    return word & (mhi & ~mlo) & bits;
}

// Per floe: the sums of its flagged pair records (own row, partner row) and
// of its bond records, in that order, FP32.  Few registers, so that many
// floes' dependent loads are in flight at once.
template <bool DIAG>
__global__ void __launch_bounds__(256, 8) k_floe_sums(Views V, MixedBufs B)
{
    step_kernel_entry();
    constexpr bool diag = DIAG;
    // the work list of the next step starts empty (the pair kernels of this
    // step have completed)
    if (blockIdx.x == 0 && threadIdx.x == 0) *B.nwork = 0;
    if (*(volatile int *)V.status & ST_ABORT) return;
    const int stride = gridDim.x * blockDim.x;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < V.N; g += stride) {
        const bool shel = V.P[V.inst[g]].shelter != 0;
        // contact and bond sums (FP32) in the order: own row, partner row,
        // own bonds, partner bonds
        float fcx = 0.f, fcy = 0.f, mc = 0.f, fbx = 0.f, fby = 0.f, mb = 0.f;
        float sca = 1.f, scw = 1.f, rex = 0.f;
        float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f), q1 = make_float4(0.f, 0.f, 0.f, 0.f);   // tac pc sxx syy | sxy syx
        float tab = 0.f, pbs = 0.f;
        // flag bytes are read eight at a time; most pairs leave no record
        const unsigned long long want = diag ? 0x0e0e0e0e0e0e0e0eULL : 0x0a0a0a0a0a0a0a0aULL;
        const int e0 = V.up_off[g], e1 = V.up_off[g + 1];
        const int l0 = V.lo_off[g], l1 = V.lo_off[g + 1];
        for (int w = e0 >> 3; e1 > e0 && w <= (e1 - 1) >> 3; w++) {
            unsigned long long bits = flag_word(B.pfl, w, e0, e1, want);
            while (bits) {
                const int byte = (__ffsll((long long)bits) - 1) >> 3;
                const unsigned f = (unsigned)(bits >> (8 * byte)) & 0xffu;
                bits &= ~(0xffULL << (8 * byte));
                const int e = (w << 3) + byte;
                if (f & PF_REC) {
                    const float4 r0 = B.rec[2 * (size_t)e];
                    fcx += r0.x; fcy += r0.y; mc += r0.z;
                    if (shel) {
                        const float4 r1 = B.rec[2 * (size_t)e + 1];
                        sca = fminf(sca, r1.x); scw = fminf(scw, r1.y);
                    }
                    if (f & PF_REX) { const float o = B.rx[e].x; rex = (rex + o) + rex * o; }
                }
                if (f & PF_DG) { add4(q0, B.pdg[2 * (size_t)e]); add4(q1, B.pdg[2 * (size_t)e + 1]); }
            }
        }
        for (int w = l0 >> 3; l1 > l0 && w <= (l1 - 1) >> 3; w++) {
            unsigned long long bits = flag_word(B.lfl, w, l0, l1, want);
            while (bits) {
                const int byte = (__ffsll((long long)bits) - 1) >> 3;
                const unsigned f = (unsigned)(bits >> (8 * byte)) & 0xffu;
                bits &= ~(0xffULL << (8 * byte));
                const int p = V.ent_lo[(w << 3) + byte].y;
                if (f & PF_REC) {
                    const float4 r0 = B.rec[2 * (size_t)p];
                    fcx -= r0.x; fcy -= r0.y; mc += r0.w;
                    if (shel) {
                        const float4 r1 = B.rec[2 * (size_t)p + 1];
                        sca = fminf(sca, r1.z); scw = fminf(scw, r1.w);
                    }
                    if (f & PF_REX) { const float o = B.rx[p].y; rex = (rex + o) + rex * o; }
                }
                if (f & PF_DG) { add4(q0, B.pdg[2 * (size_t)p]); add4(q1, B.pdg[2 * (size_t)p + 1]); }
            }
        }
        for (int k = B.bfo[g]; k < B.bfo[g + 1]; k++) {
            const float4 rb = B.brec[k];
            fbx += rb.x; fby += rb.y; mb += rb.z;
            if (diag) {
                const float4 d0 = B.bdg[2 * (size_t)k], d1 = B.bdg[2 * (size_t)k + 1];
                tab += d0.x; pbs += d0.y; q0.z += d0.z; q0.w += d0.w; q1.x += d1.x; q1.y += d1.y;
            }
        }
        B.fsum[2 * (size_t)g] = make_float4(fcx, fcy, mc, fbx);
        B.fsum[2 * (size_t)g + 1] = make_float4(fby, mb, sca, scw);
        B.frex[g] = rex;
        if (diag) {
            B.fdg[2 * (size_t)g] = make_float4(q0.x, q0.y, tab, pbs);
            B.fdg[2 * (size_t)g + 1] = make_float4(q0.z, q0.w, q1.x, q1.y);
        }
    }
}

// Per floe: walls, ridging, drag, Coriolis and the FP64 update from the
// sums; every load is the floe's own, so they are all in flight together.
// Fields without walls (periodic or open on every side) neither read nor
// write the wall histories (they stay zero on both sides).  A batch without
// any wall runs the WALLS = false instance, which needs far fewer registers.
template <bool DIAG, bool WALLS>
__global__ void __launch_bounds__(256, WALLS ? 2 : 4) k_floes_mixed(Views V, int cur, int sic, MixedBufs B)
{
    step_kernel_entry();
    if (floe_update_stopped(V, sic)) return;
    const int nxt = cur ^ 1;
    const int stride = gridDim.x * blockDim.x;
    unsigned dmx = 0;      // largest squared step of this thread's floes (FP32 bits)
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < V.N; g += stride) {
        const int ig = V.inst[g];
        const InstParams &P = V.P[ig];
        const bool px = P.boundary & BC_PERIODIC_X, py = P.boundary & BC_PERIODIC_Y;
        const bool shel = P.shelter != 0;
        const bool walls = WALLS && has_walls(P.boundary);
        const float4 s0 = B.fsum[2 * (size_t)g], s1 = B.fsum[2 * (size_t)g + 1];
        const float rex = B.frex[g];
        const float fcx = s0.x, fcy = s0.y, mc = s0.z, fbx = s0.w, fby = s1.x, mb = s1.y;
        const float sca = s1.z, scw = s1.w;
        const double x = V.x[cur][g], y = V.y[cur][g], th = V.th[cur][g];
        const double u = V.u[cur][g], v = V.v[cur][g], om = V.om[cur][g];
        const double r = V.r[cur][g], h = V.h[cur][g];
        double dtb1 = 0.0, dtb2 = 0.0, thb1 = 0.0, thb2 = 0.0;
        if (walls) {
            dtb1 = V.dtb1[cur][g]; dtb2 = V.dtb2[cur][g];
            thb1 = V.thb1[cur][g]; thb2 = V.thb2[cur][g];
        }
        // ridging of this floe's pairs (volume pi r^2 h kept)
        Shape run = shape_mixed(P, r, h);
        if (rex != 0.f) {
            const double h1 = h + h * (double)rex;
            run = shape_mixed(P, r * sqrt(h / h1), h1);
        }
        WallOut W;
        int wev = 0;
        if (walls) {
            verify_bc(P, x, y, u, v, om, run, dtb1, dtb2, thb1, thb2, W, wev);
        } else {
            W.fx_bc = W.fy_bc = W.m_bc = 0.0;
            W.sxx = W.syy = W.sxy = W.syx = 0.0;
            W.ta_bc = W.p_bc = 0.0;
        }
        double ua, va, uw, vw;
        wind_at(P, V.field, x, y, ua, va, uw, vw);
        const Drag<float> D = forcing<float>(P, run, u, v, om, ua, va, uw, vw, shel ? sca : 0.f, shel ? scw : 0.f);
        const double fax = D.fax, fay = D.fay, fwx = D.fwx, fwy = D.fwy;
        const double tfx = (((((double)fcx + (double)fbx) + fax) + fwx) + (double)D.fcorx) + W.fx_bc;
        const double tfy = (((((double)fcy + (double)fby) + fay) + fwy) + (double)D.fcory) + W.fy_bc;
        const double mt = ((((double)mc + (double)mb) + (double)D.ma) + (double)D.mw) + W.m_bc;
        const double dt = P.dt;
        // FP64 update, the divisions by mass and inertia as two reciprocals
        const double inv_m = 1.0 / run.mass, inv_i = 1.0 / run.inertia;
        const double u1 = u + (tfx * inv_m) * dt;
        const double v1 = v + (tfy * inv_m) * dt;
        const double om1 = om + (mt * inv_i) * dt;
        double x1 = x + u1 * dt;
        double y1 = y + v1 * dt;
        const double th1 = th + om1 * dt;
        if (px) { if (x1 < 0.0) x1 = x1 + P.nx; else if (x1 >= P.nx) x1 = x1 - P.nx; }
        if (py) { if (y1 < 0.0) y1 = y1 + P.ny; else if (y1 >= P.ny) y1 = y1 - P.ny; }
        V.x[nxt][g] = x1; V.y[nxt][g] = y1; V.th[nxt][g] = th1;
        V.u[nxt][g] = u1; V.v[nxt][g] = v1; V.om[nxt][g] = om1;
        V.r[nxt][g] = run.r; V.h[nxt][g] = run.h;
        if (walls) {
            V.dtb1[nxt][g] = dtb1; V.dtb2[nxt][g] = dtb2;
            V.thb1[nxt][g] = thb1; V.thb2[nxt][g] = thb2;
        }
        V.snap[nxt][g] = pack_snap(x1, y1, run, u1, v1, om1, ig);
        const double ddx = wrap_d(x1 - V.x0[cur][g], P.nx, px), ddy = wrap_d(y1 - V.y0[cur][g], P.ny, py);
        const double half = 0.5 * P.skin;
        if (ddx * ddx + ddy * ddy > half * half) {
            atomicOr(V.status, ST_EXPIRED);
            atomicMin(V.expired_at, global_step(V, sic));
        }
        const double sdx = wrap_d(x1 - x, P.nx, px), sdy = wrap_d(y1 - y, P.ny, py);
        dmx = max(dmx, __float_as_uint(__double2float_ru(sdx * sdx + sdy * sdy)));
        if (!(isfinite(x1) && isfinite(y1) && isfinite(u1) && isfinite(v1) && isfinite(om1) && isfinite(th1)))
            atomicOr(V.status, ST_NAN);
        if (DIAG) {
            const float4 d0 = B.fdg[2 * (size_t)g], d1 = B.fdg[2 * (size_t)g + 1];   // tac pc tab pb | sxx syy sxy syx
            const size_t N = (size_t)V.N;
            const double rr = run.r;
            const double tac = d0.x;
            const double pa = tac != 0.0 ? (double)d0.y / tac : 0.0;
            const double pbv = d0.z != 0.f ? (double)d0.w / (double)d0.z : 0.0;
            const double pw = W.ta_bc != 0.0 ? W.p_bc / W.ta_bc : 0.0;
            double *D0 = V.diag;
            D0[0 * N + g] = tfx; D0[1 * N + g] = tfy; D0[2 * N + g] = fcx; D0[3 * N + g] = fcy;
            D0[4 * N + g] = fbx; D0[5 * N + g] = fby; D0[6 * N + g] = mt; D0[7 * N + g] = mc;
            D0[8 * N + g] = mb;
            D0[9 * N + g] = ((double)d1.x + W.sxx) + (fax + fwx) * rr;
            D0[10 * N + g] = ((double)d1.y + W.syy) + (fay + fwy) * rr;
            D0[11 * N + g] = ((double)d1.z + W.sxy) + 0.0;
            D0[12 * N + g] = ((double)d1.w + W.syx) + 0.0;
            D0[13 * N + g] = (pa + pbv) + pw;
        }
    }
    // the largest step, which the next step's screening adds to its bound:
    // one atomic per warp, and only where it raises the maximum
    const unsigned am = __activemask();
    const unsigned wm = __reduce_max_sync(am, dmx);
    if ((int)(threadIdx.x & 31) == __ffs(am) - 1 && wm > __ldcg(B.dsp + cur)) atomicMax(B.dsp + cur, wm);
}

// Row (slot) of every entry of a CSR.
__global__ void k_fill_erow(const int *off, int N, unsigned *erow)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < N; s += gridDim.x * blockDim.x)
        for (int e = off[s]; e < off[s + 1]; e++) erow[e] = (unsigned)s;
}

__global__ void k_pack_snap(Views V, int side)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < V.N; g += gridDim.x * blockDim.x)
        V.snap[side][g] = pack_snap(V.x[side][g], V.y[side][g], make_shape(V.P[V.inst[g]], V.r[side][g], V.h[side][g]),
                                    V.u[side][g], V.v[side][g], V.om[side][g], V.inst[g]);
}

void launch_fill_erow(const int *off, int N, unsigned *erow, cudaStream_t st)
{
    const int grid = N > 0 ? std::min((N + 255) / 256, 148 * 16) : 1;
    k_fill_erow<<<grid, 256, 0, st>>>(off, N, erow);
}

void launch_pack_snap(const Views &V, int side, cudaStream_t st)
{
    const int grid = V.N > 0 ? std::min((V.N + 255) / 256, 148 * 16) : 1;
    k_pack_snap<<<grid, 256, 0, st>>>(V, side);
}


// Per rebuild: the partner index of every owner entry, the pair flags from
// the migrated histories, no records.
__global__ void k_mixed_rows_init(int P, const int2 *ent_lo, const Hist4<float> *hist, int *lo_of,
                                  unsigned char *pfl, unsigned char *lfl)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P; k += gridDim.x * blockDim.x) {
        const int p = ent_lo[k].y;
        if (p >= 0 && p < P) lo_of[p] = k;
        lfl[k] = 0;
        const Hist4<float> H = hist[k];
        pfl[k] = (H.deltat != 0.f || H.thetarelc != 0.f) ? PF_HIST : 0;
    }
}

// Slot of every floe by global id (instance offset + reference id), then the
// slots of both floes of every bond.
__global__ void k_slot_of(Views V, int side, int *slot_of)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x)
        slot_of[V.P[V.inst[s]].off + V.id[side][s]] = s;
}

__global__ void k_bond_slots(Views V, int side, const int *slot_of, int4 *bsp, uint32_t *pkey, int *pval)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const int off = V.P[V.inst[s]].off;
        const int gl = off + V.id[side][s];
        for (int b = V.bond_off[gl]; b < V.bond_off[gl + 1]; b++) {
            const int gj = off + V.bond_hi[b];
            reinterpret_cast<int2 *>(&bsp[b])[0] = make_int2(s, slot_of[gj]);
            if (pkey) { pkey[b] = (uint32_t)gj; pval[b] = b; }
        }
    }
}

// Per slot: the number of bond records (bonds where the floe is the lower
// id, then those where it is the higher id); after the scan bfo, the record
// positions of every bond.
__global__ void k_bond_counts(Views V, int side, const int *blo_start, const int *blo_end, int *cnt)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const int gl = V.P[V.inst[s]].off + V.id[side][s];
        cnt[s] = (V.bond_off[gl + 1] - V.bond_off[gl]) + (blo_end[gl] - blo_start[gl]);
    }
}

__global__ void k_bond_pos(Views V, int side, const int *blo_start, const int *blo_end, const int *blo_idx,
                           const int *bfo, int4 *bsp)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const int gl = V.P[V.inst[s]].off + V.id[side][s];
        const int b0 = V.bond_off[gl], b1 = V.bond_off[gl + 1];
        const int base = bfo[s];
        for (int b = b0; b < b1; b++) bsp[b].z = base + (b - b0);
        const int k0 = blo_start[gl], k1 = blo_end[gl];
        for (int k = k0; k < k1; k++) bsp[blo_idx[k]].w = base + (b1 - b0) + (k - k0);
    }
}

// Per rebuild: the bonds' working order, by the slot of the lower-id floe
// (wfo: first working index of every slot), and per working index the
// dynamic record, the FP32 copy of the static record, slots and record
// positions, both sides of the live-bond flag, and the inverse map.
__global__ void k_bond_own_counts(Views V, int side, int *cnt)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const int gl = V.P[V.inst[s]].off + V.id[side][s];
        cnt[s] = V.bond_off[gl + 1] - V.bond_off[gl];
    }
}

__global__ void k_bond_perm(Views V, int side, const int *wfo, int *perm)
{
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V.N; s += gridDim.x * blockDim.x) {
        const int gl = V.P[V.inst[s]].off + V.id[side][s];
        const int b0 = V.bond_off[gl], b1 = V.bond_off[gl + 1], base = wfo[s];
        for (int b = b0; b < b1; b++) perm[base + (b - b0)] = b;
    }
}

__global__ void k_bond_work_gather(Views V, const int *perm, int nb, const BondStat *in, const BondDyn *dyn,
                                   const int4 *bsp, BondGeom32 *wst, BondDyn *wdyn, int4 *wsp, int *winv,
                                   unsigned char *wflag)
{
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nb; w += gridDim.x * blockDim.x) {
        const int b = perm[w];
        winv[b] = w;
        const BondDyn d = dyn[b];
        wdyn[w] = d;
        wsp[w] = bsp[b];
        wflag[w] = wflag[nb + w] = (unsigned char)(d.flag == 1);
        const BondStat s = in[b];
        BondGeom32 o;
        o.rb = (float)s.rb; o.hb = (float)s.hb; o.lb = (float)s.lb;
        o.inv_l = (float)(1.0 / s.lb);
        wst[w] = o;
    }
}

// Writes the working dynamic records back to the bond table (before a
// rebuild, a relayout or a read of the bond table).
__global__ void k_bond_work_scatter(const int *perm, int nb, const BondDyn *wdyn, BondDyn *dyn)
{
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nb; w += gridDim.x * blockDim.x)
        dyn[perm[w]] = wdyn[w];
}

// Per rebuild: the owner entries that can take part in a contact before the
// next rebuild - distance at the rebuild within min(r_i + r_j, r_i + rtree)
// plus the skin (each floe then moves at most half the skin) - together
// with every entry that carries a contact history and every entry of a
// sheltering field (whose candidates all leave records).
__global__ void k_contact_mark(Views V, int side, int P, const unsigned *erow, const unsigned char *pfl, int *mark)
{
    const Snap *S = V.snap[side];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < P; e += gridDim.x * blockDim.x) {
        const int s = (int)erow[e];
        const int t = V.ent_up[e].x;
        const Snap Si = S[s], Sj = S[t];
        const InstParams &Pm = V.P[Si.inst];
        int m = 1;
        if (!Pm.shelter && !(pfl[e] & PF_HIST)) {
            const bool px = Pm.boundary & BC_PERIODIC_X, py = Pm.boundary & BC_PERIODIC_Y;
            const double dx = wrap_d(Si.x - Sj.x, Pm.nx, px), dy = wrap_d(Si.y - Sj.y, Pm.ny, py);
            const double R = fmin(Si.r + Sj.r, Si.r + Pm.rtree) + Pm.skin;
            m = dx * dx + dy * dy <= (R * R) * (1.0 + 1e-9) ? 1 : 0;
        }
        mark[e] = m;
    }
}

// The list item: the entry, the two slots and the pair's gap at the rebuild
// (the bound of k_pairs_screen with D = 0).  A pair that carries a contact
// history gets a bound of at most -1, so that the screen always tests it
// (the screen reads a pair's flags only for the items it tests).
// side: the rows' side, whose positions are the floes' rebuild origins.
__global__ void k_contact_fill(Views V, int side, int P, const unsigned *erow, const unsigned char *pfl,
                               const int *mark, const int *pos, int2 *eb, int2 *stl)
{
    const Snap *S = V.snap[side];
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < P; e += gridDim.x * blockDim.x) {
        if (!mark[e]) continue;
        const int s = (int)erow[e];
        const int t = V.ent_up[e].x;
        const Snap Si = S[s], Sj = S[t];
        const InstParams &Pm = V.P[Si.inst];
        float gap = -INFINITY;
        if (!Pm.shelter && !Pm.ridging) {
            const bool px = Pm.boundary & BC_PERIODIC_X, py = Pm.boundary & BC_PERIODIC_Y;
            const double dx = wrap_d(Si.x - Sj.x, Pm.nx, px), dy = wrap_d(Si.y - Sj.y, Pm.ny, py);
            const double g = sqrt(dx * dx + dy * dy) - (Si.r + Sj.r) * (1.0 + 1e-9);
            gap = __double2float_rd(g);
        }
        if (pfl[e] & PF_HIST) gap = fminf(gap, -1.f);
        eb[pos[e]] = make_int2(e, __float_as_int(gap));
        stl[pos[e]] = make_int2(s, t);
    }
}

// Enough blocks for two full waves at any block size (148 SMs x 2048
// threads), so that small blocks do not cap the resident warps; the kernels
// stride over the rest.
static int grid_of(long long n, int block)
{
    return (int)std::max(1LL, std::min<long long>((n + block - 1) / block, 148LL * (4096 / block)));
}

void launch_mixed_rows_init(int P, const int2 *ent_lo, const void *hist, int *lo_of, unsigned char *pfl,
                            unsigned char *lfl, cudaStream_t st)
{
    if (P > 0)
        k_mixed_rows_init<<<grid_of(P, 256), 256, 0, st>>>(P, ent_lo, (const Hist4<float> *)hist, lo_of, pfl, lfl);
}

void launch_bond_slots(const Views &V, int side, int *slot_of, int4 *bsp, uint32_t *pkey, int *pval,
                       cudaStream_t st)
{
    k_slot_of<<<grid_of(V.N, 256), 256, 0, st>>>(V, side, slot_of);
    k_bond_slots<<<grid_of(V.N, 128), 128, 0, st>>>(V, side, slot_of, bsp, pkey, pval);
}

void launch_contact_list(const Views &V, int side, int P, const unsigned *erow, const unsigned char *pfl, int *mark,
                         int *pos, int *scan_scratch, int2 *eb, int2 *stl, cudaStream_t st)
{
    if (P <= 0) return;
    k_contact_mark<<<grid_of(P, 256), 256, 0, st>>>(V, side, P, erow, pfl, mark);
    scan_excl(mark, pos, P, scan_scratch, st);
    k_contact_fill<<<grid_of(P, 256), 256, 0, st>>>(V, side, P, erow, pfl, mark, pos, eb, stl);
}

void launch_bond_work(const Views &V, int side, int nb, int *cnt, int *wfo, int *scan_scratch, int *perm,
                      const BondStat *in, const BondDyn *dyn, const int4 *bsp, BondGeom32 *wst, BondDyn *wdyn,
                      int4 *wsp, int *winv, unsigned char *wflag, cudaStream_t st)
{
    if (nb <= 0) return;
    k_bond_own_counts<<<grid_of(V.N, 256), 256, 0, st>>>(V, side, cnt);
    scan_excl(cnt, wfo, V.N, scan_scratch, st);
    k_bond_perm<<<grid_of(V.N, 128), 128, 0, st>>>(V, side, wfo, perm);
    k_bond_work_gather<<<grid_of(nb, 256), 256, 0, st>>>(V, perm, nb, in, dyn, bsp, wst, wdyn, wsp, winv, wflag);
}

void launch_bond_work_scatter(const int *perm, int nb, const BondDyn *wdyn, BondDyn *dyn, cudaStream_t st)
{
    if (nb > 0) k_bond_work_scatter<<<grid_of(nb, 256), 256, 0, st>>>(perm, nb, wdyn, dyn);
}

void launch_bond_positions(const Views &V, int side, const int *blo_start, const int *blo_end, const int *blo_idx,
                           int *cnt, int *bfo, int *scan_scratch, int4 *bsp, cudaStream_t st)
{
    k_bond_counts<<<grid_of(V.N, 256), 256, 0, st>>>(V, side, blo_start, blo_end, cnt);
    scan_excl(cnt, bfo, V.N, scan_scratch, st);
    k_bond_pos<<<grid_of(V.N, 128), 128, 0, st>>>(V, side, blo_start, blo_end, blo_idx, bfo, bsp);
}

void launch_pairs_screen(const Views &V, int cur, int diag, int P, int2 *eb, const int2 *stl,
                         MixedBufs B, int block, int variant, cudaStream_t st)
{
    if (P <= 0) return;
    // a diagnostic step only advances the displacement bound here
    const int grid = diag ? 1 : grid_of(P, block);
    if (variant == 1) launch_step(V.pdl != 0, k_pairs_screen<4>, grid, block, st, V, cur, diag, P, eb, stl, B);
    else if (variant == 2) launch_step(V.pdl != 0, k_pairs_screen<16>, grid, block, st, V, cur, diag, P, eb, stl, B);
    else launch_step(V.pdl != 0, k_pairs_screen<8>, grid, block, st, V, cur, diag, P, eb, stl, B);
}

bool step_pdl()
{
    static const bool on = [] {
        const char *e = getenv("GODAR_PDL");
        return !e || atoi(e) != 0;
    }();
    return on;
}

void launch_pairs_work(const Views &V, int cur, int diag, int P, const unsigned *erow_up, MixedBufs B, int block,
                       cudaStream_t st)
{
    // the list length is only known on the device: a grid of a few CTAs per
    // SM strides over it
    if (P > 0) launch_step(V.pdl != 0, k_pairs_mixed, 148 * (1024 / block), block, st, V, cur, diag, P, erow_up, B);
}

void launch_bonds_mixed(const Views &V, int cur, int diag, int NB, MixedBufs B, int block, int variant,
                        unsigned test_spins, cudaStream_t st)
{
    if (NB <= 0) return;
    if (variant == 1) {
        // a persistent grid: up to eight blocks per SM, each streaming its tiles
        const int ntiles = (NB + BT - 1) / BT;
        const int grid = std::max(1, std::min(ntiles, 148 * 8));
        launch_step(V.pdl != 0, k_bonds_tma, grid, BT, st, V, cur, diag, NB, B.bsp, B.bst, B.brec, B.bdg, B.bfl_wr, B.wdyn,
                                         test_spins);
        return;
    }
    launch_step(V.pdl != 0, k_bonds_mixed, grid_of(NB, block), block, st, V, cur, diag, NB, B.bsp, B.bst, B.brec,
                                                        B.bdg, B.bfl_wr, B.wdyn);
}

void launch_floe_sums(const Views &V, int diag, MixedBufs B, int block, cudaStream_t st)
{
    if (diag) launch_step(V.pdl != 0, k_floe_sums<true>, grid_of(V.N, block), block, st, V, B);
    else launch_step(V.pdl != 0, k_floe_sums<false>, grid_of(V.N, block), block, st, V, B);
}

void launch_floes_mixed(const Views &V, int cur, int diag, int sic, int walls, MixedBufs B, int block,
                        cudaStream_t st)
{
    if (!walls) {
        if (diag) launch_step(V.pdl != 0, k_floes_mixed<true, false>, grid_of(V.N, block), block, st, V, cur, sic, B);
        else launch_step(V.pdl != 0, k_floes_mixed<false, false>, grid_of(V.N, block), block, st, V, cur, sic, B);
        return;
    }
    if (diag) launch_step(V.pdl != 0, k_floes_mixed<true, true>, grid_of(V.N, block), block, st, V, cur, sic, B);
    else launch_step(V.pdl != 0, k_floes_mixed<false, true>, grid_of(V.N, block), block, st, V, cur, sic, B);
}

}  // namespace godar
