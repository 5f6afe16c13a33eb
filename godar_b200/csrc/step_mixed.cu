// The mixed-precision time step as three kernels.
//
// (b) k_pairs_own: one lane per pair (the owner rows, i.e. the lower-id
//     floe's entries), so every pair (stepper.f90:89-271) is evaluated once
//     whatever the row lengths.  The lane updates the pair's contact history
//     and bond state in place (only it touches them), adds the owner's share
//     to a warp-shuffle segmented scan keyed by the owner row (aligned windows
//     of 32 entries; the last lane of each row segment writes the window's
//     partial at its own index), and leaves the partner's share in a 32-byte
//     record with a flag (no record for pairs with no contact, bond or
//     shelter).  No atomics.
// (b') k_pairs_gather: one lane per partner-row entry; reads the records of
//     its pairs and scans them the same way.
// (c)-(e) k_floes: one thread per floe; adds the partials of the windows its
//     two rows span, then walls, ridging, drag, Coriolis and the FP64 update.
// Pair forces, sheltering and drag are FP32; geometry that cancels, bond
// strain/damage, ridging bookkeeping and integration are FP64.
#include <algorithm>

#include "step_kernel.cuh"
#include "kernels.h"

namespace godar {

struct BondM {
    int flag;
    double dmg, dnb, dtb, thji, thij;
};

// stepper.f90:89-271 for one candidate pair in the mixed precision: FP32
// forces from FP32 velocities, masses and precomputed beam coefficients; the
// overlap, chord length, ridged volume, bond strain and damage in FP64.
GD_DEV PairRes<float> pair_mixed(const InstParams &P, const BondStat *BS, double dx, double dy, double dist,
                                 const Snap &I, const Snap &J, float uai, float vai, float uwi, float vwi,
                                 Hist4<float> &H, BondM *B, bool want_shelter, bool diag)
{
    PairRes<float> R;
    const float dt = P.f_dt;
    const float fd = (float)dist;
    const float cosa = (float)(-dx) / fd;
    const float sina = (float)(-dy) / fd;
    const float omegarel = J.om - I.om;
    const float du = J.u - I.u, dv = J.v - I.v;
    const float veln = du * cosa + dv * sina;
    const float veltb = -(du * sina) + dv * cosa;
    float ri = (float)I.r, rj = (float)J.r;
    const float velt = veltb - (I.om * ri + J.om * rj);
    const double deltan = (I.r + J.r) - dist;
    const float dn = (float)deltan;
    R.cosa = cosa; R.sina = sina; R.deltan = deltan;
    R.who = 0; R.vol = 0.0;
    float hi_l = I.h, hj_l = J.h;
    R.contact = deltan > 0.0;
    if (R.contact) {
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
            if (hm2 == si.h) { R.who = 1; apply_dh(P, si, Vol); }
            else if (hm2 == sj.h) { R.who = 2; apply_dh(P, sj, Vol); }
            R.vol = Vol;
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
        if (!(B && B->flag == 1)) {
            float mrolling = krc * H.thetarelc - gamr * omegarel;
            if (fabsf(H.thetarelc) > ((2.f * fabsf(fcn)) / knc) / dr) mrolling = 0.f;
            mcc = mrolling;
        }
        H.fcn = fcn;
        H.fct = fct;
        R.fcn = fcn; R.fct = fct; R.fcr = fcr; R.mcc = mcc;
        R.ac = dr * fminf(hi_l, hj_l);
    } else {
        H.thetarelc = 0.f;
        H.deltat = 0.f;
        R.fcn = R.fct = R.fcr = R.mcc = R.ac = 0.f;
    }
    R.ri_l = ri;
    R.rj_l = rj;
    R.bond_on = false;
    R.fbn = R.fbt = R.mji = R.mij = R.sbt = 0.f;
    float sfbn = 0.f, sfbt = 0.f;
    if (B) {
        if (B->flag == 1) {
            // bond_forces_euler (bonds.f90:74-161): strain in FP64, beam
            // coefficients = (1 - D) x undamaged ones
            B->dnb = (double)veln * P.dt + B->dnb;
            B->dtb = (double)veltb * P.dt + B->dtb;
            B->thji = (double)I.om * P.dt + B->thji;
            B->thij = (double)J.om * P.dt + B->thij;
            const float omd = (float)(1.0 - B->dmg);
            const float m_redu = (I.mass * J.mass) / (I.mass + J.mass);
            const float i_redu = (I.inertia * J.inertia) / (I.inertia + J.inertia);
            const float k_axial = omd * BS->k_ax, k_shear1 = omd * BS->k_sh1, k_shear2 = omd * BS->k_sh2;
            const float k_rot1 = omd * BS->k_r1, k_rot2 = omd * BS->k_r2;
            const float il = BS->inv_l;
            const float eta_i = 2.f * sqrtf(omd * BS->ei_l) * sqrtf(i_redu);
            const float eta_a = 2.f * sqrtf(omd * BS->ea_l) * sqrtf(m_redu);
            const float gam_axial = eta_a * il;
            const float gam_shear1 = ((12.f * eta_i) * il) * (il * il);
            const float gam_shear2 = ((6.f * eta_i) * il) * il;
            const float gam_rot1 = (4.f * eta_i) * il, gam_rot2 = (2.f * eta_i) * il;
            const float dnb = (float)B->dnb, dtb = (float)B->dtb, thji = (float)B->thji, thij = (float)B->thij;
            float fbn = k_axial * dnb + gam_axial * veln;
            float fbt = ((k_shear1 * dtb + k_shear2 * (thji + thij)) + gam_shear1 * veltb) + gam_shear2 * (I.om + J.om);
            float mji = ((((k_rot1 * thji + k_rot2 * thij) - k_shear2 * dtb) + gam_rot1 * I.om) + gam_rot2 * J.om)
                        - gam_shear2 * veltb;
            float mij = ((((k_rot2 * thji + k_rot1 * thij) - k_shear2 * dtb) + gam_rot2 * I.om) + gam_rot1 * J.om)
                        - gam_shear2 * veltb;
            // bond_breaking (bonds.f90:164-212)
            const float sb = (float)BS->sb, rb = (float)BS->rb, ib = (float)BS->ib, hb = (float)BS->hb;
            const float taub = fabsf(fbt) / sb;
            const float bend = (fabsf(mji) * rb) / ib;
            const float sigmatb = -(fbn / sb) + bend;
            const float sigmacb = fbn / sb + bend;
            const float t1 = taub / (P.f_tau * hb);
            float phi = t1 * t1;
            if (sigmacb > 0.f) { const float t2 = sigmacb / (P.f_sigcb * hb); phi = phi + t2 * t2; }
            if (sigmatb > 0.f) { const float t3 = sigmatb / (P.f_sigtb * hb); phi = phi + t3 * t3; }
            const float psi = fminf(1.f, rsqrtf(phi));
            double D = B->dmg;
            D = (D + (((1.0 - (double)psi) * (1.0 - D)) * P.dt) / P.dtd) - (D * P.dt) / P.dth;
            B->dmg = D;
            if (D >= P.dmax) {
                B->flag = 0;
                fbn = 0.f; fbt = 0.f; mji = 0.f;
                B->dmg = 1.0;
            }
            sfbn = fbn; sfbt = fbt;
            if (B->flag == 1) {
                R.bond_on = true;
                R.fbn = fbn; R.fbt = fbt; R.mji = mji; R.mij = mij; R.sbt = sb;
            }
        } else {
            B->thji = 0.0; B->thij = 0.0; B->dnb = 0.0; B->dtb = 0.0;
        }
    }
    if (want_shelter) {
        const float hfai = P.f_hfa * hi_l, hfaj = P.f_hfa * hj_l, hfwi = P.f_hfw * hi_l, hfwj = P.f_hfw * hj_l;
        R.a_ij = S_shelter<float>(hfai, hfaj, dn, cosa, sina, uai, vai);
        R.w_ij = S_shelter<float>(hfwi, hfwj, dn, cosa, sina, uwi, vwi);
        R.a_ji = S_shelter<float>(hfaj, hfai, dn, -cosa, -sina, uai, vai);
        R.w_ji = S_shelter<float>(hfwj, hfwi, dn, -cosa, -sina, uwi, vwi);
    }
    R.S = diag ? sqrtf(H.fcn * H.fcn + H.fct * H.fct) + sqrtf(sfbn * sfbn + sfbt * sfbt) : 0.f;
    return R;
}

// Warp-shuffle segmented inclusive scans over a 32-entry window, keyed by the
// row: sums of the force terms, minima of the shelter factors, the
// diagnostic sums on diagnostic steps and the ridging product.
struct Share {
    float f0, f1, f2, f3, f4, f5, amin, wmin;
    float d0, d1, d2, d3, d4, d5, d6, d7;
    float rex;
};

GD_DEV void share_zero(Share &a)
{
    a.f0 = a.f1 = a.f2 = a.f3 = a.f4 = a.f5 = 0.f;
    a.amin = a.wmin = 3.0e38f;
    a.d0 = a.d1 = a.d2 = a.d3 = a.d4 = a.d5 = a.d6 = a.d7 = 0.f;
    a.rex = 0.f;
}

GD_DEV void scan_window(Share &a, int s, int lane, bool diag)
{
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int su = __shfl_up_sync(0xffffffffu, s, d);
        const bool same = lane >= d && su == s;
        float o;
        o = __shfl_up_sync(0xffffffffu, a.f0, d); if (same) a.f0 += o;
        o = __shfl_up_sync(0xffffffffu, a.f1, d); if (same) a.f1 += o;
        o = __shfl_up_sync(0xffffffffu, a.f2, d); if (same) a.f2 += o;
        o = __shfl_up_sync(0xffffffffu, a.f3, d); if (same) a.f3 += o;
        o = __shfl_up_sync(0xffffffffu, a.f4, d); if (same) a.f4 += o;
        o = __shfl_up_sync(0xffffffffu, a.f5, d); if (same) a.f5 += o;
        o = __shfl_up_sync(0xffffffffu, a.amin, d); if (same) a.amin = fminf(a.amin, o);
        o = __shfl_up_sync(0xffffffffu, a.wmin, d); if (same) a.wmin = fminf(a.wmin, o);
    }
    if (diag) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int su = __shfl_up_sync(0xffffffffu, s, d);
            const bool same = lane >= d && su == s;
            float o;
            o = __shfl_up_sync(0xffffffffu, a.d0, d); if (same) a.d0 += o;
            o = __shfl_up_sync(0xffffffffu, a.d1, d); if (same) a.d1 += o;
            o = __shfl_up_sync(0xffffffffu, a.d2, d); if (same) a.d2 += o;
            o = __shfl_up_sync(0xffffffffu, a.d3, d); if (same) a.d3 += o;
            o = __shfl_up_sync(0xffffffffu, a.d4, d); if (same) a.d4 += o;
            o = __shfl_up_sync(0xffffffffu, a.d5, d); if (same) a.d5 += o;
            o = __shfl_up_sync(0xffffffffu, a.d6, d); if (same) a.d6 += o;
            o = __shfl_up_sync(0xffffffffu, a.d7, d); if (same) a.d7 += o;
        }
    }
    // ridging keeps pi r^2 h of the recipient, so a floe's events compose as
    // h -> h prod(1 + Vol_k / V0); carried as the excess over one
    if (__any_sync(0xffffffffu, a.rex != 0.f)) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int su = __shfl_up_sync(0xffffffffu, s, d);
            const float o = __shfl_up_sync(0xffffffffu, a.rex, d);
            if (lane >= d && su == s) a.rex = (a.rex + o) + a.rex * o;
        }
    }
}

GD_DEV void put_partial(const Share &a, int e, bool diag, float4 *part, float4 *pdg, float *prx)
{
    part[2 * (size_t)e] = make_float4(a.f0, a.f1, a.f2, a.f3);
    part[2 * (size_t)e + 1] = make_float4(a.f4, a.f5, a.amin, a.wmin);
    if (diag) {
        pdg[2 * (size_t)e] = make_float4(a.d0, a.d1, a.d2, a.d3);
        pdg[2 * (size_t)e + 1] = make_float4(a.d4, a.d5, a.d6, a.d7);
    }
    prx[e] = a.rex;
}

GD_DEV void share_from(Share &a, const Acc<float> &A)
{
    a.f0 = A.fcx; a.f1 = A.fcy; a.f2 = A.mc; a.f3 = A.fbx; a.f4 = A.fby; a.f5 = A.mb;
    a.amin = A.hsfa; a.wmin = A.hsfw;
    a.d0 = A.tac; a.d1 = A.pc; a.d2 = A.tab; a.d3 = A.pb; a.d4 = A.sxx; a.d5 = A.syy; a.d6 = A.sxy; a.d7 = A.syx;
}

GD_DEV void acc_zero(Acc<float> &A)
{
    A.fcx = A.fcy = A.mc = A.fbx = A.fby = A.mb = 0.f;
    A.tac = A.pc = A.tab = A.pb = 0.f;
    A.sxx = A.syy = A.sxy = A.syx = 0.f;
    A.hsfa = A.hsfw = 3.0e38f;
}

__global__ void __launch_bounds__(256, 2) k_pairs_own(Views V, int cur, int diag, int P, const unsigned *erow,
                                                     float4 *part, float4 *pdg, float *prx, float4 *jrec,
                                                     float4 *jdiag, float *jrex, unsigned char *jflag)
{
    if (*(volatile int *)V.status & (ST_EXPIRED | ST_NAN | ST_ROW_OVERFLOW)) return;
    Hist4<float> *Hh = (Hist4<float> *)V.hist[0];
    BondDyn *BD = V.bdyn[0];
    const Snap *S = V.snap[cur];
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    const int nwin = (P + 31) >> 5;
    unsigned long long n_cand = 0, n_cont = 0, n_bond = 0, n_plast = 0;
    for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < nwin; w += nwarps) {
        const int e = (w << 5) + lane;
        const bool valid = e < P;
        const int s = valid ? (int)erow[e] : -1 - lane;
        Share a;
        share_zero(a);
        if (valid) {
            const int2 en = V.ent_up[e];
            const int t = en.x, p = en.y;
            const InstParams &Pm = V.P[V.inst[s]];
            const bool px = Pm.boundary & BC_PERIODIC_X, py = Pm.boundary & BC_PERIODIC_Y;
            const bool shel = Pm.shelter != 0;
            const Snap Si = S[s], Sj = S[t];      // s has the lower id: the reference's "i"
            const double dx = wrap_d(Si.x - Sj.x, Pm.nx, px), dy = wrap_d(Si.y - Sj.y, Pm.ny, py);
            const double dist = sqrt(dx * dx + dy * dy);
            unsigned char act = 0;
            if (dist <= Si.r + Pm.rtree) {
                Hist4<float> H = Hh[p];
                const bool had = H.deltat != 0.f || H.thetarelc != 0.f;
                const int bi = V.bidx[p];
                BondM BM;
                if (bi >= 0) {
                    const BondDyn bd = BD[bi];
                    BM.flag = bd.flag; BM.dmg = bd.dmg; BM.dnb = bd.dnb; BM.dtb = bd.dtb;
                    BM.thji = bd.thji; BM.thij = bd.thij;
                }
                float ua = 0.f, va = 0.f, uw = 0.f, vw = 0.f;
                if (shel) {
                    double a0, a1, a2, a3;
                    wind_at(Pm, V.field, Si.x, Si.y, a0, a1, a2, a3);
                    ua = (float)a0; va = (float)a1; uw = (float)a2; vw = (float)a3;
                }
                const PairRes<float> R = pair_mixed(Pm, bi >= 0 ? &V.bstat[bi] : nullptr, dx, dy, dist, Si, Sj,
                                                    ua, va, uw, vw, H, bi >= 0 ? &BM : nullptr, shel, diag != 0);
                if (R.contact || had) Hh[p] = H;
                if (bi >= 0) {
                    BondDyn bd;
                    bd.dnb = BM.dnb; bd.dtb = BM.dtb; bd.thji = BM.thji; bd.thij = BM.thij; bd.dmg = BM.dmg;
                    bd.flag = BM.flag; bd.pad = 0;
                    BD[bi] = bd;
                }
                const float llb = Pm.f_llb;
                Acc<float> A;
                acc_zero(A);
                acc_side_i(A, R, llb, shel, diag != 0);
                share_from(a, A);
                if (R.who == 1) a.rex = (float)(R.vol / ((Pm.pi * (Si.r * Si.r)) * (double)Si.h));
                // the partner's share, for the gather kernel
                if (R.contact || R.bond_on || shel || R.who == 2 || (diag && R.S != 0.f)) {
                    Acc<float> B;
                    acc_zero(B);
                    acc_side_j(B, R, llb, shel, diag != 0);
                    jrec[2 * (size_t)p] = make_float4(B.fcx, B.fcy, B.mc, B.fbx);
                    jrec[2 * (size_t)p + 1] = make_float4(B.fby, B.mb, B.hsfa, B.hsfw);
                    if (diag) {
                        jdiag[2 * (size_t)p] = make_float4(B.tac, B.pc, B.tab, B.pb);
                        jdiag[2 * (size_t)p + 1] = make_float4(B.sxx, B.syy, B.sxy, B.syx);
                    }
                    jrex[p] = R.who == 2 ? (float)(R.vol / ((Pm.pi * (Sj.r * Sj.r)) * (double)Sj.h)) : 0.f;
                    act = 1;
                }
                if (diag) {
                    V.pdn[p] = (float)R.deltan;
                    n_cand++;
                    n_cont += R.contact;
                    n_bond += R.bond_on;
                    n_plast += R.who != 0;
                }
            } else if (diag) {
                V.pdn[p] = __int_as_float(0x7fc00000);
            }
            jflag[p] = act;
        }
        scan_window(a, s, lane, diag != 0);
        const int sd = __shfl_down_sync(0xffffffffu, s, 1);
        if (valid && (lane == 31 || sd != s || e + 1 >= P)) put_partial(a, e, diag != 0, part, pdg, prx);
    }
    if (diag) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            n_cand += __shfl_down_sync(0xffffffffu, n_cand, o);
            n_cont += __shfl_down_sync(0xffffffffu, n_cont, o);
            n_bond += __shfl_down_sync(0xffffffffu, n_bond, o);
            n_plast += __shfl_down_sync(0xffffffffu, n_plast, o);
        }
        if (lane == 0) {
            atomicAdd(&V.counters[0], n_cand);
            atomicAdd(&V.counters[1], n_cont);
            atomicAdd(&V.counters[2], n_bond);
            atomicAdd(&V.counters[3], n_plast);
        }
    }
}

__global__ void __launch_bounds__(256) k_pairs_gather(Views V, int diag, int P, const unsigned *erow, float4 *part,
                                                     float4 *pdg, float *prx, const float4 *jrec,
                                                     const float4 *jdiag, const float *jrex,
                                                     const unsigned char *jflag)
{
    if (*(volatile int *)V.status & (ST_EXPIRED | ST_NAN | ST_ROW_OVERFLOW)) return;
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    const int nwin = (P + 31) >> 5;
    for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < nwin; w += nwarps) {
        const int e = (w << 5) + lane;
        const bool valid = e < P;
        const int s = valid ? (int)erow[e] : -1 - lane;
        Share a;
        share_zero(a);
        if (valid) {
            const int p = V.ent_lo[e].y;
            if (jflag[p]) {
                const float4 r0 = jrec[2 * (size_t)p], r1 = jrec[2 * (size_t)p + 1];
                a.f0 = r0.x; a.f1 = r0.y; a.f2 = r0.z; a.f3 = r0.w;
                a.f4 = r1.x; a.f5 = r1.y; a.amin = r1.z; a.wmin = r1.w;
                a.rex = jrex[p];
                if (diag) {
                    const float4 q0 = jdiag[2 * (size_t)p], q1 = jdiag[2 * (size_t)p + 1];
                    a.d0 = q0.x; a.d1 = q0.y; a.d2 = q0.z; a.d3 = q0.w;
                    a.d4 = q1.x; a.d5 = q1.y; a.d6 = q1.z; a.d7 = q1.w;
                }
            }
        }
        scan_window(a, s, lane, diag != 0);
        const int sd = __shfl_down_sync(0xffffffffu, s, 1);
        if (valid && (lane == 31 || sd != s || e + 1 >= P)) put_partial(a, e, diag != 0, part, pdg, prx);
    }
}

GD_DEV Snap pack_snap(double x, double y, const Shape &sh, double u, double v, double om)
{
    Snap s;
    s.x = x; s.y = y; s.r = sh.r;
    s.h = (float)sh.h; s.u = (float)u; s.v = (float)v; s.om = (float)om;
    s.mass = (float)sh.mass;
    s.inertia = (float)sh.inertia;
    return s;
}

GD_DEV void add_partials(int e0, int e1, bool diag, const float4 *pm, const float4 *pd, const float *prx,
                         float4 &a0, float4 &a1, float4 &q0, float4 &q1, float &rex)
{
    if (e1 <= e0) return;
    for (int w = e0 >> 5; w <= (e1 - 1) >> 5; w++) {
        const int pos = min(e1, (w + 1) << 5) - 1;
        const float4 b0 = pm[2 * (size_t)pos], b1 = pm[2 * (size_t)pos + 1];
        a0.x += b0.x; a0.y += b0.y; a0.z += b0.z; a0.w += b0.w;
        a1.x += b1.x; a1.y += b1.y; a1.z = fminf(a1.z, b1.z); a1.w = fminf(a1.w, b1.w);
        if (diag) {
            const float4 c0 = pd[2 * (size_t)pos], c1 = pd[2 * (size_t)pos + 1];
            q0.x += c0.x; q0.y += c0.y; q0.z += c0.z; q0.w += c0.w;
            q1.x += c1.x; q1.y += c1.y; q1.z += c1.z; q1.w += c1.w;
        }
        const float o = prx[pos];
        rex = (rex + o) + rex * o;
    }
}

__global__ void __launch_bounds__(256, 2) k_floes_mixed(Views V, int cur, int diag, int sic,
                                                       const float4 *pm_up, const float4 *pd_up,
                                                       const float *prx_up, const float4 *pm_lo,
                                                       const float4 *pd_lo, const float *prx_lo)
{
    if (*(volatile int *)V.status & (ST_EXPIRED | ST_NAN | ST_ROW_OVERFLOW)) return;
    const int nxt = cur ^ 1;
    const int stride = gridDim.x * blockDim.x;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < V.N; g += stride) {
        const InstParams &P = V.P[V.inst[g]];
        const bool px = P.boundary & BC_PERIODIC_X, py = P.boundary & BC_PERIODIC_Y;
        const bool shel = P.shelter != 0;
        const double x = V.x[cur][g], y = V.y[cur][g], th = V.th[cur][g];
        const double u = V.u[cur][g], v = V.v[cur][g], om = V.om[cur][g];
        const double r = V.r[cur][g], h = V.h[cur][g];
        double dtb1 = V.dtb1[cur][g], dtb2 = V.dtb2[cur][g];
        double thb1 = V.thb1[cur][g], thb2 = V.thb2[cur][g];
        float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = make_float4(0.f, 0.f, 1.f, 1.f);
        float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f), q1 = make_float4(0.f, 0.f, 0.f, 0.f);
        float rex = 0.f;
        add_partials(V.up_off[g], V.up_off[g + 1], diag != 0, pm_up, pd_up, prx_up, a0, a1, q0, q1, rex);
        add_partials(V.lo_off[g], V.lo_off[g + 1], diag != 0, pm_lo, pd_lo, prx_lo, a0, a1, q0, q1, rex);
        // ridging of this floe's pairs (volume pi r^2 h kept)
        Shape run = make_shape(P, r, h);
        if (rex != 0.f) {
            const double h1 = h + h * (double)rex;
            run = make_shape(P, r * sqrt(h / h1), h1);
        }
        WallOut W;
        int wev = 0;
        verify_bc(P, x, y, u, v, om, run, dtb1, dtb2, thb1, thb2, W, wev);
        double ua, va, uw, vw;
        wind_at(P, V.field, x, y, ua, va, uw, vw);
        const float sca = shel ? a1.z : 0.f, scw = shel ? a1.w : 0.f;
        const Drag<float> D = forcing<float>(P, run, u, v, om, ua, va, uw, vw, sca, scw);
        const double fcx = a0.x, fcy = a0.y, mc = a0.z, fbx = a0.w, fby = a1.x, mb = a1.y;
        const double fax = D.fax, fay = D.fay, fwx = D.fwx, fwy = D.fwy;
        const double tfx = ((((fcx + fbx) + fax) + fwx) + (double)D.fcorx) + W.fx_bc;
        const double tfy = ((((fcy + fby) + fay) + fwy) + (double)D.fcory) + W.fy_bc;
        const double mt = (((mc + mb) + (double)D.ma) + (double)D.mw) + W.m_bc;
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
        V.snap[nxt][g] = pack_snap(x1, y1, run, u1, v1, om1);
        const double ddx = wrap_d(x1 - V.x0[cur][g], P.nx, px), ddy = wrap_d(y1 - V.y0[cur][g], P.ny, py);
        const double half = 0.5 * P.skin;
        if (ddx * ddx + ddy * ddy > half * half) {
            atomicOr(V.status, ST_EXPIRED);
            atomicMin(V.expired_at, sic);
        }
        if (!(isfinite(x1) && isfinite(y1) && isfinite(u1) && isfinite(v1) && isfinite(om1) && isfinite(th1)))
            atomicOr(V.status, ST_NAN);
        if (diag) {
            const size_t N = (size_t)V.N;
            const double rr = run.r;
            const double tac = q0.x, tab = q0.z;
            const double pa = tac != 0.0 ? (double)q0.y / tac : 0.0;
            const double pbv = tab != 0.0 ? (double)q0.w / tab : 0.0;
            const double pw = W.ta_bc != 0.0 ? W.p_bc / W.ta_bc : 0.0;
            double *D0 = V.diag;
            D0[0 * N + g] = tfx; D0[1 * N + g] = tfy; D0[2 * N + g] = fcx; D0[3 * N + g] = fcy;
            D0[4 * N + g] = fbx; D0[5 * N + g] = fby; D0[6 * N + g] = mt; D0[7 * N + g] = mc;
            D0[8 * N + g] = mb;
            D0[9 * N + g] = ((double)q1.x + W.sxx) + (fax + fwx) * rr;
            D0[10 * N + g] = ((double)q1.y + W.syy) + (fay + fwy) * rr;
            D0[11 * N + g] = ((double)q1.z + W.sxy) + 0.0;
            D0[12 * N + g] = ((double)q1.w + W.syx) + 0.0;
            D0[13 * N + g] = (pa + pbv) + pw;
        }
    }
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
                                    V.u[side][g], V.v[side][g], V.om[side][g]);
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

static int window_grid(int P, int block)
{
    const long long nwin = ((long long)P + 31) / 32;
    const int wpb = block / 32;
    return (int)std::max(1LL, std::min<long long>((nwin + wpb - 1) / wpb, 148LL * 32));
}

void launch_pairs_own(const Views &V, int cur, int diag, int P, const unsigned *erow_up, MixedBufs B, int block,
                      cudaStream_t st)
{
    k_pairs_own<<<window_grid(P, block), block, 0, st>>>(V, cur, diag, P, erow_up, B.part_up, B.pdg_up, B.prx_up,
                                                         B.jrec, B.jdiag, B.jrex, B.jflag);
}

void launch_pairs_gather(const Views &V, int diag, int P, const unsigned *erow_lo, MixedBufs B, int block,
                         cudaStream_t st)
{
    k_pairs_gather<<<window_grid(P, block), block, 0, st>>>(V, diag, P, erow_lo, B.part_lo, B.pdg_lo, B.prx_lo,
                                                            B.jrec, B.jdiag, B.jrex, B.jflag);
}

void launch_floes_mixed(const Views &V, int cur, int diag, int sic, MixedBufs B, int block, cudaStream_t st)
{
    const int grid = (int)std::max(1LL, std::min<long long>(((long long)V.N + block - 1) / block, 148LL * 16));
    k_floes_mixed<<<grid, block, 0, st>>>(V, cur, diag, sic, B.part_up, B.pdg_up, B.prx_up, B.part_lo, B.pdg_lo,
                                          B.prx_lo);
}

}  // namespace godar
