// Per-pair, per-wall and per-floe physics of one time step, as device
// functions.  Each function restates the reference routine named beside it;
// in the FP64 instantiation (T = double, file compiled with --fmad=false) every
// expression keeps the reference's operand order so that the result is
// bit-identical to the CPU oracle.  In the mixed instantiation (T = float) the
// pair forces, sheltering and drag run in FP32, while geometry that cancels
// (distance, overlap, chord length, ridged area), bond strain/damage and all
// shape bookkeeping stay in FP64.
#pragma once
#include "common.cuh"
#include "detmath.cuh"

namespace godar {

template <typename T> struct M;
template <> struct M<double> {
    static GD_DEV double sqrt_(double x) { return ::sqrt(x); }
    static GD_DEV double exp_(double x) { return dm::exp(x); }
    static GD_DEV double log_(double x) { return dm::log(x); }
};
// FP32 is the mixed path's force arithmetic: the hardware's approximate
// exponential and logarithm are within its tolerance
template <> struct M<float> {
    static GD_DEV float sqrt_(float x) { return sqrtf(x); }
    static GD_DEV float exp_(float x) { return __expf(x); }
    static GD_DEV float log_(float x) { return __logf(x); }
};

template <typename T> GD_DEV T tmax(T a, T b) { return a > b ? a : b; }
template <typename T> GD_DEV T tmin(T a, T b) { return a < b ? a : b; }

// fit (contact_forces.f90:247-266)
template <typename T> GD_DEV T fit(T xi)
{
    const T p1 = (T)9117e-4, p2 = (T)2722e-4, p3 = (T)3324e-6, q1 = (T)1524e-3, q2 = (T)3159e-5;
    return ((p1 * (xi * xi) + p2 * xi) + p3) / (((xi * xi) + q1 * xi) + q2);
}

// heaviside (forcing.f90:226-236): sign(0.5, x) + 0.5 with IEEE signed zero
template <typename T> GD_DEV T heaviside(T x) { return copysign((T)0.5, x) + (T)0.5; }

// S_shelter (forcing.f90:238-270); 0.18 is a default-kind REAL literal there
template <typename T>
GD_DEV T S_shelter(T hfi, T hfj, T deltan, T cosa, T sina, T uf, T vf)
{
    const T wnorm = M<T>::sqrt_(uf * uf + vf * vf) + (T)1e-20;
    const T costheta = (uf * cosa + vf * sina) / wnorm;
    const T c018 = (T)(double)0.18f;
    const T ex = M<T>::exp_(-((c018 * fabs(deltan / costheta)) / hfj));
    const T D = ((T)1 - ((T)1 - heaviside(deltan)) * ((T)1 - ex))
                - (heaviside(deltan) * heaviside(hfi - hfj)) * ((T)1 - hfj / hfi);
    const T G = heaviside(costheta) * costheta;
    return (T)1 - D * G;
}

// ridging.f90:88-99 / 74-86: thickness increase of one floe (FP64 always)
GD_DEV void apply_dh(const InstParams &P, Shape &s, double Vol)
{
    const double dh = Vol / (P.pi * (s.r * s.r));
    s.r = s.r * ::sqrt(s.h / (s.h + dh));
    s.h = s.h + dh;
    s = make_shape(P, s.r, s.h);
}

struct BondLocal {
    int flag;
    double dmg, dnb, dtb, thji, thij;   // dynamic (bonds.f90:94-99, 197-199)
    double rb, hb, lb, sb, ib;          // static (bonds.f90:255-262)
};

template <typename T> struct PairRes {
    T cosa, sina;
    bool contact;
    T fcn, fct, fcr, mcc, ac;
    bool bond_on;
    T fbn, fbt, mji, mij, sbt;
    T a_ij, a_ji, w_ij, w_ji;
    T S;
    T ri_l, rj_l;      // r(i), r(j) after the pair's own ridging event
    int who;           // 0 none, 1 lower-id floe, 2 higher-id floe
    double vol;
    double deltan;
};

// stepper.f90:89-271 for one candidate pair with lower-id floe "i" and
// higher-id floe "j".  dx, dy = x_i - x_j, y_i - y_j (minimum image), dist
// their FP64 norm.  si, sj: start-of-step shapes.  H and B are updated in
// place (the caller owns the storage).  CONTACT = false compiles the
// contact branch out, for callers that know the pair is not in contact
// ((r_i + r_j) - dist <= 0, the same expression as below).
template <typename T, bool CONTACT = true>
GD_DEV PairRes<T> pair_compute(const InstParams &P, double dx, double dy, double dist,
                               double ui, double vi, double oi, double uj, double vj, double oj,
                               Shape si, Shape sj, double uai, double vai, double uwi, double vwi,
                               Hist4<T> &H, BondLocal *B, bool want_shelter)
{
    PairRes<T> R;
    const T dt = (T)P.dt;
    // rel_pos_vel (physics.f90:73-114)
    const T cosa = (T)(-dx) / (T)dist;
    const T sina = (T)(-dy) / (T)dist;
    const T omegarel = (T)(oj - oi);
    const T du = (T)(uj - ui), dv = (T)(vj - vi);
    const T veln = du * cosa + dv * sina;
    const T veltb = -(du * sina) + dv * cosa;
    const T velt = veltb - ((T)oi * (T)si.r + (T)oj * (T)sj.r);
    const double deltan = (si.r + sj.r) - dist;
    const T dn = (T)deltan;
    R.cosa = cosa; R.sina = sina; R.deltan = deltan;
    R.who = 0; R.vol = 0.0;

    R.contact = CONTACT && deltan > 0.0;
    if (R.contact) {
        // contact_forces (contact_forces.f90:1-87)
        H.deltat = -(velt * dt) + H.deltat;
        double q = ((dist * dist - sj.r * sj.r) + si.r * si.r) / (2.0 * dist);
        double drd = 2.0 * ::sqrt(si.r * si.r - q * q);
        T dr = (T)drd;
        H.thetarelc = -(omegarel * dt) + H.thetarelc;
        const T m_redu = (T)((si.mass * sj.mass) / (si.mass + sj.mass));
        const T r_redu = (T)((si.r * sj.r) / (si.r + sj.r));
        const T hmin = (T)(si.h < sj.h ? si.h : sj.h);
        const T pi = (T)P.pi, ec = (T)P.ec, gc = (T)P.gc, beta = (T)P.beta;
        const T knc = ((pi * ec) * hmin) * fit<T>((dn * r_redu) / ((T)2 * (hmin * hmin)));
        T ktc = (((T)6 * gc) / ec) * knc;
        T krc = (knc * (dr * dr)) / (T)12;
        T gamn = -(beta * M<T>::sqrt_(((T)4 * knc) * m_redu));
        T gamt = -(((T)2 * beta) * M<T>::sqrt_((((T)2 / (T)3) * ktc) * m_redu));
        T gamr = (gamn * (dr * dr)) / (T)12;
        T fcn = tmax<T>(knc * dn - gamn * veln, (T)0);
        T fct = ktc * H.deltat - gamt * velt;
        if (P.ridging) {
            const T sig = (T)P.sigmanc_crit;
            if (sig * hmin <= (fcn / dr) / hmin) {
                // plastic_contact (ridging.f90:1-33)
                const T knp = ((sig * (hmin * hmin)) * dr) / dn;
                ktc = (((T)6 * gc) / ec) * knp;
                krc = (knp * (dr * dr)) / (T)12;
                gamn = -(beta * M<T>::sqrt_(((T)4 * knp) * m_redu));
                gamt = -(((T)2 * beta) * M<T>::sqrt_((((T)2 / (T)3) * ktc) * m_redu));
                gamr = (gamn * (dr * dr)) / (T)12;
                fcn = tmin<T>(fcn, (sig * (hmin * hmin)) * dr);
                fct = ktc * H.deltat - gamt * velt;
                // update_shape (ridging.f90:36-99), FP64
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
                drd = 2.0 * ::sqrt(si.r * si.r - q2 * q2);
                dr = (T)drd;
            }
        }
        // coulomb (physics.f90:1-33)
        T fcr;
        const T mu = (T)P.mu;
        if (fabs(fct) > mu * fabs(fcn)) {
            fct = -((mu * fabs(fcn)) * copysign((T)1, velt));
            fcr = fct;
            if (P.slipping) H.deltat = (fct + gamt * velt) / ktc;
        } else {
            fcr = fct;
        }
        T mcc = (T)0;
        if (!(B && B->flag == 1)) {
            T mrolling = krc * H.thetarelc - gamr * omegarel;
            if (fabs(H.thetarelc) > (((T)2 * fabs(fcn)) / knc) / dr) mrolling = (T)0;
            mcc = mrolling;
        }
        H.fcn = fcn;
        H.fct = fct;
        R.fcn = fcn; R.fct = fct; R.fcr = fcr; R.mcc = mcc;
        R.ac = (T)(drd * (si.h < sj.h ? si.h : sj.h));
    } else {
        // reset_contact (reset.f90:1-15)
        H.thetarelc = (T)0;
        H.deltat = (T)0;
        R.fcn = R.fct = R.fcr = R.mcc = R.ac = (T)0;
    }
    R.ri_l = (T)si.r;
    R.rj_l = (T)sj.r;

    R.bond_on = false;
    R.fbn = R.fbt = R.mji = R.mij = R.sbt = (T)0;
    T sfbn = (T)0, sfbt = (T)0;
    if (B) {
        if (B->flag == 1) {
            // bond_forces_euler (bonds.f90:74-161); strain state in FP64
            B->dnb = (double)veln * P.dt + B->dnb;
            B->dtb = (double)veltb * P.dt + B->dtb;
            B->thji = oi * P.dt + B->thji;
            B->thij = oj * P.dt + B->thij;
            const double m_redu = (si.mass * sj.mass) / (si.mass + sj.mass);
            const double i_redu = (si.inertia * sj.inertia) / (si.inertia + sj.inertia);
            const double L = B->lb;
            const double EA = ((1.0 - B->dmg) * P.eb) * B->sb;
            const double EI = ((1.0 - B->dmg) * P.eb) * B->ib;
            const T k_axial = (T)(EA / L);
            const T k_shear1 = (T)((12.0 * EI) / ((L * L) * L));
            const T k_shear2 = (T)((6.0 * EI) / (L * L));
            const T k_rot1 = (T)((4.0 * EI) / L);
            const T k_rot2 = (T)((2.0 * EI) / L);
            const double eta_i = 2.0 * ::sqrt((EI * i_redu) / L);
            const double eta_a = 2.0 * ::sqrt((EA * m_redu) * L);
            const T gam_axial = (T)(eta_a / L);
            const T gam_shear1 = (T)((12.0 * eta_i) / ((L * L) * L));
            const T gam_shear2 = (T)((6.0 * eta_i) / (L * L));
            const T gam_rot1 = (T)((4.0 * eta_i) / L);
            const T gam_rot2 = (T)((2.0 * eta_i) / L);
            const T dnb = (T)B->dnb, dtb = (T)B->dtb, thji = (T)B->thji, thij = (T)B->thij;
            const T Toi = (T)oi, Toj = (T)oj;
            T fbn = k_axial * dnb + gam_axial * veln;
            T fbt = ((k_shear1 * dtb + k_shear2 * (thji + thij)) + gam_shear1 * veltb)
                    + gam_shear2 * (Toi + Toj);
            T mji = ((((k_rot1 * thji + k_rot2 * thij) - k_shear2 * dtb) + gam_rot1 * Toi)
                     + gam_rot2 * Toj) - gam_shear2 * veltb;
            T mij = ((((k_rot2 * thji + k_rot1 * thij) - k_shear2 * dtb) + gam_rot2 * Toi)
                     + gam_rot1 * Toj) - gam_shear2 * veltb;
            // bond_breaking (bonds.f90:164-212); damage in FP64
            const T sb = (T)B->sb, rb = (T)B->rb, ib = (T)B->ib, hb = (T)B->hb;
            const T taub = fabs(fbt) / sb;
            const T sigmatb = -(fbn / sb) + (fabs(mji) * rb) / ib;
            const T sigmacb = fbn / sb + (fabs(mji) * rb) / ib;
            const T t1 = taub / ((T)P.tau_crit * hb);
            T phi = t1 * t1;
            if (sigmacb > (T)0) { const T t2 = sigmacb / ((T)P.sigmacb_crit * hb); phi = phi + t2 * t2; }
            if (sigmatb > (T)0) { const T t3 = sigmatb / ((T)P.sigmatb_crit * hb); phi = phi + t3 * t3; }
            const T psi = tmin<T>((T)1, (T)1 / M<T>::sqrt_(phi));
            double D = B->dmg;
            D = (D + (((1.0 - (double)psi) * (1.0 - D)) * P.dt) / P.dtd) - (D * P.dt) / P.dth;
            B->dmg = D;
            if (D >= P.dmax) {
                B->flag = 0;
                fbn = (T)0; fbt = (T)0; mji = (T)0;
                B->dmg = 1.0;
            }
            sfbn = fbn; sfbt = fbt;
            if (B->flag == 1) {
                R.bond_on = true;
                R.fbn = fbn; R.fbt = fbt; R.mji = mji; R.mij = mij; R.sbt = sb;
            }
        } else {
            // reset_bond (reset.f90:18-34)
            B->thji = 0.0; B->thij = 0.0; B->dnb = 0.0; B->dtb = 0.0;
        }
    }

    if (want_shelter) {
        // sheltering (forcing.f90:162-186), wind of the lower-id floe
        const T hfai = (T)si.hfa, hfaj = (T)sj.hfa, hfwi = (T)si.hfw, hfwj = (T)sj.hfw;
        const T ua = (T)uai, va = (T)vai, uw = (T)uwi, vw = (T)vwi;
        R.a_ij = S_shelter<T>(hfai, hfaj, dn, cosa, sina, ua, va);
        R.w_ij = S_shelter<T>(hfwi, hfwj, dn, cosa, sina, uw, vw);
        R.a_ji = S_shelter<T>(hfaj, hfai, dn, -cosa, -sina, ua, va);
        R.w_ji = S_shelter<T>(hfwj, hfwi, dn, -cosa, -sina, uw, vw);
    }
    // stress magnitude of stepper.f90:238-271 (last contact forces of the pair)
    R.S = M<T>::sqrt_(H.fcn * H.fcn + H.fct * H.fct) + M<T>::sqrt_(sfbn * sfbn + sfbt * sfbt);
    return R;
}

// Per-floe accumulators of one step.
template <typename T> struct Acc {
    T fcx, fcy, mc, fbx, fby, mb;
    T tac, pc, tab, pb;
    T sxx, syy, sxy, syx;
    T hsfa, hsfw;
};

// stepper.f90:113-129, 139-146, 165-198, 215-223, 238-271 for the
// lower-id floe ("i" side)
template <typename T>
GD_DEV void acc_side_i(Acc<T> &A, const PairRes<T> &R, T lambda_lb, bool shelter, bool diag)
{
    if (R.contact) {
        A.fcx = (A.fcx - R.fcn * R.cosa) + R.fcr * R.sina;
        A.fcy = (A.fcy - R.fcn * R.sina) - R.fcr * R.cosa;
        A.mc = (A.mc - R.ri_l * R.fct) - R.mcc;
        if (diag) { A.tac = A.tac + R.ac; A.pc = A.pc - R.fcn * R.ac; }
    }
    if (R.bond_on) {
        A.fbx = (A.fbx + R.fbn * R.cosa) - R.fbt * R.sina;
        A.fby = (A.fby + R.fbn * R.sina) + R.fbt * R.cosa;
        A.mb = (A.mb - (lambda_lb * R.ri_l) * R.fbt) - R.mji;
        if (diag) { A.tab = A.tab + R.sbt; A.pb = A.pb - R.fbn * R.sbt; }
    }
    if (shelter) {
        A.hsfa = tmin<T>(A.hsfa, R.a_ji);
        A.hsfw = tmin<T>(A.hsfw, R.w_ji);
    }
    if (diag) {
        A.sxx = A.sxx - ((R.S * R.cosa) * R.ri_l) * R.cosa;
        A.syy = A.syy - ((R.S * R.sina) * R.ri_l) * R.sina;
        A.sxy = A.sxy - ((R.S * R.sina) * R.ri_l) * R.cosa;
        A.syx = A.syx - ((R.S * R.cosa) * R.ri_l) * R.sina;
    }
}

template <typename T>
GD_DEV void acc_side_j(Acc<T> &A, const PairRes<T> &R, T lambda_lb, bool shelter, bool diag)
{
    if (R.contact) {
        A.fcx = (A.fcx + R.fcn * R.cosa) - R.fcr * R.sina;
        A.fcy = (A.fcy + R.fcn * R.sina) + R.fcr * R.cosa;
        A.mc = (A.mc - R.rj_l * R.fct) + R.mcc;
        if (diag) { A.tac = A.tac + R.ac; A.pc = A.pc - R.fcn * R.ac; }
    }
    if (R.bond_on) {
        A.fbx = (A.fbx - R.fbn * R.cosa) + R.fbt * R.sina;
        A.fby = (A.fby - R.fbn * R.sina) - R.fbt * R.cosa;
        A.mb = (A.mb - (lambda_lb * R.rj_l) * R.fbt) - R.mij;
        if (diag) { A.tab = A.tab + R.sbt; A.pb = A.pb - R.fbn * R.sbt; }
    }
    if (shelter) {
        A.hsfa = tmin<T>(A.hsfa, R.a_ij);
        A.hsfw = tmin<T>(A.hsfw, R.w_ij);
    }
    if (diag) {
        A.sxx = A.sxx - ((R.S * R.cosa) * R.ri_l) * R.cosa;
        A.syy = A.syy - ((R.S * R.sina) * R.ri_l) * R.sina;
        A.sxy = A.sxy - ((R.S * R.sina) * R.ri_l) * R.cosa;
        A.syx = A.syx - ((R.S * R.cosa) * R.ri_l) * R.sina;
    }
}

// Wall contacts of one floe: verify_bc / check_wall / contact_bc /
// coulomb_bc / plastic_contact_bc / update_shape_bc / reset_boundary
// (boundaries.f90:1-146, contact_forces.f90:90-244, physics.f90:36-70,
// ridging.f90:102-180, reset.f90:37-69).  FP64 in both precisions.
struct WallOut {
    double fx_bc, fy_bc, m_bc;
    double sxx, syy, sxy, syx;
    double ta_bc, p_bc;
};

GD_DEV void wall_one(const InstParams &P, int dir1, int dir2, int bd, double x, double y,
                     double u, double v, double om, Shape &s, double &dtb, double &thb,
                     WallOut &W, int &events)
{
    const double dt = P.dt;
    const double d1 = (double)dir1, d2 = (double)dir2;
    const double cosa_bc = (double)(dir1 * (dir2 - (1 - dir2)));
    const double sina_bc = (double)((1 - dir1) * (dir2 - (1 - dir2)));
    const double veln_bc = -(u * cosa_bc) - v * sina_bc;
    const double velt_bc = (u * sina_bc - v * cosa_bc) - om * s.r;
    const double deltan_bc = ((1.0 - d2) * (s.r - x) + d2 * ((s.r + x) - P.nx)) * d1
                             + ((1.0 - d2) * (s.r - y) + d2 * ((s.r + y) - P.ny)) * (1.0 - d1);
    double t0 = s.r - deltan_bc;
    double dr = 2.0 * ::sqrt(s.r * s.r - t0 * t0);
    dtb = -(velt_bc * dt) + dtb;
    const double deltat_bc = dtb;
    thb = -(om * dt) + thb;
    const double h = s.h, r = s.r;
    const double knc = ((P.pi * P.ec) * h) * fit<double>((deltan_bc * r) / ((1.0 * 2.0) * (h * h)));
    double ktc = ((6.0 * P.gc) / P.ec) * knc;
    double krc = (knc * (dr * dr)) / 12.0;
    double gamn = -(P.beta * ::sqrt(((4.0 * knc) * s.mass) / 1.0));
    double gamt = -((2.0 * P.beta) * ::sqrt((((2.0 / 3.0) * ktc) * s.mass) / 1.0));
    double gamr = (gamn * (dr * dr)) / 12.0;
    double fn = knc * deltan_bc - gamn * veln_bc;
    fn = fn > 0.0 ? fn : 0.0;
    double ft = ktc * deltat_bc - gamt * velt_bc;
    if (P.ridging) {
        if (P.sigmanc_crit * h <= (fn / dr) / h) {
            // plastic_contact_bc: m(i) is the total moment, zero during the
            // pair loop (reset.f90:97), so its damping vanishes
            const double mtot = 0.0;
            const double knp = ((P.sigmanc_crit * (h * h)) * dr) / deltan_bc;
            ktc = ((6.0 * P.gc) / P.ec) * knp;
            krc = (knp * (dr * dr)) / 12.0;
            gamn = -(P.beta * ::sqrt(((4.0 * knp) * mtot) / 1.0));
            gamt = -((2.0 * P.beta) * ::sqrt((((2.0 / 3.0) * ktc) * mtot) / 1.0));
            gamr = (gamn * (dr * dr)) / 12.0;
            const double cap = (P.sigmanc_crit * (h * h)) * dr;
            fn = fn < cap ? fn : cap;
            ft = ktc * deltat_bc - gamt * velt_bc;
            // update_shape_bc
            const double Area = (r * r) * dm::asin((dr / 2.0) / r) - (dr * (r - deltan_bc)) / 2.0;
            const double a2 = Area * h;
            const double Vol = a2 > 0.0 ? a2 : 0.0;
            apply_dh(P, s, Vol);
            events++;
            t0 = s.r - deltan_bc;
            dr = 2.0 * ::sqrt(s.r * s.r - t0 * t0);
        }
    }
    // coulomb_bc
    double fr;
    if (fabs(ft) > P.mu * fabs(fn)) {
        ft = -((P.mu * fabs(fn)) * copysign(1.0, velt_bc));
        fr = ft;
        if (P.slipping) dtb = (ft + gamt * velt_bc) / ktc;
    } else {
        fr = ft;
    }
    double mroll = krc * thb - gamr * om;
    if (fabs(thb) > ((2.0 * fabs(fn)) / knc) / dr) mroll = 0.0;
    // check_wall
    W.fx_bc = (W.fx_bc - fn * cosa_bc) + fr * sina_bc;
    W.fy_bc = (W.fy_bc - fn * sina_bc) - fr * cosa_bc;
    W.m_bc = (W.m_bc - mroll) - s.r * ft;
    const double q = ::sqrt(fn * fn + ft * ft);
    W.sxx = -((q * s.r) * (cosa_bc * cosa_bc));
    W.syy = -((q * s.r) * (sina_bc * sina_bc));
    W.sxy = -(((q * s.r) * cosa_bc) * sina_bc);
    W.syx = -(((q * s.r) * sina_bc) * cosa_bc);
    W.ta_bc = W.ta_bc + dr * s.h;
    W.p_bc = W.p_bc - (fn * dr) * s.h;
}

GD_DEV void verify_bc(const InstParams &P, double x, double y, double u, double v, double om,
                      Shape &s, double &dtb1, double &dtb2, double &thb1, double &thb2,
                      WallOut &W, int &events)
{
    W.fx_bc = W.fy_bc = W.m_bc = 0.0;
    W.sxx = W.syy = W.sxy = W.syx = 0.0;
    W.ta_bc = W.p_bc = 0.0;
    const int b = P.boundary;
    const bool wb = !(b & BC_PERIODIC_Y) && !(b & BC_OPEN_BOTTOM);
    const bool wt = !(b & BC_PERIODIC_Y) && !(b & BC_OPEN_TOP);
    const bool wl = !(b & BC_PERIODIC_X) && !(b & BC_OPEN_LEFT);
    const bool wr = !(b & BC_PERIODIC_X) && !(b & BC_OPEN_RIGHT);
    int t1 = 0, t2 = 0;
    if (wb && y - s.r < 0.0) { t1 = 1; wall_one(P, 0, 0, 1, x, y, u, v, om, s, dtb1, thb1, W, events); }
    if (wt && y + s.r > P.ny) { t1 = 1; wall_one(P, 0, 1, 1, x, y, u, v, om, s, dtb1, thb1, W, events); }
    if (wl && x - s.r < 0.0) { t2 = 1; wall_one(P, 1, 0, 2, x, y, u, v, om, s, dtb2, thb2, W, events); }
    if (wr && x + s.r > P.nx) { t2 = 1; wall_one(P, 1, 1, 2, x, y, u, v, om, s, dtb2, thb2, W, events); }
    if (t2 == 0) { thb2 = 0.0; dtb2 = 0.0; }
    if (t1 == 0) { thb1 = 0.0; dtb1 = 0.0; }
}

// forcing (forcing.f90:32-159) and coriolis (forcing.f90:189-206)
template <typename T> struct Drag { T fax, fay, fwx, fwy, ma, mw, fcorx, fcory; };

template <typename T>
GD_DEV Drag<T> forcing(const InstParams &P, const Shape &s, double u, double v, double om,
                       double ua_i, double va_i, double uw_i, double vw_i, T sca, T scw)
{
    Drag<T> D;
    const T pi = (T)P.pi, rhoair = (T)P.rhoair, rhowater = (T)P.rhowater;
    const T dua = (T)(ua_i - u), dva = (T)(va_i - v);
    const T duw = (T)(uw_i - u), dvw = (T)(vw_i - v);
    const T an = M<T>::sqrt_(dua * dua + dva * dva);
    const T on = M<T>::sqrt_(duw * duw + dvw * dvw);
    const T l10 = sizeof(T) == 8 ? (T)P.log10z0 : (T)P.log10z0f;
    const T la = M<T>::log_((T)s.hfa / (T)P.z0w) / l10;
    const T lw = M<T>::log_((T)s.hfw / (T)P.z0w) / l10;
    const T alog = la * la, olog = lw * lw;
    const T r = (T)s.r, hfa = (T)s.hfa, hfw = (T)s.hfw;
    const T Tom = (T)om, aom = fabs(Tom);
    const T r2 = r * r;
    T fdax, fday, fsax, fsay, fdwx, fdwy, fswx, fswy;
    if (an == (T)0) {
        fdax = fday = fsax = fsay = (T)0;
    } else {
        fdax = (((((((rhoair * (T)P.Cdair) * hfa) * r) * dua) * an) * alog) * sca) * pi / (T)2;
        fday = (((((((rhoair * (T)P.Cdair) * hfa) * r) * dva) * an) * alog) * sca) * pi / (T)2;
        const T g = an * an + (r2 * (aom * aom)) / (T)4;
        fsax = (((((rhoair * pi) * r2) * (T)P.Csair) * dua) / an) * g;
        fsay = (((((rhoair * pi) * r2) * (T)P.Csair) * dva) / an) * g;
    }
    if (on == (T)0) {
        fdwx = fdwy = fswx = fswy = (T)0;
    } else {
        fdwx = (((((((rhowater * (T)P.Cdwater) * hfw) * r) * duw) * on) * olog) * scw) * pi / (T)2;
        fdwy = (((((((rhowater * (T)P.Cdwater) * hfw) * r) * dvw) * on) * olog) * scw) * pi / (T)2;
        const T g = on * on + (r2 * (aom * aom)) / (T)4;
        fswx = (((((rhowater * pi) * r2) * (T)P.Cswater) * duw) / on) * g;
        fswy = (((((rhowater * pi) * r2) * (T)P.Cswater) * dvw) / on) * g;
    }
    D.fax = fdax + fsax; D.fay = fday + fsay;
    D.fwx = fdwx + fswx; D.fwy = fdwy + fswy;
    const T r4 = r2 * r2, r5 = (r2 * r) * r2;
    if (an < (T)1e-2)
        D.ma = -((((((((T)2 * pi) / (T)5) * r5) * rhoair) * (T)P.Csair) * Tom) * aom);
    else
        D.ma = -((((((((T)3 / (T)4) * pi) * rhoair) * (T)P.Csair) * an) * Tom) * r4);
    if (on < (T)1e-3)
        D.mw = -((((((((T)2 * pi) / (T)5) * r5) * rhowater) * (T)P.Cswater) * Tom) * aom);
    else
        D.mw = -((((((((T)3 / (T)4) * pi) * rhowater) * (T)P.Cswater) * on) * Tom) * r4);
    const T oe = (T)7.2921e-5;
    const T mass = (T)s.mass, sl = (T)P.sin_lat;
    D.fcorx = (((mass * (T)2) * oe) * sl) * (T)v;
    D.fcory = -((((mass * (T)2) * oe) * sl) * (T)u);
    return D;
}

}  // namespace godar
