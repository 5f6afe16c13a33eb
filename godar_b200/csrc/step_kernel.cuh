// One time step of every floe of a batch: the body of `stepper`
// (stepper.f90:44-343) as a single kernel.  One thread per floe walks the
// floe's neighbour row:
//   (b) pair forces: contact (contact_forces.f90:1-87), bonds
//       (bonds.f90:74-212), sheltering (forcing.f90:162-186) and stress /
//       pressure diagnostics for every candidate pair, accumulated in the
//       reference's own order - partners of lower id (the floe is the "j" of
//       rows processed earlier, ascending id), then its own row ("i",
//       ascending distance as returned by the kd-tree), so the FP64 sums are
//       bit-identical to the sequential reference order; each pair is
//       evaluated by both its floes, only the lower-id floe writes its
//       history (two-sided storage, so no floe reads state another thread is
//       writing and no atomics are needed);
//   (d) ridging: the plastic events of the floe's pairs, applied to its
//       radius/thickness in that order (update_shape, ridging.f90:36-99),
//       before its wall contacts (verify_bc, boundaries.f90:1-97);
//   (c) drag, Coriolis and the shelter minimum (forcing.f90:32-206);
//   (e) totals (stepper.f90:312-332) and the symplectic Euler update
//       (integration.f90:1-38), FP64.
// Neighbours read the start-of-step state (side cur); the floe writes side
// cur ^ 1.
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

template <typename T, bool EXACT>
__global__ void __launch_bounds__(128) k_step(Views V, int cur, int diag, int sic)
{
    if (*(volatile int *)V.status & ST_ABORT) return;
    const int nxt = cur ^ 1;
    const Hist4<T> *Hc = (const Hist4<T> *)V.hist[cur];
    Hist4<T> *Hn = (Hist4<T> *)V.hist[nxt];
    unsigned long long n_cand = 0, n_cont = 0, n_bond = 0, n_plast = 0;
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
        const Shape s0 = make_shape(P, r, h);
        double ua, va, uw, vw;
        wind_at(P, V.field, x, y, ua, va, uw, vw);
        Acc<T> A;
        A.fcx = A.fcy = A.mc = A.fbx = A.fby = A.mb = (T)0;
        A.tac = A.pc = A.tab = A.pb = (T)0;
        A.sxx = A.syy = A.sxy = A.syx = (T)0;
        A.hsfa = A.hsfw = shel ? (T)1 : (T)0;
        Shape run = s0;
        const T llb = (T)P.lambda_lb;
        const int l0 = V.lo_off[g], l1 = V.lo_off[g + 1];
        const int el = V.up_off[g], e1 = V.up_off[g + 1];

        // ---- partners of lower id: this floe is the reference's "j"
        for (int e = l0; e < l1; e++) {
            const int2 en = V.ent_lo[e];
            const int t = en.x, p = en.y;
            const double xt = V.x[cur][t], yt = V.y[cur][t], rt = V.r[cur][t];
            const double dx = wrap_d(xt - x, P.nx, px), dy = wrap_d(yt - y, P.ny, py);
            const double dist = sqrt(dx * dx + dy * dy);
            if (!(dist <= rt + P.rtree)) continue;
            const Shape st = make_shape(P, rt, V.h[cur][t]);
            double uat = 0.0, vat = 0.0, uwt = 0.0, vwt = 0.0;
            if (shel) wind_at(P, V.field, xt, yt, uat, vat, uwt, vwt);
            Hist4<T> H = Hc[p];
            const int bi = V.bidx[p];
            BondLocal BL;
            if (bi >= 0) bond_load(V, bi, cur, BL);
            const PairRes<T> R = pair_compute<T>(P, dx, dy, dist, V.u[cur][t], V.v[cur][t], V.om[cur][t],
                                                 u, v, om, st, s0, uat, vat, uwt, vwt, H,
                                                 bi >= 0 ? &BL : nullptr, shel);
            acc_side_j(A, R, llb, shel, diag != 0);
            if (R.who == 2) apply_dh(P, run, R.vol);
        }

        // ---- own row (partners of higher id): this floe is the reference's "i"
        if (EXACT) {
            // kd-tree order: ascending distance, ties by id; rows are nearly
            // sorted from the previous step, so insertion sort is linear
            for (int e = el; e < e1; e++) {
                const int t = V.ent_up[e].x;
                const double dx = wrap_d(x - V.x[cur][t], P.nx, px), dy = wrap_d(y - V.y[cur][t], P.ny, py);
                V.edist[e] = sqrt(dx * dx + dy * dy);
            }
            for (int a = el + 1; a < e1; a++) {
                const int2 ea = V.ent_up[a];
                const double da = V.edist[a];
                int b = a - 1;
                double db = V.edist[b];
                if (db < da) continue;
                const int ida = V.id[cur][ea.x];
                while (b >= el) {
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
        for (int e = el; e < e1; e++) {
            const int2 en = V.ent_up[e];
            const int t = en.x, p = en.y;
            const double xt = V.x[cur][t], yt = V.y[cur][t];
            const double dx = wrap_d(x - xt, P.nx, px), dy = wrap_d(y - yt, P.ny, py);
            const double dist = EXACT ? V.edist[e] : sqrt(dx * dx + dy * dy);
            Hist4<T> H = Hc[p];
            const int bi = V.bidx[p];
            BondLocal BL;
            if (bi >= 0) bond_load(V, bi, cur, BL);
            if (!(dist <= r + P.rtree)) {
                Hn[p] = H;
                if (bi >= 0) bond_store(V, bi, nxt, BL);
                if (diag) V.pdn[p] = __int_as_float(0x7fc00000);
                continue;
            }
            const Shape st = make_shape(P, V.r[cur][t], V.h[cur][t]);
            const PairRes<T> R = pair_compute<T>(P, dx, dy, dist, u, v, om, V.u[cur][t], V.v[cur][t],
                                                 V.om[cur][t], s0, st, ua, va, uw, vw, H,
                                                 bi >= 0 ? &BL : nullptr, shel);
            Hn[p] = H;
            if (bi >= 0) bond_store(V, bi, nxt, BL);
            acc_side_i(A, R, llb, shel, diag != 0);
            if (R.who == 1) apply_dh(P, run, R.vol);
            if (diag) {
                V.pdn[p] = (float)R.deltan;
                n_cand++;
                n_cont += R.contact;
                n_bond += R.bond_on;
                n_plast += R.who != 0;
            }
        }

        // ---- walls with the shape after this floe's pair events
        WallOut W;
        int wev = 0;
        verify_bc(P, x, y, u, v, om, run, dtb1, dtb2, thb1, thb2, W, wev);
        n_plast += diag ? wev : 0;

        // ---- drag and Coriolis with the final shape
        const Drag<T> D = forcing<T>(P, run, u, v, om, ua, va, uw, vw, A.hsfa, A.hsfw);

        // ---- totals and integration (FP64)
        const double fcx = (double)A.fcx, fcy = (double)A.fcy, fbx = (double)A.fbx, fby = (double)A.fby;
        const double mc = (double)A.mc, mb = (double)A.mb;
        const double fax = (double)D.fax, fay = (double)D.fay, fwx = (double)D.fwx, fwy = (double)D.fwy;
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

        // ---- neighbour-list validity and finiteness
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
            const double sxx = ((double)A.sxx + W.sxx) + (fax + fwx) * rr;
            const double syy = ((double)A.syy + W.syy) + (fay + fwy) * rr;
            const double sxy = ((double)A.sxy + W.sxy) + 0.0;
            const double syx = ((double)A.syx + W.syx) + 0.0;
            const double tac = (double)A.tac, tab = (double)A.tab;
            const double pa = tac != 0.0 ? (double)A.pc / tac : 0.0;
            const double pbv = tab != 0.0 ? (double)A.pb / tab : 0.0;
            const double pw = W.ta_bc != 0.0 ? W.p_bc / W.ta_bc : 0.0;
            double *D0 = V.diag;
            D0[0 * N + g] = tfx; D0[1 * N + g] = tfy; D0[2 * N + g] = fcx; D0[3 * N + g] = fcy;
            D0[4 * N + g] = fbx; D0[5 * N + g] = fby; D0[6 * N + g] = mt; D0[7 * N + g] = mc;
            D0[8 * N + g] = mb; D0[9 * N + g] = sxx; D0[10 * N + g] = syy; D0[11 * N + g] = sxy;
            D0[12 * N + g] = syx; D0[13 * N + g] = (pa + pbv) + pw;
        }
    }

    // bonds that no neighbour row references keep their state
    const int nc = *V.ncarry;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += stride) {
        const int bi = V.carry[k];
        V.bdyn[nxt][bi] = V.bdyn[cur][bi];
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

}  // namespace godar
