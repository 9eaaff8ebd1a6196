// cumc_adjoint.cuh — hand-written discrete adjoint of the FP64 RK3 step
// (Cartesian, cylindrical and spherical grids, models NONE and RIEMANN, PPM or
// TVD reconstruction, HLL, CT, every boundary flag).
//
// The forward stage s (solver/rungekutta.f90:38-66 and the kernels of
// cumc_kernels.cuh) is, per stage,
//   P_{s-1}   primitives with ghosts (utop + boundary of the previous combine)
//   F         = sweeps(P_{s-1})             face fluxes (PPM/TVD + HLL)
//   E         = emf(F, P_{s-1})             edge EMFs
//   L         = combine's flux difference and CT curl of (F, E)
//   Upre_s    = a U0 + b U_{s-1} + c dt L   on (0:n)^3
//   (U_s,P_s) = utop(Upre_s) + boundary
// with dt frozen (recorded in the forward pass). The reverse sweep of a stage
// applies the transposes in the opposite order:
//   boundary^T   ghost adjoints folded onto the active cells they copy
//   utop^T       adjoint of Upre_s from those of U_s and P_s
//   combine^T    a, b parts to U0, U_{s-1}; c dt part to L
//   CT^T, emf^T  edge and cell-EMF adjoints
//   sweep^T      HLL^T and PPM^T per face, limiter and solver branches
//                frozen by recomputing the forward values
// Cells outside 1:n and face fields outside their live positions are
// overwritten by the forward boundary, so their adjoints are folded onto
// their sources and then zero.
#pragma once
#include "cumc_kernels.cuh"
#include "cumc_walk.cuh"

namespace cumc {

// device pointer sets passed by value
struct Arr8 {
    double* a[8];
};
struct Arr3 {
    double* a[3];
};

// adjoint of the primitive fields of one stage (with ghosts)
struct AdjPrim {
    double* w[5];   // rho, vx, vy, vz, p
    double* bc[3];  // cell-centred B
    double* eps;
};

// ---------------------------------------------------------------------------
// reconstruction transposes (branches frozen by recomputation)
// ---------------------------------------------------------------------------

// ppm_slope's value (bit-identical: the same expression) and its partial
// derivatives with respect to (vm, vc, vp), on the branch the value took
struct SlopeGrad {
    double d, gm, gc, gp;
};
__device__ __forceinline__ SlopeGrad ppm_slope_grad(double vm, double vc, double vp, double b0, double b1) {
    SlopeGrad s{0.0, 0.0, 0.0, 0.0};
    const double delta = b0 * (vp - vc) + b1 * (vc - vm);
    if ((vp - vc) * (vc - vm) > 0.0) {
        const double m1 = fabs(delta), m2 = 2.0 * fabs(vc - vm), m3 = 2.0 * fabs(vc - vp);
        const double sd = copysign(1.0, delta);
        const double m12 = fmin(m1, m2);
        s.d = fmin(m12, m3) * sd;
        if (m12 <= m3 && m1 <= m2) {  // slope = delta
            s.gm = -b1;
            s.gc = b1 - b0;
            s.gp = b0;
        } else if (m12 <= m3) {  // slope = sd 2 |vc - vm|
            const double g = sd * 2.0 * copysign(1.0, vc - vm);
            s.gm = -g;
            s.gc = g;
        } else {  // slope = sd 2 |vc - vp|
            const double g = sd * 2.0 * copysign(1.0, vc - vp);
            s.gc = g;
            s.gp = -g;
        }
    }
    return s;
}

// transpose of the reconstruction of one cell from v[0..4] = cells c-2..c+2:
// seeds lvm, lvp on (vm_out, vp_out); adds to lv[0..4]
template <int RECON>
__device__ __forceinline__ void recon_adj(const AxisTabs& A, int c, const double v[5], double lvm, double lvp,
                                          double lv[5]) {
    if (lvm == 0.0 && lvp == 0.0) return;
    if (RECON == 4) {
        const SlopeGrad sm = ppm_slope_grad(v[0], v[1], v[2], A.s0[c - 1], A.s1[c - 1]);
        const SlopeGrad sc = ppm_slope_grad(v[1], v[2], v[3], A.s0[c], A.s1[c]);
        const SlopeGrad sp = ppm_slope_grad(v[2], v[3], v[4], A.s0[c + 1], A.s1[c + 1]);
        const double dmm = sm.d, dmc = sc.d, dmp = sp.d;
        const double vl = ppm_face(v[1], v[2], dmm, dmc, A.a0[c - 1], A.a1[c - 1], A.a2[c - 1], A.a3[c - 1]);
        const double vr = ppm_face(v[2], v[3], dmc, dmp, A.a0[c], A.a1[c], A.a2[c], A.a3[c]);
        const double vc = v[2];
        // ppm_fix transpose
        double lvc = 0.0, lvl = 0.0, lvr = 0.0;
        if ((vr - vc) * (vc - vl) <= 0.0) {
            lvc += lvm + lvp;
        } else {
            double vm1 = vl;
            if ((vr - vl) * ((vl - 3.0 * vc) + 2.0 * vr) < 0.0) {
                vm1 = 3.0 * vc - 2.0 * vr;
                lvc += 3.0 * lvm;
                lvr -= 2.0 * lvm;
            } else {
                lvl += lvm;
            }
            if ((vr - vm1) * ((3.0 * vc - 2.0 * vl) - vr) < 0.0) {
                lvc += 3.0 * lvp;
                lvl -= 2.0 * lvp;
            } else {
                lvr += lvp;
            }
        }
        // interface values: V = vc' + (a0 + a1)(vp' - vc') + a2 dmp' + a3 dmc'
        double ldmm = 0.0, ldmc = 0.0, ldmp = 0.0;
        {
            const double s = A.a0[c - 1] + A.a1[c - 1];
            lv[1] += (1.0 - s) * lvl;
            lv[2] += s * lvl;
            ldmc += A.a2[c - 1] * lvl;
            ldmm += A.a3[c - 1] * lvl;
        }
        {
            const double s = A.a0[c] + A.a1[c];
            lv[2] += (1.0 - s) * lvr;
            lv[3] += s * lvr;
            ldmp += A.a2[c] * lvr;
            ldmc += A.a3[c] * lvr;
        }
        lv[2] += lvc;
        lv[0] += ldmm * sm.gm;
        lv[1] += ldmm * sm.gc + ldmc * sc.gm;
        lv[2] += ldmm * sm.gp + ldmc * sc.gc + ldmp * sp.gm;
        lv[3] += ldmc * sc.gp + ldmp * sp.gc;
        lv[4] += ldmp * sp.gp;
    } else {
        // vm = vc - sl/2, vp = vc + sl/2, sl = minmod of dqf = 2(vp-vc)/cf, dqb = 2(vc-vm)/cb
        lv[2] += lvm + lvp;
        const double lsl = 0.5 * (lvp - lvm);
        const double cf = A.tcf[c], cb = A.tcb[c];
        const double dqf = (2.0 * (v[3] - v[2])) / cf;
        const double dqb = (2.0 * (v[2] - v[1])) / cb;
        const double sf = copysign(1.0, dqf), sb = copysign(1.0, dqb);
        if (sf != sb) return;  // slope 0
        if (fabs(dqf) <= fabs(dqb)) {  // slope = dqf
            lv[3] += 2.0 * lsl / cf;
            lv[2] -= 2.0 * lsl / cf;
        } else {  // slope = dqb
            lv[2] += 2.0 * lsl / cb;
            lv[1] -= 2.0 * lsl / cb;
        }
    }
}

// ---------------------------------------------------------------------------
// HLL transpose (hll_flux7 of cumc_device.cuh, branches frozen)
// ---------------------------------------------------------------------------
template <int DIR>
struct SideAdj {
    // forward values here only weight derivatives, so reciprocals replace
    // the forward's divisions (no branch depends on them)
    double rho, irho, v[3], p, b[3], e, vsq, bsq, E, hb2, vdotb;
    double Lrho, Lv[3], Lp, Lb[3], LE, Lhb2, Lvdotb;
    __device__ __forceinline__ void init(const double w[8], double ig1) {
        rho = w[IRHO];
        irho = 1.0 / rho;
        v[0] = w[IVX]; v[1] = w[IVY]; v[2] = w[IVZ];
        p = w[ITAU];
        b[0] = w[IBX]; b[1] = w[IBY]; b[2] = w[IBZ];
        e = (p * irho) * ig1;
        vsq = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
        bsq = (b[0] * b[0] + b[1] * b[1]) + b[2] * b[2];
        E = rho * (e + 0.5 * vsq) + 0.5 * bsq;
        hb2 = 0.5 * bsq;
        vdotb = (b[0] * v[0] + b[1] * v[1]) + b[2] * v[2];
        Lrho = Lp = LE = Lhb2 = Lvdotb = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) Lv[i] = Lb[i] = 0.0;
    }
    __device__ __forceinline__ double u(int q) const {
        return q == IRHO ? rho : q <= IVZ ? v[q - IVX] * rho : q == ITAU ? E : b[q - IBX];
    }
    __device__ __forceinline__ double f(int q) const {
        constexpr int t1 = (DIR + 1) % 3, t2 = (DIR + 2) % 3;
        const double vn = v[DIR], bn = b[DIR];
        if (q == IRHO) return rho * vn;
        if (q == IVX + DIR) return ((v[DIR] * rho * vn + p) + hb2) - bn * bn;
        if (q == IVX + t1) return v[t1] * rho * vn - bn * b[t1];
        if (q == IVX + t2) return v[t2] * rho * vn - bn * b[t2];
        if (q == ITAU) return (E * vn + (p + hb2) * vn) - bn * vdotb;
        if (q == IBX + t1) return vn * b[t1] - v[t1] * bn;
        return vn * b[t2] - v[t2] * bn;
    }
    __device__ __forceinline__ void u_adj(int q, double lam) {
        if (q == IRHO) Lrho += lam;
        else if (q <= IVZ) { Lv[q - IVX] += lam * rho; Lrho += lam * v[q - IVX]; }
        else if (q == ITAU) LE += lam;
        else Lb[q - IBX] += lam;
    }
    __device__ __forceinline__ void f_adj(int q, double lam) {
        const double vn = v[DIR], bn = b[DIR];
        if (q == IRHO) {
            Lrho += lam * vn;
            Lv[DIR] += lam * rho;
        } else if (q == IVX + DIR) {
            Lv[DIR] += lam * 2.0 * rho * vn;
            Lrho += lam * vn * vn;
            Lp += lam;
            Lhb2 += lam;
            Lb[DIR] -= lam * 2.0 * bn;
        } else if (q >= IVX && q <= IVZ) {
            const int t = q - IVX;
            Lv[t] += lam * rho * vn;
            Lrho += lam * v[t] * vn;
            Lv[DIR] += lam * v[t] * rho;
            Lb[DIR] -= lam * b[t];
            Lb[t] -= lam * bn;
        } else if (q == ITAU) {
            LE += lam * vn;
            Lv[DIR] += lam * (E + p + hb2);
            Lp += lam * vn;
            Lhb2 += lam * vn;
            Lb[DIR] -= lam * vdotb;
            Lvdotb -= lam * bn;
        } else {
            const int t = q - IBX;
            Lv[DIR] += lam * b[t];
            Lb[t] += lam * vn;
            Lv[t] -= lam * bn;
            Lb[DIR] -= lam * v[t];
        }
    }
    // fold E, hb2, vdotb, e into the primitive adjoints; out[8] in natural order
    __device__ __forceinline__ void finish(double ig1, double out[8]) {
        const double Le = LE * rho;
        const double Lvsq = LE * 0.5 * rho;
        const double Lbsq = LE * 0.5 + 0.5 * Lhb2;
        Lrho += LE * (e + 0.5 * vsq);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            Lb[i] += Lvdotb * v[i] + 2.0 * b[i] * Lbsq;
            Lv[i] += Lvdotb * b[i] + 2.0 * v[i] * Lvsq;
        }
        Lp += Le * irho * ig1;
        Lrho -= Le * e * irho;
        out[IRHO] += Lrho;
        out[IVX] += Lv[0]; out[IVY] += Lv[1]; out[IVZ] += Lv[2];
        out[ITAU] += Lp;
        out[IBX] += Lb[0]; out[IBY] += Lb[1]; out[IBZ] += Lb[2];
    }
};

// adjoint of cf = signalspeed(cs, bn, bt1, bt2, rho): adds to the arguments' adjoints
__device__ __forceinline__ void signalspeed_adj(double cs, double bn, double bt1, double bt2, double rho, double cf,
                                                double lcf, double& lcs, double& lbn, double& lbt1, double& lbt2,
                                                double& lrho) {
    if (lcf == 0.0 || !(cf > 0.0)) return;
    const double irho = 1.0 / rho;
    const double a2 = cs * cs;
    const double b2n = (bn * bn) * irho, b2t1 = (bt1 * bt1) * irho, b2t2 = (bt2 * bt2) * irho;
    const double b2 = (b2n + b2t1) + b2t2;
    const double inner = ((a2 * a2 + b2 * b2) + (2.0 * b2) * a2) - (4.0 * a2) * b2n;
    const double lsum = lcf * 0.25 / cf;  // d cf / d (a2 + b2 + s)
    double la2 = lsum, lb2 = lsum, lb2n = 0.0;
    if (inner > 0.0) {
        const double ls = lsum * 0.5 / sqrt(inner);  // d sqrt(inner) / d inner
        la2 += ls * (2.0 * (a2 + b2) - 4.0 * b2n);
        lb2 += ls * 2.0 * (a2 + b2);
        lb2n += ls * (-4.0 * a2);
    }
    lb2n += lb2;
    lcs += 2.0 * cs * la2;
    lbn += 2.0 * bn * irho * lb2n;
    lbt1 += 2.0 * bt1 * irho * lb2;
    lbt2 += 2.0 * bt2 * irho * lb2;
    lrho -= (b2n * lb2n + (b2t1 + b2t2) * lb2) * irho;
}

// adjoint of out[7] = hll_flux7<DIR>(wl, wr): lout[7] -> lwl[8], lwr[8] (added)
template <int DIR>
__device__ __forceinline__ void hll_adj(const double wl[8], const double wr[8], double g, const double lout[7],
                                        double lwl[8], double lwr[8]) {
    constexpr int ivn = IVX + DIR;
    constexpr int ibn = IBX + DIR, ibt1 = IBX + (DIR + 1) % 3, ibt2 = IBX + (DIR + 2) % 3;
    constexpr int bt_a = DIR == 0 ? IBY : IBX;
    constexpr int bt_b = DIR == 2 ? IBY : IBZ;
    const int comp[7] = {IRHO, IVX, IVY, IVZ, ITAU, bt_a, bt_b};
    const double ig1 = 1.0 / (g - 1.0);
    SideAdj<DIR> L, R;
    L.init(wl, ig1);
    R.init(wr, ig1);
    const double csL = sqrt((g * wl[ITAU]) / wl[IRHO]);
    const double csR = sqrt((g * wr[ITAU]) / wr[IRHO]);
    const double cfL = signalspeed(csL, wl[ibn], wl[ibt1], wl[ibt2], wl[IRHO]);
    const double cfR = signalspeed(csR, wr[ibn], wr[ibt1], wr[ibt2], wr[IRHO]);
    const double sqL = sqrt(wl[IRHO]), sqR = sqrt(wr[IRHO]);
    const double ubar = roe_avg(wl[ivn], wr[ivn], sqL, sqR);
    const double cbar = roe_avg(cfL, cfR, sqL, sqR);
    const double aL = wl[ivn] - cfL, bL = ubar - cbar;
    const double aR = wr[ivn] + cfR, bR = ubar + cbar;
    const double sL = fmin(aL, bL), sR = fmax(aR, bR);
    double lsL = 0.0, lsR = 0.0;
    if (sL >= 0.0) {
#pragma unroll
        for (int c = 0; c < 7; ++c) L.f_adj(comp[c], lout[c]);
    } else if (sL <= 0.0 && sR >= 0.0) {
        const double id = 1.0 / (sR - sL);
        double ld = 0.0;
#pragma unroll
        for (int c = 0; c < 7; ++c) {
            const int q = comp[c];
            const double fl = L.f(q), fr = R.f(q), ul = L.u(q), ur = R.u(q);
            const double out = ((sR * fl - sL * fr) + (sL * sR) * (ur - ul)) * id;
            const double ln = lout[c] * id;
            ld -= ln * out;
            L.f_adj(q, sR * ln);
            R.f_adj(q, -sL * ln);
            R.u_adj(q, sL * sR * ln);
            L.u_adj(q, -sL * sR * ln);
            lsR += ln * (fl + sL * (ur - ul));
            lsL += ln * (-fr + sR * (ur - ul));
        }
        lsR += ld;
        lsL -= ld;
    } else {
#pragma unroll
        for (int c = 0; c < 7; ++c) R.f_adj(comp[c], lout[c]);
    }
    // sL = min(aL, bL), sR = max(aR, bR)
    double lvnL = 0.0, lvnR = 0.0, lcfL = 0.0, lcfR = 0.0, lubar = 0.0, lcbar = 0.0;
    if (aL <= bL) { lvnL += lsL; lcfL -= lsL; } else { lubar += lsL; lcbar -= lsL; }
    if (aR >= bR) { lvnR += lsR; lcfR += lsR; } else { lubar += lsR; lcbar += lsR; }
    // Roe averages
    const double iss = 1.0 / (sqL + sqR);
    double lsqL = (lubar * (wl[ivn] - ubar) + lcbar * (cfL - cbar)) * iss;
    double lsqR = (lubar * (wr[ivn] - ubar) + lcbar * (cfR - cbar)) * iss;
    lvnL += lubar * sqL * iss;
    lvnR += lubar * sqR * iss;
    lcfL += lcbar * sqL * iss;
    lcfR += lcbar * sqR * iss;
    // fast speeds
    double lcsL = 0.0, lcsR = 0.0;
    signalspeed_adj(csL, wl[ibn], wl[ibt1], wl[ibt2], wl[IRHO], cfL, lcfL, lcsL, L.Lb[DIR], L.Lb[(DIR + 1) % 3],
                    L.Lb[(DIR + 2) % 3], L.Lrho);
    signalspeed_adj(csR, wr[ibn], wr[ibt1], wr[ibt2], wr[IRHO], cfR, lcfR, lcsR, R.Lb[DIR], R.Lb[(DIR + 1) % 3],
                    R.Lb[(DIR + 2) % 3], R.Lrho);
    // cs = sqrt(g p / rho): d cs = cs/2 (dp/p - drho/rho); sq = sqrt(rho): d sq = drho / (2 sq)
    if (csL > 0.0) {
        const double h = 0.5 * lcsL * csL;
        L.Lp += h / wl[ITAU];
        L.Lrho -= h * L.irho;
    }
    if (csR > 0.0) {
        const double h = 0.5 * lcsR * csR;
        R.Lp += h / wr[ITAU];
        R.Lrho -= h * R.irho;
    }
    L.Lrho += 0.5 * lsqL / sqL;
    R.Lrho += 0.5 * lsqR / sqR;
    L.Lv[DIR] += lvnL;
    R.Lv[DIR] += lvnR;
    L.finish(ig1, lwl);
    R.finish(ig1, lwr);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
struct AdjStage {
    const double* mu[8];    // adjoint of the combine's output (Upre), live entries only
    const double* lamE[3];  // edge-EMF adjoints (k_adj_ct)
    const double* dt;       // device dt of the step
    double gam;             // combine's coefficient on dt L
};

__device__ __forceinline__ bool inside(int j, int k, int l, const Box& b) {
    return j >= 1 && j <= b.nx && k >= 1 && k <= b.ny && l >= 1 && l <= b.nz;
}
__device__ __forceinline__ bool in0n(int j, int k, int l, const Box& b) {
    return j >= 0 && j <= b.nx && k >= 0 && k <= b.ny && l >= 0 && l <= b.nz;
}

// CT^T: edge-EMF adjoints on (0:n)^3 from the field part of mu (solver/mhd.f90
// :137-148, with the GEOM_CT factors of solver/coords.f90:310-415). Each face
// field's l_rk is (E_a p - E_a' m)/c - (E_b p - E_b' m)/c over the triple's
// factors, so an edge collects p/c from its own triple and m/c from the
// triples above it.
template <int COORD>
__global__ void __launch_bounds__(256) k_adj_ct(Box b, Tabs T, AdjStage a, double* lex, double* ley, double* lez) {
    const int n0 = b.nx + 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int j = (int)(t % n0), k = (int)((t / n0) % n1), l = (int)(t / ((long long)n0 * n1));
    const int i = b.idx(j, k, l);
    const int sj = 1, sk = b.SX, sl = b.SX * b.SY;
    const double cdt = a.gam * *a.dt;
    const double* mx = a.mu[IBX];
    const double* my = a.mu[IBY];
    const double* mz = a.mu[IBZ];
    // the face triple's own CT factors (the edge is its upper one) ...
    CTf g;
    geom_ct<COORD>(T, j, k, l, g);
    double ez = -(mx[i] * g.bx_ez_p) / g.bx_ez_c + (my[i] * g.by_ez_p) / g.by_ez_c;
    double ey = (mx[i] * g.bx_ey_p) / g.bx_ey_c - (mz[i] * g.bz_ey_p) / g.bz_ey_c;
    double ex = -(my[i] * g.by_ex_p) / g.by_ex_c + (mz[i] * g.bz_ex_p) / g.bz_ex_c;
    // ... and those of the triples above it, where the edge is the lower one
    if (k + 1 <= b.ny) {
        geom_ct<COORD>(T, j, k + 1, l, g);
        ez += (mx[i + sk] * g.bx_ez_m) / g.bx_ez_c;
        ex -= (mz[i + sk] * g.bz_ex_m) / g.bz_ex_c;
    }
    if (j + 1 <= b.nx) {
        geom_ct<COORD>(T, j + 1, k, l, g);
        ez -= (my[i + sj] * g.by_ez_m) / g.by_ez_c;
        ey += (mz[i + sj] * g.bz_ey_m) / g.bz_ey_c;
    }
    if (l + 1 <= b.nz) {
        geom_ct<COORD>(T, j, k, l + 1, g);
        ey -= (mx[i + sl] * g.bx_ey_m) / g.bx_ey_c;
        ex += (my[i + sl] * g.by_ex_m) / g.by_ex_c;
    }
    lex[i] = cdt * ex;
    ley[i] = cdt * ey;
    lez[i] = cdt * ez;
}

// emf^T, cell part: ecell = -v x B on (0:n+1)^3 enters four edges with -1/4
// (solver/mhd.f90:95-125); adds to the velocity and cell-field adjoints
__global__ void __launch_bounds__(256) k_adj_ecell(Box b, Prim pr, const double* lex, const double* ley,
                                                   const double* lez, AdjPrim o) {
    const int n0 = b.nx + 2, n1 = b.ny + 2, n2 = b.nz + 2;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int j = (int)(t % n0), k = (int)((t / n0) % n1), l = (int)(t / ((long long)n0 * n1));
    const int i = b.idx(j, k, l);
    const int sj = 1, sk = b.SX, sl = b.SX * b.SY;
    auto E = [&](const double* e, int dj, int dk, int dl) -> double {
        const int jj = j - dj, kk = k - dk, ll = l - dl;
        return in0n(jj, kk, ll, b) ? e[i - dj * sj - dk * sk - dl * sl] : 0.0;
    };
    const double lx = -0.25 * (((E(lex, 0, 0, 0) + E(lex, 0, 0, 1)) + E(lex, 0, 1, 0)) + E(lex, 0, 1, 1));
    const double ly = -0.25 * (((E(ley, 0, 0, 0) + E(ley, 0, 0, 1)) + E(ley, 1, 0, 0)) + E(ley, 1, 0, 1));
    const double lz = -0.25 * (((E(lez, 0, 0, 0) + E(lez, 0, 1, 0)) + E(lez, 1, 0, 0)) + E(lez, 1, 1, 0));
    if (lx == 0.0 && ly == 0.0 && lz == 0.0) return;
    const double vx = pr.w[1][i], vy = pr.w[2][i], vz = pr.w[3][i];
    const double bx = pr.bc[0][i], by = pr.bc[1][i], bz = pr.bc[2][i];
    // ex = vz by - vy bz, ey = vx bz - vz bx, ez = vy bx - vx by
    o.w[1][i] += ly * bz - lz * by;
    o.w[2][i] += lz * bx - lx * bz;
    o.w[3][i] += lx * by - ly * bx;
    o.bc[0][i] += lz * vy - ly * vz;
    o.bc[1][i] += lx * vz - lz * vx;
    o.bc[2][i] += ly * vx - lx * vy;
}

// GEOM_SOURCE^T (solver/coords.f90:127-161) on the interior cells: the
// geometric source, added geom_repeat times to l_rk of the cell's momentum
// (and so to Upre with weight gam dt), differentiated with respect to the
// stage's primitives (rho, v, p, bcell) at the cell.
template <int COORD>
__global__ void __launch_bounds__(256) k_adj_source(Box b, Tabs T, Prim pr, AdjStage a, int repeat, AdjPrim o) {
    const long long total = (long long)b.nx * b.ny * b.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int j = (int)(t % b.nx) + 1, k = (int)((t / b.nx) % b.ny) + 1, l = (int)(t / ((long long)b.nx * b.ny)) + 1;
    const int i = b.idx(j, k, l);
    const double f = (a.gam * *a.dt) * repeat;
    const double lx = f * a.mu[IVX][i], ly = f * a.mu[IVY][i], lz = f * a.mu[IVZ][i];
    const double rho = pr.w[0][i], vx = pr.w[1][i], vy = pr.w[2][i], vz = pr.w[3][i];
    const double bx = pr.bc[0][i], by = pr.bc[1][i], bz = pr.bc[2][i];
    const double ix = 1.0 / T.ax[0].c[j];
    double lrho, lvx, lvy, lvz, lp, lbx, lby, lbz;
    if (COORD == 2) {
        // sx = ((p + rho vy^2) + |B|^2/2 - by^2)/R, sy = -(rho vx vy - bx by)/R
        lrho = (lx * (vy * vy) - ly * (vx * vy)) * ix;
        lvx = -ly * (rho * vy) * ix;
        lvy = (lx * (2.0 * rho * vy) - ly * (rho * vx)) * ix;
        lvz = 0.0;
        lp = lx * ix;
        lbx = (lx * bx + ly * by) * ix;
        lby = (ly * bx - lx * by) * ix;
        lbz = lx * bz * ix;
    } else {
        // sx = ((2p + bx^2) + rho (vy^2 + vz^2))/r
        // sy = ((p + rho vz^2) + |B|^2/2 - bz^2)/(r tan) - (rho vx vy - bx by)/r
        // sz = -(rho vx vz - bx bz)/r - (rho vy vz - by bz)/(r tan)
        const double it = ix / T.tanc[k];
        lrho = lx * (vy * vy + vz * vz) * ix + ly * ((vz * vz) * it - (vx * vy) * ix) -
               lz * ((vx * vz) * ix + (vy * vz) * it);
        lvx = -(ly * vy + lz * vz) * rho * ix;
        lvy = lx * (2.0 * rho * vy) * ix - ly * (rho * vx) * ix - lz * (rho * vz) * it;
        lvz = lx * (2.0 * rho * vz) * ix + ly * (2.0 * rho * vz) * it - lz * ((rho * vx) * ix + (rho * vy) * it);
        lp = 2.0 * lx * ix + ly * it;
        lbx = 2.0 * lx * bx * ix + ly * (bx * it + by * ix) + lz * bz * ix;
        lby = ly * (by * it + bx * ix) + lz * bz * it;
        lbz = -ly * bz * it + lz * (bx * ix + by * it);
    }
    o.w[0][i] += lrho;
    o.w[1][i] += lvx;
    o.w[2][i] += lvy;
    o.w[3][i] += lvz;
    o.w[4][i] += lp;
    o.bc[0][i] += lbx;
    o.bc[1][i] += lby;
    o.bc[2][i] += lbz;
}

// adjoints of the reconstructed left and right states of each face (the 7
// reconstructed fields in sweep order), stored at the face's left cell
struct FaceAdj {
    double* l[7];
    double* r[7];
};

// sweep^T, pass A: per face (normal 0:n_d, transverse 0:n+1), the flux
// adjoints from mu (flux difference) and the edge adjoints (emf), the forward
// left/right states, and HLL^T. Writes the state adjoints to fa and adds the
// normal-field adjoint of the face to lambf. Five 128-thread blocks per SM:
// 96 registers with some spilled to L1 beat 166 registers at three blocks.
// FROM_STATES: fa already holds the forward states (the forward sweep's
// STATES form, one reconstruction per cell); each face reads its two states
// and overwrites them with their adjoints. Otherwise the face reconstructs
// its two cells itself.
template <int COORD, int DIR, int RECON, bool FROM_STATES = false>
__global__ void __launch_bounds__(128, 5) k_adj_hll(Box b, Tabs T, Prim pr, double ggas, AdjStage a, FaceAdj fa,
                                                double* lambf) {
    const int n0 = (DIR == 0 ? b.nx : b.nx + 1) + 1;
    const int n1 = (DIR == 1 ? b.ny : b.ny + 1) + 1;
    const int n2 = (DIR == 2 ? b.nz : b.nz + 1) + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int j = (int)(t % n0), k = (int)((t / n0) % n1), l = (int)(t / ((long long)n0 * n1));
    const int base = b.idx(j, k, l);
    const int sj = 1, sk = b.SX, sl = b.SX * b.SY;
    const int s = DIR == 0 ? sj : DIR == 1 ? sk : sl;
    const int c = DIR == 0 ? j : DIR == 1 ? k : l;
    const int nd = DIR == 0 ? b.nx : DIR == 1 ? b.ny : b.nz;
    const AxisTabs A = T.ax[DIR];

    // flux adjoints
    double lf[7];
    const double cdt = a.gam * *a.dt;
    {
        const bool tin = DIR == 0 ? (k >= 1 && k <= b.ny && l >= 1 && l <= b.nz)
                                  : DIR == 1 ? (j >= 1 && j <= b.nx && l >= 1 && l <= b.nz)
                                             : (j >= 1 && j <= b.nx && k >= 1 && k <= b.ny);
        const bool lin = tin && c >= 1, rin = tin && c + 1 <= nd;
        // the face enters its left cell's flux difference as -F g+/g_c and
        // its right cell's as +F g-/g_c (Cartesian: 1/dx of each cell)
        double il = 0.0, ir = 0.0;
        if (COORD == 1) {
            il = lin ? 1.0 / A.d[c] : 0.0;
            ir = rin ? 1.0 / A.d[c + 1] : 0.0;
        } else {
            double gp, gc, gm;
            if (lin) {
                geom_flux<COORD, DIR>(T, j, k, l, gp, gc, gm);
                il = gp / gc;
            }
            if (rin) {
                geom_flux<COORD, DIR>(T, j + (DIR == 0), k + (DIR == 1), l + (DIR == 2), gp, gc, gm);
                ir = gm / gc;
            }
        }
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double ml = lin ? a.mu[q][base] : 0.0, mr = rin ? a.mu[q][base + s] : 0.0;
            lf[q] = cdt * (mr * ir - ml * il);
        }
        auto E = [&](const double* e, int dj, int dk, int dl) -> double {
            return in0n(j - dj, k - dk, l - dl, b) ? e[base - dj * sj - dk * sk - dl * sl] : 0.0;
        };
        if (DIR == 0) {  // x faces: by enters ez (-1/2), bz enters ey (+1/2)
            lf[5] = -0.5 * (E(a.lamE[2], 0, 0, 0) + E(a.lamE[2], 0, 1, 0));
            lf[6] = 0.5 * (E(a.lamE[1], 0, 0, 0) + E(a.lamE[1], 0, 0, 1));
        } else if (DIR == 1) {  // y faces: bx enters ez (+1/2), bz enters ex (-1/2)
            lf[5] = 0.5 * (E(a.lamE[2], 0, 0, 0) + E(a.lamE[2], 1, 0, 0));
            lf[6] = -0.5 * (E(a.lamE[0], 0, 0, 0) + E(a.lamE[0], 0, 0, 1));
        } else {  // z faces: bx enters ey (-1/2), by enters ex (+1/2)
            lf[5] = -0.5 * (E(a.lamE[1], 0, 0, 0) + E(a.lamE[1], 1, 0, 0));
            lf[6] = 0.5 * (E(a.lamE[0], 0, 0, 0) + E(a.lamE[0], 0, 1, 0));
        }
    }
    bool any = false;
#pragma unroll
    for (int q = 0; q < 7; ++q) any |= lf[q] != 0.0;
    if (!any) {
#pragma unroll
        for (int v = 0; v < 7; ++v) fa.l[v][base] = fa.r[v][base] = 0.0;
        return;
    }

    constexpr int bt_a = DIR == 0 ? 1 : 0;
    constexpr int bt_b = DIR == 2 ? 1 : 2;
    const double* src[7] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[bt_a], pr.bc[bt_b]};
    const int slot[7] = {IRHO, IVX, IVY, IVZ, ITAU, IBX + bt_a, IBX + bt_b};

    // forward states (the forward sweep's values: vp_out of cell c, vm_out of cell c+1)
    double wl[8], wr[8];
#pragma unroll
    for (int v = 0; v < 7; ++v) {
        if (FROM_STATES) {
            wl[slot[v]] = fa.l[v][base];
            wr[slot[v]] = fa.r[v][base];
            continue;
        }
        const double* q = src[v] + base;
        double cv[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) cv[m] = q[(m - 2) * s];  // cells c-2..c+3
        double vm, vp;
        if (RECON == 4) {
            const double dmm = ppm_slope(cv[0], cv[1], cv[2], A.s0[c - 1], A.s1[c - 1]);
            const double dmc = ppm_slope(cv[1], cv[2], cv[3], A.s0[c], A.s1[c]);
            const double dmp = ppm_slope(cv[2], cv[3], cv[4], A.s0[c + 1], A.s1[c + 1]);
            const double dmq = ppm_slope(cv[3], cv[4], cv[5], A.s0[c + 2], A.s1[c + 2]);
            const double V0 = ppm_face(cv[1], cv[2], dmm, dmc, A.a0[c - 1], A.a1[c - 1], A.a2[c - 1], A.a3[c - 1]);
            const double V1 = ppm_face(cv[2], cv[3], dmc, dmp, A.a0[c], A.a1[c], A.a2[c], A.a3[c]);
            const double V2 = ppm_face(cv[3], cv[4], dmp, dmq, A.a0[c + 1], A.a1[c + 1], A.a2[c + 1], A.a3[c + 1]);
            double vm0, vp1;
            ppm_fix(cv[2], V0, V1, vm0, vp);
            ppm_fix(cv[3], V1, V2, vm, vp1);
        } else {
            vp = cv[2] + 0.5 * tvd_slope(cv[1], cv[2], cv[3], A.tcf[c], A.tcb[c]);
            vm = cv[3] - 0.5 * tvd_slope(cv[2], cv[3], cv[4], A.tcf[c + 1], A.tcb[c + 1]);
        }
        wl[slot[v]] = vp;
        wr[slot[v]] = vm;
    }
    const double bn = pr.bf[DIR][base];
    wl[IBX + DIR] = bn;
    wr[IBX + DIR] = bn;

    double lwl[8] = {0, 0, 0, 0, 0, 0, 0, 0}, lwr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    hll_adj<DIR>(wl, wr, ggas, lf, lwl, lwr);
    lambf[base] += lwl[IBX + DIR] + lwr[IBX + DIR];
#pragma unroll
    for (int v = 0; v < 7; ++v) {
        fa.l[v][base] = lwl[slot[v]];
        fa.r[v][base] = lwr[slot[v]];
    }
}

// field v (0..6) of a sweep along DIR: source and adjoint arrays
template <int DIR>
__device__ __forceinline__ void sweep_field(const Prim& pr, const AdjPrim& o, int v, const double*& src, double*& dst) {
    constexpr int bt_a = DIR == 0 ? 1 : 0;
    constexpr int bt_b = DIR == 2 ? 1 : 2;
    if (v < 5) {
        src = pr.w[v];
        dst = o.w[v];
    } else {
        src = pr.bc[v == 5 ? bt_a : bt_b];
        dst = o.bc[v == 5 ? bt_a : bt_b];
    }
}

// sweep^T, pass B along y or z: the reconstruction transpose. One thread
// per (column, field, segment of RC_SEG cells) walks its segment: cell c's
// reconstruction (vm_out, vp_out) took its seeds from faces c-1 and c; its
// transpose adds to cells c-2..c+2, kept in a five-cell ring, and a cell is
// complete once the walk has passed it by two. A segment writes cells
// c0-2 .. c1+1, so the four cells next to each end of a segment also receive
// from the neighbouring segment. The even segments run in one launch and
// the odd ones in a second (`parity`): within a launch no two threads write
// the same cell, every add is a plain one, and each cell takes its
// contributions in a fixed order, so the result is the same bits on every
// run. The next cell and face seeds are loaded one cell ahead.
constexpr int RC_SEG = 32;

template <int DIR, int RECON>
__global__ void __launch_bounds__(128) k_adj_recon_col(Box b, Tabs T, Prim pr, FaceAdj fa, AdjPrim o, int parity) {
    using G = WalkGeom<DIR>;
    const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= G::ncols(b)) return;
    const int v = blockIdx.y;
    const int nd = G::nd(b);
    const int c0 = (2 * (int)blockIdx.z + parity) * RC_SEG;
    if (c0 > nd + 1) return;
    const int c1 = min(c0 + RC_SEG, nd + 2);  // reconstructed cells 0..nd+1
    const int a = (int)(col % G::wa(b)), cc = (int)(col / G::wa(b));
    const int s = G::stride(b);
    const int base = G::idx(b, a, cc, 0);
    const AxisTabs A = T.ax[DIR];
    const double* src;
    double* dst;
    sweep_field<DIR>(pr, o, v, src, dst);
    src += base;
    dst += base;
    const double* fl = fa.l[v] + base;
    const double* fr = fa.r[v] + base;
    auto emit = [&](int q, double val) {
        if (val != 0.0) dst[q * s] += val;
    };
    double x[5] = {src[(c0 - 2) * s], src[(c0 - 1) * s], src[c0 * s], src[(c0 + 1) * s], src[(c0 + 2) * s]};
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // cells c-2..c+2
    double lvm = c0 >= 1 ? fr[(c0 - 1) * s] : 0.0;
    double lvp = c0 <= nd ? fl[c0 * s] : 0.0;
    for (int c = c0; c < c1; ++c) {
        const double xn = c + 3 <= nd + 3 ? src[(c + 3) * s] : 0.0;
        const double lvm_n = fr[c * s];  // face c seeds vm_out of cell c+1
        const double lvp_n = c + 1 <= nd ? fl[(c + 1) * s] : 0.0;
        recon_adj<RECON>(A, c, x, lvm, lvp, acc);
        emit(c - 2, acc[0]);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            acc[m] = acc[m + 1];
            x[m] = x[m + 1];
        }
        acc[4] = 0.0;
        x[4] = xn;
        lvm = lvm_n;
        lvp = lvp_n;
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) emit(c1 - 2 + m, acc[m]);
}

// sweep^T, pass B along x: the reconstruction transpose with one lane per
// cell. A warp covers cells 28w-4 .. 28w+27 of a row and owns the middle 28
// (lanes 2..29): each lane transposes its own cell's reconstruction, and the
// five contributions to each owned cell are summed through warp shuffles.
template <int RECON>
__global__ void __launch_bounds__(128) k_adj_recon_x(Box b, Tabs T, Prim pr, FaceAdj fa, AdjPrim o) {
    const int nw = (b.nx + 6 + 27) / 28;  // warps per row
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long rows = (long long)(b.ny + 2) * (b.nz + 2);
    if (warp >= rows * nw) return;  // whole warp
    const int w = (int)(warp % nw);
    const long long row = warp / nw;
    const int k = (int)(row % (b.ny + 2)), l = (int)(row / (b.ny + 2));
    const int c = 28 * w + lane - 4;
    const AxisTabs A = T.ax[0];
    const int base = b.idx(0, k, l);
    const bool mine = c >= 0 && c <= b.nx + 1;                  // a reconstructed cell
    const bool owned = lane >= 2 && lane <= 29 && c >= -2 && c <= b.nx + 3;
#pragma unroll 1
    for (int v = 0; v < 7; ++v) {
        const double* src;
        double* dst;
        sweep_field<0>(pr, o, v, src, dst);
        double lv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (mine) {
            const double* q = src + base + c;
            const double x[5] = {q[-2], q[-1], q[0], q[1], q[2]};
            const double lvm = c >= 1 ? fa.r[v][base + c - 1] : 0.0;
            const double lvp = c <= b.nx ? fa.l[v][base + c] : 0.0;
            recon_adj<RECON>(A, c, x, lvm, lvp, lv);
        }
        const double tot = lv[2] + __shfl_down_sync(0xffffffffu, lv[0], 2) + __shfl_down_sync(0xffffffffu, lv[1], 1) +
                           __shfl_up_sync(0xffffffffu, lv[3], 1) + __shfl_up_sync(0xffffffffu, lv[4], 2);
        if (owned && tot != 0.0) dst[base + c] += tot;
    }
}

// boundary^T: the transpose of k_boundary, in gather form. k_boundary copies
// each ghost from one source (an active cell, or a live face), with the
// parity sign, and sets the ghost pressure p = rho eps (gamma-1)
// (solver/update.f90:27-35). So the transpose adds to each source the signed
// adjoints of every ghost copied from it, each ghost's density and eps
// adjoints first taking in its pressure adjoint. k_adj_boundary_gather runs
// one thread per possible source and enumerates its ghost images direction
// by direction (at most 6 per direction), so there are no atomics and the
// summation order is fixed. k_adj_boundary_clear then zeroes every ghost
// adjoint that was moved. fw holds the forward primitives of the stage.

// ghost indices along one direction whose gmap source is a; count returned
__device__ __forceinline__ int ghost_images(int a, int n, int fin, int fout, int* g, int* side) {
    int c = 0;
    if (a < 1 || a > n) return 0;
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        const int i = t < 3 ? t - 2 : n + t - 2;
        int src, sd;
        gmap(i, n, fin, fout, src, sd);
        if (src == a) {
            g[c] = i;
            side[c] = sd;
            ++c;
        }
    }
    return c;
}

// parity factor of a ghost image (side < 0: identity)
__device__ __forceinline__ int bsign(const BoundArgs& fw, int dir, int side, int q) {
    if (side < 0 || fw.flag[2 * dir + side] < 2) return 1;
    return fw.fac[2 * dir + side][q];
}

__global__ void __launch_bounds__(256) k_adj_boundary_gather(Box b, BoundArgs fw, AdjPrim o, double* lbx, double* lby,
                                                             double* lbz) {
    int j, k, l, i;
    if (!box1_index(b, j, k, l, i)) return;
    // index lists per direction: entry 0 is the identity, then the ghost images
    int gx[7], sx[7], gy[7], sy[7], gz[7], sz[7], gye[7], sye[7];
    gx[0] = j, gy[0] = k, gz[0] = l, gye[0] = k;
    sx[0] = sy[0] = sz[0] = sye[0] = -1;
    const int cx = 1 + ghost_images(j, b.nx, fw.flag[0], fw.flag[1], gx + 1, sx + 1);
    const int cy = 1 + ghost_images(k, b.ny, fw.flag[2], fw.flag[3], gy + 1, sy + 1);
    const int cz = 1 + ghost_images(l, b.nz, fw.flag[4], fw.flag[5], gz + 1, sz + 1);
    const int cye = 1 + ghost_images(k, b.ny, fw.flag[2], fw.eps_yout, gye + 1, sye + 1);
    if (cx == 1 && cy == 1 && cz == 1 && cye == 1) return;
    const double gm1 = fw.ggas - 1.0;
    if (j >= 1 && k >= 1 && l >= 1) {  // cell-centred quantities
        double acc[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int z = 0; z < cz; ++z)
            for (int y = 0; y < cy; ++y)
                for (int x = 0; x < cx; ++x) {
                    if (x == 0 && y == 0 && z == 0) continue;
                    const int g = b.idx(gx[x], gy[y], gz[z]);
                    const double lp = o.w[4][g];
                    const double lw[7] = {o.w[0][g] + lp * fw.eps[g] * gm1, o.w[1][g], o.w[2][g], o.w[3][g],
                                          o.bc[0][g], o.bc[1][g], o.bc[2][g]};
#pragma unroll
                    for (int q = 0; q < 7; ++q) {
                        const int qq = q < 4 ? q : IBX + q - 4;
                        const int s = bsign(fw, 0, sx[x], qq) * bsign(fw, 1, sy[y], qq) * bsign(fw, 2, sz[z], qq);
                        acc[q] += s * lw[q];
                    }
                }
        double acce = 0.0;
        for (int z = 0; z < cz; ++z)
            for (int y = 0; y < cye; ++y)
                for (int x = 0; x < cx; ++x) {
                    if (x == 0 && y == 0 && z == 0) continue;
                    const int g = b.idx(gx[x], gye[y], gz[z]);
                    acce += o.eps[g] + o.w[4][g] * fw.w[0][g] * gm1;
                }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (acc[q] != 0.0) o.w[q][i] += acc[q];
#pragma unroll
        for (int q = 0; q < 3; ++q)
            if (acc[4 + q] != 0.0) o.bc[q][i] += acc[4 + q];
        if (acce != 0.0) o.eps[i] += acce;
    }
    // face fields: only the components tangential to a ghost direction move
    if (k >= 1 && l >= 1 && (cy > 1 || cz > 1)) {
        double acc = 0.0;
        for (int z = 0; z < cz; ++z)
            for (int y = 0; y < cy; ++y)
                if (y || z) acc += (bsign(fw, 1, sy[y], IBX) * bsign(fw, 2, sz[z], IBX)) * lbx[b.idx(j, gy[y], gz[z])];
        if (acc != 0.0) lbx[i] += acc;
    }
    if (j >= 1 && l >= 1 && (cx > 1 || cz > 1)) {
        double acc = 0.0;
        for (int z = 0; z < cz; ++z)
            for (int x = 0; x < cx; ++x)
                if (x || z) acc += (bsign(fw, 0, sx[x], IBY) * bsign(fw, 2, sz[z], IBY)) * lby[b.idx(gx[x], k, gz[z])];
        if (acc != 0.0) lby[i] += acc;
    }
    if (j >= 1 && k >= 1 && (cx > 1 || cy > 1)) {
        double acc = 0.0;
        for (int y = 0; y < cy; ++y)
            for (int x = 0; x < cx; ++x)
                if (x || y) acc += (bsign(fw, 0, sx[x], IBZ) * bsign(fw, 1, sy[y], IBZ)) * lbz[b.idx(gx[x], gy[y], l)];
        if (acc != 0.0) lbz[i] += acc;
    }
}

// zero the ghost adjoints k_adj_boundary_gather moved (one thread per ghost,
// the ghost order of k_boundary)
__global__ void __launch_bounds__(256) k_adj_boundary_clear(Box b, BoundArgs fw, AdjPrim o, double* lbx, double* lby,
                                                            double* lbz) {
    const long long zsl = 6LL * b.SX * b.SY, ysl = 6LL * b.SX * b.nz, xsl = 6LL * b.ny * b.nz;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int j, k, l;
    if (t < zsl) {
        const int s = (int)(t / ((long long)b.SX * b.SY));
        const int r = (int)(t % ((long long)b.SX * b.SY));
        l = s < 3 ? s - 2 : b.nz + s - 2;
        k = r / b.SX - 2;
        j = r % b.SX - 2;
    } else if ((t -= zsl) < ysl) {
        const int s = (int)(t / ((long long)b.SX * b.nz));
        const int r = (int)(t % ((long long)b.SX * b.nz));
        k = s < 3 ? s - 2 : b.ny + s - 2;
        l = r / b.SX + 1;
        j = r % b.SX - 2;
    } else if ((t -= ysl) < xsl) {
        const int s = (int)(t / ((long long)b.ny * b.nz));
        const int r = (int)(t % ((long long)b.ny * b.nz));
        j = s < 3 ? s - 2 : b.nx + s - 2;
        l = r / b.ny + 1;
        k = r % b.ny + 1;
    } else {
        return;
    }
    const int i = b.idx(j, k, l);
    const bool gx = j < 1 || j > b.nx, gy = k < 1 || k > b.ny, gz = l < 1 || l > b.nz;
#pragma unroll
    for (int q = 0; q < 5; ++q) o.w[q][i] = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) o.bc[q][i] = 0.0;
    o.eps[i] = 0.0;
    if (j >= 0 && j <= b.nx && (gy || gz)) lbx[i] = 0.0;
    if (k >= 0 && k <= b.ny && (gx || gz)) lby[i] = 0.0;
    if (l >= 0 && l <= b.nz && (gx || gy)) lbz[i] = 0.0;
}

// utop^T on the active cells: from the adjoints of the re-derived conserved
// hydro variables (lu) and of the primitives (o), the adjoint of the
// combine's output Upre (hydro part, mu) and of the cell-centred field
// (lb, folded onto the faces by k_adj_bface). FROMUTORVE, CHECKRHO (RIEMANN:
// eps >= 0, branch frozen), FROMRVETOU and UPDATE's pressure
// (solver/fromrvetou.f90:21-127, solver/update.f90:27-35). FROM_CONS=false is
// initial_update, whose inputs are the uploaded rho, v and eps: mu then
// receives (rho, vx, vy, vz, eps) adjoints.
template <int MODEL, bool FROM_CONS>
__global__ void __launch_bounds__(256) k_adj_utop(Box b, Arr8 u, Arr8 w0, const double* eps0, Arr8 lu,
                                                  AdjPrim o, double ggas, Arr8 mu, Arr3 lb, double alpha,
                                                  double beta, Arr8 lam0) {
    const int n0 = b.nx + 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int j = (int)(t % n0), k = (int)((t / n0) % n1), l = (int)(t / ((long long)n0 * n1));
    const int i = b.idx(j, k, l);
    if (!(j >= 1 && k >= 1 && l >= 1)) {
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            mu.a[q][i] = 0.0;
            if (beta != 0.0) lu.a[q][i] = 0.0;
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) lb.a[q][i] = 0.0;
        return;
    }
    const double bx = 0.5 * (u.a[IBX][i] + u.a[IBX][i - 1]);
    const double by = 0.5 * (u.a[IBY][i] + u.a[IBY][i - b.SX]);
    const double bz = 0.5 * (u.a[IBZ][i] + u.a[IBZ][i - b.SX * b.SY]);
    const double bsquare = (bx * bx + by * by) + bz * bz;
    double rho, vx, vy, vz, e_raw;
    if (FROM_CONS) {
        rho = u.a[IRHO][i];
        vx = u.a[IVX][i] / rho;
        vy = u.a[IVY][i] / rho;
        vz = u.a[IVZ][i] / rho;
        const double vsq = (vx * vx + vy * vy) + vz * vz;
        e_raw = (u.a[ITAU][i] - 0.5 * bsquare) / rho - 0.5 * vsq;
    } else {
        rho = w0.a[0][i];
        vx = w0.a[1][i];
        vy = w0.a[2][i];
        vz = w0.a[3][i];
        e_raw = eps0[i];
    }
    const bool clamped = MODEL == 1 && !(e_raw >= 0.0);
    const double e = clamped ? 0.0 : e_raw;
    const double vsquare = (vx * vx + vy * vy) + vz * vz;
    const double g1 = ggas - 1.0;
    // adjoint inputs
    const double lu0 = lu.a[IRHO][i], lu1 = lu.a[IVX][i], lu2 = lu.a[IVY][i], lu3 = lu.a[IVZ][i], lu4 = lu.a[ITAU][i];
    const double lp = o.w[4][i];
    double Lrho = lu0 + o.w[0][i] + lu1 * vx + lu2 * vy + lu3 * vz + lu4 * (e + 0.5 * vsquare) + lp * e * g1;
    double Lvx = o.w[1][i] + lu1 * rho, Lvy = o.w[2][i] + lu2 * rho, Lvz = o.w[3][i] + lu3 * rho;
    double Le = o.eps[i] + lu4 * rho + lp * rho * g1;
    double Lvsq = lu4 * 0.5 * rho;
    double Lbsq = 0.5 * lu4;
    if (clamped) Le = 0.0;
    if (FROM_CONS) {
        // e_raw = (E - bsq/2)/rho - vsq/2
        const double E = u.a[ITAU][i];
        const double LE = Le / rho;
        Lbsq -= 0.5 * Le / rho;
        Lrho -= Le * (E - 0.5 * bsquare) / (rho * rho);
        Lvsq -= 0.5 * Le;
        Lvx += 2.0 * vx * Lvsq;
        Lvy += 2.0 * vy * Lvsq;
        Lvz += 2.0 * vz * Lvsq;
        // v = m / rho
        mu.a[IVX][i] = Lvx / rho;
        mu.a[IVY][i] = Lvy / rho;
        mu.a[IVZ][i] = Lvz / rho;
        Lrho -= (Lvx * vx + Lvy * vy + Lvz * vz) / rho;
        mu.a[IRHO][i] = Lrho;
        mu.a[ITAU][i] = LE;
    } else {
        Lvx += 2.0 * vx * Lvsq;
        Lvy += 2.0 * vy * Lvsq;
        Lvz += 2.0 * vz * Lvsq;
        mu.a[0][i] = Lrho;
        mu.a[1][i] = Lvx;
        mu.a[2][i] = Lvy;
        mu.a[3][i] = Lvz;
        mu.a[4][i] = Le;  // adjoint of the uploaded eps
    }
    lb.a[0][i] = o.bc[0][i] + 2.0 * bx * Lbsq;
    lb.a[1][i] = o.bc[1][i] + 2.0 * by * Lbsq;
    lb.a[2][i] = o.bc[2][i] + 2.0 * bz * Lbsq;
    // combine^T of the hydro part: Upre = alpha U0 + beta U_prev + ...; the
    // adjoint of U_prev replaces lu (read above by this thread only)
    if (FROM_CONS && (alpha != 0.0 || beta != 0.0)) {
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double m = mu.a[q][i];
            lam0.a[q][i] += alpha * m;
            if (beta != 0.0) lu.a[q][i] = beta * m;
        }
    }
}

// face-field adjoint on (0:n)^3: the pass-through adjoint of the live face
// values plus half the adjoints of the two active cells whose bcell average
// reads the face (solver/fromrvetou.f90:97-107); zero on every other entry
__global__ void __launch_bounds__(256) k_adj_bface(Box b, Arr3 lbf, Arr3 lb, Arr3 out, double alpha, double beta,
                                                   Arr3 lam0) {
    const int n0 = b.nx + 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int j = (int)(t % n0), k = (int)((t / n0) % n1), l = (int)(t / ((long long)n0 * n1));
    const int i = b.idx(j, k, l);
    const int st[3] = {1, b.SX, b.SX * b.SY};
    const int own[3] = {j, k, l};
    const int nn[3] = {b.nx, b.ny, b.nz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        bool live = true;
#pragma unroll
        for (int e = 0; e < 3; ++e)
            if (e != d && (own[e] < 1 || own[e] > nn[e])) live = false;
        double v = 0.0;
        if (live) {
            v = lbf.a[d][i];
            const double left = own[d] >= 1 ? lb.a[d][i] : 0.0;
            const double right = own[d] + 1 <= nn[d] ? lb.a[d][i + st[d]] : 0.0;
            v += 0.5 * (left + right);
        }
        out.a[d][i] = v;
        // combine^T of the field part (lbf, read above by this thread only,
        // becomes the adjoint of the previous stage's face field)
        if (alpha != 0.0) lam0.a[d][i] += alpha * v;
        if (beta != 0.0) lbf.a[d][i] = beta * v;
    }
}

// objective at the final state, per-block partial sums (deterministic order)
// and its adjoint seed. kind 1: magnetic energy 0.5 sum |bcell|^2 dV; kind 2:
// kinetic energy 0.5 sum rho |v|^2 dV; kind 3: sum of weights . cons over the
// live entries (weights in lamu on entry).
__global__ void __launch_bounds__(256) k_adj_objective(Box b, Tabs T, int coord, Prim pr, Arr8 u, int kind, AdjPrim o,
                                                       Arr8 lamu, double* partial) {
    const long long total = (long long)b.nx * b.ny * b.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (t < total) {
        const int j = (int)(t % b.nx) + 1, k = (int)((t / b.nx) % b.ny) + 1, l = (int)(t / ((long long)b.nx * b.ny)) + 1;
        const int i = b.idx(j, k, l);
        // cell volume: dx dy dz; R dR dphi dz; (r^3)/3 d(-cos theta) dphi
        const double dv = coord == CUMC_CARTESIAN     ? (T.ax[0].d[j] * T.ax[1].d[k]) * T.ax[2].d[l]
                          : coord == CUMC_CYLINDRICAL ? ((T.ax[0].c[j] * T.ax[0].d[j]) * T.ax[1].d[k]) * T.ax[2].d[l]
                                                      : (T.r3d3[j] * T.dcos[k]) * T.ax[2].d[l];
        if (kind == 1) {
            const double bx = pr.bc[0][i], by = pr.bc[1][i], bz = pr.bc[2][i];
            acc = 0.5 * ((bx * bx + by * by) + bz * bz) * dv;
            o.bc[0][i] += bx * dv;
            o.bc[1][i] += by * dv;
            o.bc[2][i] += bz * dv;
        } else if (kind == 2) {
            const double rho = pr.w[0][i], vx = pr.w[1][i], vy = pr.w[2][i], vz = pr.w[3][i];
            const double vsq = (vx * vx + vy * vy) + vz * vz;
            acc = 0.5 * rho * vsq * dv;
            o.w[0][i] += 0.5 * vsq * dv;
            o.w[1][i] += rho * vx * dv;
            o.w[2][i] += rho * vy * dv;
            o.w[3][i] += rho * vz * dv;
        } else {
            for (int q = 0; q < 5; ++q) acc += lamu.a[q][i] * u.a[q][i];
            // face fields: the cell's own faces (index 1:n) plus the lower boundary faces (index 0)
            const int st[3] = {1, b.SX, b.SX * b.SY};
            const int own[3] = {j, k, l};
            for (int d = 0; d < 3; ++d) {
                acc += lamu.a[IBX + d][i] * u.a[IBX + d][i];
                if (own[d] == 1) acc += lamu.a[IBX + d][i - st[d]] * u.a[IBX + d][i - st[d]];
            }
        }
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[w];
        partial[blockIdx.x] = v;
    }
}

// clears the weights of a linear objective off its live entries
__global__ void __launch_bounds__(256) k_adj_mask_live(Box b, Arr8 lamu) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.count()) return;
    const int j = (int)(t % b.SX) - 2, k = (int)((t / b.SX) % b.SY) - 2, l = (int)(t / ((long long)b.SX * b.SY)) - 2;
    const int own[3] = {j, k, l};
    const int nn[3] = {b.nx, b.ny, b.nz};
    const bool cell = inside(j, k, l, b);
    for (int q = 0; q < 5; ++q)
        if (!cell) lamu.a[q][t] = 0.0;
    for (int d = 0; d < 3; ++d) {
        bool live = own[d] >= 0 && own[d] <= nn[d];
        for (int e = 0; e < 3; ++e)
            if (e != d && (own[e] < 1 || own[e] > nn[e])) live = false;
        if (!live) lamu.a[IBX + d][t] = 0.0;
    }
}

// one block: sum of n partial sums in a fixed order
__global__ void __launch_bounds__(256) k_adj_sum(const double* partial, int n, double* out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[w];
        *out = v;
    }
}

}  // namespace cumc
