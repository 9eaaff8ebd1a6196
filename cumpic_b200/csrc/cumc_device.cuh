// cumc_device.cuh — device-side data layout and per-cell arithmetic of the
// CUMC3D hot path on B200 (sm_100a).
//
// Layout in HBM: structure of arrays. Every field is one FP64 array over the
// ghosted box (-2:n+3)^3 with x fastest, so a warp reads 32 consecutive x
// cells (256 B) per variable. The reference keeps the 8 equations
// interleaved per cell (AoS, solver/setup.f90:257); the library transposes
// once at upload/download.
//
// Every arithmetic expression below keeps the operation order of the
// reference subroutine it cites; the parity build uses --fmad=false so that
// no multiply-add is contracted and the FP64 path reproduces the FP64 CPU
// restatement bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cumc {

constexpr int NG = 3;  // ghost layers (solver/definition.f90:54)

// Box geometry: strides of the ghosted SoA arrays.
struct Box {
    int nx, ny, nz;
    int SX, SY, SZ;  // nx+6, ny+6, nz+6
    const int* skip;  // device flag: when non-null and set, kernels return at once
                      // (the time loop has reached t_end inside a captured graph)
    __host__ __device__ __forceinline__ int idx(int j, int k, int l) const {
        return (j + 2) + SX * ((k + 2) + SY * (l + 2));
    }
    __host__ __device__ __forceinline__ long long count() const { return (long long)SX * SY * SZ; }
};

// Per-axis 1-D tables (pointers pre-offset so that t[i] is valid for
// i in -3..n+3). All values are computed on the host with the formulas of the
// reference so that the device reads the same doubles the reference would
// recompute inline.
struct AxisTabs {
    const double* f;    // face coordinate xF(i)                   (solver/coords.f90:24-32)
    const double* d;    // cell width  xF(i)-xF(i-1)               (COORD_DX, :91-93)
    const double* c;    // cell centre 0.5*(xF(i)+xF(i-1))         (GET_COORD, :63-65)
    const double* s0;   // PPM slope weight b0c of cell i          (solver/reconstruct.f90:246)
    const double* s1;   // PPM slope weight b1c of cell i          (:247)
    const double* a0;   // PPM interface weights a0p..a3p of the   (:240-243)
    const double* a1;   //   face between cell i and i+1; equal to
    const double* a2;   //   a0m..a3m of cell i+1
    const double* a3;
    const double* tcf;  // TVD_MM cf of cell i                     (:110)
    const double* tcb;  // TVD_MM cb of cell i                     (:111)
};

struct Tabs {
    AxisTabs ax[3];
    // x-axis metric factors (solver/coords.f90:173-415)
    const double* r2;     // xF(j)*xF(j)
    const double* r3d3;   // (xF(j)^3 - xF(j-1)^3)/3
    const double* rfac;   // (2*(xF(j)^3-xF(j-1)^3)/3)/(xF(j)^2-xF(j-1)^2)
    const double* hr2;    // 0.5*(xF(j)^2 - xF(j-1)^2)
    // y-axis metric factors
    const double* sinf;   // sin(yF(k))
    const double* dcos;   // cos(yF(k-1)) - cos(yF(k))
    const double* tanc;   // tan(y-centre of cell k)
    const double* sinc;   // sin(y-centre of cell k)
};

// Equation identifiers (solver/setup.f90:49-116), zero-based here.
enum { IRHO = 0, IVX = 1, IVY = 2, IVZ = 3, ITAU = 4, IBX = 5, IBY = 6, IBZ = 7 };

// ---------------------------------------------------------------------------
// reconstruction
// ---------------------------------------------------------------------------

// van Leer-limited PPM slope of a cell from its neighbours
// (solver/reconstruct.f90:254-280). The reference evaluates this three times
// per call (dmm1, dmc, dmp1); the three forms are the same expression of the
// cell's own (vm, vc, vp) and weights, so it is computed once per cell.
template <typename R>
__device__ __forceinline__ R ppm_slope(R vm, R vc, R vp, R b0, R b1) {
    const R delta = b0 * (vp - vc) + b1 * (vc - vm);
    if ((vp - vc) * (vc - vm) > R(0))
        return fmin(fmin(fabs(delta), R(2) * fabs(vc - vm)), R(2) * fabs(vc - vp)) * copysign(R(1), delta);
    return R(0);
}

// Unlimited PPM value at the face between cell c and c+1
// (solver/reconstruct.f90:285; identical to :286 evaluated by cell c+1).
template <typename R>
__device__ __forceinline__ R ppm_face(R vc, R vp, R dmc, R dmp, R a0, R a1, R a2, R a3) {
    return (((vc + a0 * (vp - vc)) + a1 * (vp - vc)) + a2 * dmp) + a3 * dmc;
}

// Extremum and overshoot fixes of one cell (solver/reconstruct.f90:289-307).
// The second test reads the already-modified left value, as the reference does.
template <typename R>
__device__ __forceinline__ void ppm_fix(R vc, R vl, R vr, R& vm_out, R& vp_out) {
    vm_out = vl;
    vp_out = vr;
    if ((vr - vc) * (vc - vl) <= R(0)) {
        vp_out = vc;
        vm_out = vc;
    } else {
        if ((vr - vl) * ((vl - R(3) * vc) + R(2) * vr) < R(0)) vm_out = R(3) * vc - R(2) * vr;
        if ((vp_out - vm_out) * ((R(3) * vc - R(2) * vl) - vr) < R(0)) vp_out = R(3) * vc - R(2) * vl;
    }
}

// TVD minmod slope of a cell (solver/reconstruct.f90:110-118).
template <typename R>
__device__ __forceinline__ R tvd_slope(R vm, R vc, R vp, R cf, R cb) {
    const R dqf = (R(2) * (vp - vc)) / cf;
    const R dqb = (R(2) * (vc - vm)) / cb;
    return (R(0.5) * (copysign(R(1), dqf) + copysign(R(1), dqb))) * fmin(fabs(dqf), fabs(dqb));
}

// ---------------------------------------------------------------------------
// HLL Riemann solver at one face (solver/rsolver.f90:43-130)
// ---------------------------------------------------------------------------

// compute_signalspeed (solver/definition.f90:394-410)
template <typename R>
__device__ __forceinline__ R signalspeed(R cs, R bn, R bt1, R bt2, R rho) {
    const R a2 = cs * cs;
    const R a4 = a2 * a2;
    const R b2n = (bn * bn) / rho;
    const R b2t1 = (bt1 * bt1) / rho;
    const R b2t2 = (bt2 * bt2) / rho;
    const R b2 = (b2n + b2t1) + b2t2;
    const R b4 = b2 * b2;
    return sqrt(R(0.5) * ((a2 + b2) + sqrt(fmax(((a4 + b4) + (R(2) * b2) * a2) - (R(4) * a2) * b2n, R(0)))));
}

// compute_signalspeed with the quotients by rho formed as products with
// irho = 1/rho (the CUMC_FP64_FAST form: not bit-compatible with the reference)
template <typename R>
__device__ __forceinline__ R signalspeed_recip(R cs, R bn, R bt1, R bt2, R irho) {
    const R a2 = cs * cs;
    const R a4 = a2 * a2;
    const R b2n = (bn * bn) * irho;
    const R b2t1 = (bt1 * bt1) * irho;
    const R b2t2 = (bt2 * bt2) * irho;
    const R b2 = (b2n + b2t1) + b2t2;
    const R b4 = b2 * b2;
    return sqrt(R(0.5) * ((a2 + b2) + sqrt(fmax(((a4 + b4) + (R(2) * b2) * a2) - (R(4) * a2) * b2n, R(0)))));
}

// compute_roe (solver/definition.f90:387-392)
template <typename R>
__device__ __forceinline__ R roe_avg(R xl, R xr, R sl, R sr) {
    // sl, sr = sqrt(rhoL), sqrt(rhoR): the reference takes each DSQRT again
    // per call; the value is the same.
    return (sl * xl + sr * xr) / (sl + sr);
}

// compute_fluxhll (solver/definition.f90:380-385)
template <typename R>
__device__ __forceinline__ R fluxhll(R yl, R yr, R xl, R xr, R sl, R sr) {
    return ((sr * yl - sl * yr) + (sl * sr) * (xr - xl)) / (sr - sl);
}

// One side of the face (PtoU_MHD_face, solver/ptou_face.f90:34-88, and
// Ptof_MHD, solver/flux.f90:163-262), kept as the few scalars every conserved
// and flux component is formed from, so that the HLL combination below can
// form one component at a time (each with the reference's expression tree)
// instead of holding four 8-vectors live.
template <int DIR, typename R>
struct FaceSide {
    static constexpr int t1 = (DIR + 1) % 3, t2 = (DIR + 2) % 3;
    R rho, v[3], p, b[3], E, hb2, vdotb;
    struct GivenEps {};
    __device__ __forceinline__ FaceSide(const R w[8], R ggas)
        : FaceSide(w, (w[ITAU] / w[IRHO]) / (ggas - R(1)), GivenEps{}) {}
    // e: the side's specific internal energy, EOS_EPSILON (model/riemann/src/eos.f90:194)
    __device__ __forceinline__ FaceSide(const R w[8], R e, GivenEps) {
        rho = w[IRHO];
        v[0] = w[IVX]; v[1] = w[IVY]; v[2] = w[IVZ];
        p = w[ITAU];
        b[0] = w[IBX]; b[1] = w[IBY]; b[2] = w[IBZ];
        const R vsquare = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
        const R bsquare = (b[0] * b[0] + b[1] * b[1]) + b[2] * b[2];
        E = rho * (e + R(0.5) * vsquare) + R(0.5) * bsquare;
        hb2 = R(0.5) * bsquare;
        vdotb = (b[0] * v[0] + b[1] * v[1]) + b[2] * v[2];
    }
    // conserved component q
    __device__ __forceinline__ R u(int q) const {
        return q == IRHO ? rho : q <= IVZ ? v[q - IVX] * rho : q == ITAU ? E : b[q - IBX];
    }
    // flux component q along DIR (q != IBX+DIR, whose flux is 0)
    __device__ __forceinline__ R f(int q) const {
        const R vn = v[DIR], bn = b[DIR];
        if (q == IRHO) return rho * vn;
        if (q == IVX + DIR) return ((v[DIR] * rho * vn + p) + hb2) - bn * bn;
        if (q == IVX + t1) return v[t1] * rho * vn - bn * b[t1];
        if (q == IVX + t2) return v[t2] * rho * vn - bn * b[t2];
        if (q == ITAU) return (E * vn + (p + hb2) * vn) - bn * vdotb;
        if (q == IBX + t1) return vn * b[t1] - v[t1] * bn;
        return vn * b[t2] - v[t2] * bn;  // IBX + t2
    }
};

// HLL flux at a face from the left and right primitive states (8 each,
// natural order). out receives the 7 stored components: rho, rho v, E and
// the two tangential fields in natural (x, y, z) order.
//
// RECIP (the CUMC_FP64_FAST form, not bit-compatible with the reference):
// the 21 quotients of a face share five divisors (rho of either side,
// ggas - 1, the Roe weight sum, sR - sL), so each divisor's reciprocal is
// formed once and the quotients become products; the values differ from the
// reference's by a few units in the last place.
template <int DIR, typename R, bool RECIP = false>
__device__ __forceinline__ void hll_flux7(const R wl[8], const R wr[8], R ggas, R out[7]) {
    constexpr int ivn = IVX + DIR;
    constexpr int ibn = IBX + DIR, ibt1 = IBX + (DIR + 1) % 3, ibt2 = IBX + (DIR + 2) % 3;
    using Side = FaceSide<DIR, R>;
    R sL, sR;
    Side L = RECIP ? Side(wl, wl[ITAU] * (R(1) / wl[IRHO]) * (R(1) / (ggas - R(1))), typename Side::GivenEps{})
                   : Side(wl, ggas);
    Side Rs = RECIP ? Side(wr, wr[ITAU] * (R(1) / wr[IRHO]) * (R(1) / (ggas - R(1))), typename Side::GivenEps{})
                    : Side(wr, ggas);
    if (RECIP) {
        const R irL = R(1) / wl[IRHO], irR = R(1) / wr[IRHO];
        const R csL = sqrt((ggas * wl[ITAU]) * irL);
        const R csR = sqrt((ggas * wr[ITAU]) * irR);
        const R cfsL = signalspeed_recip(csL, wl[ibn], wl[ibt1], wl[ibt2], irL);
        const R cfsR = signalspeed_recip(csR, wr[ibn], wr[ibt1], wr[ibt2], irR);
        const R sqL = sqrt(wl[IRHO]), sqR = sqrt(wr[IRHO]);
        const R isq = R(1) / (sqL + sqR);
        const R ubar = (sqL * wl[ivn] + sqR * wr[ivn]) * isq;
        const R cbar = (sqL * cfsL + sqR * cfsR) * isq;
        sL = fmin(wl[ivn] - cfsL, ubar - cbar);
        sR = fmax(wr[ivn] + cfsR, ubar + cbar);
    } else {
        // EOS_SOUNDSPEED (model/riemann/src/eos.f90:168)
        const R csL = sqrt((ggas * wl[ITAU]) / wl[IRHO]);
        const R csR = sqrt((ggas * wr[ITAU]) / wr[IRHO]);
        const R cfsL = signalspeed(csL, wl[ibn], wl[ibt1], wl[ibt2], wl[IRHO]);
        const R cfsR = signalspeed(csR, wr[ibn], wr[ibt1], wr[ibt2], wr[IRHO]);
        const R sqL = sqrt(wl[IRHO]), sqR = sqrt(wr[IRHO]);
        const R ubar = roe_avg(wl[ivn], wr[ivn], sqL, sqR);
        const R cbar = roe_avg(cfsL, cfsR, sqL, sqR);
        sL = fmin(wl[ivn] - cfsL, ubar - cbar);
        sR = fmax(wr[ivn] + cfsR, ubar + cbar);
    }
    constexpr int bt_a = DIR == 0 ? IBY : IBX;  // stored tangential components
    constexpr int bt_b = DIR == 2 ? IBY : IBZ;
    const int comp[7] = {IRHO, IVX, IVY, IVZ, ITAU, bt_a, bt_b};
    if (sL >= R(0)) {
#pragma unroll
        for (int c = 0; c < 7; ++c) out[c] = L.f(comp[c]);
    } else if (sL <= R(0) && sR >= R(0)) {
        if (RECIP) {
            const R ids = R(1) / (sR - sL);
#pragma unroll
            for (int c = 0; c < 7; ++c) {
                const R yl = L.f(comp[c]), yr = Rs.f(comp[c]), xl = L.u(comp[c]), xr = Rs.u(comp[c]);
                out[c] = ((sR * yl - sL * yr) + (sL * sR) * (xr - xl)) * ids;
            }
        } else {
#pragma unroll
            for (int c = 0; c < 7; ++c)
                out[c] = fluxhll(L.f(comp[c]), Rs.f(comp[c]), L.u(comp[c]), Rs.u(comp[c]), sL, sR);
        }
    } else {
#pragma unroll
        for (int c = 0; c < 7; ++c) out[c] = Rs.f(comp[c]);
    }
}

// ---------------------------------------------------------------------------
// CFL time step of one cell (finddt, solver/rungekutta.f90:201-250)
// ---------------------------------------------------------------------------

// the fast magnetosonic speed along each axis from the cell's primitives and
// bcell, then cfl * min(dx, dy, dz) / max_d(|v_d| + c_f,d); the inner square
// root has no MAX(., 0) guard, as in the reference. dxl, dyl, dzl are the
// cell's lengths along the three axes (cfl_lengths). Every caller of the CFL
// step (finddt, its fusion into stage 3, cumc_cfl_dt_static) evaluates this
// one function, so they give the same double.
__host__ __device__ __forceinline__ double cfl_cell_dt(double rho, double p, double vx, double vy, double vz,
                                                       double bcx, double bcy, double bcz, double dxl, double dyl,
                                                       double dzl, double ggas, double cfl) {
    const double cs = sqrt((ggas * p) / rho);
    const double a2 = cs * cs;
    const double a4 = a2 * a2;
    const double b2x = (bcx * bcx) / rho;
    const double b2y = (bcy * bcy) / rho;
    const double b2z = (bcz * bcz) / rho;
    const double b2 = (b2x + b2y) + b2z;
    const double b4 = b2 * b2;
    const double base = (a4 + (2.0 * a2) * b2) + b4;
    const double cfx = sqrt(0.5 * ((a2 + b2) + sqrt(base - (4.0 * a2) * b2x)));
    const double cfy = sqrt(0.5 * ((a2 + b2) + sqrt(base - (4.0 * a2) * b2y)));
    const double cfz = sqrt(0.5 * ((a2 + b2) + sqrt(base - (4.0 * a2) * b2z)));
    const double lambda = fmax(fmax(fabs(vx) + cfx, fabs(vy) + cfy), fabs(vz) + cfz);
    return (fmin(fmin(dxl, dyl), dzl) * cfl) / lambda;
}

// the cell's lengths along the axes (solver/rungekutta.f90:237-243): the
// widths, with dy -> r dy on cylindrical and spherical grids and
// dz -> r sin(theta) dz on spherical ones; xc is the cell-centre radius and
// sinyc the sine of the polar cell centre. coordinate: 1 Cartesian,
// 2 cylindrical, 3 spherical.
__host__ __device__ __forceinline__ void cfl_lengths(int coordinate, double xc, double sinyc, double& dyl,
                                                     double& dzl) {
    if (coordinate == 2) {
        dyl = xc * dyl;
    } else if (coordinate == 3) {
        dyl = xc * dyl;
        dzl = (xc * sinyc) * dzl;
    }
}

// ---------------------------------------------------------------------------
// geometry (solver/coords.f90) from the 1-D tables
// ---------------------------------------------------------------------------

// GEOM_FLUX (solver/coords.f90:231-302) for direction DIR at cell (j,k,l)
template <int COORD, int DIR>
__device__ __forceinline__ void geom_flux(const Tabs& T, int j, int k, int l, double& gp, double& gc, double& gm) {
    if (COORD == 1) {
        gp = 1.0;
        gm = 1.0;
        gc = DIR == 0 ? T.ax[0].d[j] : DIR == 1 ? T.ax[1].d[k] : T.ax[2].d[l];
    } else if (COORD == 2) {
        if (DIR == 0) { gp = T.ax[0].f[j]; gm = T.ax[0].f[j - 1]; gc = T.ax[0].c[j] * T.ax[0].d[j]; }
        else if (DIR == 1) { gp = 1.0; gm = 1.0; gc = T.ax[0].c[j] * T.ax[1].d[k]; }
        else { gp = 1.0; gm = 1.0; gc = T.ax[2].d[l]; }
    } else {
        if (DIR == 0) { gp = T.r2[j]; gm = T.r2[j - 1]; gc = T.r3d3[j]; }
        else if (DIR == 1) { gp = T.sinf[k]; gm = T.sinf[k - 1]; gc = T.rfac[j] * T.dcos[k]; }
        else { gp = 1.0; gm = 1.0; gc = ((T.rfac[j] * T.dcos[k]) * T.ax[2].d[l]) / T.ax[1].d[k]; }
    }
}

// GEOM_CT (solver/coords.f90:310-415)
struct CTf {
    double bx_ez_m, bx_ez_c, bx_ez_p, bx_ey_m, bx_ey_c, bx_ey_p;
    double by_ex_m, by_ex_c, by_ex_p, by_ez_m, by_ez_c, by_ez_p;
    double bz_ex_m, bz_ex_c, bz_ex_p, bz_ey_m, bz_ey_c, bz_ey_p;
};
template <int COORD>
__device__ __forceinline__ void geom_ct(const Tabs& T, int j, int k, int l, CTf& g) {
    const double dxl = T.ax[0].d[j], dyl = T.ax[1].d[k], dzl = T.ax[2].d[l];
    if (COORD == 1) {
        g.bx_ez_m = 1.0; g.bx_ez_c = dyl; g.bx_ez_p = 1.0;
        g.bx_ey_m = 1.0; g.bx_ey_c = dzl; g.bx_ey_p = 1.0;
        g.by_ex_m = 1.0; g.by_ex_c = dzl; g.by_ex_p = 1.0;
        g.by_ez_m = 1.0; g.by_ez_c = dxl; g.by_ez_p = 1.0;
        g.bz_ey_m = 1.0; g.bz_ey_c = dxl; g.bz_ey_p = 1.0;
        g.bz_ex_m = 1.0; g.bz_ex_c = dyl; g.bz_ex_p = 1.0;
    } else if (COORD == 2) {
        const double x = T.ax[0].c[j];
        g.bx_ez_m = 1.0; g.bx_ez_c = dyl * T.ax[0].f[j]; g.bx_ez_p = 1.0;
        g.bx_ey_m = 1.0; g.bx_ey_c = dzl; g.bx_ey_p = 1.0;
        g.by_ex_m = 1.0; g.by_ex_c = dzl; g.by_ex_p = 1.0;
        g.by_ez_m = 1.0; g.by_ez_c = dxl; g.by_ez_p = 1.0;
        g.bz_ey_m = T.ax[0].f[j - 1]; g.bz_ey_c = x * dxl; g.bz_ey_p = T.ax[0].f[j];
        g.bz_ex_m = 1.0; g.bz_ex_c = x * dyl; g.bz_ex_p = 1.0;
    } else {
        const double x = T.ax[0].c[j];
        const double dc = T.dcos[k];
        g.bx_ez_m = T.sinf[k - 1]; g.bx_ez_c = T.ax[0].f[j] * dc; g.bx_ez_p = T.sinf[k];
        g.bx_ey_m = 1.0; g.bx_ey_c = ((T.ax[0].f[j] * dc) * dzl) / dyl; g.bx_ey_p = 1.0;
        g.by_ex_m = 1.0; g.by_ex_c = (x * T.sinf[k]) * dzl; g.by_ex_p = 1.0;
        g.by_ez_m = T.ax[0].f[j - 1]; g.by_ez_c = x * dxl; g.by_ez_p = T.ax[0].f[j];
        g.bz_ey_m = T.ax[0].f[j - 1]; g.bz_ey_c = x * dxl; g.bz_ey_p = T.ax[0].f[j];
        g.bz_ex_m = 1.0; g.bz_ex_c = x * dyl; g.bz_ex_p = 1.0;
    }
}

// ---------------------------------------------------------------------------
// HLL of the mixed form (float states). The wave speeds and the two stored
// tangential-field components are formed in FP32, in the reciprocal form of
// hll_flux7 (five divisors, each reciprocal formed once); the five hydro
// components (rho, rho v, E) take their side fluxes, conserved values and HLL
// combination in FP64 from the FP32 states, with each side's internal energy,
// E, B^2/2 and v.B in FP64. Measured on Orszag-Tang 256^3 to t = 0.5, the
// all-FP32 form leaves the density 1.06e-5 (relative L1) from the FP64 run,
// this form 8.0e-6: the side fluxes' and the combination's FP32 rounding is
// the largest error left once the states are FP32.
//
// The FP64 quotients (by rho, by gamma-1, by sR-sL) start from the FP32
// reciprocal and take one Newton-Raphson step for 1/x, r' = r (2 - x r),
// which squares its relative error (6e-8 -> ~4e-15): FP64 accuracy without
// an FP64 division.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rcp_newton(double x, float r0) {
    const double r = (double)r0;
    return r * (2.0 - x * r);
}

// one side's flux (F) or conserved value (U) of component q, in T from the
// FP32 side primitives and the side's derived scalars
template <typename T, int DIR>
__device__ __forceinline__ T side_f(const FaceSide<DIR, float>& s, int q, double Ex, double hb2x, double vdotbx) {
    constexpr int t1 = (DIR + 1) % 3, t2 = (DIR + 2) % 3;
    const T rho = s.rho, vn = s.v[DIR], bn = s.b[DIR], p = s.p, hb2 = (T)hb2x, E = (T)Ex, vdotb = (T)vdotbx;
    if (q == IRHO) return rho * vn;
    if (q == IVX + DIR) return ((vn * rho * vn + p) + hb2) - bn * bn;
    if (q == IVX + t1) return (T)s.v[t1] * rho * vn - bn * (T)s.b[t1];
    if (q == IVX + t2) return (T)s.v[t2] * rho * vn - bn * (T)s.b[t2];
    if (q == ITAU) return (E * vn + (p + hb2) * vn) - bn * vdotb;
    if (q == IBX + t1) return vn * (T)s.b[t1] - (T)s.v[t1] * bn;
    return vn * (T)s.b[t2] - (T)s.v[t2] * bn;
}
template <typename T, int DIR>
__device__ __forceinline__ T side_u(const FaceSide<DIR, float>& s, int q, double Ex) {
    return q == IRHO ? (T)s.rho : q <= IVZ ? (T)s.v[q - IVX] * (T)s.rho : q == ITAU ? (T)Ex : (T)s.b[q - IBX];
}

// a side's internal energy, E, B^2/2 and v.B in FP64 from its FP32 primitives
// (the FaceSide expressions); irho32, ig32: FP32 reciprocals of rho and gamma-1
struct SideScalars {
    double E, hb2, vdotb;
};
__device__ __forceinline__ SideScalars side_scalars64(const float (&w)[8], float irho32, double ig) {
    const double rho = w[IRHO], vx = w[IVX], vy = w[IVY], vz = w[IVZ], bx = w[IBX], by = w[IBY], bz = w[IBZ];
    const double e = (double)w[ITAU] * rcp_newton(rho, irho32) * ig;
    const double vsq = (vx * vx + vy * vy) + vz * vz, bsq = (bx * bx + by * by) + bz * bz;
    return {rho * (e + 0.5 * vsq) + 0.5 * bsq, 0.5 * bsq, (bx * vx + by * vy) + bz * vz};
}

template <int DIR>
__device__ __forceinline__ void hll_flux7_mixed(const float (&wl)[8], const float (&wr)[8], float ggas,
                                                float (&out)[7]) {
    constexpr int ivn = IVX + DIR;
    constexpr int ibn = IBX + DIR, ibt1 = IBX + (DIR + 1) % 3, ibt2 = IBX + (DIR + 2) % 3;
    constexpr int HYDRO = 5;  // components 0..4 in FP64
    const float irL = 1.0f / wl[IRHO], irR = 1.0f / wr[IRHO];
    float sL, sR;
    {
        const float csL = sqrtf((ggas * wl[ITAU]) * irL);
        const float csR = sqrtf((ggas * wr[ITAU]) * irR);
        const float cfsL = signalspeed_recip<float>(csL, wl[ibn], wl[ibt1], wl[ibt2], irL);
        const float cfsR = signalspeed_recip<float>(csR, wr[ibn], wr[ibt1], wr[ibt2], irR);
        const float sqL = sqrtf(wl[IRHO]), sqR = sqrtf(wr[IRHO]);
        const float isq = 1.0f / (sqL + sqR);
        const float ubar = (sqL * wl[ivn] + sqR * wr[ivn]) * isq;
        const float cbar = (sqL * cfsL + sqR * cfsR) * isq;
        sL = fminf(wl[ivn] - cfsL, ubar - cbar);
        sR = fmaxf(wr[ivn] + cfsR, ubar + cbar);
    }
    using Side = FaceSide<DIR, float>;
    const float ig = 1.0f / (ggas - 1.0f);
    const double igd = rcp_newton((double)ggas - 1.0, ig);
    const SideScalars aL = side_scalars64(wl, irL, igd), aR = side_scalars64(wr, irR, igd);
    // the FP32 side (tangential-field components only read rho, v, b)
    const Side L(wl, wl[ITAU] * irL * ig, typename Side::GivenEps{});
    const Side Rs(wr, wr[ITAU] * irR * ig, typename Side::GivenEps{});
    constexpr int bt_a = DIR == 0 ? IBY : IBX;
    constexpr int bt_b = DIR == 2 ? IBY : IBZ;
    const int comp[7] = {IRHO, IVX, IVY, IVZ, ITAU, bt_a, bt_b};
    if (sL >= 0.0f) {
#pragma unroll
        for (int q = 0; q < 7; ++q)
            out[q] = q < HYDRO ? (float)side_f<double>(L, comp[q], aL.E, aL.hb2, aL.vdotb) : L.f(comp[q]);
    } else if (sR >= 0.0f) {
        const float idsf = 1.0f / (sR - sL), lrf = sL * sR;
        const double cl = sL, cr = sR, ids = rcp_newton(cr - cl, idsf), lr = cl * cr;
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            if (q < HYDRO) {
                const double yl = side_f<double>(L, comp[q], aL.E, aL.hb2, aL.vdotb);
                const double yr = side_f<double>(Rs, comp[q], aR.E, aR.hb2, aR.vdotb);
                const double xl = side_u<double>(L, comp[q], aL.E), xr = side_u<double>(Rs, comp[q], aR.E);
                out[q] = (float)(((cr * yl - cl * yr) + lr * (xr - xl)) * ids);
            } else {
                const float yl = L.f(comp[q]), yr = Rs.f(comp[q]), xl = L.u(comp[q]), xr = Rs.u(comp[q]);
                out[q] = ((sR * yl - sL * yr) + lrf * (xr - xl)) * idsf;
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < 7; ++q)
            out[q] = q < HYDRO ? (float)side_f<double>(Rs, comp[q], aR.E, aR.hb2, aR.vdotb) : Rs.f(comp[q]);
    }
}

// the sweeps' HLL solve: hll_flux7 in FP64 (RECIP: the CUMC_FP64_FAST form).
// For the mixed form's float states, RECIP selects the all-FP32 reciprocal
// form of hll_flux7 (faster; density 1.06e-5 from the FP64 run at t_end above)
// and its absence hll_flux7_mixed (the default).
template <int DIR, typename R, bool RECIP>
__device__ __forceinline__ void sweep_hll(const R (&wl)[8], const R (&wr)[8], R ggas, R (&fx)[7]) {
    if constexpr (sizeof(R) == 4) {
        if constexpr (RECIP) hll_flux7<DIR, R, true>(wl, wr, ggas, fx);
        else hll_flux7_mixed<DIR>(wl, wr, ggas, fx);
    } else {
        hll_flux7<DIR, R, RECIP>(wl, wr, ggas, fx);
    }
}

}  // namespace cumc
