// cumc_kernels.cuh — the per-stage kernels of the CUMC3D hot path.
//
// One SSP-RK3 stage (solver/rungekutta.f90:38-66) runs as
//   k_sweep<x>, k_sweep<y>, k_sweep<z>   face fluxes (GET_FLUXES interpolate + RIEMANN)
//   k_emf                                edge EMFs (GET_FLUXES EMF sums + flux_ct ecell/ecorn)
//   k_ct                                 CT curl + RK combine of the face fields
//   k_combine_utop                       flux difference + sources + RK combine of the hydro
//                                        cons, then FROMUTORVE, CUSTOM_CHECKRHO, FROMRVETOU,
//                                        UPDATE (interior)
//   k_boundary                           BOUNDARY (+CUSTOM_BOUNDARY) and UPDATE on the ghosts
// (k_combine stores l_rk for SPATIAL alone; k_utop serves initial_update.)
// The reference's intermediates primL/primR/consL/consR/fluxL/fluxR/l_rk/sc/
// ecell never reach HBM here; only the face fluxes and edge EMFs do.
#pragma once
#include "../../include/cumc.h"
#include "cumc_device.cuh"

namespace cumc {

template <typename R>
struct PrimT {         // stage-start primitive state (with ghosts), storage type R
    const R* w[5];     // rho, vx, vy, vz, p
    const R* bc[3];    // cell-centred B (bcell)
    const R* bf[3];    // face B (prim(ibx:ibz) == cons(ibx:ibz))
};
using Prim = PrimT<double>;

template <typename R>
struct FaceFluxT {     // fluxes of one direction, stored at the index of the face's left cell
    R* f[7];           // rho, mx, my, mz, E, B_t(first in x,y,z order), B_t(second)
};
using FaceFlux = FaceFluxT<double>;

struct Cons {
    double* u[8];
};

// ----------------------------------------------------------------------------
// k_sweep: HLL fluxes on the faces of one direction.
// Faces: normal index 0:n_d, transverse 0:n+1 (solver/spatial.f90:157-168,
// 235-246, 313-324). Each thread owns one face; it reconstructs the 5 hydro
// primitives and the 2 transverse cell-centred fields of the two adjacent
// cells (INTERPOLATE, solver/spatial.f90:131-154) and solves the Riemann
// problem (HLL_SOLVER).
// ----------------------------------------------------------------------------
template <int DIR, int RECON, typename R = double>
__global__ void __launch_bounds__(128) k_sweep(Box b, Tabs T, PrimT<R> pr, R ggas, FaceFluxT<R> out) {
    const int n0 = (DIR == 0 ? b.nx : b.nx + 1) + 1;
    const int n1 = (DIR == 1 ? b.ny : b.ny + 1) + 1;
    const int n2 = (DIR == 2 ? b.nz : b.nz + 1) + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total || (b.skip && *b.skip)) return;
    const int j = (int)(t % n0);
    const int k = (int)((t / n0) % n1);
    const int l = (int)(t / ((long long)n0 * n1));
    const int base = b.idx(j, k, l);
    const int s = DIR == 0 ? 1 : DIR == 1 ? b.SX : b.SX * b.SY;
    const int c = DIR == 0 ? j : DIR == 1 ? k : l;  // face between cell c and c+1
    const AxisTabs A = T.ax[DIR];

    // variables reconstructed along DIR, in natural order
    constexpr int bt_a = DIR == 0 ? 1 : 0;  // first transverse field component
    constexpr int bt_b = DIR == 2 ? 1 : 2;  // second transverse field component
    const R* src[7] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[bt_a], pr.bc[bt_b]};
    const int slot[7] = {IRHO, IVX, IVY, IVZ, ITAU, IBX + bt_a, IBX + bt_b};

    R wl[8], wr[8];
#pragma unroll
    for (int v = 0; v < 7; ++v) {
        const R* q = src[v] + base;
        R w[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) w[m] = q[(m - 2) * s];  // cells c-2 .. c+3
        R left, right;
        if (RECON == 4) {
            const R d1 = ppm_slope(w[0], w[1], w[2], (R)A.s0[c - 1], (R)A.s1[c - 1]);
            const R d2 = ppm_slope(w[1], w[2], w[3], (R)A.s0[c], (R)A.s1[c]);
            const R d3 = ppm_slope(w[2], w[3], w[4], (R)A.s0[c + 1], (R)A.s1[c + 1]);
            const R d4 = ppm_slope(w[3], w[4], w[5], (R)A.s0[c + 2], (R)A.s1[c + 2]);
            const R f0 = ppm_face(w[1], w[2], d1, d2, (R)A.a0[c - 1], (R)A.a1[c - 1], (R)A.a2[c - 1], (R)A.a3[c - 1]);
            const R f1 = ppm_face(w[2], w[3], d2, d3, (R)A.a0[c], (R)A.a1[c], (R)A.a2[c], (R)A.a3[c]);
            const R f2 = ppm_face(w[3], w[4], d3, d4, (R)A.a0[c + 1], (R)A.a1[c + 1], (R)A.a2[c + 1], (R)A.a3[c + 1]);
            R vm, vp;
            ppm_fix(w[2], f0, f1, vm, vp);
            left = vp;   // primL at face c = vp_out of cell c
            ppm_fix(w[3], f1, f2, vm, vp);
            right = vm;  // primR at face c = vm_out of cell c+1
        } else {
            const R sl = tvd_slope(w[1], w[2], w[3], (R)A.tcf[c], (R)A.tcb[c]);
            const R sr = tvd_slope(w[2], w[3], w[4], (R)A.tcf[c + 1], (R)A.tcb[c + 1]);
            left = w[2] + R(0.5) * sl;
            right = w[3] - R(0.5) * sr;
        }
        wl[slot[v]] = left;
        wr[slot[v]] = right;
    }
    // normal field: the shared face value (solver/spatial.f90:148-149)
    const R bn = pr.bf[DIR][base];
    wl[IBX + DIR] = bn;
    wr[IBX + DIR] = bn;

    R fx[7];
    sweep_hll<DIR, R, false>(wl, wr, ggas, fx);
#pragma unroll
    for (int i = 0; i < 7; ++i) out.f[i][base] = fx[i];
}

// ----------------------------------------------------------------------------
// k_emf: edge EMFs on 0:n (solver/spatial.f90:190-203,268-281,346-359 then
// solver/mhd.f90:95-125). ecorn is accumulated in the reference's sweep
// order starting from zero, then ecorn = 2*ecorn - average of the four cell
// EMFs E = -v x B.
// ----------------------------------------------------------------------------
template <typename R>
struct EdgeET {
    R* e[3];
};
using EdgeE = EdgeET<double>;

template <typename R>
__device__ __forceinline__ R ecell_x(const PrimT<R>& p, int i) { return p.w[3][i] * p.bc[1][i] - p.w[2][i] * p.bc[2][i]; }
template <typename R>
__device__ __forceinline__ R ecell_y(const PrimT<R>& p, int i) { return p.w[1][i] * p.bc[2][i] - p.w[3][i] * p.bc[0][i]; }
template <typename R>
__device__ __forceinline__ R ecell_z(const PrimT<R>& p, int i) { return p.w[2][i] * p.bc[0][i] - p.w[1][i] * p.bc[1][i]; }

template <typename R>
__global__ void __launch_bounds__(256) k_emf(Box b, PrimT<R> pr, FaceFluxT<R> fx, FaceFluxT<R> fy, FaceFluxT<R> fz,
                                             EdgeET<R> out) {
    const int n0 = b.nx + 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total || (b.skip && *b.skip)) return;
    const int j = (int)(t % n0);
    const int k = (int)((t / n0) % n1);
    const int l = (int)(t / ((long long)n0 * n1));
    const int i = b.idx(j, k, l);
    const int sj = 1, sk = b.SX, sl = b.SX * b.SY;
    // x-faces carry (by, bz) fluxes, y-faces (bx, bz), z-faces (bx, by)
    const R* Fx_by = fx.f[5]; const R* Fx_bz = fx.f[6];
    const R* Fy_bx = fy.f[5]; const R* Fy_bz = fy.f[6];
    const R* Fz_bx = fz.f[5]; const R* Fz_by = fz.f[6];
    const R q = R(0.25);
    R ex = R(0) + q * (-Fy_bz[i] - Fy_bz[i + sl]);
    ex = ex + q * (Fz_by[i] + Fz_by[i + sk]);
    R ey = R(0) + q * (Fx_bz[i] + Fx_bz[i + sl]);
    ey = ey + q * (-Fz_bx[i] - Fz_bx[i + sj]);
    R ez = R(0) + q * (-Fx_by[i] - Fx_by[i + sk]);
    ez = ez + q * (Fy_bx[i] + Fy_bx[i + sj]);
    ex = ex * R(2) - q * (((ecell_x(pr, i) + ecell_x(pr, i + sl)) + ecell_x(pr, i + sk)) + ecell_x(pr, i + sk + sl));
    ey = ey * R(2) - q * (((ecell_y(pr, i) + ecell_y(pr, i + sl)) + ecell_y(pr, i + sj)) + ecell_y(pr, i + sj + sl));
    ez = ez * R(2) - q * (((ecell_z(pr, i) + ecell_z(pr, i + sk)) + ecell_z(pr, i + sj)) + ecell_z(pr, i + sj + sk));
    out.e[0][i] = ex;
    out.e[1][i] = ey;
    out.e[2][i] = ez;
}

// CFL step of one interior cell (solver/rungekutta.f90:201-250)
template <int COORD>
__device__ __forceinline__ double cell_dt(const Tabs& T, int j, int k, int l, double rho, double p, double vx,
                                          double vy, double vz, double bcx, double bcy, double bcz, double ggas,
                                          double cfl) {
    double dyl = T.ax[1].d[k], dzl = T.ax[2].d[l];
    if (COORD != 1) cfl_lengths(COORD, T.ax[0].c[j], COORD == 3 ? T.sinc[k] : 0.0, dyl, dzl);
    return cfl_cell_dt(rho, p, vx, vy, vz, bcx, bcy, bcz, T.ax[0].d[j], dyl, dzl, ggas, cfl);
}

// block minimum of dt (every thread of the block calls it), then one 64-bit
// atomicMin on the non-negative bit pattern; fmin drops NaN, as MIN does for
// the reference's non-NaN path
__device__ __forceinline__ void block_min_dt(double dt, unsigned long long* dtmin) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dt;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 1.0e10;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0 && v >= 0.0) atomicMin(dtmin, (unsigned long long)__double_as_longlong(v));
    }
}

// ----------------------------------------------------------------------------
// The RK stage combine on (0:n)^3 (solver/rungekutta.f90:41-51,75-85,109-119).
// Hydro l_rk (interior only) is the x, y, z flux differences in that order
// plus the source (solver/spatial.f90:171-187,365-375); the field l_rk is the
// CT curl (solver/mhd.f90:130-153).
//
// Stages 1-3 run as two kernels. k_ct updates the face fields. k_combine_utop
// then combines the hydro cons in registers and converts them at once
// (FROMUTORVE, CUSTOM_CHECKRHO, P_to_U, UPDATE's pressure): the cell-centred
// field it needs averages face fields at i, i-1, i-SX and i-SX*SY, which k_ct
// has all written by then. The combined hydro cons therefore never make a
// round trip through HBM between the combine and the conversion. Every value
// is computed by the same expressions, in the same order, as the combine and
// k_utop would in sequence. k_combine (STAGE 0 only) stores l_rk for
// cumc_spatial.
// ----------------------------------------------------------------------------
struct CombineArgs {
    const double* u0[8];  // u_old
    const double* uc[8];  // cons entering the combine (stages 2 and 3)
    double* ud[8];        // result (may alias u0 or uc: pointwise)
    double* lrk[8];       // STAGE 0 output
    double* tape[8];      // when set: a copy of the combine's output, before the conversion
    const double* dt;     // device scalar
    const double* ecorn[3];
    int geom_repeat;
    double rho_floor, r_sh;
};

// source terms sc of cell (j, k, l) at index i (solver/spatial.f90:75-102:
// GEOM_SOURCE `geom_repeat` times, then CUSTOM_SOURCE) from the stage's
// primitives
template <int COORD, int MODEL>
__device__ __forceinline__ void cell_sources(const Tabs& T, const Prim& pr, int geom_repeat, double rho_floor,
                                             double r_sh, int j, int k, int l, int i, double* sc) {
#pragma unroll
    for (int q = 0; q < 5; ++q) sc[q] = 0.0;
    if (COORD == 1 && MODEL < 2) return;
    const double rho = pr.w[0][i], vx = pr.w[1][i], vy = pr.w[2][i], vz = pr.w[3][i], p = pr.w[4][i];
    const double bx = pr.bc[0][i], by = pr.bc[1][i], bz = pr.bc[2][i];
    const double x = T.ax[0].c[j];
    if (COORD == 2) {  // GEOM_SOURCE cylindrical (solver/coords.f90:127-136)
        const double bsquare = (bx * bx + by * by) + bz * bz;
        for (int r = 0; r < geom_repeat; ++r) {
            sc[IVX] = sc[IVX] + (((p + (rho * vy) * vy) + 0.5 * bsquare) - by * by) / (x);
            sc[IVY] = sc[IVY] - ((rho * vx) * vy - bx * by) / (x);
        }
    } else if (COORD == 3) {  // GEOM_SOURCE spherical (solver/coords.f90:139-161)
        const double bsquare = (bx * bx + by * by) + bz * bz;
        const double tany = T.tanc[k];
        for (int r = 0; r < geom_repeat; ++r) {
            sc[IVX] = sc[IVX] + ((2.0 * p + bx * bx) + rho * (vy * vy + vz * vz)) / (x);
            sc[IVY] = (sc[IVY] + (((p + (rho * vz) * vz) + 0.5 * bsquare) - bz * bz) / (x * tany)) -
                      ((rho * vx) * vy - bx * by) / (x);
            sc[IVZ] = (sc[IVZ] - ((rho * vx) * vz - bx * bz) / (x)) - ((rho * vy) * vz - by * bz) / (x * tany);
        }
    }
    if (MODEL == 2) {  // point-mass gravity (model/torus_sph/src/custom.f90:132-146)
        const double diff = rho - rho_floor;
        const double factor = fmax(copysign(1.0, diff), 0.0);
        const double dphidr = 1.0 / ((x - r_sh) * (x - r_sh));
        sc[IVX] = sc[IVX] + (((-factor) * rho) * dphidr);
        sc[ITAU] = sc[ITAU] + ((((-factor) * rho) * vx) * dphidr);
    } else if (MODEL == 3) {  // gravity in (R, z) (model/torus_cyn/src/custom.f90)
        const double z = T.ax[2].c[l];
        const double diff = rho - rho_floor;
        const double factor = fmax(copysign(1.0, diff), 0.0);
        const double radius = sqrt(x * x + z * z);
        const double dphidr = (x / radius) / ((radius - r_sh) * (radius - r_sh));
        const double dphidz = (z / radius) / ((radius - r_sh) * (radius - r_sh));
        sc[IVX] = sc[IVX] + (((-factor) * rho) * dphidr);
        sc[IVZ] = sc[IVZ] + (((-factor) * rho) * dphidz);
        sc[ITAU] = sc[ITAU] + (((-factor) * rho) * (vx * dphidr + vz * dphidz));
    }
}

// one direction's share of a cell's hydro l_rk: the flux difference of the
// faces above (fp) and below (fm) with the geometry factors of GEOM_FLUX
// (solver/spatial.f90:171-187)
__device__ __forceinline__ double flux_diff(double L, double fp, double fm, double gp, double gm, double gc) {
    return L - (fp * gp - fm * gm) / gc;
}

// hydro l_rk of cell (j, k, l): zero outside the interior; inside, the x, y, z
// flux differences in that order, then the sources (solver/spatial.f90:365-375)
template <int COORD, int MODEL>
__device__ __forceinline__ void hydro_lrk(const Tabs& T, const Prim& pr, const FaceFlux& fx, const FaceFlux& fy,
                                          const FaceFlux& fz, const CombineArgs& a, int j, int k, int l, int i,
                                          int sk, int sl, double* L) {
    constexpr int sj = 1;
#pragma unroll
    for (int q = 0; q < 5; ++q) L[q] = 0.0;
    if (j >= 1 && k >= 1 && l >= 1) {
        double gp, gc, gm;
        geom_flux<COORD, 0>(T, j, k, l, gp, gc, gm);
#pragma unroll
        for (int q = 0; q < 5; ++q) L[q] = flux_diff(L[q], fx.f[q][i], fx.f[q][i - sj], gp, gm, gc);
        geom_flux<COORD, 1>(T, j, k, l, gp, gc, gm);
#pragma unroll
        for (int q = 0; q < 5; ++q) L[q] = flux_diff(L[q], fy.f[q][i], fy.f[q][i - sk], gp, gm, gc);
        geom_flux<COORD, 2>(T, j, k, l, gp, gc, gm);
#pragma unroll
        for (int q = 0; q < 5; ++q) L[q] = flux_diff(L[q], fz.f[q][i], fz.f[q][i - sl], gp, gm, gc);

        double sc[5];
        cell_sources<COORD, MODEL>(T, pr, a.geom_repeat, a.rho_floor, a.r_sh, j, k, l, i, sc);
#pragma unroll
        for (int q = 0; q < 5; ++q) L[q] = L[q] + sc[q];
    }
}

template <int COORD>
__device__ __forceinline__ void ct_lrk(const Tabs& T, const double* const* ecorn, int j, int k, int l, int i, int sk,
                                       int sl, double* L) {
    constexpr int sj = 1;
    CTf g;
    geom_ct<COORD>(T, j, k, l, g);
    const double* Ex = ecorn[0];
    const double* Ey = ecorn[1];
    const double* Ez = ecorn[2];
    L[0] = -((Ez[i] * g.bx_ez_p - Ez[i - sk] * g.bx_ez_m) / g.bx_ez_c -
             (Ey[i] * g.bx_ey_p - Ey[i - sl] * g.bx_ey_m) / g.bx_ey_c);
    L[1] = -((Ex[i] * g.by_ex_p - Ex[i - sl] * g.by_ex_m) / g.by_ex_c -
             (Ez[i] * g.by_ez_p - Ez[i - sj] * g.by_ez_m) / g.by_ez_c);
    L[2] = -((Ey[i] * g.bz_ey_p - Ey[i - sj] * g.bz_ey_m) / g.bz_ey_c -
             (Ex[i] * g.bz_ex_p - Ex[i - sk] * g.bz_ex_m) / g.bz_ex_c);
}

// u_new of one value for RK stage STAGE (u_c is not read at stage 1)
template <int STAGE>
__device__ __forceinline__ double rk_point(double u0, double uc, double dt, double L) {
    constexpr double rk20 = 3.0 / 4.0, rk21 = 1.0 / 4.0, rk22 = 1.0 / 4.0;
    constexpr double rk30 = 1.0 / 3.0, rk31 = 2.0 / 3.0, rk32 = 2.0 / 3.0;
    if (STAGE == 1) return u0 + dt * L;
    if (STAGE == 2) return (rk20 * u0 + rk21 * uc) + (rk22 * dt) * L;
    return (rk30 * u0 + rk31 * uc) + (rk32 * dt) * L;
}

// flat thread index -> (j, k, l) on (0:n)^3; false past the end or when skipped
__device__ __forceinline__ bool box1_index(const Box& b, int& j, int& k, int& l, int& i) {
    const int n0 = b.nx + 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total || (b.skip && *b.skip)) return false;
    j = (int)(t % n0);
    k = (int)((t / n0) % n1);
    l = (int)(t / ((long long)n0 * n1));
    i = b.idx(j, k, l);
    return true;
}

// SPATIAL alone (cumc_spatial): l_rk of all 8 variables
template <int COORD, int MODEL>
__global__ void __launch_bounds__(256) k_combine(Box b, Tabs T, Prim pr, FaceFlux fx, FaceFlux fy, FaceFlux fz,
                                                 CombineArgs a) {
    int j, k, l, i;
    if (!box1_index(b, j, k, l, i)) return;
    const int sk = b.SX, sl = b.SX * b.SY;
    double L[8];
    hydro_lrk<COORD, MODEL>(T, pr, fx, fy, fz, a, j, k, l, i, sk, sl, L);
    ct_lrk<COORD>(T, a.ecorn, j, k, l, i, sk, sl, L + IBX);
#pragma unroll
    for (int q = 0; q < 8; ++q) a.lrk[q][i] = L[q];
}

// face fields of RK stage STAGE. Each thread reads u0, uc and writes ud at its
// own index only, so ud may alias u0 or uc.
// (8 blocks of 256 per SM: these two kernels wait on memory, and a full SM
// of warps hides more of it than 5 blocks without spills: 1.44 -> 1.23 ms and
// 0.47 -> 0.36 ms at 256^3)
template <int COORD, int STAGE>
__global__ void __launch_bounds__(256, 8) k_ct(Box b, Tabs T, CombineArgs a) {
    int j, k, l, i;
    if (!box1_index(b, j, k, l, i)) return;
    double L[3];
    ct_lrk<COORD>(T, a.ecorn, j, k, l, i, b.SX, b.SX * b.SY, L);
    const double dt = *a.dt;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double r = rk_point<STAGE>(a.u0[IBX + q][i], STAGE == 1 ? 0.0 : a.uc[IBX + q][i], dt, L[q]);
        a.ud[IBX + q][i] = r;
        if (a.tape[IBX + q]) a.tape[IBX + q][i] = r;
    }
}

// ----------------------------------------------------------------------------
// k_utop: on (0:n)^3, FROMUTORVE (solver/fromrvetou.f90:75-127, UtoP_MHD
// solver/utop.f90:33-68), CUSTOM_CHECKRHO (interior), FROMRVETOU's P_to_U
// (solver/ptou.f90:33-66) and UPDATE's pressure on the interior
// (solver/update.f90:27-35). FROM_CONS=false is initial_update: the
// primitives come from the uploaded model instead of from cons.
// ----------------------------------------------------------------------------
struct UtopArgs {
    double* u[8];       // cons: read, hydro part rewritten
    double* w[5];       // rho, vx, vy, vz, p
    double* bc[3];
    double* eps;
    double ggas, rho_floor, eps_floor;
    unsigned int* flag;  // bit 0: non-finite value seen
    unsigned long long* dtmin = nullptr;  // k_combine_utop, stage 3: the next step's CFL dt (finddt fused)
    double cfl = 0.0;
};

// bcell of cell i: the face-field average on the interior (solver/fromrvetou.f90
// :97-107, 40-50, stored), the stored bcell elsewhere
__device__ __forceinline__ void bcell_point(const Box& b, const UtopArgs& a, int i, bool interior, double& bx,
                                            double& by, double& bz) {
    if (interior) {
        bx = 0.5 * (a.u[IBX][i] + a.u[IBX][i - 1]);
        by = 0.5 * (a.u[IBY][i] + a.u[IBY][i - b.SX]);
        bz = 0.5 * (a.u[IBZ][i] + a.u[IBZ][i - b.SX * b.SY]);
        a.bc[0][i] = bx;
        a.bc[1][i] = by;
        a.bc[2][i] = bz;
    } else {
        bx = a.bc[0][i];
        by = a.bc[1][i];
        bz = a.bc[2][i];
    }
}

// the conversions of one cell as values: from the hydro cons uh and the cell
// field (FROMUTORVE's primitives, CUSTOM_CHECKRHO on the interior, P_to_U's
// cons and UPDATE's pressure); FROM_CONS false starts from the primitives
// rho, v and eps given in uh instead (initial_update)
struct CellConv {
    double u[5];      // cons after the floors
    double w[4];      // rho, vx, vy, vz
    double eps, p;    // p on the interior only
    bool bad;         // non-finite density, velocity or pressure (interior)
};
template <int MODEL, bool FROM_CONS>
__device__ __forceinline__ CellConv utop_of(const double* uh, bool interior, double bx, double by, double bz,
                                            double ggas, double rho_floor, double eps_floor) {
    CellConv o;
    const double bsquare = (bx * bx + by * by) + bz * bz;
    double rho, vx, vy, vz, e;
    if (FROM_CONS) {
        rho = uh[IRHO];
        vx = uh[IVX] / rho;
        vy = uh[IVY] / rho;
        vz = uh[IVZ] / rho;
        const double vsquare = (vx * vx + vy * vy) + vz * vz;
        e = (uh[ITAU] - 0.5 * bsquare) / rho - 0.5 * vsquare;
    } else {
        rho = uh[0];
        vx = uh[1];
        vy = uh[2];
        vz = uh[3];
        e = uh[4];
    }
    if (interior) {  // CUSTOM_CHECKRHO
        if (MODEL == 1) {
            e = fmax(e, 0.0);
        } else if (MODEL == 2 || MODEL == 3) {
            if (rho < rho_floor) rho = rho_floor;
            if (e < eps_floor) e = eps_floor;
        }
    }
    const double vsquare = (vx * vx + vy * vy) + vz * vz;
    o.u[IRHO] = rho;
    o.u[IVX] = vx * rho;
    o.u[IVY] = vy * rho;
    o.u[IVZ] = vz * rho;
    o.u[ITAU] = rho * (e + 0.5 * vsquare) + 0.5 * bsquare;
    o.w[0] = rho;
    o.w[1] = vx;
    o.w[2] = vy;
    o.w[3] = vz;
    o.eps = e;
    o.p = 0.0;
    o.bad = false;
    if (interior) {
        o.p = (rho * e) * (ggas - 1.0);  // EOS_PRESSURE
        o.bad = !(isfinite(o.p) && isfinite(vsquare) && isfinite(rho));
    }
    return o;
}

// the conversions of one cell; with FROM_CONS the hydro cons come in uh
template <int MODEL, bool FROM_CONS>
__device__ __forceinline__ void utop_point(const UtopArgs& a, int i, bool interior, const double* uh, double bx,
                                           double by, double bz, double* prim_out = nullptr) {
    double in[5];
    if (FROM_CONS) {
#pragma unroll
        for (int q = 0; q < 5; ++q) in[q] = uh[q];
    } else {
        in[0] = a.w[0][i];
        in[1] = a.w[1][i];
        in[2] = a.w[2][i];
        in[3] = a.w[3][i];
        in[4] = a.eps[i];
    }
    const CellConv o = utop_of<MODEL, FROM_CONS>(in, interior, bx, by, bz, a.ggas, a.rho_floor, a.eps_floor);
#pragma unroll
    for (int q = 0; q < 5; ++q) a.u[q][i] = o.u[q];
#pragma unroll
    for (int q = 0; q < 4; ++q) a.w[q][i] = o.w[q];
    a.eps[i] = o.eps;
    if (interior) {
        a.w[4][i] = o.p;
        if (o.bad) atomicOr(a.flag, 1u);
        if (prim_out) {
            prim_out[0] = o.w[0];
            prim_out[1] = o.w[1];
            prim_out[2] = o.w[2];
            prim_out[3] = o.w[3];
            prim_out[4] = o.p;
        }
    }
}

template <int MODEL, bool FROM_CONS>
__global__ void __launch_bounds__(256) k_utop(Box b, UtopArgs a) {
    int j, k, l, i;
    if (!box1_index(b, j, k, l, i)) return;
    const bool interior = j >= 1 && k >= 1 && l >= 1;
    double bx, by, bz;
    bcell_point(b, a, i, interior, bx, by, bz);
    double uh[5];
    if (FROM_CONS) {
#pragma unroll
        for (int q = 0; q < 5; ++q) uh[q] = a.u[q][i];
    }
    utop_point<MODEL, FROM_CONS>(a, i, interior, uh, bx, by, bz);
}

// hydro part of RK stage STAGE and the conversions, after k_ct of the same
// stage. o.u is a.ud; w, bc and eps of o are the arrays pr reads, each at the
// thread's own index only, before the thread writes them.
// At stage 3, when o.dtmin is set, the kernel also forms the next step's CFL
// dt from the primitives it has just made (the finddt of the following main-
// loop iteration, solver/main.f90:130, fused): every thread then stays to
// the block's min reduction.
template <int COORD, int MODEL, int STAGE>
__global__ void __launch_bounds__(256, 8) k_combine_utop(Box b, Tabs T, Prim pr, FaceFlux fx, FaceFlux fy, FaceFlux fz,
                                                      CombineArgs a, UtopArgs o) {
    if (b.skip && *b.skip) return;
    int j, k, l, i;
    const bool live = box1_index(b, j, k, l, i);
    const bool fuse_dt = STAGE == 3 && o.dtmin;
    if (!live && !fuse_dt) return;
    double dt_cell = 1.0e10;
    if (live) {
        double L[5];
        hydro_lrk<COORD, MODEL>(T, pr, fx, fy, fz, a, j, k, l, i, b.SX, b.SX * b.SY, L);
        const double dt = *a.dt;
        double uh[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            uh[q] = rk_point<STAGE>(a.u0[q][i], STAGE == 1 ? 0.0 : a.uc[q][i], dt, L[q]);
            if (a.tape[q]) a.tape[q][i] = uh[q];
        }
        const bool interior = j >= 1 && k >= 1 && l >= 1;
        double bx, by, bz;
        bcell_point(b, o, i, interior, bx, by, bz);
        double pw[5];
        utop_point<MODEL, true>(o, i, interior, uh, bx, by, bz, fuse_dt ? pw : nullptr);
        if (fuse_dt && interior)
            dt_cell = cell_dt<COORD>(T, j, k, l, pw[0], pw[4], pw[1], pw[2], pw[3], bx, by, bz, o.ggas, o.cfl);
    }
    if (fuse_dt) block_min_dt(dt_cell, o.dtmin);
}

// k_combine_utop on two cells of a row per thread: cells j and j+1 with j
// even, so that with an even row stride SX every pair index i = idx(j, k, l)
// is even and each array is read and written as 16-byte pairs. The x
// neighbour i-1 comes from the pair at i-2; the y and z neighbours i-SX and
// i-SX*SY are pairs too. Every cell's value is the same expression, in the
// same order, as in k_combine_utop (flux_diff, rk_point, utop_of), so the
// results are bit for bit the scalar kernel's. A pair whose second cell lies
// past nx (odd number of cells in the row) reads that in-box ghost index and
// stores only the first cell; cells outside the interior keep their stored
// bcell and pressure as in the scalar kernel. Needs SX even and every array
// 16-byte aligned (checked by the launcher, which otherwise uses the scalar
// kernel).
__device__ __forceinline__ double2 ld2(const double* p, int i) {
    return *reinterpret_cast<const double2*>(p + i);
}
__device__ __forceinline__ void st2(double* p, int i, double x, double y) {
    *reinterpret_cast<double2*>(p + i) = make_double2(x, y);
}

template <int COORD, int MODEL, int STAGE>
__global__ void __launch_bounds__(256, 4) k_combine_utop2(Box b, Tabs T, Prim pr, FaceFlux fx, FaceFlux fy,
                                                       FaceFlux fz, CombineArgs a, UtopArgs o) {
    if (b.skip && *b.skip) return;
    const int np = (b.nx + 2) >> 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = t < (long long)np * n1 * n2;
    const bool fuse_dt = STAGE == 3 && o.dtmin;
    if (!live && !fuse_dt) return;
    double dt_cell = 1.0e10;
    if (live) {
        const int j = (int)(t % np) * 2, k = (int)((t / np) % n1), l = (int)(t / ((long long)np * n1));
        const int i = b.idx(j, k, l);
        const int sk = b.SX, sl = b.SX * b.SY;
        const bool two = j + 1 <= b.nx;
        const bool kl = k >= 1 && l >= 1;
        const bool in0 = kl && j >= 1, in1 = kl && two;  // interior cells of the pair
        double L0[5], L1[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) L0[q] = L1[q] = 0.0;
        if (kl) {
            double gp0, gc0, gm0, gp1, gc1, gm1;
            geom_flux<COORD, 0>(T, j, k, l, gp0, gc0, gm0);
            geom_flux<COORD, 0>(T, j + 1, k, l, gp1, gc1, gm1);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double2 c = ld2(fx.f[q], i), m = ld2(fx.f[q], i - 2);
                L0[q] = flux_diff(L0[q], c.x, m.y, gp0, gm0, gc0);
                L1[q] = flux_diff(L1[q], c.y, c.x, gp1, gm1, gc1);
            }
            geom_flux<COORD, 1>(T, j, k, l, gp0, gc0, gm0);
            geom_flux<COORD, 1>(T, j + 1, k, l, gp1, gc1, gm1);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double2 c = ld2(fy.f[q], i), m = ld2(fy.f[q], i - sk);
                L0[q] = flux_diff(L0[q], c.x, m.x, gp0, gm0, gc0);
                L1[q] = flux_diff(L1[q], c.y, m.y, gp1, gm1, gc1);
            }
            geom_flux<COORD, 2>(T, j, k, l, gp0, gc0, gm0);
            geom_flux<COORD, 2>(T, j + 1, k, l, gp1, gc1, gm1);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double2 c = ld2(fz.f[q], i), m = ld2(fz.f[q], i - sl);
                L0[q] = flux_diff(L0[q], c.x, m.x, gp0, gm0, gc0);
                L1[q] = flux_diff(L1[q], c.y, m.y, gp1, gm1, gc1);
            }
            double sc[5];
            if (in0) {
                cell_sources<COORD, MODEL>(T, pr, a.geom_repeat, a.rho_floor, a.r_sh, j, k, l, i, sc);
#pragma unroll
                for (int q = 0; q < 5; ++q) L0[q] = L0[q] + sc[q];
            } else {
#pragma unroll
                for (int q = 0; q < 5; ++q) L0[q] = 0.0;
            }
            if (in1) {
                cell_sources<COORD, MODEL>(T, pr, a.geom_repeat, a.rho_floor, a.r_sh, j + 1, k, l, i + 1, sc);
#pragma unroll
                for (int q = 0; q < 5; ++q) L1[q] = L1[q] + sc[q];
            } else {
#pragma unroll
                for (int q = 0; q < 5; ++q) L1[q] = 0.0;
            }
        }
        const double dt = *a.dt;
        double uh0[5], uh1[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double2 u0 = ld2(a.u0[q], i);
            const double2 uc = STAGE == 1 ? make_double2(0.0, 0.0) : ld2(a.uc[q], i);
            uh0[q] = rk_point<STAGE>(u0.x, uc.x, dt, L0[q]);
            uh1[q] = rk_point<STAGE>(u0.y, uc.y, dt, L1[q]);
            if (a.tape[q]) {
                if (two) st2(a.tape[q], i, uh0[q], uh1[q]);
                else a.tape[q][i] = uh0[q];
            }
        }
        // cell fields: the face averages on the interior, the stored bcell elsewhere
        double bx0, by0, bz0, bx1, by1, bz1;
        {
            const double2 fxc = ld2(o.u[IBX], i), fxm = ld2(o.u[IBX], i - 2);
            const double2 fyc = ld2(o.u[IBY], i), fym = ld2(o.u[IBY], i - sk);
            const double2 fzc = ld2(o.u[IBZ], i), fzm = ld2(o.u[IBZ], i - sl);
            double2 s0 = make_double2(0.0, 0.0), s1 = s0, s2 = s0;
            if (!(in0 && in1)) {
                s0 = ld2(o.bc[0], i);
                s1 = ld2(o.bc[1], i);
                s2 = ld2(o.bc[2], i);
            }
            bx0 = in0 ? 0.5 * (fxc.x + fxm.y) : s0.x;
            by0 = in0 ? 0.5 * (fyc.x + fym.x) : s1.x;
            bz0 = in0 ? 0.5 * (fzc.x + fzm.x) : s2.x;
            bx1 = in1 ? 0.5 * (fxc.y + fxc.x) : s0.y;
            by1 = in1 ? 0.5 * (fyc.y + fym.y) : s1.y;
            bz1 = in1 ? 0.5 * (fzc.y + fzm.y) : s2.y;
            if (in0 && in1) {
                st2(o.bc[0], i, bx0, bx1);
                st2(o.bc[1], i, by0, by1);
                st2(o.bc[2], i, bz0, bz1);
            } else if (in0) {
                o.bc[0][i] = bx0;
                o.bc[1][i] = by0;
                o.bc[2][i] = bz0;
            } else if (in1) {
                o.bc[0][i + 1] = bx1;
                o.bc[1][i + 1] = by1;
                o.bc[2][i + 1] = bz1;
            }
        }
        const CellConv c0 = utop_of<MODEL, true>(uh0, in0, bx0, by0, bz0, o.ggas, o.rho_floor, o.eps_floor);
        const CellConv c1 = utop_of<MODEL, true>(uh1, in1, bx1, by1, bz1, o.ggas, o.rho_floor, o.eps_floor);
        if (two) {
#pragma unroll
            for (int q = 0; q < 5; ++q) st2(o.u[q], i, c0.u[q], c1.u[q]);
#pragma unroll
            for (int q = 0; q < 4; ++q) st2(o.w[q], i, c0.w[q], c1.w[q]);
            st2(o.eps, i, c0.eps, c1.eps);
        } else {
#pragma unroll
            for (int q = 0; q < 5; ++q) o.u[q][i] = c0.u[q];
#pragma unroll
            for (int q = 0; q < 4; ++q) o.w[q][i] = c0.w[q];
            o.eps[i] = c0.eps;
        }
        if (in0 && in1) st2(o.w[4], i, c0.p, c1.p);
        else if (in0) o.w[4][i] = c0.p;
        else if (in1) o.w[4][i + 1] = c1.p;
        if ((in0 && c0.bad) || (in1 && c1.bad)) atomicOr(o.flag, 1u);
        if (fuse_dt) {
            if (in0)
                dt_cell = cell_dt<COORD>(T, j, k, l, c0.w[0], c0.p, c0.w[1], c0.w[2], c0.w[3], bx0, by0, bz0, o.ggas,
                                         o.cfl);
            if (in1)
                dt_cell = fmin(dt_cell, cell_dt<COORD>(T, j + 1, k, l, c1.w[0], c1.p, c1.w[1], c1.w[2], c1.w[3], bx1,
                                                       by1, bz1, o.ggas, o.cfl));
        }
    }
    if (fuse_dt) block_min_dt(dt_cell, o.dtmin);
}

// ----------------------------------------------------------------------------
// k_boundary: ghost shell of BOUNDARY (solver/boundary.f90:5-13) and UPDATE
// (solver/update.f90) on the ghosts.
//
// The reference fills x, then y, then z ghosts, each pass copying (with the
// parity signs bfac) from cells the previous passes already filled. Because
// each pass only reads indices inside 1:n along its own direction, the final
// value of any ghost equals the product of the three per-direction maps
// applied to one active cell. Each thread therefore gathers its ghost
// directly from active cells; no ghost is read, so one launch suffices.
// Face fields: only the components tangential to a ghost direction are
// filled (solver/boundary.f90:372-373,472-473,572-573); normal components
// outside 0:n along their own axis are never read and are left alone.
// ----------------------------------------------------------------------------
template <typename R>
struct BoundArgsT {
    R* w[5];
    R* bc[3];
    double* eps;            // FP64 path: gathered, then p = rho*eps*(ggas-1); mixed path: null, p gathered
    R* bf[3];
    int flag[6];            // boundary_flag
    int eps_yout;           // effective y-outer flag of BOUNDARY1D (solver/boundary.f90:211)
    signed char fac[6][8];  // bfac_xin, xout, yin, yout, zin, zout (solver/setup.f90:121-230)
    double ggas;
};

// source index and sign of one direction's ghost map; returns false if the
// index is active (identity)
__device__ __forceinline__ bool gmap(int i, int n, int fin, int fout, int& src, int& side) {
    if (i < 1) {
        side = 0;
        src = fin == 0 ? i + n : fin == 1 ? 1 : 1 - i;
        return true;
    }
    if (i > n) {
        side = 1;
        src = fout == 0 ? i - n : fout == 1 ? n : 2 * n + 1 - i;
        return true;
    }
    src = i;
    side = -1;
    return false;
}

using BoundArgs = BoundArgsT<double>;

template <int MODEL, typename R>
__global__ void __launch_bounds__(256) k_boundary(Box b, BoundArgsT<R> a) {
    const long long zsl = 6LL * b.SX * b.SY, ysl = 6LL * b.SX * b.nz, xsl = 6LL * b.ny * b.nz;
    if (b.skip && *b.skip) return;
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
        // the six x ghosts of a row on six consecutive threads, so that a warp
        // reads and writes a few row segments instead of 32 rows
        const int s = (int)(t % 6);
        const long long r = t / 6;
        j = s < 3 ? s - 2 : b.nx + s - 2;
        l = (int)(r / b.ny) + 1;
        k = (int)(r % b.ny) + 1;
    } else {
        return;
    }
    const int i = b.idx(j, k, l);
    int sj, sk, sl, dj, dk, dl;
    const bool gx = gmap(j, b.nx, a.flag[0], a.flag[1], sj, dj);
    const bool gy = gmap(k, b.ny, a.flag[2], a.flag[3], sk, dk);
    const bool gz = gmap(l, b.nz, a.flag[4], a.flag[5], sl, dl);
    // z ghost planes of a face shared with a neighbouring slab come from the
    // halo exchange; only Bz on the face l = 0 itself, a live face whose
    // x/y ghost copies are local, is filled here
    const bool exch = (l < 1 && a.flag[4] == CUMC_BC_EXCHANGE) || (l > b.nz && a.flag[5] == CUMC_BC_EXCHANGE);
    if (!exch) {
        // parity sign of equation q across the mapped directions (bfac is 1
        // except at reflecting faces, flags >= 2)
        auto sgn = [&](int q) -> int {
            int s = 1;
            if (gx && a.flag[dj] >= 2) s *= a.fac[dj][q];
            if (gy && a.flag[2 + dk] >= 2) s *= a.fac[2 + dk][q];
            if (gz && a.flag[4 + dl] >= 2) s *= a.fac[4 + dl][q];
            return s;
        };
        const int src = b.idx(sj, sk, sl);
        R w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const R v = a.w[q][src];
            w[q] = sgn(q) == 1 ? v : -v;
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const R v = a.bc[q][src];
            a.bc[q][i] = sgn(IBX + q) == 1 ? v : -v;
        }
        // torus ghost clamps (CUSTOM_BOUNDARY) act after all copies
        if (MODEL == 2 || MODEL == 3) {
            if (j < 1) w[1] = fmin(w[1], R(0));
            if (j > b.nx) w[1] = fmax(w[1], R(0));
        }
        if (MODEL == 3) {
            if (l < 1) w[3] = fmin(w[3], R(0));
            if (l > b.nz) w[3] = fmax(w[3], R(0));
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) a.w[q][i] = w[q];
        if (a.eps) {
            // eps: BOUNDARY1D with even parity; its y-outer branch keys on flag(3)
            int ej = j, ek = k, el = l, dd;
            gmap(j, b.nx, a.flag[0], a.flag[1], ej, dd);
            gmap(k, b.ny, a.flag[2], a.eps_yout, ek, dd);
            gmap(l, b.nz, a.flag[4], a.flag[5], el, dd);
            const double e = a.eps[b.idx(ej, ek, el)];
            a.eps[i] = e;
            a.w[4][i] = (R)(((double)w[0] * e) * (a.ggas - 1.0));  // UPDATE on the ghost
        } else {
            a.w[4][i] = a.w[4][src];  // pressure is even under every map
        }
        // tangential face fields
        if (j >= 0 && j <= b.nx && (gy || gz)) {  // Bx: map y and z only
            int s = 1;
            if (gy && a.flag[2 + dk] >= 2) s *= a.fac[2 + dk][IBX];
            if (gz && a.flag[4 + dl] >= 2) s *= a.fac[4 + dl][IBX];
            const R v = a.bf[0][b.idx(j, sk, sl)];
            a.bf[0][i] = s == 1 ? v : -v;
        }
        if (k >= 0 && k <= b.ny && (gx || gz)) {  // By: map x and z only
            int s = 1;
            if (gx && a.flag[dj] >= 2) s *= a.fac[dj][IBY];
            if (gz && a.flag[4 + dl] >= 2) s *= a.fac[4 + dl][IBY];
            const R v = a.bf[1][b.idx(sj, k, sl)];
            a.bf[1][i] = s == 1 ? v : -v;
        }
    }
    if (l >= 0 && l <= b.nz && (gx || gy)) {  // Bz: map x and y only
        int s = 1;
        if (gx && a.flag[dj] >= 2) s *= a.fac[dj][IBZ];
        if (gy && a.flag[2 + dk] >= 2) s *= a.fac[2 + dk][IBZ];
        const R v = a.bf[2][b.idx(sj, sk, l)];
        a.bf[2][i] = s == 1 ? v : -v;
    }
}

// ----------------------------------------------------------------------------
// k_finddt: CFL time step (solver/rungekutta.f90:201-261), block min then one
// 64-bit atomicMin on the (non-negative) bit pattern.
// ----------------------------------------------------------------------------
template <int COORD, typename R = double>
__global__ void __launch_bounds__(256) k_finddt(Box b, Tabs T, PrimT<R> pr, double ggas, double cfl,
                                                unsigned long long* dtmin) {
    if (b.skip && *b.skip) return;
    const long long total = (long long)b.nx * b.ny * b.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dt_out = 1.0e10;
    if (t < total) {
        const int j = (int)(t % b.nx) + 1;
        const int k = (int)((t / b.nx) % b.ny) + 1;
        const int l = (int)(t / ((long long)b.nx * b.ny)) + 1;
        const int i = b.idx(j, k, l);
        dt_out = cell_dt<COORD>(T, j, k, l, pr.w[0][i], (double)pr.w[4][i], pr.w[1][i], pr.w[2][i], pr.w[3][i],
                                pr.bc[0][i], pr.bc[1][i], pr.bc[2][i], ggas, cfl);
    }
    block_min_dt(dt_out, dtmin);
}

// ----------------------------------------------------------------------------
// small device-side scalar kernels for the time loop
// ----------------------------------------------------------------------------
struct Clock {
    double* dt;                // dt used by the stage kernels
    unsigned long long* dtmin; // finddt result (bit pattern)
    double* t;                 // simulation time
    int* steps;                // steps taken
    int* done;                 // 1 once t >= t_end
};

static __global__ void k_set_scalar(double* p, double v) { *p = v; }
static __global__ void k_reset_dtmin(unsigned long long* p) { *p = (unsigned long long)__double_as_longlong(1.0e10); }
// loop condition of solver/main.f90:127
static __global__ void k_check_done(Clock c, double t_end) { *c.done = (*c.t < t_end) ? 0 : 1; }
// dt = finddt, clipped to t_end (solver/main.f90:133-135)
static __global__ void k_clip_dt(Clock c, double t_end) {
    if (*c.done) return;
    double dt = __longlong_as_double((long long)*c.dtmin);
    const double t = *c.t;
    if (t + dt > t_end) dt = t_end - t;
    *c.dt = dt;
}
static __global__ void k_advance_time(Clock c) {
    if (*c.done) return;
    *c.t = *c.t + *c.dt;
    *c.steps = *c.steps + 1;
}

// ----------------------------------------------------------------------------
// layout transposes between the reference's AoS arrays and the SoA fields
// ----------------------------------------------------------------------------
static __global__ void k_aos_to_soa(long long n, int nv, const double* __restrict__ aos, double* const* soa) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    for (int v = 0; v < nv; ++v)
        if (soa[v]) soa[v][t] = aos[t * nv + v];
}
static __global__ void k_soa_to_aos(long long n, int nv, double* __restrict__ aos, const double* const* soa) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    for (int v = 0; v < nv; ++v) aos[t * nv + v] = soa[v] ? soa[v][t] : 0.0;
}

// ----------------------------------------------------------------------------
// find_divb (solver/mhd.f90:40-52) with GEOM_AREA (solver/coords.f90:173-223):
// per-block signed max, |div|max and the largest sum of |A B| over a cell's
// faces, combined on the host.
// ----------------------------------------------------------------------------
template <int COORD>
__global__ void __launch_bounds__(256) k_divb(Box b, Tabs T, const double* bx, const double* by, const double* bz,
                                              double* part) {
    const long long total = (long long)b.nx * b.ny * b.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double smax = -1.0e300, amax = 0.0, fmaxv = 0.0;
    if (t < total) {
        const int j = (int)(t % b.nx) + 1;
        const int k = (int)((t / b.nx) % b.ny) + 1;
        const int l = (int)(t / ((long long)b.nx * b.ny)) + 1;
        const int i = b.idx(j, k, l);
        const double dxl = T.ax[0].d[j], dyl = T.ax[1].d[k], dzl = T.ax[2].d[l];
        double axp, axm, ayp, aym, azp, azm;
        if (COORD == 1) {
            axp = dyl * dzl; axm = dyl * dzl;
            ayp = dxl * dzl; aym = dxl * dzl;
            azp = dxl * dyl; azm = dxl * dyl;
        } else if (COORD == 2) {
            axp = (T.ax[0].f[j] * dyl) * dzl;
            axm = (T.ax[0].f[j - 1] * dyl) * dzl;
            ayp = dxl * dzl; aym = dxl * dzl;
            azp = T.hr2[j] * dyl; azm = azp;
        } else {
            axp = (T.r2[j] * T.dcos[k]) * dzl;
            axm = (T.r2[j - 1] * T.dcos[k]) * dzl;
            ayp = (T.hr2[j] * T.sinf[k]) * dzl;
            aym = (T.hr2[j] * T.sinf[k - 1]) * dzl;
            azp = T.hr2[j] * dyl; azm = azp;
        }
        const double fxp = axp * bx[i], fxm = axm * bx[i - 1];
        const double fyp = ayp * by[i], fym = aym * by[i - b.SX];
        const double fzp = azp * bz[i], fzm = azm * bz[i - b.SX * b.SY];
        const double div = ((fxp - fxm) + (fyp - fym)) + (fzp - fzm);
        smax = div;
        amax = fabs(div);
        fmaxv = ((fabs(fxp) + fabs(fxm)) + (fabs(fyp) + fabs(fym))) + (fabs(fzp) + fabs(fzm));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
        amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        fmaxv = fmax(fmaxv, __shfl_xor_sync(0xffffffffu, fmaxv, o));
    }
    __shared__ double red[3][32];
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = smax;
        red[1][threadIdx.x >> 5] = amax;
        red[2][threadIdx.x >> 5] = fmaxv;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            smax = fmax(smax, red[0][w]);
            amax = fmax(amax, red[1][w]);
            fmaxv = fmax(fmaxv, red[2][w]);
        }
        part[3 * blockIdx.x + 0] = smax;
        part[3 * blockIdx.x + 1] = amax;
        part[3 * blockIdx.x + 2] = fmaxv;
    }
}

}  // namespace cumc
