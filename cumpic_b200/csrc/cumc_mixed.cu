// cumc_mixed.cu — mixed-precision form of the CUMC3D step (CUMC_MIXED).
//
// Compiled separately from the FP64 path, with FMA contraction (IEEE-rounded
// FP32 division and square root): nothing here is meant to be bit-compatible
// with the reference.
//
// What runs in which precision:
//   * reconstruction, the HLL wave speeds, the HLL flux of the tangential
//     fields, EMFs, flux differences, sources: FP32 (the sweep and EMF
//     templates shared with the FP64 path); the HLL flux of the five hydro
//     components is combined in FP64 from the FP32 states (hll_flux7_mixed,
//     cumc_walk.cuh), which halves the largest FP32 error left;
//   * the CT curl of the FP32 edge EMFs and the face-field increments: FP64,
//     so that div B stays at round-off;
//   * the RK3 accumulation of rho and rho v: U^n is kept as a hi/lo pair of
//     FP32 values and updated with Knuth's TwoSum and Dekker's FastTwoSum;
//     stage states are stored as the FP32 increment d_s = U_s - U^n, so their
//     rounding error scales with the increment, not with U;
//   * total energy and its stage combine, and the pressure recovery
//     p = (g-1) rho ((E - B^2/2)/rho - v^2/2) (solver/utop.f90:63-65), which
//     cancels catastrophically at low plasma beta: FP64.
// SSP-RK3 (solver/rungekutta.f90:46,80,114) in increment form:
//   d1 = dt L1,  d2 = (d1 + dt L2)/4,  U^{n+1} = U^n + 2/3 (d2 + dt L3)
// which equals u1 = u0 + dt L1, u2 = 3/4 u0 + 1/4 u1 + 1/4 dt L2,
// u3 = 1/3 u0 + 2/3 u2 + 2/3 dt L3 in exact arithmetic.
// A stage is the three sweeps, k_emf_ct_mx, k_combine_utop_mx and the
// boundary fill (CUMC_MX_STAGE=split runs k_emf, k_combine_mx and k_utop_mx
// instead, for A/B timing).
#include "cumc_mixed.h"
#include "cumc_emfct.cuh"
#include "cumc_sweep.cuh"
#include "cumc_walk.cuh"

namespace cumc {
namespace {

// Knuth's TwoSum: s + e == a + b exactly
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
// Dekker's FastTwoSum (|a| >= |b|)
__device__ __forceinline__ void fast_two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    e = __fsub_rn(b, __fsub_rn(s, a));
}
// (hi, lo) += x
__device__ __forceinline__ void df_add(float& hi, float& lo, float x) {
    float s, e;
    two_sum(hi, x, s, e);
    e = __fadd_rn(e, lo);
    fast_two_sum(s, e, hi, lo);
}
__device__ __forceinline__ void df_split(double v, float& hi, float& lo) {
    hi = __double2float_rn(v);
    lo = __double2float_rn(v - (double)hi);
}
__device__ __forceinline__ double df_val(float hi, float lo) { return (double)hi + (double)lo; }

// x / y in FP64 through the FP32 reciprocal of y and one Newton-Raphson step
// for 1/y (rcp_newton): within a few units in the last place of the IEEE
// quotient, without an FP64 division. The fused stage's CT curl and its
// conversions use it (0.90 -> 0.84 ms and 0.59 -> 0.54 ms a stage at 256^3);
// a build with CUMC_MX_IEEE_DIV defined takes the IEEE quotient instead.
__device__ __forceinline__ double qdiv(double x, double y) {
#ifdef CUMC_MX_IEEE_DIV
    return x / y;
#else
    return x * rcp_newton(y, 1.0f / (float)y);
#endif
}

template <typename K, typename... Args>
void run(const Launcher& L, int cls, dim3 grid, int block, size_t smem, K kern, Args... args) {
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return;
    if (L.pre) L.pre(L.user, cls);
    kern<<<grid, block, smem, L.stream>>>(args...);
    if (L.post) L.post(L.user, cls);
}
inline dim3 g1(long long n, int block) { return dim3((unsigned)((n + block - 1) / block)); }

// ---------------------------------------------------------------------------
// flux difference + sources + CT curl in FP32, then the increment-form combine
// ---------------------------------------------------------------------------
struct CombineMx {
    float* uh[8];
    float* ul[8];
    double* e0;
    float* d[8];
    double* db[3];
    double* es;
    const float* w[5];
    const float* bc[3];
    const float* ecorn[3];
    const double* dt;
    int geom_repeat;
    float rho_floor, r_sh;
};

// k_combine_mx and k_utop_mx wait on memory: 8 blocks of 256 per SM (a full
// SM of warps, a few registers spilled) beat 5 unspilled ones (1.05 -> 0.77 ms
// and 0.63 -> 0.54 ms at 256^3)
// hydro l_rk of cell (j, k, l) in FP32: flux differences and sources (zero
// outside the interior)
template <int COORD, int MODEL>
__device__ __forceinline__ void hydro_l_mx(const Box& b, const Tabs& T, const FaceFluxT<float>& fx,
                                           const FaceFluxT<float>& fy, const FaceFluxT<float>& fz, const CombineMx& a,
                                           int j, int k, int l, int i, float* L) {
    const int sj = 1, sk = b.SX, sl = b.SX * b.SY;
#pragma unroll
    for (int q = 0; q < 5; ++q) L[q] = 0.f;
    if (j >= 1 && k >= 1 && l >= 1) {
        double gp, gc, gm;
        geom_flux<COORD, 0>(T, j, k, l, gp, gc, gm);
        float fp = (float)gp, fm = (float)gm, fi = (float)(1.0 / gc);
#pragma unroll
        for (int q = 0; q < 5; ++q) L[q] -= (fx.f[q][i] * fp - fx.f[q][i - sj] * fm) * fi;
        geom_flux<COORD, 1>(T, j, k, l, gp, gc, gm);
        fp = (float)gp; fm = (float)gm; fi = (float)(1.0 / gc);
#pragma unroll
        for (int q = 0; q < 5; ++q) L[q] -= (fy.f[q][i] * fp - fy.f[q][i - sk] * fm) * fi;
        geom_flux<COORD, 2>(T, j, k, l, gp, gc, gm);
        fp = (float)gp; fm = (float)gm; fi = (float)(1.0 / gc);
#pragma unroll
        for (int q = 0; q < 5; ++q) L[q] -= (fz.f[q][i] * fp - fz.f[q][i - sl] * fm) * fi;
        const float rho = a.w[0][i], vx = a.w[1][i], vy = a.w[2][i], vz = a.w[3][i], p = a.w[4][i];
        const float bx = a.bc[0][i], by = a.bc[1][i], bz = a.bc[2][i];
        const float x = (float)T.ax[0].c[j];
        const float rep = (float)a.geom_repeat;
        if (COORD == 2) {
            const float bsq = bx * bx + by * by + bz * bz;
            L[IVX] += rep * ((p + rho * vy * vy + 0.5f * bsq - by * by) / x);
            L[IVY] -= rep * ((rho * vx * vy - bx * by) / x);
        } else if (COORD == 3) {
            const float bsq = bx * bx + by * by + bz * bz;
            const float tany = (float)T.tanc[k];
            L[IVX] += rep * ((2.f * p + bx * bx + rho * (vy * vy + vz * vz)) / x);
            L[IVY] += rep * ((p + rho * vz * vz + 0.5f * bsq - bz * bz) / (x * tany) - (rho * vx * vy - bx * by) / x);
            L[IVZ] -= rep * ((rho * vx * vz - bx * bz) / x + (rho * vy * vz - by * bz) / (x * tany));
        }
        if (MODEL == 2) {
            const float factor = rho >= a.rho_floor ? 1.f : 0.f;
            const float dphidr = 1.f / ((x - a.r_sh) * (x - a.r_sh));
            L[IVX] -= factor * rho * dphidr;
            L[ITAU] -= factor * rho * vx * dphidr;
        } else if (MODEL == 3) {
            const float z = (float)T.ax[2].c[l];
            const float factor = rho >= a.rho_floor ? 1.f : 0.f;
            const float radius = sqrtf(x * x + z * z);
            const float inv = 1.f / (radius * (radius - a.r_sh) * (radius - a.r_sh));
            L[IVX] -= factor * rho * x * inv;
            L[IVZ] -= factor * rho * z * inv;
            L[ITAU] -= factor * rho * (vx * x + vz * z) * inv;
        }
    }
}

#ifndef CUMC_MXC_MINB
#define CUMC_MXC_MINB 8
#endif
#ifndef CUMC_MXU_MINB
#define CUMC_MXU_MINB 8
#endif
template <int COORD, int MODEL, int STAGE>
__global__ void __launch_bounds__(256, CUMC_MXC_MINB) k_combine_mx(Box b, Tabs T, FaceFluxT<float> fx, FaceFluxT<float> fy,
                                                    FaceFluxT<float> fz, CombineMx a) {
    const int n0 = b.nx + 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total || (b.skip && *b.skip)) return;
    const int j = (int)(t % n0);
    const int k = (int)((t / n0) % n1);
    const int l = (int)(t / ((long long)n0 * n1));
    const int i = b.idx(j, k, l);
    const int sj = 1, sk = b.SX, sl = b.SX * b.SY;
    float L[8];
#pragma unroll
    for (int q = 5; q < 8; ++q) L[q] = 0.f;
    hydro_l_mx<COORD, MODEL>(b, T, fx, fy, fz, a, j, k, l, i, L);
    // CT curl of the FP32 edge EMFs, formed in FP64 (solver/mhd.f90:137-148)
    double LB[3];
    {
        CTf g;
        geom_ct<COORD>(T, j, k, l, g);
        const float* Ex = a.ecorn[0];
        const float* Ey = a.ecorn[1];
        const float* Ez = a.ecorn[2];
        auto e = [](const float* E, int at) { return (double)E[at]; };
        LB[0] = -((e(Ez, i) * g.bx_ez_p - e(Ez, i - sk) * g.bx_ez_m) / g.bx_ez_c -
                  (e(Ey, i) * g.bx_ey_p - e(Ey, i - sl) * g.bx_ey_m) / g.bx_ey_c);
        LB[1] = -((e(Ex, i) * g.by_ex_p - e(Ex, i - sl) * g.by_ex_m) / g.by_ex_c -
                  (e(Ez, i) * g.by_ez_p - e(Ez, i - sj) * g.by_ez_m) / g.by_ez_c);
        LB[2] = -((e(Ey, i) * g.bz_ey_p - e(Ey, i - sj) * g.bz_ey_m) / g.bz_ey_c -
                  (e(Ex, i) * g.bz_ex_p - e(Ex, i - sk) * g.bz_ex_m) / g.bz_ex_c);
    }
    const double dt = *a.dt;
    const float dtf = (float)dt;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        double* db = a.db[q];
        if (STAGE == 1) {
            db[i] = dt * LB[q];
        } else if (STAGE == 2) {
            db[i] = 0.25 * (db[i] + dt * LB[q]);
        } else {
            const double v = df_val(a.uh[IBX + q][i], a.ul[IBX + q][i]) + (2.0 / 3.0) * (db[i] + dt * LB[q]);
            float hi, lo;
            df_split(v, hi, lo);
            a.uh[IBX + q][i] = hi;
            a.ul[IBX + q][i] = lo;
        }
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        if (q == ITAU) continue;
        if (STAGE == 1) {
            a.d[q][i] = dtf * L[q];
        } else if (STAGE == 2) {
            a.d[q][i] = 0.25f * (a.d[q][i] + dtf * L[q]);
        } else {
            const float inc = (2.f / 3.f) * (a.d[q][i] + dtf * L[q]);
            float hi = a.uh[q][i], lo = a.ul[q][i];
            df_add(hi, lo, inc);
            a.uh[q][i] = hi;
            a.ul[q][i] = lo;
        }
    }
    const double LE = (double)L[ITAU];
    constexpr double rk20 = 3.0 / 4.0, rk21 = 1.0 / 4.0, rk22 = 1.0 / 4.0;
    constexpr double rk30 = 1.0 / 3.0, rk31 = 2.0 / 3.0, rk32 = 2.0 / 3.0;
    if (STAGE == 1) a.es[i] = a.e0[i] + dt * LE;
    else if (STAGE == 2) a.es[i] = (rk20 * a.e0[i] + rk21 * a.es[i]) + (rk22 * dt) * LE;
    else a.e0[i] = (rk30 * a.e0[i] + rk31 * a.es[i]) + (rk32 * dt) * LE;
}

// ---------------------------------------------------------------------------
// The fused stage (default): k_emf_ct_mx forms the FP32 edge EMFs of a tile
// in shared memory (the tiles and z march of k_emf_ct) and applies the CT
// curl in FP64 to the face-field increments; k_combine_utop_mx then forms
// the hydro combine of a cell in registers and converts it at once, as
// k_combine_mx followed by k_utop_mx would (the same expressions in the same
// order), so the hydro increments and the stage energy do not make a round
// trip through HBM between the two and the edge EMFs never reach it.
// ---------------------------------------------------------------------------
struct CtMx {
    float* uh[3];   // U^n face fields, high parts
    float* ul[3];   // low parts
    double* db[3];  // stage increments of the face fields
    const double* dt;
};

#ifndef CUMC_ECMX_MINB
#define CUMC_ECMX_MINB 6
#endif
template <int COORD, int STAGE>
__global__ void __launch_bounds__(EC_TX * EC_TY, CUMC_ECMX_MINB) k_emf_ct_mx(Box b, Tabs T, PrimT<float> pr, FaceFluxT<float> fx,
                                                               FaceFluxT<float> fy, FaceFluxT<float> fz, CtMx a,
                                                               int seg) {
    extern __shared__ __align__(16) unsigned char ecm_raw[];
    EmfCtSmemT<float>& S = *reinterpret_cast<EmfCtSmemT<float>*>(ecm_raw);
    if (b.skip && *b.skip) return;
    constexpr int NE = EC_EX * EC_EY, NT = EC_TX * EC_TY;
    const int j0 = blockIdx.x * EC_TX, k0 = blockIdx.y * EC_TY;
    const int l0 = blockIdx.z * seg, l1 = min(l0 + seg, b.nz + 1);
    const int tj = threadIdx.x % EC_TX, tk = threadIdx.x / EC_TX;
    const int j = j0 + tj, k = k0 + tk;
    const bool mine = j <= b.nx && k <= b.ny;
    const int e0 = threadIdx.x, e1 = threadIdx.x + NT;
    const double dt = *a.dt;

    ec_cells(b, pr, S, j0, k0, l0 - 1);
    ec_cells(b, pr, S, j0, k0, l0);
    __syncthreads();
    ec_edges(b, fx, fy, fz, S, j0, k0, l0 - 1, false);
    __syncthreads();
    for (int l = l0; l < l1; ++l) {
        const EdgePart<float> p0 = ec_edge_part(b, fx, fy, fz, j0, k0, l, e0);
        const EdgePart<float> p1 = e1 < NE ? ec_edge_part(b, fx, fy, fz, j0, k0, l, e1) : EdgePart<float>{0.f, 0.f, 0.f};
        const int i = b.idx(j, k, l);
        double dbv[3] = {0.0, 0.0, 0.0};
        float hv[3] = {0.f, 0.f, 0.f}, lv[3] = {0.f, 0.f, 0.f};
        if (mine) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (STAGE != 1) dbv[c] = a.db[c][i];
                if (STAGE == 3) {
                    hv[c] = a.uh[c][i];
                    lv[c] = a.ul[c][i];
                }
            }
        }
        ec_cells(b, pr, S, j0, k0, l + 1);
        __syncthreads();
        ec_edge_finish(b, S, p0, j0, k0, l, e0);
        if (e1 < NE) ec_edge_finish(b, S, p1, j0, k0, l, e1);
        __syncthreads();
        if (mine) {
            // CT curl of the FP32 edge EMFs, formed in FP64 (solver/mhd.f90:137-148)
            const int ej = tj + 1, ek = tk + 1, e = l & 1, em = (l - 1) & 1;
            const double Ez = S.ez[ek][ej], Ez_km = S.ez[ek - 1][ej], Ez_jm = S.ez[ek][ej - 1];
            const double Ey = S.ey[e][ek][ej], Ey_lm = S.ey[em][ek][ej], Ey_jm = S.ey[e][ek][ej - 1];
            const double Ex = S.ex[e][ek][ej], Ex_lm = S.ex[em][ek][ej], Ex_km = S.ex[e][ek - 1][ej];
            CTf g;
            geom_ct<COORD>(T, j, k, l, g);
            double LB[3];
            LB[0] = -(qdiv(Ez * g.bx_ez_p - Ez_km * g.bx_ez_m, g.bx_ez_c) -
                      qdiv(Ey * g.bx_ey_p - Ey_lm * g.bx_ey_m, g.bx_ey_c));
            LB[1] = -(qdiv(Ex * g.by_ex_p - Ex_lm * g.by_ex_m, g.by_ex_c) -
                      qdiv(Ez * g.by_ez_p - Ez_jm * g.by_ez_m, g.by_ez_c));
            LB[2] = -(qdiv(Ey * g.bz_ey_p - Ey_jm * g.bz_ey_m, g.bz_ey_c) -
                      qdiv(Ex * g.bz_ex_p - Ex_km * g.bz_ex_m, g.bz_ex_c));
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (STAGE == 1) {
                    a.db[c][i] = dt * LB[c];
                } else if (STAGE == 2) {
                    a.db[c][i] = 0.25 * (dbv[c] + dt * LB[c]);
                } else {
                    const double v = df_val(hv[c], lv[c]) + (2.0 / 3.0) * (dbv[c] + dt * LB[c]);
                    float hi, lo;
                    df_split(v, hi, lo);
                    a.uh[c][i] = hi;
                    a.ul[c][i] = lo;
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// conserved -> primitive with FP64 pressure recovery; floors; FP32 prims out
// ---------------------------------------------------------------------------
struct UtopMx {
    float* uh[8];
    float* ul[8];
    double* e0;
    float* d[8];
    double* db[3];
    double* es;
    float* w[5];
    float* bc[3];
    float* bf[3];
    double ggas, rho_floor, eps_floor;
    unsigned int* flag;
    unsigned long long* dtmin = nullptr;  // FINAL: the next step's CFL dt (finddt fused)
    double cfl = 0.0;
};

// FINAL: the state is U^n (after stage 3); otherwise U^n + d. With a.dtmin
// set (FINAL only) the kernel also forms the next step's CFL dt from the FP32
// primitives it stores, widened as k_finddt<float> reads them; every thread
// then stays to the block's min reduction.
// one cell (flat index t on (0:n)^3); returns its CFL dt when fuse_dt, else 1e10
template <int COORD, int MODEL, bool FINAL>
__device__ __forceinline__ double utop_mx_cell(const Box& b, const Tabs& T, const UtopMx& a, long long t, bool fuse_dt) {
    const int n0 = b.nx + 1, n1 = b.ny + 1;
    const int j = (int)(t % n0);
    const int k = (int)((t / n0) % n1);
    const int l = (int)(t / ((long long)n0 * n1));
    const int i = b.idx(j, k, l);
    const bool interior = j >= 1 && k >= 1 && l >= 1;
    auto U = [&](int q, int at) -> double {
        const double v = df_val(a.uh[q][at], a.ul[q][at]);
        if (FINAL) return v;
        return v + (q >= IBX ? a.db[q - IBX][at] : (double)a.d[q][at]);
    };
    const int off[3] = {1, b.SX, b.SX * b.SY};
    double bcv[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double face = U(IBX + q, i);
        a.bf[q][i] = (float)face;
        if (interior) {
            bcv[q] = 0.5 * (face + U(IBX + q, i - off[q]));
            a.bc[q][i] = (float)bcv[q];
        } else {
            bcv[q] = a.bc[q][i];
        }
    }
    const double bsq = (bcv[0] * bcv[0] + bcv[1] * bcv[1]) + bcv[2] * bcv[2];
    const double rho = U(IRHO, i);
    const double vx = U(IVX, i) / rho, vy = U(IVY, i) / rho, vz = U(IVZ, i) / rho;
    const double vsq = (vx * vx + vy * vy) + vz * vz;
    const double E = FINAL ? a.e0[i] : a.es[i];
    double e = (E - 0.5 * bsq) / rho - 0.5 * vsq;
    double rn = rho;
    bool changed = false;
    if (interior) {
        if (MODEL == 1) {
            if (e < 0.0) { e = 0.0; changed = true; }
        } else if (MODEL == 2 || MODEL == 3) {
            if (rn < a.rho_floor) { rn = a.rho_floor; changed = true; }
            if (e < a.eps_floor) { e = a.eps_floor; changed = true; }
        }
    }
    if (changed) {  // FROMRVETOU after CUSTOM_CHECKRHO: re-derive U from the floored prims
        const double un[4] = {rn, vx * rn, vy * rn, vz * rn};
        const double En = rn * (e + 0.5 * vsq) + 0.5 * bsq;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (FINAL) {
                float hi, lo;
                df_split(un[q], hi, lo);
                a.uh[q][i] = hi;
                a.ul[q][i] = lo;
            } else {
                a.d[q][i] = (float)(un[q] - df_val(a.uh[q][i], a.ul[q][i]));
            }
        }
        if (FINAL) a.e0[i] = En;
        else a.es[i] = En;
    }
    const double p = (rn * e) * (a.ggas - 1.0);
    a.w[0][i] = (float)rn;
    a.w[1][i] = (float)vx;
    a.w[2][i] = (float)vy;
    a.w[3][i] = (float)vz;
    double dt_cell = 1.0e10;
    if (interior) {
        a.w[4][i] = (float)p;
        if (!(isfinite(p) && isfinite(vsq) && isfinite(rn))) atomicOr(a.flag, 1u);
        if (fuse_dt)
            dt_cell = cell_dt<COORD>(T, j, k, l, (double)(float)rn, (double)(float)p, (double)(float)vx,
                                     (double)(float)vy, (double)(float)vz, (double)a.bc[0][i], (double)a.bc[1][i],
                                     (double)a.bc[2][i], a.ggas, a.cfl);
    }
    return dt_cell;
}

// the block reduction has one call site, which every thread of the block
// reaches (its warp shuffles and barrier need all of them)
template <int COORD, int MODEL, bool FINAL>
__global__ void __launch_bounds__(256, CUMC_MXU_MINB) k_utop_mx(Box b, Tabs T, UtopMx a) {
    const long long total = (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b.skip && *b.skip) return;  // the same for every thread
    const bool fuse_dt = FINAL && a.dtmin;
    if (t >= total && !fuse_dt) return;
    double dt_cell = 1.0e10;
    if (t < total) dt_cell = utop_mx_cell<COORD, MODEL, FINAL>(b, T, a, t, fuse_dt);
    if (fuse_dt) block_min_dt(dt_cell, a.dtmin);
}

// k_combine_mx's hydro part and k_utop_mx's conversion of one cell in one
// pass: the new increments (or, at stage 3, the new hi/lo state) and stage
// energy stay in registers between the two. The face fields come from
// k_emf_ct_mx, which has written all of them (the cell field averages the
// neighbours at i-1, i-SX and i-SX*SY). Every thread stays to the block's min
// reduction when the stage-3 launch forms the next step's dt.
#ifndef CUMC_CUMX_MINB
#define CUMC_CUMX_MINB 6
#endif
template <int COORD, int MODEL, int STAGE>
__global__ void __launch_bounds__(256, CUMC_CUMX_MINB) k_combine_utop_mx(Box b, Tabs T, FaceFluxT<float> fx, FaceFluxT<float> fy,
                                                         FaceFluxT<float> fz, CombineMx c, UtopMx a) {
    constexpr bool FINAL = STAGE == 3;
    const int n0 = b.nx + 1, n1 = b.ny + 1;
    const long long total = (long long)n0 * n1 * (b.nz + 1);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b.skip && *b.skip) return;
    const bool fuse_dt = FINAL && a.dtmin;
    if (t >= total && !fuse_dt) return;
    double dt_cell = 1.0e10;
    if (t < total) {
        const int j = (int)(t % n0);
        const int k = (int)((t / n0) % n1);
        const int l = (int)(t / ((long long)n0 * n1));
        const int i = b.idx(j, k, l);
        const bool interior = j >= 1 && k >= 1 && l >= 1;
        float L[5];
        hydro_l_mx<COORD, MODEL>(b, T, fx, fy, fz, c, j, k, l, i, L);
        const double dt = *c.dt;
        const float dtf = (float)dt;
        // the combine (k_combine_mx): new increments dn (stages 1, 2) or the new
        // hi/lo state (stage 3) of rho and rho v; the stage energy
        float uh4[4], ul4[4], dn[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uh4[q] = a.uh[q][i];
            ul4[q] = a.ul[q][i];
            if (STAGE == 1) {
                dn[q] = dtf * L[q];
            } else if (STAGE == 2) {
                dn[q] = 0.25f * (a.d[q][i] + dtf * L[q]);
            } else {
                const float inc = (2.f / 3.f) * (a.d[q][i] + dtf * L[q]);
                df_add(uh4[q], ul4[q], inc);
                dn[q] = 0.f;
            }
        }
        const double LE = (double)L[ITAU];
        constexpr double rk20 = 3.0 / 4.0, rk21 = 1.0 / 4.0, rk22 = 1.0 / 4.0;
        constexpr double rk30 = 1.0 / 3.0, rk31 = 2.0 / 3.0, rk32 = 2.0 / 3.0;
        double E;
        if (STAGE == 1) E = a.e0[i] + dt * LE;
        else if (STAGE == 2) E = (rk20 * a.e0[i] + rk21 * a.es[i]) + (rk22 * dt) * LE;
        else E = (rk30 * a.e0[i] + rk31 * a.es[i]) + (rk32 * dt) * LE;
        // the conversion (utop_mx_cell)
        auto U = [&](int q) -> double {
            const double v = df_val(uh4[q], ul4[q]);
            return FINAL ? v : v + (double)dn[q];
        };
        auto UB = [&](int q, int at) -> double {
            const double v = df_val(a.uh[IBX + q][at], a.ul[IBX + q][at]);
            return FINAL ? v : v + a.db[q][at];
        };
        const int off[3] = {1, b.SX, b.SX * b.SY};
        double bcv[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double face = UB(q, i);
            a.bf[q][i] = (float)face;
            if (interior) {
                bcv[q] = 0.5 * (face + UB(q, i - off[q]));
                a.bc[q][i] = (float)bcv[q];
            } else {
                bcv[q] = a.bc[q][i];
            }
        }
        const double bsq = (bcv[0] * bcv[0] + bcv[1] * bcv[1]) + bcv[2] * bcv[2];
        const double rho = U(IRHO);
        const double vx = qdiv(U(IVX), rho), vy = qdiv(U(IVY), rho), vz = qdiv(U(IVZ), rho);
        const double vsq = (vx * vx + vy * vy) + vz * vz;
        double e = qdiv(E - 0.5 * bsq, rho) - 0.5 * vsq;
        double rn = rho;
        bool changed = false;
        if (interior) {
            if (MODEL == 1) {
                if (e < 0.0) { e = 0.0; changed = true; }
            } else if (MODEL == 2 || MODEL == 3) {
                if (rn < a.rho_floor) { rn = a.rho_floor; changed = true; }
                if (e < a.eps_floor) { e = a.eps_floor; changed = true; }
            }
        }
        if (changed) {  // FROMRVETOU after CUSTOM_CHECKRHO: re-derive U from the floored prims
            const double un[4] = {rn, vx * rn, vy * rn, vz * rn};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (FINAL) {
                    df_split(un[q], uh4[q], ul4[q]);
                } else {
                    dn[q] = (float)(un[q] - df_val(uh4[q], ul4[q]));
                }
            }
            E = rn * (e + 0.5 * vsq) + 0.5 * bsq;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (FINAL) {
                a.uh[q][i] = uh4[q];
                a.ul[q][i] = ul4[q];
            } else {
                a.d[q][i] = dn[q];
            }
        }
        if (FINAL) a.e0[i] = E;
        else a.es[i] = E;
        const double p = (rn * e) * (a.ggas - 1.0);
        a.w[0][i] = (float)rn;
        a.w[1][i] = (float)vx;
        a.w[2][i] = (float)vy;
        a.w[3][i] = (float)vz;
        if (interior) {
            a.w[4][i] = (float)p;
            if (!(isfinite(p) && isfinite(vsq) && isfinite(rn))) atomicOr(a.flag, 1u);
            if (fuse_dt)
                dt_cell = cell_dt<COORD>(T, j, k, l, (double)(float)rn, (double)(float)p, (double)(float)vx,
                                         (double)(float)vy, (double)(float)vz, (double)(float)bcv[0],
                                         (double)(float)bcv[1], (double)(float)bcv[2], a.ggas, a.cfl);
        }
    }
    if (fuse_dt) block_min_dt(dt_cell, a.dtmin);
}

// initial_update from the uploaded FP64 model (AoS staging): CUSTOM_CHECKRHO,
// bcell, P_to_U into hi/lo + FP64 energy, FP32 prims
template <int MODEL>
__global__ void __launch_bounds__(256) k_initial_mx(Box b, UtopMx a, const double* __restrict__ prim,
                                                    const double* __restrict__ eps) {
    const int n0 = b.nx + 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long total = (long long)n0 * n1 * n2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int j = (int)(t % n0);
    const int k = (int)((t / n0) % n1);
    const int l = (int)(t / ((long long)n0 * n1));
    const int i = b.idx(j, k, l);
    const bool interior = j >= 1 && k >= 1 && l >= 1;
    const int off[3] = {1, b.SX, b.SX * b.SY};
    double bcv[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const double face = prim[8LL * i + IBX + q];
        float hi, lo;
        df_split(face, hi, lo);
        a.uh[IBX + q][i] = hi;
        a.ul[IBX + q][i] = lo;
        a.bf[q][i] = hi;
        if (interior) {
            bcv[q] = 0.5 * (face + prim[8LL * (i - off[q]) + IBX + q]);
            a.bc[q][i] = (float)bcv[q];
        } else {
            bcv[q] = 0.0;
        }
    }
    double rho = prim[8LL * i + IRHO];
    const double vx = prim[8LL * i + IVX], vy = prim[8LL * i + IVY], vz = prim[8LL * i + IVZ];
    double e = eps[i];
    if (interior) {
        if (MODEL == 1) e = fmax(e, 0.0);
        else if (MODEL == 2 || MODEL == 3) {
            if (rho < a.rho_floor) rho = a.rho_floor;
            if (e < a.eps_floor) e = a.eps_floor;
        }
    }
    const double bsq = (bcv[0] * bcv[0] + bcv[1] * bcv[1]) + bcv[2] * bcv[2];
    const double vsq = (vx * vx + vy * vy) + vz * vz;
    const double un[4] = {rho, vx * rho, vy * rho, vz * rho};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float hi, lo;
        df_split(un[q], hi, lo);
        a.uh[q][i] = hi;
        a.ul[q][i] = lo;
    }
    a.e0[i] = rho * (e + 0.5 * vsq) + 0.5 * bsq;
    a.w[0][i] = (float)rho;
    a.w[1][i] = (float)vx;
    a.w[2][i] = (float)vy;
    a.w[3][i] = (float)vz;
    const double p = (rho * e) * (a.ggas - 1.0);
    a.w[4][i] = (float)p;
    if (interior && !(isfinite(p) && isfinite(vsq) && isfinite(rho))) atomicOr(a.flag, 1u);
}

// state -> FP64 AoS in the reference layout
template <int WHAT>
__global__ void __launch_bounds__(256) k_export_mx(Box b, UtopMx a, double* __restrict__ out) {
    const long long n = b.count();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = (int)t;
    if (WHAT == 0) {  // prim
        for (int q = 0; q < 5; ++q) out[8 * t + q] = a.w[q][i];
        for (int q = 0; q < 3; ++q) out[8 * t + 5 + q] = a.bf[q][i];
    } else if (WHAT == 1) {  // cons
        for (int q = 0; q < 8; ++q)
            out[8 * t + q] = q == ITAU ? a.e0[i] : df_val(a.uh[q][i], a.ul[q][i]);
    } else if (WHAT == 2) {  // eps = p / rho / (g-1)
        out[t] = ((double)a.w[4][i] / (double)a.w[0][i]) / (a.ggas - 1.0);
    } else if (WHAT == 3) {
        for (int q = 0; q < 3; ++q) out[3 * t + q] = a.bc[q][i];
    } else {  // face fields as three SoA arrays
        for (int q = 0; q < 3; ++q) out[q * n + t] = df_val(a.uh[IBX + q][i], a.ul[IBX + q][i]);
    }
}

template <int DIR>
void sweep_mx(const Launcher& L, const Box& b, const Tabs& T, const PrimT<float>& pr, float ggas, const MixedBufs& m,
              int recon, int sm_count, bool fp32) {
    FaceFluxT<float> out;
    for (int q = 0; q < 7; ++q) out.f[q] = m.F[DIR][q];
    const bool ppm = recon == 4;
    if (DIR > 0) {  // column walker along y or z, window in shared memory
        constexpr int D = DIR > 0 ? DIR : 1;
        int nseg;
        const int seg = walk_segment_for<D>(b, WalkGeom<D>::ncols(b), sm_count, &nseg);
        const dim3 grid((unsigned)((WalkGeom<D>::ncols(b) + WK_THREADS - 1) / WK_THREADS), (unsigned)nseg);
        const size_t sm = walk_smem<float>(D);
        if (fp32)
            run(L, DIR, grid, WK_THREADS, sm,
                ppm ? k_sweep_walk_sm<D, 4, float, false, true> : k_sweep_walk_sm<D, 1, float, false, true>, b, T, pr,
                ggas, out, seg, out, 0, -1);
        else
            run(L, DIR, grid, WK_THREADS, sm, ppm ? k_sweep_walk_sm<D, 4, float> : k_sweep_walk_sm<D, 1, float>, b, T,
                pr, ggas, out, seg, out, 0, -1);
        return;
    }
    // x: one lane per cell
    const long long n = xwarp_threads(b);
    if (fp32)
        run(L, DIR, g1(n, 128), 128, 0, ppm ? k_sweep_xwarp<4, float, false, true> : k_sweep_xwarp<1, float, false, true>,
            b, T, pr, ggas, out, out, 0, -1);
    else
        run(L, DIR, g1(n, 128), 128, 0, ppm ? k_sweep_xwarp<4, float> : k_sweep_xwarp<1, float>, b, T, pr, ggas, out,
            out, 0, -1);
}

UtopMx utop_args(const MixedBufs& m, const MixedParams& p) {
    UtopMx a;
    for (int q = 0; q < 8; ++q) { a.uh[q] = m.uh[q]; a.ul[q] = m.ul[q]; a.d[q] = m.d[q]; }
    for (int q = 0; q < 3; ++q) a.db[q] = m.db[q];
    a.e0 = m.e0;
    a.es = m.es;
    for (int q = 0; q < 5; ++q) a.w[q] = m.w[q];
    for (int q = 0; q < 3; ++q) { a.bc[q] = m.bc[q]; a.bf[q] = m.bf[q]; }
    a.ggas = p.ggas;
    a.rho_floor = p.rho_floor;
    a.eps_floor = p.eps_floor;
    a.flag = m.flag;
    return a;
}

void boundary_mx(const Launcher& L, const Box& b, const MixedBufs& m, const MixedParams& p) {
    BoundArgsT<float> a;
    for (int q = 0; q < 5; ++q) a.w[q] = m.w[q];
    for (int q = 0; q < 3; ++q) { a.bc[q] = m.bc[q]; a.bf[q] = m.bf[q]; }
    a.eps = nullptr;
    for (int q = 0; q < 6; ++q) a.flag[q] = p.flag[q];
    a.eps_yout = p.eps_yout;
    for (int s = 0; s < 6; ++s)
        for (int q = 0; q < 8; ++q) a.fac[s][q] = p.fac[s][q];
    a.ggas = p.ggas;
    const long long n = 6LL * b.SX * b.SY + 6LL * b.SX * b.nz + 6LL * b.ny * b.nz;
    switch (p.model) {
        case 2: run(L, 6, g1(n, 256), 256, 0, k_boundary<2, float>, b, a); break;
        case 3: run(L, 6, g1(n, 256), 256, 0, k_boundary<3, float>, b, a); break;
        default: run(L, 6, g1(n, 256), 256, 0, k_boundary<0, float>, b, a); break;
    }
}

template <int COORD, int MODEL>
void combine_mx(const Launcher& L, const Box& b, const Tabs& T, const MixedBufs& m, const MixedParams& p, int stage) {
    FaceFluxT<float> ff[3];
    for (int d = 0; d < 3; ++d)
        for (int q = 0; q < 7; ++q) ff[d].f[q] = m.F[d][q];
    CombineMx a;
    for (int q = 0; q < 8; ++q) { a.uh[q] = m.uh[q]; a.ul[q] = m.ul[q]; a.d[q] = m.d[q]; }
    for (int q = 0; q < 3; ++q) a.db[q] = m.db[q];
    a.e0 = m.e0;
    a.es = m.es;
    for (int q = 0; q < 5; ++q) a.w[q] = m.w[q];
    for (int q = 0; q < 3; ++q) { a.bc[q] = m.bc[q]; a.ecorn[q] = m.E[q]; }
    a.dt = m.dt;
    a.geom_repeat = p.geom_repeat;
    a.rho_floor = (float)p.rho_floor;
    a.r_sh = (float)p.r_sh;
    const dim3 g = g1((long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256);
    if (stage == 1) run(L, 4, g, 256, 0, k_combine_mx<COORD, MODEL, 1>, b, T, ff[0], ff[1], ff[2], a);
    else if (stage == 2) run(L, 4, g, 256, 0, k_combine_mx<COORD, MODEL, 2>, b, T, ff[0], ff[1], ff[2], a);
    else run(L, 4, g, 256, 0, k_combine_mx<COORD, MODEL, 3>, b, T, ff[0], ff[1], ff[2], a);
}

template <int COORD>
void combine_model_mx(const Launcher& L, const Box& b, const Tabs& T, const MixedBufs& m, const MixedParams& p,
                      int stage) {
    switch (p.model) {
        case 0: combine_mx<COORD, 0>(L, b, T, m, p, stage); break;
        case 1: combine_mx<COORD, 1>(L, b, T, m, p, stage); break;
        case 2: combine_mx<COORD, 2>(L, b, T, m, p, stage); break;
        default: combine_mx<COORD, 3>(L, b, T, m, p, stage); break;
    }
}

CombineMx combine_args(const MixedBufs& m, const MixedParams& p) {
    CombineMx a;
    for (int q = 0; q < 8; ++q) { a.uh[q] = m.uh[q]; a.ul[q] = m.ul[q]; a.d[q] = m.d[q]; }
    for (int q = 0; q < 3; ++q) a.db[q] = m.db[q];
    a.e0 = m.e0;
    a.es = m.es;
    for (int q = 0; q < 5; ++q) a.w[q] = m.w[q];
    for (int q = 0; q < 3; ++q) { a.bc[q] = m.bc[q]; a.ecorn[q] = m.E[q]; }
    a.dt = m.dt;
    a.geom_repeat = p.geom_repeat;
    a.rho_floor = (float)p.rho_floor;
    a.r_sh = (float)p.r_sh;
    return a;
}

template <int COORD, int MODEL, int STAGE>
void fused_tail_t(const Launcher& L, const Box& b, const Tabs& T, const PrimT<float>& pr, const FaceFluxT<float>* ff,
                  const MixedBufs& m, const MixedParams& p, unsigned long long* dtmin) {
    CtMx ct;
    for (int q = 0; q < 3; ++q) {
        ct.uh[q] = m.uh[IBX + q];
        ct.ul[q] = m.ul[IBX + q];
        ct.db[q] = m.db[q];
    }
    ct.dt = m.dt;
    int seg;
    const dim3 g = emf_ct_grid(b, (long long)p.sm_count * CUMC_ECMX_MINB, &seg);
    run(L, CUMC_K_CT, g, EC_TX * EC_TY, sizeof(EmfCtSmemT<float>), k_emf_ct_mx<COORD, STAGE>, b, T, pr, ff[0], ff[1],
        ff[2], ct, seg);
    UtopMx a = utop_args(m, p);
    if (STAGE == 3 && dtmin) {  // the following iteration's finddt, fused (dtmin reset by the caller)
        a.dtmin = dtmin;
        a.cfl = p.cfl;
    }
    run(L, CUMC_K_COMBINE, g1((long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256), 256, 0,
        k_combine_utop_mx<COORD, MODEL, STAGE>, b, T, ff[0], ff[1], ff[2], combine_args(m, p), a);
}

template <int COORD, int MODEL>
void fused_tail_s(const Launcher& L, const Box& b, const Tabs& T, const PrimT<float>& pr, const FaceFluxT<float>* ff,
                  const MixedBufs& m, const MixedParams& p, int stage, unsigned long long* dtmin) {
    if (stage == 1) fused_tail_t<COORD, MODEL, 1>(L, b, T, pr, ff, m, p, dtmin);
    else if (stage == 2) fused_tail_t<COORD, MODEL, 2>(L, b, T, pr, ff, m, p, dtmin);
    else fused_tail_t<COORD, MODEL, 3>(L, b, T, pr, ff, m, p, dtmin);
}

template <int COORD>
void fused_tail_c(const Launcher& L, const Box& b, const Tabs& T, const PrimT<float>& pr, const FaceFluxT<float>* ff,
                  const MixedBufs& m, const MixedParams& p, int stage, unsigned long long* dtmin) {
    switch (p.model) {
        case 0: fused_tail_s<COORD, 0>(L, b, T, pr, ff, m, p, stage, dtmin); break;
        case 1: fused_tail_s<COORD, 1>(L, b, T, pr, ff, m, p, stage, dtmin); break;
        case 2: fused_tail_s<COORD, 2>(L, b, T, pr, ff, m, p, stage, dtmin); break;
        default: fused_tail_s<COORD, 3>(L, b, T, pr, ff, m, p, stage, dtmin); break;
    }
}

// the stage after the sweeps: k_emf_ct_mx, then k_combine_utop_mx
void fused_tail(const Launcher& L, const Box& b, const Tabs& T, const PrimT<float>& pr, const FaceFluxT<float>* ff,
                const MixedBufs& m, const MixedParams& p, int stage, unsigned long long* dtmin) {
    switch (p.coord) {
        case 1: fused_tail_c<1>(L, b, T, pr, ff, m, p, stage, dtmin); break;
        case 2: fused_tail_c<2>(L, b, T, pr, ff, m, p, stage, dtmin); break;
        default: fused_tail_c<3>(L, b, T, pr, ff, m, p, stage, dtmin); break;
    }
}

}  // namespace

cudaError_t mixed_attributes() {
    const void* k[6] = {(const void*)k_sweep_tile<0, 4, float>, (const void*)k_sweep_tile<1, 4, float>,
                        (const void*)k_sweep_tile<2, 4, float>, (const void*)k_sweep_tile<0, 1, float>,
                        (const void*)k_sweep_tile<1, 1, float>, (const void*)k_sweep_tile<2, 1, float>};
    for (const void* f : k) {
        cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw_smem<float>());
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void mixed_stage(const Launcher& L, const Box& b, const Tabs& T, const MixedBufs& m, const MixedParams& p, int stage,
                 unsigned long long* dtmin) {
    PrimT<float> pr;
    for (int q = 0; q < 5; ++q) pr.w[q] = m.w[q];
    for (int q = 0; q < 3; ++q) { pr.bc[q] = m.bc[q]; pr.bf[q] = m.bf[q]; }
    const float ggas = (float)p.ggas;
    sweep_mx<0>(L, b, T, pr, ggas, m, p.recon, p.sm_count, p.hll_fp32 != 0);
    sweep_mx<1>(L, b, T, pr, ggas, m, p.recon, p.sm_count, p.hll_fp32 != 0);
    sweep_mx<2>(L, b, T, pr, ggas, m, p.recon, p.sm_count, p.hll_fp32 != 0);
    FaceFluxT<float> ff[3];
    for (int d = 0; d < 3; ++d)
        for (int q = 0; q < 7; ++q) ff[d].f[q] = m.F[d][q];
    if (p.fused) {
        fused_tail(L, b, T, pr, ff, m, p, stage, dtmin);
        boundary_mx(L, b, m, p);
        return;
    }
    EdgeET<float> ee;
    for (int q = 0; q < 3; ++q) ee.e[q] = m.E[q];
    run(L, 3, g1((long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256), 256, 0, k_emf<float>, b, pr, ff[0], ff[1],
        ff[2], ee);
    switch (p.coord) {
        case 1: combine_model_mx<1>(L, b, T, m, p, stage); break;
        case 2: combine_model_mx<2>(L, b, T, m, p, stage); break;
        default: combine_model_mx<3>(L, b, T, m, p, stage); break;
    }
    UtopMx a = utop_args(m, p);
    if (stage == 3 && dtmin) {  // the following iteration's finddt, fused (dtmin reset by the caller)
        a.dtmin = dtmin;
        a.cfl = p.cfl;
    }
    const dim3 g = g1((long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256);
#define CUMC_MX_UTOP(C, M)                                                          \
    if (stage == 3) run(L, 5, g, 256, 0, k_utop_mx<C, M, true>, b, T, a);           \
    else run(L, 5, g, 256, 0, k_utop_mx<C, M, false>, b, T, a);
#define CUMC_MX_UTOP_MODEL(C)                    \
    switch (p.model) {                           \
        case 0: CUMC_MX_UTOP(C, 0) break;        \
        case 1: CUMC_MX_UTOP(C, 1) break;        \
        case 2: CUMC_MX_UTOP(C, 2) break;        \
        default: CUMC_MX_UTOP(C, 3) break;       \
    }
    switch (p.coord) {
        case 1: CUMC_MX_UTOP_MODEL(1) break;
        case 2: CUMC_MX_UTOP_MODEL(2) break;
        default: CUMC_MX_UTOP_MODEL(3) break;
    }
#undef CUMC_MX_UTOP_MODEL
#undef CUMC_MX_UTOP
    boundary_mx(L, b, m, p);
}

void mixed_initial(const Launcher& L, const Box& b, const Tabs& T, const MixedBufs& m, const MixedParams& p,
                   const double* prim_aos, const double* eps_aos) {
    (void)T;
    const UtopMx a = utop_args(m, p);
    const dim3 g = g1((long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256);
    switch (p.model) {
        case 0: run(L, -1, g, 256, 0, k_initial_mx<0>, b, a, prim_aos, eps_aos); break;
        case 1: run(L, -1, g, 256, 0, k_initial_mx<1>, b, a, prim_aos, eps_aos); break;
        case 2: run(L, -1, g, 256, 0, k_initial_mx<2>, b, a, prim_aos, eps_aos); break;
        default: run(L, -1, g, 256, 0, k_initial_mx<3>, b, a, prim_aos, eps_aos); break;
    }
    boundary_mx(L, b, m, p);
}

void mixed_finddt(const Launcher& L, const Box& b, const Tabs& T, const MixedBufs& m, const MixedParams& p,
                  unsigned long long* dtmin) {
    PrimT<float> pr;
    for (int q = 0; q < 5; ++q) pr.w[q] = m.w[q];
    for (int q = 0; q < 3; ++q) { pr.bc[q] = m.bc[q]; pr.bf[q] = m.bf[q]; }
    const dim3 g = g1((long long)b.nx * b.ny * b.nz, 256);
    switch (p.coord) {
        case 1: run(L, 7, g, 256, 0, k_finddt<1, float>, b, T, pr, p.ggas, p.cfl, dtmin); break;
        case 2: run(L, 7, g, 256, 0, k_finddt<2, float>, b, T, pr, p.ggas, p.cfl, dtmin); break;
        default: run(L, 7, g, 256, 0, k_finddt<3, float>, b, T, pr, p.ggas, p.cfl, dtmin); break;
    }
}

void mixed_export(const Launcher& L, const Box& b, const MixedBufs& m, const MixedParams& p, int what, double* aos) {
    const UtopMx a = utop_args(m, p);
    const dim3 g = g1(b.count(), 256);
    switch (what) {
        case 0: run(L, -1, g, 256, 0, k_export_mx<0>, b, a, aos); break;
        case 1: run(L, -1, g, 256, 0, k_export_mx<1>, b, a, aos); break;
        case 2: run(L, -1, g, 256, 0, k_export_mx<2>, b, a, aos); break;
        case 3: run(L, -1, g, 256, 0, k_export_mx<3>, b, a, aos); break;
        default: run(L, -1, g, 256, 0, k_export_mx<4>, b, a, aos); break;
    }
}

}  // namespace cumc
