// cumc_oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the CUMC3D per-step hot path (leon-astrophy/CUMPIC,
// solver/*.f90 and model/*/src/{eos,custom}.f90), written as a checker for the
// CUDA library. Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline may load it; the product never links or calls it.
//
// Parity status: the reference is Fortran 90 + OpenACC and this image has no
// Fortran compiler, MPI or HDF5, and the reference ships no tests or golden
// vectors. This restatement is pinned against a mechanical Fortran-to-C
// translation of the reference's own sources (oracle/f2c_ref.py, fixtures in
// tests/golden/); where that translation is unavailable, parity is unpinned.
//
// Layout and loop structure follow the reference one to one: every array is
// REAL*8 A(1:8, -2:n+3, -2:n+3, -2:n+3) in column-major order with the
// variable index fastest (solver/setup.f90:257-292), every parallel region of
// the reference is one loop nest here with the same bounds, and every per-cell
// leaf keeps the reference's operation order. Floating point is compiled with
// -ffp-contract=off so that no multiply-add is fused.
//
// Choices where the reference is undefined or processor dependent:
//  * ALLOCATE does not initialise memory; every array starts at zero here.
//  * SIGN(1d0, x) follows copysign (x = -0.0 gives -1).
//  * MIN/MAX follow C fmin/fmax.
//  * x**2 and x**3 are x*x and (x*x)*x.
//  * Left-to-right evaluation of every sum and product (Fortran compilers may
//    reassociate under -fast; the reference build is therefore not
//    bit-defined, solver/../make.inc:36).

#include "../include/cumc.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// equation indices (solver/setup.f90:49-116)
constexpr int irho = 1, ivx = 2, ivy = 3, ivz = 4, itau = 5, ibx = 6, iby = 7, ibz = 8;
constexpr int imin = 1, imax = 8;
constexpr int iex = 1, iey = 2, iez = 3;
constexpr int x_dir = 1, y_dir = 2, z_dir = 3;
constexpr int NGHOST = 3;

// Runge-Kutta coefficients (solver/definition.f90:180-185)
constexpr double rk20 = 3.0 / 4.0, rk21 = 1.0 / 4.0, rk22 = 1.0 / 4.0;
constexpr double rk30 = 1.0 / 3.0, rk31 = 2.0 / 3.0, rk32 = 2.0 / 3.0;

inline double SIGN1(double b) { return std::copysign(1.0, b); }
inline double MIN2(double a, double b) { return std::fmin(a, b); }
inline double MAX2(double a, double b) { return std::fmax(a, b); }
inline double MIN3(double a, double b, double c) { return std::fmin(std::fmin(a, b), c); }
inline double MAX3(double a, double b, double c) { return std::fmax(std::fmax(a, b), c); }
inline double sqrt_(double a) { return std::sqrt(a); }
inline double fabs_(double a) { return std::fabs(a); }
inline double val(double a) { return a; }

// Tangent-linear scalar: a value and one directional derivative. Values are
// computed with exactly the double operations above, so a Dual run follows
// the same branches as the double run on the same inputs (limiter, extremum
// and HLL choices frozen at the base point) and its derivative parts are the
// exact directional derivative of the discrete map.
struct Dual {
    double v, d;
    Dual() : v(0.0), d(0.0) {}
    Dual(double x) : v(x), d(0.0) {}  // constants carry no derivative
    Dual(double x, double t) : v(x), d(t) {}
};
inline Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(const Dual& a, const Dual& b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline double SIGN1(const Dual& b) { return std::copysign(1.0, b.v); }
inline Dual MIN2(const Dual& a, const Dual& b) { return b.v < a.v ? b : a; }
inline Dual MAX2(const Dual& a, const Dual& b) { return b.v > a.v ? b : a; }
inline Dual MIN3(const Dual& a, const Dual& b, const Dual& c) { return MIN2(MIN2(a, b), c); }
inline Dual MAX3(const Dual& a, const Dual& b, const Dual& c) { return MAX2(MAX2(a, b), c); }
inline Dual sqrt_(const Dual& a) {
    const double s = std::sqrt(a.v);
    return Dual(s, s > 0.0 ? a.d / (2.0 * s) : 0.0);
}
inline Dual fabs_(const Dual& a) { return a.v < 0.0 ? -a : a; }
inline double val(const Dual& a) { return a.v; }

template <typename T>
struct OracleT {
    cumc_config cfg{};
    int nx = 0, ny = 0, nz = 0;
    size_t SX = 0, SY = 0, SZ = 0, NT = 0;
    int coordinate = CUMC_CARTESIAN;
    int boundary_flag[6]{};
    int bfac_xin[9], bfac_xout[9], bfac_yin[9], bfac_yout[9], bfac_zin[9], bfac_zout[9];
    double ggas = 5.0 / 3.0, cfl = 0.4;
    int recon = CUMC_PPMC;
    int model = CUMC_MODEL_RIEMANN;
    double rho_floor = 0, eps_floor = 0, r_sh = 0;
    int geom_repeat = 8;

    std::vector<double> xF, yF, zF;  // index -3..n+3 stored at [i+3]
    std::vector<T> prim, cons, primL, primR, consL, consR, fluxL, fluxR, flux;
    std::vector<T> l_rk, u_old, sc, bcell, ecell, ecorn, eps;
    double dt = 0;

    // ---- indexing (Fortran column-major, lower bound -2 on space) ----
    inline size_t ix(int j, int k, int l) const {
        return (size_t)(j + 2) + SX * ((size_t)(k + 2) + SY * (size_t)(l + 2));
    }
    inline T& A8(std::vector<T>& a, int i, int j, int k, int l) {
        return a[(size_t)(i - 1) + 8 * ix(j, k, l)];
    }
    inline T& B3(int i, int j, int k, int l) { return bcell[(size_t)(i - ibx) + 3 * ix(j, k, l)]; }
    inline T& E3(std::vector<T>& a, int i, int j, int k, int l) {
        return a[(size_t)(i - 1) + 3 * ix(j, k, l)];
    }
    inline T& EPS(int j, int k, int l) { return eps[ix(j, k, l)]; }
    inline double XF(int j) const { return xF[(size_t)(j + 3)]; }
    inline double YF(int k) const { return yF[(size_t)(k + 3)]; }
    inline double ZF(int l) const { return zF[(size_t)(l + 3)]; }

    // ---- geometry (solver/coords.f90) ----
    // GET_COORD (solver/coords.f90:49-69)
    void get_coord(int j, int k, int l, double& x, double& y, double& z) const {
        x = 0.5 * (XF(j) + XF(j - 1));
        y = 0.5 * (YF(k) + YF(k - 1));
        z = 0.5 * (ZF(l) + ZF(l - 1));
    }
    // COORD_DX (solver/coords.f90:77-97)
    void coord_dx(int j, int k, int l, double& dx, double& dy, double& dz) const {
        dx = (XF(j) - XF(j - 1));
        dy = (YF(k) - YF(k - 1));
        dz = (ZF(l) - ZF(l - 1));
    }

    // GEOM_SOURCE (solver/coords.f90:105-165)
    void geom_source(int j, int k, int l) {
        double x, y, z, dxl, dyl, dzl;
        get_coord(j, k, l, x, y, z);
        coord_dx(j, k, l, dxl, dyl, dzl);
        const T bx = B3(ibx, j, k, l), by = B3(iby, j, k, l), bz = B3(ibz, j, k, l);
        const T rho = A8(prim, irho, j, k, l), vx = A8(prim, ivx, j, k, l);
        const T vy = A8(prim, ivy, j, k, l), vz = A8(prim, ivz, j, k, l);
        const T p = A8(prim, itau, j, k, l);
        if (coordinate == CUMC_CYLINDRICAL) {
            const T bsquare = bx * bx + by * by + bz * bz;
            A8(sc, ivx, j, k, l) = A8(sc, ivx, j, k, l) + (((p + (rho * vy) * vy) + 0.5 * bsquare) - by * by) / (x);
            A8(sc, ivy, j, k, l) = A8(sc, ivy, j, k, l) - ((rho * vx) * vy - bx * by) / (x);
        } else if (coordinate == CUMC_SPHERICAL) {
            const T bsquare = bx * bx + by * by + bz * bz;
            const double tany = std::tan(y);
            A8(sc, ivx, j, k, l) = A8(sc, ivx, j, k, l) + ((2.0 * p + bx * bx) + rho * (vy * vy + vz * vz)) / (x);
            A8(sc, ivy, j, k, l) = (A8(sc, ivy, j, k, l) + (((p + (rho * vz) * vz) + 0.5 * bsquare) - bz * bz) / (x * tany))
                                   - ((rho * vx) * vy - bx * by) / (x);
            A8(sc, ivz, j, k, l) = (A8(sc, ivz, j, k, l) - ((rho * vx) * vz - bx * bz) / (x))
                                   - ((rho * vy) * vz - by * bz) / (x * tany);
        }
    }

    // GEOM_AREA (solver/coords.f90:173-223)
    void geom_area(int j, int k, int l, double& axp, double& axm, double& ayp, double& aym, double& azp,
                   double& azm) const {
        double x, y, z, dxl, dyl, dzl;
        get_coord(j, k, l, x, y, z);
        coord_dx(j, k, l, dxl, dyl, dzl);
        if (coordinate == CUMC_CARTESIAN) {
            axp = dyl * dzl; axm = dyl * dzl;
            ayp = dxl * dzl; aym = dxl * dzl;
            azp = dxl * dyl; azm = dxl * dyl;
        } else if (coordinate == CUMC_CYLINDRICAL) {
            axp = (XF(j) * dyl) * dzl;
            axm = (XF(j - 1) * dyl) * dzl;
            ayp = dxl * dzl; aym = dxl * dzl;
            azp = (0.5 * (XF(j) * XF(j) - XF(j - 1) * XF(j - 1))) * dyl;
            azm = azp;
        } else {
            const double dcos = std::cos(YF(k - 1)) - std::cos(YF(k));
            axp = ((XF(j) * XF(j)) * dcos) * dzl;
            axm = ((XF(j - 1) * XF(j - 1)) * dcos) * dzl;
            const double half = 0.5 * (XF(j) * XF(j) - XF(j - 1) * XF(j - 1));
            ayp = (half * std::sin(YF(k))) * dzl;
            aym = (half * std::sin(YF(k - 1))) * dzl;
            azp = half * dyl;
            azm = half * dyl;
        }
    }

    // GEOM_FLUX (solver/coords.f90:231-302)
    void geom_flux(int dir, int j, int k, int l, double& gp, double& gc, double& gm) const {
        double x, y, z, dxl, dyl, dzl;
        get_coord(j, k, l, x, y, z);
        coord_dx(j, k, l, dxl, dyl, dzl);
        if (coordinate == CUMC_CARTESIAN) {
            gp = 1.0; gm = 1.0;
            gc = dir == x_dir ? dxl : dir == y_dir ? dyl : dzl;
        } else if (coordinate == CUMC_CYLINDRICAL) {
            if (dir == x_dir) { gp = XF(j); gm = XF(j - 1); gc = x * dxl; }
            else if (dir == y_dir) { gp = 1.0; gm = 1.0; gc = x * dyl; }
            else { gp = 1.0; gm = 1.0; gc = dzl; }
        } else {
            const double xp = XF(j), xm = XF(j - 1);
            if (dir == x_dir) {
                gp = xp * xp; gm = xm * xm;
                gc = ((xp * xp) * xp - (xm * xm) * xm) / 3.0;
            } else {
                const double rfac = ((2.0 * ((xp * xp) * xp - (xm * xm) * xm)) / 3.0) / (xp * xp - xm * xm);
                const double dcos = std::cos(YF(k - 1)) - std::cos(YF(k));
                if (dir == y_dir) {
                    gp = std::sin(YF(k)); gm = std::sin(YF(k - 1));
                    gc = rfac * dcos;
                } else {
                    gp = 1.0; gm = 1.0;
                    gc = ((rfac * dcos) * dzl) / dyl;
                }
            }
        }
    }

    // GEOM_CT (solver/coords.f90:310-415): g[face][edge][m,c,p]
    struct CT { double bx_ez_m, bx_ez_c, bx_ez_p, bx_ey_m, bx_ey_c, bx_ey_p,
                       by_ex_m, by_ex_c, by_ex_p, by_ez_m, by_ez_c, by_ez_p,
                       bz_ex_m, bz_ex_c, bz_ex_p, bz_ey_m, bz_ey_c, bz_ey_p; };
    void geom_ct(int j, int k, int l, CT& g) const {
        double x, y, z, dxl, dyl, dzl;
        get_coord(j, k, l, x, y, z);
        coord_dx(j, k, l, dxl, dyl, dzl);
        if (coordinate == CUMC_CARTESIAN) {
            g.bx_ez_m = 1.0; g.bx_ez_c = dyl; g.bx_ez_p = 1.0;
            g.bx_ey_m = 1.0; g.bx_ey_c = dzl; g.bx_ey_p = 1.0;
            g.by_ex_m = 1.0; g.by_ex_c = dzl; g.by_ex_p = 1.0;
            g.by_ez_m = 1.0; g.by_ez_c = dxl; g.by_ez_p = 1.0;
            g.bz_ey_m = 1.0; g.bz_ey_c = dxl; g.bz_ey_p = 1.0;
            g.bz_ex_m = 1.0; g.bz_ex_c = dyl; g.bz_ex_p = 1.0;
        } else if (coordinate == CUMC_CYLINDRICAL) {
            g.bx_ez_m = 1.0; g.bx_ez_c = dyl * XF(j); g.bx_ez_p = 1.0;
            g.bx_ey_m = 1.0; g.bx_ey_c = dzl; g.bx_ey_p = 1.0;
            g.by_ex_m = 1.0; g.by_ex_c = dzl; g.by_ex_p = 1.0;
            g.by_ez_m = 1.0; g.by_ez_c = dxl; g.by_ez_p = 1.0;
            g.bz_ey_m = XF(j - 1); g.bz_ey_c = x * dxl; g.bz_ey_p = XF(j);
            g.bz_ex_m = 1.0; g.bz_ex_c = x * dyl; g.bz_ex_p = 1.0;
        } else {
            const double dcos = std::cos(YF(k - 1)) - std::cos(YF(k));
            g.bx_ez_m = std::sin(YF(k - 1)); g.bx_ez_c = XF(j) * dcos; g.bx_ez_p = std::sin(YF(k));
            g.bx_ey_m = 1.0; g.bx_ey_c = ((XF(j) * dcos) * dzl) / dyl; g.bx_ey_p = 1.0;
            g.by_ex_m = 1.0; g.by_ex_c = (x * std::sin(YF(k))) * dzl; g.by_ex_p = 1.0;
            g.by_ez_m = XF(j - 1); g.by_ez_c = x * dxl; g.by_ez_p = XF(j);
            g.bz_ey_m = XF(j - 1); g.bz_ey_c = x * dxl; g.bz_ey_p = XF(j);
            g.bz_ex_m = 1.0; g.bz_ex_c = x * dyl; g.bz_ex_p = 1.0;
        }
    }

    // ---- EOS (model/riemann/src/eos.f90:126-200) ----
    inline T eos_pressure(const T& rho, const T& e) const { return (rho * e) * (ggas - 1.0); }
    inline T eos_soundspeed(const T& p, const T& rho) const { return sqrt_((ggas * p) / rho); }
    inline T eos_epsilon(const T& p, const T& rho) const { return (p / rho) / (ggas - 1.0); }

    // ---- reconstruction (solver/reconstruct.f90) ----
    void dh3(int dir, int j, int k, int l, int off, double& d) const {
        double a, b, c;
        if (dir == x_dir) { coord_dx(j + off, k, l, a, b, c); d = a; }
        else if (dir == y_dir) { coord_dx(j, k + off, l, a, b, c); d = b; }
        else { coord_dx(j, k, l + off, a, b, c); d = c; }
    }

    // TVD_MM (solver/reconstruct.f90:58-128)
    void tvd_mm(int dir, int j, int k, int l, T vm2, T vm1, T vc, T vp1, T vp2, T& vm_out, T& vp_out) const {
        (void)vm2; (void)vp2;
        double dh_m1, dh_c, dh_p1;
        dh3(dir, j, k, l, -1, dh_m1);
        dh3(dir, j, k, l, 0, dh_c);
        dh3(dir, j, k, l, 1, dh_p1);
        const double cf = (dh_c + dh_p1) / dh_c;
        const double cb = (dh_c + dh_m1) / dh_c;
        const T dqf = (2.0 * (vp1 - vc)) / cf;
        const T dqb = (2.0 * (vc - vm1)) / cb;
        const T slope = (0.5 * (SIGN1(dqf) + SIGN1(dqb))) * MIN2(fabs_(dqf), fabs_(dqb));
        vp_out = vc + 0.5 * slope;
        vm_out = vc - 0.5 * slope;
    }

    // PPM (solver/reconstruct.f90:137-311)
    void ppm(int dir, int j, int k, int l, T vm2, T vm1, T vc, T vp1, T vp2, T& vm_out, T& vp_out) const {
        double dm2, dm1, dc, dp1, dp2;
        dh3(dir, j, k, l, -2, dm2);
        dh3(dir, j, k, l, -1, dm1);
        dh3(dir, j, k, l, 0, dc);
        dh3(dir, j, k, l, 1, dp1);
        dh3(dir, j, k, l, 2, dp2);
        // :211-231
        const double a1R = dc / (dc + dp1);
        const double a1L = dm1 / (dm1 + dc);
        const double aR = ((2.0 * dp1) * dc) / (dp1 + dc);
        const double aL = ((2.0 * dc) * dm1) / (dc + dm1);
        const double deltaXR = ((dm1 + dc) + dp1) + dp2;
        const double deltaXL = ((dm2 + dm1) + dc) + dp1;
        const double z1R = (dm1 + dc) / (2.0 * dc + dp1);
        const double z1L = (dm2 + dm1) / (2.0 * dm1 + dc);
        const double zR = (dp2 + dp1) / (2.0 * dp1 + dc);
        const double zL = (dp1 + dc) / (2.0 * dc + dm1);
        const double cc1 = dc / ((dm1 + dc) + dp1);
        const double cp1 = dp1 / ((dc + dp1) + dp2);
        const double cm1 = dm1 / ((dm2 + dm1) + dc);
        const double cc2 = (2.0 * dm1 + dc) / (dp1 + dc);
        const double cp2 = (2.0 * dc + dp1) / (dp2 + dp1);
        const double cm2 = (2.0 * dm2 + dm1) / (dc + dm1);
        const double cc3 = (dc + 2.0 * dp1) / (dm1 + dc);
        const double cp3 = (dp1 + 2.0 * dp2) / (dc + dp1);
        const double cm3 = (dm1 + 2.0 * dc) / (dm2 + dm1);
        // :236-249
        const double a0m = a1L;
        const double a1m = (aL * (z1L - zL)) / deltaXL;
        const double a2m = ((-dm1) * z1L) / deltaXL;
        const double a3m = (dc * zL) / deltaXL;
        const double a0p = a1R;
        const double a1p = (aR * (z1R - zR)) / deltaXR;
        const double a2p = ((-dc) * z1R) / deltaXR;
        const double a3p = (dp1 * zR) / deltaXR;
        const double b0m = cm1 * cm2, b1m = cm1 * cm3;
        const double b0c = cc1 * cc2, b1c = cc1 * cc3;
        const double b0p = cp1 * cp2, b1p = cp1 * cp3;
        // :254-256
        const T deltap1 = b0p * (vp2 - vp1) + b1p * (vp1 - vc);
        const T deltac = b0c * (vp1 - vc) + b1c * (vc - vm1);
        const T deltam1 = b0m * (vc - vm1) + b1m * (vm1 - vm2);
        // :261-280 van Leer limiter
        T dmc, dmp1, dmm1;
        if ((vp1 - vc) * (vc - vm1) > 0.0)
            dmc = MIN3(fabs_(deltac), 2.0 * fabs_(vc - vm1), 2.0 * fabs_(vc - vp1)) * SIGN1(deltac);
        else
            dmc = 0.0;
        if ((vp2 - vp1) * (vp1 - vc) > 0.0)
            dmp1 = MIN3(fabs_(deltap1), 2.0 * fabs_(vp1 - vc), 2.0 * fabs_(vp1 - vp2)) * SIGN1(deltap1);
        else
            dmp1 = 0.0;
        if ((vc - vm1) * (vm1 - vm2) > 0.0)
            dmm1 = MIN3(fabs_(deltam1), 2.0 * fabs_(vm1 - vm2), 2.0 * fabs_(vm1 - vc)) * SIGN1(deltam1);
        else
            dmm1 = 0.0;
        // :285-286
        vp_out = (((vc + a0p * (vp1 - vc)) + a1p * (vp1 - vc)) + a2p * dmp1) + a3p * dmc;
        vm_out = (((vm1 + a0m * (vc - vm1)) + a1m * (vc - vm1)) + a2m * dmc) + a3m * dmm1;
        const T vl = vm_out, vr = vp_out;
        // :295-307 extremum and overshoot fixes; the second test reads the
        // already-modified vm_out
        if ((vr - vc) * (vc - vl) <= 0.0) {
            vp_out = vc;
            vm_out = vc;
        } else {
            if ((vr - vl) * ((vl - 3.0 * vc) + 2.0 * vr) < 0.0) vm_out = 3.0 * vc - 2.0 * vr;
            if ((vp_out - vm_out) * ((3.0 * vc - 2.0 * vl) - vr) < 0.0) vp_out = 3.0 * vc - 2.0 * vl;
        }
    }

    // INTERPOLATE (solver/reconstruct.f90:18-51)
    void interpolate(int dir, int j, int k, int l, T vm2, T vm1, T vc, T vp1, T vp2, T& vm_out, T& vp_out) const {
        if (recon == CUMC_TVDMM) tvd_mm(dir, j, k, l, vm2, vm1, vc, vp1, vp2, vm_out, vp_out);
        else ppm(dir, j, k, l, vm2, vm1, vc, vp1, vp2, vm_out, vp_out);
    }

    // ---- Riemann solver (solver/rsolver.f90, flux.f90, ptou_face.f90) ----
    // PtoU_MHD_face (solver/ptou_face.f90:34-88)
    void ptou_face(std::vector<T>& P, std::vector<T>& U, int j, int k, int l, const T& e) {
        const T vx = A8(P, ivx, j, k, l), vy = A8(P, ivy, j, k, l), vz = A8(P, ivz, j, k, l);
        const T bx = A8(P, ibx, j, k, l), by = A8(P, iby, j, k, l), bz = A8(P, ibz, j, k, l);
        const T rho = A8(P, irho, j, k, l);
        const T vsquare = (vx * vx + vy * vy) + vz * vz;
        const T bsquare = (bx * bx + by * by) + bz * bz;
        A8(U, irho, j, k, l) = rho;
        A8(U, ivx, j, k, l) = vx * rho;
        A8(U, ivy, j, k, l) = vy * rho;
        A8(U, ivz, j, k, l) = vz * rho;
        A8(U, itau, j, k, l) = rho * (e + 0.5 * vsquare) + 0.5 * bsquare;
        A8(U, ibx, j, k, l) = bx;
        A8(U, iby, j, k, l) = by;
        A8(U, ibz, j, k, l) = bz;
    }

    // Ptof_MHD, one side (solver/flux.f90:163-262)
    void ptof_side(std::vector<T>& P, std::vector<T>& U, std::vector<T>& F, int dir, int j, int k, int l) {
        int ivn, ivt1, ivt2, ibn, ibt1, ibt2;
        if (dir == x_dir) { ivn = ivx; ivt1 = ivy; ivt2 = ivz; ibn = ibx; ibt1 = iby; ibt2 = ibz; }
        else if (dir == y_dir) { ivn = ivy; ivt1 = ivz; ivt2 = ivx; ibn = iby; ibt1 = ibz; ibt2 = ibx; }
        else { ivn = ivz; ivt1 = ivx; ivt2 = ivy; ibn = ibz; ibt1 = ibx; ibt2 = iby; }
        const T bx = A8(P, ibx, j, k, l), by = A8(P, iby, j, k, l), bz = A8(P, ibz, j, k, l);
        const T vx = A8(P, ivx, j, k, l), vy = A8(P, ivy, j, k, l), vz = A8(P, ivz, j, k, l);
        const T bsquare = (bx * bx + by * by) + bz * bz;
        const T vdotb = (bx * vx + by * vy) + bz * vz;
        const T vn = A8(P, ivn, j, k, l), p = A8(P, itau, j, k, l);
        const T bn = A8(P, ibn, j, k, l);
        for (int i = imin; i <= ibx - 1; ++i) A8(F, i, j, k, l) = A8(U, i, j, k, l) * vn;
        A8(F, ivn, j, k, l) = ((A8(F, ivn, j, k, l) + p) + 0.5 * bsquare) - bn * bn;
        A8(F, ivt1, j, k, l) = A8(F, ivt1, j, k, l) - bn * A8(P, ibt1, j, k, l);
        A8(F, ivt2, j, k, l) = A8(F, ivt2, j, k, l) - bn * A8(P, ibt2, j, k, l);
        A8(F, itau, j, k, l) = (A8(F, itau, j, k, l) + (p + 0.5 * bsquare) * vn) - bn * vdotb;
        A8(F, ibn, j, k, l) = 0.0;
        A8(F, ibt1, j, k, l) = vn * A8(P, ibt1, j, k, l) - A8(P, ivt1, j, k, l) * bn;
        A8(F, ibt2, j, k, l) = vn * A8(P, ibt2, j, k, l) - A8(P, ivt2, j, k, l) * bn;
    }

    // compute_signalspeed (solver/definition.f90:394-410)
    static T signalspeed(const T& cs, const T& bn, const T& bt1, const T& bt2, const T& rho) {
        const T a2 = cs * cs;
        const T a4 = a2 * a2;
        const T b2n = (bn * bn) / rho;
        const T b2t1 = (bt1 * bt1) / rho;
        const T b2t2 = (bt2 * bt2) / rho;
        const T b2 = (b2n + b2t1) + b2t2;
        const T b4 = b2 * b2;
        return sqrt_(0.5 * ((a2 + b2) + sqrt_(MAX2(((a4 + b4) + (2.0 * b2) * a2) - (4.0 * a2) * b2n, 0.0))));
    }
    // compute_roe (solver/definition.f90:387-392)
    static T roe(const T& xl, const T& xr, const T& rl, const T& rr) {
        return (sqrt_(rl) * xl + sqrt_(rr) * xr) / (sqrt_(rl) + sqrt_(rr));
    }
    // compute_fluxhll (solver/definition.f90:380-385)
    static T fluxhll(const T& yl, const T& yr, const T& xl, const T& xr, const T& sl, const T& sr) {
        return ((sr * yl - sl * yr) + (sl * sr) * (xr - xl)) / (sr - sl);
    }

    // HLL_SOLVER (solver/rsolver.f90:43-130)
    void hll_solver(int dir, int j, int k, int l) {
        int ibn, ibt1, ibt2, ivn;
        if (dir == x_dir) { ibn = ibx; ibt1 = iby; ibt2 = ibz; ivn = ivx; }
        else if (dir == y_dir) { ibn = iby; ibt1 = ibz; ibt2 = ibx; ivn = ivy; }
        else { ibn = ibz; ibt1 = ibx; ibt2 = iby; ivn = ivz; }
        const T epsL = eos_epsilon(A8(primL, itau, j, k, l), A8(primL, irho, j, k, l));
        const T epsR = eos_epsilon(A8(primR, itau, j, k, l), A8(primR, irho, j, k, l));
        const T csL = eos_soundspeed(A8(primL, itau, j, k, l), A8(primL, irho, j, k, l));
        const T csR = eos_soundspeed(A8(primR, itau, j, k, l), A8(primR, irho, j, k, l));
        ptou_face(primL, consL, j, k, l, epsL);
        ptou_face(primR, consR, j, k, l, epsR);
        ptof_side(primL, consL, fluxL, dir, j, k, l);
        ptof_side(primR, consR, fluxR, dir, j, k, l);
        const T rhoL = A8(primL, irho, j, k, l), rhoR = A8(primR, irho, j, k, l);
        const T cfsL = signalspeed(csL, A8(primL, ibn, j, k, l), A8(primL, ibt1, j, k, l),
                                        A8(primL, ibt2, j, k, l), rhoL);
        const T cfsR = signalspeed(csR, A8(primR, ibn, j, k, l), A8(primR, ibt1, j, k, l),
                                        A8(primR, ibt2, j, k, l), rhoR);
        const T ubar = roe(A8(primL, ivn, j, k, l), A8(primR, ivn, j, k, l), rhoL, rhoR);
        const T cbar = roe(cfsL, cfsR, rhoL, rhoR);
        const T sL = MIN2(A8(primL, ivn, j, k, l) - cfsL, ubar - cbar);
        const T sR = MAX2(A8(primR, ivn, j, k, l) + cfsR, ubar + cbar);
        if (sL >= 0.0) {
            for (int i = imin; i <= imax; ++i) A8(flux, i, j, k, l) = A8(fluxL, i, j, k, l);
        } else if (sL <= 0.0 && sR >= 0.0) {
            for (int i = imin; i <= imax; ++i)
                A8(flux, i, j, k, l) = fluxhll(A8(fluxL, i, j, k, l), A8(fluxR, i, j, k, l), A8(consL, i, j, k, l),
                                              A8(consR, i, j, k, l), sL, sR);
        } else if (sR <= 0.0) {
            for (int i = imin; i <= imax; ++i) A8(flux, i, j, k, l) = A8(fluxR, i, j, k, l);
        }
    }

    // ---- model hooks ----
    // CUSTOM_CHECKRHO (model/riemann/src/custom.f90:54-76; model/torus_sph/src/custom.f90:76-106)
    void custom_checkrho() {
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    if (model == CUMC_MODEL_RIEMANN) {
                        EPS(j, k, l) = MAX2(EPS(j, k, l), 0.0);
                    } else if (model == CUMC_MODEL_TORUS_SPH || model == CUMC_MODEL_TORUS_CYN) {
                        if (A8(prim, irho, j, k, l) < rho_floor) A8(prim, irho, j, k, l) = rho_floor;
                        if (EPS(j, k, l) < eps_floor) EPS(j, k, l) = eps_floor;
                    }
                }
    }

    // CUSTOM_SOURCE (model/torus_sph/src/custom.f90:111-150; model/torus_cyn/src/custom.f90)
    void custom_source() {
        if (model != CUMC_MODEL_TORUS_SPH && model != CUMC_MODEL_TORUS_CYN) return;
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    double x, y, z;
                    get_coord(j, k, l, x, y, z);
                    const T rho = A8(prim, irho, j, k, l);
                    const T diff = rho - rho_floor;
                    const double factor = MAX2(SIGN1(diff), 0.0);
                    if (model == CUMC_MODEL_TORUS_SPH) {
                        const double dphidr = 1.0 / ((x - r_sh) * (x - r_sh));
                        A8(sc, ivx, j, k, l) = A8(sc, ivx, j, k, l) + (((-factor) * rho) * dphidr);
                        A8(sc, itau, j, k, l) =
                            A8(sc, itau, j, k, l) + ((((-factor) * rho) * A8(prim, ivx, j, k, l)) * dphidr);
                    } else {
                        const double radius = std::sqrt(x * x + z * z);
                        const double dphidr = (x / radius) / ((radius - r_sh) * (radius - r_sh));
                        const double dphidz = (z / radius) / ((radius - r_sh) * (radius - r_sh));
                        A8(sc, ivx, j, k, l) = A8(sc, ivx, j, k, l) + (((-factor) * rho) * dphidr);
                        A8(sc, ivz, j, k, l) = A8(sc, ivz, j, k, l) + (((-factor) * rho) * dphidz);
                        A8(sc, itau, j, k, l) =
                            A8(sc, itau, j, k, l) +
                            (((-factor) * rho) * (A8(prim, ivx, j, k, l) * dphidr + A8(prim, ivz, j, k, l) * dphidz));
                    }
                }
    }

    // CUSTOM_BOUNDARY (model/torus_sph/src/custom.f90:47-71; model/torus_cyn/src/custom.f90)
    void custom_boundary() {
        if (model != CUMC_MODEL_TORUS_SPH && model != CUMC_MODEL_TORUS_CYN) return;
#pragma omp parallel for collapse(2)
        for (int l = -2; l <= nz + 3; ++l)
            for (int k = -2; k <= ny + 3; ++k)
                for (int j = 1; j <= 3; ++j) {
                    A8(prim, ivx, 1 - j, k, l) = MIN2(A8(prim, ivx, 1 - j, k, l), 0.0);
                    A8(prim, ivx, nx + j, k, l) = MAX2(A8(prim, ivx, nx + j, k, l), 0.0);
                }
        if (model == CUMC_MODEL_TORUS_CYN) {
#pragma omp parallel for collapse(2)
            for (int l = 1; l <= 3; ++l)
                for (int k = -2; k <= ny + 3; ++k)
                    for (int j = -2; j <= nx + 3; ++j) {
                        A8(prim, ivz, j, k, 1 - l) = MIN2(A8(prim, ivz, j, k, 1 - l), 0.0);
                        A8(prim, ivz, j, k, nz + l) = MAX2(A8(prim, ivz, j, k, nz + l), 0.0);
                    }
        }
    }

    // ---- SPATIAL (solver/spatial.f90:11-68) ----
    void spatial() {
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j)
                    for (int i = imin; i <= imax; ++i) {
                        A8(sc, i, j, k, l) = 0.0;
                        A8(l_rk, i, j, k, l) = 0.0;
                    }
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j)
                    for (int i = iex; i <= iez; ++i) E3(ecorn, i, j, k, l) = 0.0;
        get_source();
        custom_source();
        get_fluxes();
        flux_ct();
    }

    // GET_SOURCE (solver/spatial.f90:75-102). The reference loops over
    // i = imin..imax around the call, so the source is added 8 times.
    void get_source() {
        if (coordinate == CUMC_CARTESIAN) return;  // GEOM_SOURCE has no Cartesian case
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j)
                    for (int i = 0; i < geom_repeat; ++i) geom_source(j, k, l);
    }

    // one directional sweep of GET_FLUXES (solver/spatial.f90:113-380)
    void sweep(int dir) {
        const int dj = dir == x_dir, dk = dir == y_dir, dl = dir == z_dir;
        int ibn, ibt1, ibt2;
        if (dir == x_dir) { ibn = ibx; ibt1 = iby; ibt2 = ibz; }
        else if (dir == y_dir) { ibn = iby; ibt1 = ibx; ibt2 = ibz; }
        else { ibn = ibz; ibt1 = ibx; ibt2 = iby; }
        // interpolate (:131-154, :209-232, :287-310)
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz + 1; ++l)
            for (int k = 0; k <= ny + 1; ++k)
                for (int j = 0; j <= nx + 1; ++j) {
                    for (int i = imin; i <= ibx - 1; ++i)
                        interpolate(dir, j, k, l, A8(prim, i, j - 2 * dj, k - 2 * dk, l - 2 * dl),
                                    A8(prim, i, j - dj, k - dk, l - dl), A8(prim, i, j, k, l),
                                    A8(prim, i, j + dj, k + dk, l + dl), A8(prim, i, j + 2 * dj, k + 2 * dk, l + 2 * dl),
                                    A8(primR, i, j - dj, k - dk, l - dl), A8(primL, i, j, k, l));
                    for (int ib : {ibt1, ibt2})
                        interpolate(dir, j, k, l, B3(ib, j - 2 * dj, k - 2 * dk, l - 2 * dl),
                                    B3(ib, j - dj, k - dk, l - dl), B3(ib, j, k, l), B3(ib, j + dj, k + dk, l + dl),
                                    B3(ib, j + 2 * dj, k + 2 * dk, l + 2 * dl), A8(primR, ib, j - dj, k - dk, l - dl),
                                    A8(primL, ib, j, k, l));
                    A8(primR, ibn, j - dj, k - dk, l - dl) = A8(prim, ibn, j - dj, k - dk, l - dl);
                    A8(primL, ibn, j, k, l) = A8(prim, ibn, j, k, l);
                }
        // Riemann (:157-168, :235-246, :313-324)
        const int jhi = dir == x_dir ? nx : nx + 1, khi = dir == y_dir ? ny : ny + 1, lhi = dir == z_dir ? nz : nz + 1;
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= lhi; ++l)
            for (int k = 0; k <= khi; ++k)
                for (int j = 0; j <= jhi; ++j) hll_solver(dir, j, k, l);
        // flux difference (:171-187, :249-265, :327-343)
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j)
                    for (int i = imin; i <= ibx - 1; ++i) {
                        double gp, gc, gm;
                        geom_flux(dir, j, k, l, gp, gc, gm);
                        A8(l_rk, i, j, k, l) =
                            A8(l_rk, i, j, k, l) -
                            (A8(flux, i, j, k, l) * gp - A8(flux, i, j - dj, k - dk, l - dl) * gm) / gc;
                    }
        // EMF accumulation (:190-203, :268-281, :346-359)
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j) {
                    if (dir == x_dir) {
                        E3(ecorn, iey, j, k, l) =
                            E3(ecorn, iey, j, k, l) + 0.25 * (A8(flux, ibz, j, k, l) + A8(flux, ibz, j, k, l + 1));
                        E3(ecorn, iez, j, k, l) =
                            E3(ecorn, iez, j, k, l) + 0.25 * (-A8(flux, iby, j, k, l) - A8(flux, iby, j, k + 1, l));
                    } else if (dir == y_dir) {
                        E3(ecorn, iex, j, k, l) =
                            E3(ecorn, iex, j, k, l) + 0.25 * (-A8(flux, ibz, j, k, l) - A8(flux, ibz, j, k, l + 1));
                        E3(ecorn, iez, j, k, l) =
                            E3(ecorn, iez, j, k, l) + 0.25 * (A8(flux, ibx, j, k, l) + A8(flux, ibx, j + 1, k, l));
                    } else {
                        E3(ecorn, iex, j, k, l) =
                            E3(ecorn, iex, j, k, l) + 0.25 * (A8(flux, iby, j, k, l) + A8(flux, iby, j, k + 1, l));
                        E3(ecorn, iey, j, k, l) =
                            E3(ecorn, iey, j, k, l) + 0.25 * (-A8(flux, ibx, j, k, l) - A8(flux, ibx, j + 1, k, l));
                    }
                }
    }

    // GET_FLUXES (solver/spatial.f90:113-380)
    void get_fluxes() {
        sweep(x_dir);
        sweep(y_dir);
        sweep(z_dir);
        // :365-375
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j)
                    for (int i = imin; i <= ibx - 1; ++i)
                        A8(l_rk, i, j, k, l) = A8(l_rk, i, j, k, l) + A8(sc, i, j, k, l);
    }

    // flux_ct (solver/mhd.f90:73-157)
    void flux_ct() {
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz + 1; ++l)
            for (int k = 0; k <= ny + 1; ++k)
                for (int j = 0; j <= nx + 1; ++j) {
                    const T vx = A8(prim, ivx, j, k, l), vy = A8(prim, ivy, j, k, l), vz = A8(prim, ivz, j, k, l);
                    const T bx = B3(ibx, j, k, l), by = B3(iby, j, k, l), bz = B3(ibz, j, k, l);
                    E3(ecell, iex, j, k, l) = vz * by - vy * bz;
                    E3(ecell, iey, j, k, l) = vx * bz - vz * bx;
                    E3(ecell, iez, j, k, l) = vy * bx - vx * by;
                }
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j) {
                    E3(ecorn, iex, j, k, l) = E3(ecorn, iex, j, k, l) * 2.0 -
                        0.25 * (((E3(ecell, iex, j, k, l) + E3(ecell, iex, j, k, l + 1)) + E3(ecell, iex, j, k + 1, l)) +
                                E3(ecell, iex, j, k + 1, l + 1));
                    E3(ecorn, iey, j, k, l) = E3(ecorn, iey, j, k, l) * 2.0 -
                        0.25 * (((E3(ecell, iey, j, k, l) + E3(ecell, iey, j, k, l + 1)) + E3(ecell, iey, j + 1, k, l)) +
                                E3(ecell, iey, j + 1, k, l + 1));
                    E3(ecorn, iez, j, k, l) = E3(ecorn, iez, j, k, l) * 2.0 -
                        0.25 * (((E3(ecell, iez, j, k, l) + E3(ecell, iez, j, k + 1, l)) + E3(ecell, iez, j + 1, k, l)) +
                                E3(ecell, iez, j + 1, k + 1, l));
                }
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j) {
                    CT g;
                    geom_ct(j, k, l, g);
                    A8(l_rk, ibx, j, k, l) =
                        -((E3(ecorn, iez, j, k, l) * g.bx_ez_p - E3(ecorn, iez, j, k - 1, l) * g.bx_ez_m) / g.bx_ez_c -
                          (E3(ecorn, iey, j, k, l) * g.bx_ey_p - E3(ecorn, iey, j, k, l - 1) * g.bx_ey_m) / g.bx_ey_c);
                    A8(l_rk, iby, j, k, l) =
                        -((E3(ecorn, iex, j, k, l) * g.by_ex_p - E3(ecorn, iex, j, k, l - 1) * g.by_ex_m) / g.by_ex_c -
                          (E3(ecorn, iez, j, k, l) * g.by_ez_p - E3(ecorn, iez, j - 1, k, l) * g.by_ez_m) / g.by_ez_c);
                    A8(l_rk, ibz, j, k, l) =
                        -((E3(ecorn, iey, j, k, l) * g.bz_ey_p - E3(ecorn, iey, j - 1, k, l) * g.bz_ey_m) / g.bz_ey_c -
                          (E3(ecorn, iex, j, k, l) * g.bz_ex_p - E3(ecorn, iex, j, k - 1, l) * g.bz_ex_m) / g.bz_ex_c);
                }
    }

    // ---- conversions (solver/fromrvetou.f90, ptou.f90, utop.f90) ----
    void fromrvetou() {
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    B3(ibx, j, k, l) = 0.5 * (A8(prim, ibx, j, k, l) + A8(prim, ibx, j - 1, k, l));
                    B3(iby, j, k, l) = 0.5 * (A8(prim, iby, j, k, l) + A8(prim, iby, j, k - 1, l));
                    B3(ibz, j, k, l) = 0.5 * (A8(prim, ibz, j, k, l) + A8(prim, ibz, j, k, l - 1));
                }
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j) {
                    // PtoU_MHD (solver/ptou.f90:33-66)
                    const T vx = A8(prim, ivx, j, k, l), vy = A8(prim, ivy, j, k, l), vz = A8(prim, ivz, j, k, l);
                    const T bx = B3(ibx, j, k, l), by = B3(iby, j, k, l), bz = B3(ibz, j, k, l);
                    const T rho = A8(prim, irho, j, k, l);
                    const T vsquare = (vx * vx + vy * vy) + vz * vz;
                    const T bsquare = (bx * bx + by * by) + bz * bz;
                    A8(cons, irho, j, k, l) = rho;
                    A8(cons, ivx, j, k, l) = vx * rho;
                    A8(cons, ivy, j, k, l) = vy * rho;
                    A8(cons, ivz, j, k, l) = vz * rho;
                    A8(cons, itau, j, k, l) = rho * (EPS(j, k, l) + 0.5 * vsquare) + 0.5 * bsquare;
                    for (int i = ibx; i <= ibz; ++i) A8(cons, i, j, k, l) = A8(prim, i, j, k, l);
                }
    }

    void fromutorve() {
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    B3(ibx, j, k, l) = 0.5 * (A8(cons, ibx, j, k, l) + A8(cons, ibx, j - 1, k, l));
                    B3(iby, j, k, l) = 0.5 * (A8(cons, iby, j, k, l) + A8(cons, iby, j, k - 1, l));
                    B3(ibz, j, k, l) = 0.5 * (A8(cons, ibz, j, k, l) + A8(cons, ibz, j, k, l - 1));
                }
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j) {
                    // UtoP_MHD (solver/utop.f90:33-68)
                    const T rho = A8(cons, irho, j, k, l);
                    A8(prim, irho, j, k, l) = rho;
                    A8(prim, ivx, j, k, l) = A8(cons, ivx, j, k, l) / rho;
                    A8(prim, ivy, j, k, l) = A8(cons, ivy, j, k, l) / rho;
                    A8(prim, ivz, j, k, l) = A8(cons, ivz, j, k, l) / rho;
                    for (int i = ibx; i <= ibz; ++i) A8(prim, i, j, k, l) = A8(cons, i, j, k, l);
                    const T bx = B3(ibx, j, k, l), by = B3(iby, j, k, l), bz = B3(ibz, j, k, l);
                    const T vx = A8(prim, ivx, j, k, l), vy = A8(prim, ivy, j, k, l), vz = A8(prim, ivz, j, k, l);
                    const T bsquare = (bx * bx + by * by) + bz * bz;
                    const T vsquare = (vx * vx + vy * vy) + vz * vz;
                    EPS(j, k, l) = (A8(cons, itau, j, k, l) - 0.5 * bsquare) / rho - 0.5 * vsquare;
                }
    }

    // ---- boundaries (solver/boundary.f90) ----
    // BOUNDARY1D for eps with all parities even (solver/boundary.f90:29-341).
    // Each side is its own loop nest, inner side first, as in the reference.
    void boundary1d() {
        const int* f = boundary_flag;
        const int fac = 1;  // signx_in..signz_out are all `even` (solver/boundary.f90:11)
        // x (:92-166): k, l in 1:n
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= NGHOST; ++j) {
                    if (f[0] == 0) EPS(1 - j, k, l) = EPS(nx + 1 - j, k, l);
                    else if (f[0] == 1) EPS(1 - j, k, l) = EPS(1, k, l);
                    else EPS(1 - j, k, l) = fac * EPS(j, k, l);
                }
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= NGHOST; ++j) {
                    if (f[1] == 0) EPS(nx + j, k, l) = EPS(j, k, l);
                    else if (f[1] == 1) EPS(nx + j, k, l) = EPS(nx, k, l);
                    else EPS(nx + j, k, l) = fac * EPS(nx + 1 - j, k, l);
                }
        // y (:174-246): j in -2:n+3, l in 1:n
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j) {
                    if (f[2] == 0) EPS(j, 1 - k, l) = EPS(j, ny + 1 - k, l);
                    else if (f[2] == 1) EPS(j, 1 - k, l) = EPS(j, 1, l);
                    else EPS(j, 1 - k, l) = fac * EPS(j, k, l);
                }
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j) {
                    // the outer periodic test reads boundary_flag(3), not (4) (:211)
                    if (f[2] == 0) EPS(j, ny + k, l) = EPS(j, k, l);
                    else if (f[3] == 1) EPS(j, ny + k, l) = EPS(j, ny, l);
                    else if (f[3] >= 2) EPS(j, ny + k, l) = fac * EPS(j, ny + 1 - k, l);
                }
        // z (:254-328): all j, k
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= NGHOST; ++l)
            for (int k = 1 - NGHOST; k <= ny + NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j) {
                    if (f[4] == 0) EPS(j, k, 1 - l) = EPS(j, k, nz + 1 - l);
                    else if (f[4] == 1) EPS(j, k, 1 - l) = EPS(j, k, 1);
                    else EPS(j, k, 1 - l) = fac * EPS(j, k, l);
                }
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= NGHOST; ++l)
            for (int k = 1 - NGHOST; k <= ny + NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j) {
                    if (f[5] == 0) EPS(j, k, nz + l) = EPS(j, k, l);
                    else if (f[5] == 1) EPS(j, k, nz + l) = EPS(j, k, nz);
                    else EPS(j, k, nz + l) = fac * EPS(j, k, nz + 1 - l);
                }
    }

    // one ghost copy of BOUNDARYP: hydro prims, bcell and two tangential face fields
    inline void bcopy(int jd, int kd, int ld, int js, int ks, int ls, const int* fac, int t1, int t2, bool signed_) {
        for (int i = imin; i <= ibx - 1; ++i)
            A8(prim, i, jd, kd, ld) = signed_ ? fac[i] * A8(prim, i, js, ks, ls) : A8(prim, i, js, ks, ls);
        for (int i = ibx; i <= ibz; ++i)
            B3(i, jd, kd, ld) = signed_ ? fac[i] * B3(i, js, ks, ls) : B3(i, js, ks, ls);
        A8(prim, t1, jd, kd, ld) = signed_ ? fac[t1] * A8(prim, t1, js, ks, ls) : A8(prim, t1, js, ks, ls);
        A8(prim, t2, jd, kd, ld) = signed_ ? fac[t2] * A8(prim, t2, js, ks, ls) : A8(prim, t2, js, ks, ls);
    }

    // BOUNDARYP (solver/boundary.f90:349-672); inner side before outer side
    void boundaryp() {
        const int* f = boundary_flag;
        // x (:362-454): k, l in 0:n; tangential fields iby, ibz
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 1; j <= NGHOST; ++j) {
                    if (f[0] == 0) bcopy(1 - j, k, l, nx + 1 - j, k, l, bfac_xin, iby, ibz, false);
                    else if (f[0] == 1) bcopy(1 - j, k, l, 1, k, l, bfac_xin, iby, ibz, false);
                    else bcopy(1 - j, k, l, j, k, l, bfac_xin, iby, ibz, true);
                }
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 1; j <= NGHOST; ++j) {
                    if (f[1] == 0) bcopy(nx + j, k, l, j, k, l, bfac_xout, iby, ibz, false);
                    else if (f[1] == 1) bcopy(nx + j, k, l, nx, k, l, bfac_xout, iby, ibz, false);
                    else bcopy(nx + j, k, l, nx + 1 - j, k, l, bfac_xout, iby, ibz, true);
                }
        // y (:462-554): j in -2:n+3, l in 0:n; tangential fields ibx, ibz
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 1; k <= NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j) {
                    if (f[2] == 0) bcopy(j, 1 - k, l, j, ny + 1 - k, l, bfac_yin, ibx, ibz, false);
                    else if (f[2] == 1) bcopy(j, 1 - k, l, j, 1, l, bfac_yin, ibx, ibz, false);
                    else bcopy(j, 1 - k, l, j, k, l, bfac_yin, ibx, ibz, true);
                }
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 1; k <= NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j) {
                    if (f[3] == 0) bcopy(j, ny + k, l, j, k, l, bfac_yout, ibx, ibz, false);
                    else if (f[3] == 1) bcopy(j, ny + k, l, j, ny, l, bfac_yout, ibx, ibz, false);
                    else bcopy(j, ny + k, l, j, ny + 1 - k, l, bfac_yout, ibx, ibz, true);
                }
        // z (:562-654): all j, k; tangential fields ibx, iby
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= NGHOST; ++l)
            for (int k = 1 - NGHOST; k <= ny + NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j) {
                    if (f[4] == 0) bcopy(j, k, 1 - l, j, k, nz + 1 - l, bfac_zin, ibx, iby, false);
                    else if (f[4] == 1) bcopy(j, k, 1 - l, j, k, 1, bfac_zin, ibx, iby, false);
                    else bcopy(j, k, 1 - l, j, k, l, bfac_zin, ibx, iby, true);
                }
#pragma omp parallel for collapse(2)
        for (int l = 1; l <= NGHOST; ++l)
            for (int k = 1 - NGHOST; k <= ny + NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j) {
                    if (f[5] == 0) bcopy(j, k, nz + l, j, k, l, bfac_zout, ibx, iby, false);
                    else if (f[5] == 1) bcopy(j, k, nz + l, j, k, nz, bfac_zout, ibx, iby, false);
                    else bcopy(j, k, nz + l, j, k, nz + 1 - l, bfac_zout, ibx, iby, true);
                }
        custom_boundary();
    }

    // BOUNDARY (solver/boundary.f90:5-13)
    void boundary() {
        boundaryp();
        boundary1d();
    }

    // UPDATE (solver/update.f90:12-45)
    void update() {
#pragma omp parallel for collapse(2)
        for (int l = 1 - NGHOST; l <= nz + NGHOST; ++l)
            for (int k = 1 - NGHOST; k <= ny + NGHOST; ++k)
                for (int j = 1 - NGHOST; j <= nx + NGHOST; ++j)
                    A8(prim, itau, j, k, l) = eos_pressure(A8(prim, irho, j, k, l), EPS(j, k, l));
    }

    // initial_update (solver/initial.f90:83-140)
    void initial_update() {
        custom_checkrho();
        fromrvetou();
        boundary();
        update();
    }

    // combine over (0:n)^3 and all 8 equations (solver/rungekutta.f90:41-119)
    void combine(int stage) {
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j)
                    for (int i = imin; i <= imax; ++i) {
                        T& c = A8(cons, i, j, k, l);
                        const T u0 = A8(u_old, i, j, k, l), L = A8(l_rk, i, j, k, l);
                        if (stage == 1) c = u0 + dt * L;
                        else if (stage == 2) c = (rk20 * u0 + rk21 * c) + (rk22 * dt) * L;
                        else c = (rk30 * u0 + rk31 * c) + (rk32 * dt) * L;
                    }
    }

    // RUNGEKUTTA (solver/rungekutta.f90:12-148)
    void rungekutta(double dt_in) {
        dt = dt_in;
#pragma omp parallel for collapse(2)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j)
                    for (int i = imin; i <= imax; ++i) A8(u_old, i, j, k, l) = A8(cons, i, j, k, l);
        for (int stage = 1; stage <= 3; ++stage) {
            spatial();
            combine(stage);
            fromutorve();
            custom_checkrho();
            if (stage == 3) custom_checkrho();  // OPERATOR_SPLIT is empty in every model
            fromrvetou();
            boundary();
            update();
        }
    }

    // finddt (solver/rungekutta.f90:161-265)
    double finddt() {
        double dt_temp = 1.0e10;
#pragma omp parallel for collapse(2) reduction(min : dt_temp)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    const double rho = val(A8(prim, irho, j, k, l));
                    const double cs = std::sqrt((ggas * val(A8(prim, itau, j, k, l))) / rho);
                    const double a2 = cs * cs;
                    const double a4 = a2 * a2;
                    const double b2x = (val(B3(ibx, j, k, l)) * val(B3(ibx, j, k, l))) / rho;
                    const double b2y = (val(B3(iby, j, k, l)) * val(B3(iby, j, k, l))) / rho;
                    const double b2z = (val(B3(ibz, j, k, l)) * val(B3(ibz, j, k, l))) / rho;
                    const double b2 = (b2x + b2y) + b2z;
                    const double b4 = b2 * b2;
                    const double base = (a4 + (2.0 * a2) * b2) + b4;
                    const double cfx = std::sqrt(0.5 * ((a2 + b2) + std::sqrt(base - (4.0 * a2) * b2x)));
                    const double cfy = std::sqrt(0.5 * ((a2 + b2) + std::sqrt(base - (4.0 * a2) * b2y)));
                    const double cfz = std::sqrt(0.5 * ((a2 + b2) + std::sqrt(base - (4.0 * a2) * b2z)));
                    const double lambda = MAX3(std::fabs(val(A8(prim, ivx, j, k, l))) + cfx,
                                               std::fabs(val(A8(prim, ivy, j, k, l))) + cfy,
                                               std::fabs(val(A8(prim, ivz, j, k, l))) + cfz);
                    double dxl, dyl, dzl, x, y, z;
                    coord_dx(j, k, l, dxl, dyl, dzl);
                    get_coord(j, k, l, x, y, z);
                    if (coordinate == CUMC_CYLINDRICAL) {
                        dyl = x * dyl;
                    } else if (coordinate == CUMC_SPHERICAL) {
                        dyl = x * dyl;
                        dzl = (x * std::sin(y)) * dzl;
                    }
                    const double dt_out = (MIN3(dxl, dyl, dzl) * cfl) / lambda;
                    dt_temp = MIN2(dt_out, dt_temp);
                }
        dt = dt_temp;
        return dt;
    }

    // find_divb (solver/mhd.f90:15-66)
    double find_divb() {
        double maxdb = 0.0;
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    double axp, axm, ayp, aym, azp, azm;
                    geom_area(j, k, l, axp, axm, ayp, aym, azp, azm);
                    const double div_b = ((axp * val(A8(prim, ibx, j, k, l)) - axm * val(A8(prim, ibx, j - 1, k, l))) +
                                          (ayp * val(A8(prim, iby, j, k, l)) - aym * val(A8(prim, iby, j, k - 1, l)))) +
                                         (azp * val(A8(prim, ibz, j, k, l)) - azm * val(A8(prim, ibz, j, k, l - 1)));
                    maxdb = MAX2(maxdb, div_b);
                }
        return maxdb;
    }

    bool setup(const cumc_config* c, char* err, int errlen) {
        cfg = *c;
        nx = c->nx; ny = c->ny; nz = c->nz;
        if (nx < 3 || ny < 3 || nz < 3) { snprintf(err, errlen, "every direction needs at least 3 active cells (3 ghost layers)"); return false; }
        SX = nx + 6; SY = ny + 6; SZ = nz + 6; NT = SX * SY * SZ;
        coordinate = c->coordinate;
        for (int i = 0; i < 6; ++i) boundary_flag[i] = c->boundary_flag[i];
        ggas = c->ggas; cfl = c->cfl; recon = c->recon; model = c->model;
        rho_floor = c->rho_floor; eps_floor = c->eps_floor; r_sh = c->r_sh;
        geom_repeat = c->geom_source_repeat > 0 ? c->geom_source_repeat : 8;
        // bfac tables (solver/setup.f90:121-230)
        for (int i = 0; i < 9; ++i) bfac_xin[i] = bfac_xout[i] = bfac_yin[i] = bfac_yout[i] = bfac_zin[i] = bfac_zout[i] = 1;
        auto setx = [&](int fl, int* b) -> bool {
            if (fl == 2) { b[ivx] = -1; b[ibx] = -1; }
            else if (fl == 3) { b[ivx] = -1; b[ibx] = -1; b[ivz] = -1; b[ibz] = -1; }
            else if (fl == 4) return false;
            return true;
        };
        auto sety = [&](int fl, int* b) {
            if (fl == 2) { b[ivy] = -1; b[iby] = -1; }
            else if (fl == 3) { b[ivy] = -1; b[iby] = -1; b[ivz] = -1; b[ibz] = -1; }
            else if (fl == 4) { b[ivy] = -1; b[ibx] = -1; b[ibz] = -1; }
        };
        auto setz = [&](int fl, int* b) -> bool {
            if (fl == 2) { b[ivz] = -1; b[ibz] = -1; }
            else if (fl == 3) return false;
            else if (fl == 4) { b[ivz] = -1; b[ibx] = -1; b[iby] = -1; }
            return true;
        };
        if (!setx(boundary_flag[0], bfac_xin) || !setx(boundary_flag[1], bfac_xout)) {
            snprintf(err, errlen, "equatorial symmetry is not allowed for the x-boundary"); return false;
        }
        sety(boundary_flag[2], bfac_yin); sety(boundary_flag[3], bfac_yout);
        if (!setz(boundary_flag[4], bfac_zin) || !setz(boundary_flag[5], bfac_zout)) {
            snprintf(err, errlen, "axial symmetry is not allowed for the z-boundary"); return false;
        }
        xF.assign(c->xf, c->xf + nx + 7);
        yF.assign(c->yf, c->yf + ny + 7);
        zF.assign(c->zf, c->zf + nz + 7);
        for (auto* v : {&prim, &cons, &primL, &primR, &consL, &consR, &fluxL, &fluxR, &flux, &l_rk, &u_old, &sc})
            v->assign(8 * NT, T(0.0));
        bcell.assign(3 * NT, T(0.0));
        ecell.assign(3 * NT, T(0.0));
        ecorn.assign(3 * NT, T(0.0));
        eps.assign(NT, T(0.0));
        return true;
    }
};
using Oracle = OracleT<double>;
using OracleTL = OracleT<Dual>;

}  // namespace

extern "C" {

void* orc_create(const cumc_config* cfg, char* err, int errlen) {
    auto* o = new Oracle();
    if (!o->setup(cfg, err, errlen)) { delete o; return nullptr; }
    return o;
}
void orc_free(void* h) { delete static_cast<Oracle*>(h); }
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int orc_get_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
int orc_upload(void* h, const double* prim, const double* eps) {
    auto* o = static_cast<Oracle*>(h);
    std::memcpy(o->prim.data(), prim, sizeof(double) * 8 * o->NT);
    std::memcpy(o->eps.data(), eps, sizeof(double) * o->NT);
    return 0;
}
int orc_initial_update(void* h) { static_cast<Oracle*>(h)->initial_update(); return 0; }
int orc_finddt(void* h, double* dt) { *dt = static_cast<Oracle*>(h)->finddt(); return 0; }
int orc_rungekutta(void* h, double dt) { static_cast<Oracle*>(h)->rungekutta(dt); return 0; }
int orc_spatial(void* h) { static_cast<Oracle*>(h)->spatial(); return 0; }
int orc_divb(void* h, double* maxdb) { *maxdb = static_cast<Oracle*>(h)->find_divb(); return 0; }
int orc_download(void* h, double* prim, double* cons, double* eps, double* bcell, double* lrk) {
    auto* o = static_cast<Oracle*>(h);
    if (prim) std::memcpy(prim, o->prim.data(), sizeof(double) * 8 * o->NT);
    if (cons) std::memcpy(cons, o->cons.data(), sizeof(double) * 8 * o->NT);
    if (eps) std::memcpy(eps, o->eps.data(), sizeof(double) * o->NT);
    if (bcell) std::memcpy(bcell, o->bcell.data(), sizeof(double) * 3 * o->NT);
    if (lrk) std::memcpy(lrk, o->l_rk.data(), sizeof(double) * 8 * o->NT);
    return 0;
}

// tangent-linear oracle: the same map on (value, direction) pairs
void* orc_tl_create(const cumc_config* cfg, char* err, int errlen) {
    auto* o = new OracleTL();
    if (!o->setup(cfg, err, errlen)) { delete o; return nullptr; }
    return o;
}
void orc_tl_free(void* h) { delete static_cast<OracleTL*>(h); }
int orc_tl_upload(void* h, const double* prim, const double* eps, const double* dprim, const double* deps) {
    auto* o = static_cast<OracleTL*>(h);
    for (size_t i = 0; i < 8 * o->NT; ++i) o->prim[i] = Dual(prim[i], dprim[i]);
    for (size_t i = 0; i < o->NT; ++i) o->eps[i] = Dual(eps[i], deps[i]);
    return 0;
}
int orc_tl_initial_update(void* h) { static_cast<OracleTL*>(h)->initial_update(); return 0; }
int orc_tl_rungekutta(void* h, double dt) { static_cast<OracleTL*>(h)->rungekutta(dt); return 0; }
// values and derivatives of prim, cons, eps, bcell; any pointer may be NULL
int orc_tl_download(void* h, double* prim, double* cons, double* eps, double* bcell, double* dprim, double* dcons,
                    double* deps, double* dbcell) {
    auto* o = static_cast<OracleTL*>(h);
    auto put = [](const std::vector<Dual>& a, double* v, double* d) {
        for (size_t i = 0; i < a.size(); ++i) {
            if (v) v[i] = a[i].v;
            if (d) d[i] = a[i].d;
        }
    };
    put(o->prim, prim, dprim);
    put(o->cons, cons, dcons);
    put(o->eps, eps, deps);
    put(o->bcell, bcell, dbcell);
    return 0;
}

}  // extern "C"
