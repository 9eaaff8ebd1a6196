// cumc_emfct.cuh — edge EMFs and the constrained-transport update of the
// face fields in one kernel (the EMF sums of GET_FLUXES,
// solver/spatial.f90:190-203,268-281,346-359, flux_ct's ecell/ecorn,
// solver/mhd.f90:95-125, its curl, :130-153, and the RK combine of the face
// fields, solver/rungekutta.f90:41-51,75-85,109-119).
//
// k_emf writes the three edge-EMF arrays and k_ct reads them back at six
// neighbouring edges a face triple. Here a block owns a tile of 32 x 8 face
// triples (x fastest) and marches in z over a segment of planes. Per plane
// it forms, in shared memory, the cell EMFs E = -v x B of the cells the
// plane's edges average, then the edge EMFs of the tile and of the halo row
// and column its CT reads (Ez at j-1 and k-1; Ey at j-1; Ex at k-1), and
// keeps the x and y edge EMFs of the previous plane (the l-1 edges of CT).
// Each cell EMF is formed once per plane, each edge EMF at most 1.2 times.
// Edges with an index of -1 are zero, as the never-written entries of the
// edge arrays are for k_ct. Every value is the same expression, in the same
// order, as in k_emf and k_ct, so the result is bit for bit theirs.
#pragma once
#include "cumc_kernels.cuh"

namespace cumc {

constexpr int EC_TX = 32, EC_TY = 8;           // face triples of a tile
constexpr int EC_CX = EC_TX + 2, EC_CY = EC_TY + 2;  // cells j0-1..j0+32, k0-1..k0+8
constexpr int EC_EX = EC_TX + 1, EC_EY = EC_TY + 1;  // edges j0-1..j0+31, k0-1..k0+7
constexpr int EC_SEG = 32;                     // planes a block marches over (at most; emf_ct_grid)

// shared memory of a tile; R is the EMFs' type (double, or float in the
// mixed form)
template <typename R>
struct EmfCtSmemT {
    R ec[2][3][EC_CY][EC_CX];   // cell EMFs of two planes (ring by plane parity)
    R ex[2][EC_EY][EC_EX];      // x edge EMFs of two planes (ring by plane parity)
    R ey[2][EC_EY][EC_EX];      // y edge EMFs of two planes
    R ez[EC_EY][EC_EX];         // z edge EMFs of the current plane
};
using EmfCtSmem = EmfCtSmemT<double>;

// cell EMFs of plane l for the tile's cells (zero outside -1..n+1)
template <typename R>
__device__ __forceinline__ void ec_cells(const Box& b, const PrimT<R>& pr, EmfCtSmemT<R>& S, int j0, int k0, int l) {
    const int slot = l & 1;
    for (int t = threadIdx.x; t < EC_CX * EC_CY; t += EC_TX * EC_TY) {
        const int cj = t % EC_CX, ck = t / EC_CX;
        const int j = j0 - 1 + cj, k = k0 - 1 + ck;
        R x = R(0), y = R(0), z = R(0);
        if (j <= b.nx + 1 && k <= b.ny + 1 && l >= -1 && l <= b.nz + 1) {
            const int i = b.idx(j, k, l);
            x = ecell_x(pr, i);
            y = ecell_y(pr, i);
            z = ecell_z(pr, i);
        }
        S.ec[slot][0][ck][cj] = x;
        S.ec[slot][1][ck][cj] = y;
        S.ec[slot][2][ck][cj] = z;
    }
}

// edge EMFs of plane l (x and y edges into their ring slot; z edges with `z`)
template <typename R>
__device__ __forceinline__ void ec_edges(const Box& b, const FaceFluxT<R>& fx, const FaceFluxT<R>& fy,
                                         const FaceFluxT<R>& fz, EmfCtSmemT<R>& S, int j0, int k0, int l, bool z) {
    const int sj = 1, sk = b.SX, sl = b.SX * b.SY;
    const R q = R(0.25);
    const int c0 = l & 1, c1 = (l + 1) & 1;  // cell-EMF slots of planes l and l+1
    const int e = l & 1;
    for (int t = threadIdx.x; t < EC_EX * EC_EY; t += EC_TX * EC_TY) {
        const int ej = t % EC_EX, ek = t / EC_EX;  // edge (j0 - 1 + ej, k0 - 1 + ek)
        const int j = j0 - 1 + ej, k = k0 - 1 + ek;
        const bool live = j >= 0 && k >= 0 && l >= 0 && j <= b.nx && k <= b.ny && l <= b.nz;
        const int i = live ? b.idx(j, k, l) : 0;
        // cell (j, k) of the edge is cell slot (ck, cj) = (ek, ej): the edge sits
        // at the upper faces of cells j and k
        const int cj = ej, ck = ek;
        R ex = R(0), ey = R(0), ez = R(0);
        if (live) {
            ex = R(0) + q * (-fy.f[6][i] - fy.f[6][i + sl]);
            ex = ex + q * (fz.f[6][i] + fz.f[6][i + sk]);
            ey = R(0) + q * (fx.f[6][i] + fx.f[6][i + sl]);
            ey = ey + q * (-fz.f[5][i] - fz.f[5][i + sj]);
            // k_emf's sums: cells (j,k,l), (j,k,l+1), (j,k+1,l), (j,k+1,l+1) for Ex;
            // (j,k,l), (j,k,l+1), (j+1,k,l), (j+1,k,l+1) for Ey; (j,k), (j,k+1),
            // (j+1,k), (j+1,k+1) of plane l for Ez
            ex = ex * R(2) - q * (((S.ec[c0][0][ck][cj] + S.ec[c1][0][ck][cj]) + S.ec[c0][0][ck + 1][cj]) +
                                 S.ec[c1][0][ck + 1][cj]);
            ey = ey * R(2) - q * (((S.ec[c0][1][ck][cj] + S.ec[c1][1][ck][cj]) + S.ec[c0][1][ck][cj + 1]) +
                                 S.ec[c1][1][ck][cj + 1]);
            if (z) {
                ez = R(0) + q * (-fx.f[5][i] - fx.f[5][i + sk]);
                ez = ez + q * (fy.f[5][i] + fy.f[5][i + sj]);
                ez = ez * R(2) - q * (((S.ec[c0][2][ck][cj] + S.ec[c0][2][ck + 1][cj]) + S.ec[c0][2][ck][cj + 1]) +
                                     S.ec[c0][2][ck + 1][cj + 1]);
            }
        }
        S.ex[e][ek][ej] = ex;
        S.ey[e][ek][ej] = ey;
        if (z) S.ez[ek][ej] = ez;
    }
}

// the flux half of one edge's three EMFs (the first two sums of each, k_emf's
// order); the cell-EMF half is added once the plane's cell EMFs are in
// shared memory (ec_edge_finish)
template <typename R>
struct EdgePart {
    R x, y, z;
};
template <typename R>
__device__ __forceinline__ EdgePart<R> ec_edge_part(const Box& b, const FaceFluxT<R>& fx, const FaceFluxT<R>& fy,
                                                    const FaceFluxT<R>& fz, int j0, int k0, int l, int t) {
    const int sj = 1, sk = b.SX, sl = b.SX * b.SY;
    const R q = R(0.25);
    const int j = j0 - 1 + t % EC_EX, k = k0 - 1 + t / EC_EX;
    EdgePart<R> e{R(0), R(0), R(0)};
    if (j >= 0 && k >= 0 && j <= b.nx && k <= b.ny && l <= b.nz) {
        const int i = b.idx(j, k, l);
        e.x = R(0) + q * (-fy.f[6][i] - fy.f[6][i + sl]);
        e.x = e.x + q * (fz.f[6][i] + fz.f[6][i + sk]);
        e.y = R(0) + q * (fx.f[6][i] + fx.f[6][i + sl]);
        e.y = e.y + q * (-fz.f[5][i] - fz.f[5][i + sj]);
        e.z = R(0) + q * (-fx.f[5][i] - fx.f[5][i + sk]);
        e.z = e.z + q * (fy.f[5][i] + fy.f[5][i + sj]);
    }
    return e;
}
template <typename R>
__device__ __forceinline__ void ec_edge_finish(const Box& b, EmfCtSmemT<R>& S, const EdgePart<R>& e, int j0, int k0,
                                               int l, int t) {
    const R q = R(0.25);
    const int ej = t % EC_EX, ek = t / EC_EX;
    const int j = j0 - 1 + ej, k = k0 - 1 + ek;
    const bool live = j >= 0 && k >= 0 && j <= b.nx && k <= b.ny && l <= b.nz;
    const int c0 = l & 1, c1 = (l + 1) & 1, cj = ej, ck = ek;
    R ex = R(0), ey = R(0), ez = R(0);
    if (live) {
        ex = e.x * R(2) - q * (((S.ec[c0][0][ck][cj] + S.ec[c1][0][ck][cj]) + S.ec[c0][0][ck + 1][cj]) +
                               S.ec[c1][0][ck + 1][cj]);
        ey = e.y * R(2) - q * (((S.ec[c0][1][ck][cj] + S.ec[c1][1][ck][cj]) + S.ec[c0][1][ck][cj + 1]) +
                               S.ec[c1][1][ck][cj + 1]);
        ez = e.z * R(2) - q * (((S.ec[c0][2][ck][cj] + S.ec[c0][2][ck + 1][cj]) + S.ec[c0][2][ck][cj + 1]) +
                               S.ec[c0][2][ck + 1][cj + 1]);
    }
    S.ex[l & 1][ek][ej] = ex;
    S.ey[l & 1][ek][ej] = ey;
    S.ez[ek][ej] = ez;
}

// Per plane a thread first issues its global loads (the flux half of its
// edges, u_old and u of its face triple, the cell fields of its cells of the
// next plane), so that one memory latency a plane is exposed instead of
// three. Two barriers a plane: the next plane's cell EMFs overwrite the slot
// of plane l-1's cells, read only before this plane's second barrier, and
// its edges overwrite slots that CT reads, which every thread has finished
// before it reaches the next plane's first barrier.
#ifndef CUMC_EC_MINB
#define CUMC_EC_MINB 4
#endif
template <int COORD, int STAGE>
__global__ void __launch_bounds__(EC_TX * EC_TY, CUMC_EC_MINB) k_emf_ct(Box b, Tabs T, Prim pr, FaceFlux fx,
                                                                      FaceFlux fy, FaceFlux fz, CombineArgs a,
                                                                      int seg) {
    extern __shared__ __align__(16) unsigned char ec_raw[];
    EmfCtSmem& S = *reinterpret_cast<EmfCtSmem*>(ec_raw);
    if (b.skip && *b.skip) return;
    constexpr int NE = EC_EX * EC_EY, NT = EC_TX * EC_TY;
    static_assert(NE > NT && NE <= 2 * NT, "two edges a thread at most");
    const int j0 = blockIdx.x * EC_TX, k0 = blockIdx.y * EC_TY;
    const int l0 = blockIdx.z * seg, l1 = min(l0 + seg, b.nz + 1);
    const int tj = threadIdx.x % EC_TX, tk = threadIdx.x / EC_TX;
    const int j = j0 + tj, k = k0 + tk;
    const bool mine = j <= b.nx && k <= b.ny;
    const int e0 = threadIdx.x, e1 = threadIdx.x + NT;  // the thread's edges (e1 < NE for some)
    const double dt = *a.dt;

    // prologue: the x and y edges of plane l0 - 1 (zero for l0 = 0)
    ec_cells(b, pr, S, j0, k0, l0 - 1);
    ec_cells(b, pr, S, j0, k0, l0);
    __syncthreads();
    ec_edges(b, fx, fy, fz, S, j0, k0, l0 - 1, false);
    __syncthreads();
    for (int l = l0; l < l1; ++l) {
        const EdgePart<double> p0 = ec_edge_part(b, fx, fy, fz, j0, k0, l, e0);
        const EdgePart<double> p1 = e1 < NE ? ec_edge_part(b, fx, fy, fz, j0, k0, l, e1) : EdgePart<double>{0.0, 0.0, 0.0};
        double u0v[3] = {0.0, 0.0, 0.0}, ucv[3] = {0.0, 0.0, 0.0};
        const int i = b.idx(j, k, l);
        if (mine) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                u0v[c] = a.u0[IBX + c][i];
                if (STAGE != 1) ucv[c] = a.uc[IBX + c][i];
            }
        }
        ec_cells(b, pr, S, j0, k0, l + 1);  // replaces plane l - 1's cells
        __syncthreads();
        ec_edge_finish(b, S, p0, j0, k0, l, e0);
        if (e1 < NE) ec_edge_finish(b, S, p1, j0, k0, l, e1);
        __syncthreads();
        if (mine) {
            // ct_lrk (solver/mhd.f90:137-148) on the shared-memory edges; the tile's
            // (tj, tk) is edge (tj + 1, tk + 1)
            const int ej = tj + 1, ek = tk + 1, e = l & 1, em = (l - 1) & 1;
            const double Ez = S.ez[ek][ej], Ez_km = S.ez[ek - 1][ej], Ez_jm = S.ez[ek][ej - 1];
            const double Ey = S.ey[e][ek][ej], Ey_lm = S.ey[em][ek][ej], Ey_jm = S.ey[e][ek][ej - 1];
            const double Ex = S.ex[e][ek][ej], Ex_lm = S.ex[em][ek][ej], Ex_km = S.ex[e][ek - 1][ej];
            CTf g;
            geom_ct<COORD>(T, j, k, l, g);
            double L[3];
            L[0] = -((Ez * g.bx_ez_p - Ez_km * g.bx_ez_m) / g.bx_ez_c - (Ey * g.bx_ey_p - Ey_lm * g.bx_ey_m) / g.bx_ey_c);
            L[1] = -((Ex * g.by_ex_p - Ex_lm * g.by_ex_m) / g.by_ex_c - (Ez * g.by_ez_p - Ez_jm * g.by_ez_m) / g.by_ez_c);
            L[2] = -((Ey * g.bz_ey_p - Ey_jm * g.bz_ey_m) / g.bz_ey_c - (Ex * g.bz_ex_p - Ex_km * g.bz_ex_m) / g.bz_ex_c);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double r = rk_point<STAGE>(u0v[c], ucv[c], dt, L[c]);
                a.ud[IBX + c][i] = r;
                if (a.tape[IBX + c]) a.tape[IBX + c][i] = r;
            }
        }
    }
}

// grid of a tiled EMF + CT launch and the planes a block marches over: 32,
// halved (down to 4) while the grid would not fill `slots` resident blocks
// twice (small boxes: the 128^3 adjoint box, the torus); each segment repeats
// one plane of cell and edge EMFs
inline dim3 emf_ct_grid(const Box& b, long long slots, int* seg) {
    const unsigned gx = (unsigned)((b.nx + 1 + EC_TX - 1) / EC_TX), gy = (unsigned)((b.ny + 1 + EC_TY - 1) / EC_TY);
    int s = EC_SEG;
    while (s > 4 && (long long)gx * gy * ((b.nz + 1 + s - 1) / s) < 2 * slots) s /= 2;
    *seg = s;
    return dim3(gx, gy, (unsigned)((b.nz + 1 + s - 1) / s));
}

}  // namespace cumc
