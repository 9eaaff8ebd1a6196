// cumc_sweep.cuh — tiled directional sweep: reconstruction + HLL on the faces
// of one direction (GET_FLUXES interpolate + RIEMANN, solver/spatial.f90:131-168,
// 209-246, 287-324).
//
// A block owns a tile of 16 faces along the sweep direction by 16 positions
// across it. The 7 reconstructed fields of the 21 cells the tile needs are
// staged in shared memory once; then, per field and cell, the limited PPM
// slope (once per cell), the unlimited interface value (once per face) and the
// extremum fix (once per cell) are computed in shared memory, which gives
// every face its left state vp_out(c) and right state vm_out(c+1). The reference
// evaluates the slope three times and the interface value twice per cell; the
// values are the same doubles (the weights agree, see the table builder), so
// the tile reproduces them bit for bit with a third of the arithmetic.
// Finally one thread per face solves the HLL problem and stores the fluxes.
//
// Threads are laid out with x fastest in every direction: for the y and z
// sweeps the tile is 16 x-positions wide (128-byte rows), for the x sweep the
// stencil runs along the row.
#pragma once
#include "cumc_kernels.cuh"

namespace cumc {

constexpr int SW_F = 16;             // faces per tile along the sweep direction
constexpr int SW_T = 16;             // tile width across the sweep direction
constexpr int SW_S = SW_F + 5;       // cells per tile along the sweep direction
constexpr int SW_NV = 7;             // reconstructed fields
constexpr int SW_THREADS = SW_F * SW_T;
template <typename R>
constexpr size_t sw_smem() { return sizeof(R) * (3 * SW_NV * SW_S * SW_T + 2 * SW_NV * SW_F * SW_T); }

template <int DIR>
struct SweepGeom {
    // tile origin and bounds; c = cell index along DIR, tt = index across it
    int f0, t0, third, nd, tmax;
    __device__ __forceinline__ SweepGeom(const Box& b) {
        if (DIR == 0) {
            f0 = blockIdx.x * SW_F; t0 = blockIdx.y * SW_T; third = blockIdx.z;
            nd = b.nx; tmax = b.ny + 1;
        } else if (DIR == 1) {
            t0 = blockIdx.x * SW_T; f0 = blockIdx.y * SW_F; third = blockIdx.z;
            nd = b.ny; tmax = b.nx + 1;
        } else {
            t0 = blockIdx.x * SW_T; f0 = blockIdx.y * SW_F; third = blockIdx.z;
            nd = b.nz; tmax = b.nx + 1;
        }
    }
    __device__ __forceinline__ int gidx(const Box& b, int c, int tt) const {
        if (DIR == 0) return b.idx(c, tt, third);
        if (DIR == 1) return b.idx(tt, c, third);
        return b.idx(tt, third, c);
    }
    // shared-memory slot of (s, t): x-contiguous in both layouts
    static __device__ __forceinline__ int slot(int s, int t) { return DIR == 0 ? t * SW_S + s : s * SW_T + t; }
    static __device__ __forceinline__ int fslot(int f, int t) { return DIR == 0 ? t * SW_F + f : f * SW_T + t; }
    // decode a linear work index into (s, t) with the x-direction fastest
    static __device__ __forceinline__ void decode(int idx, int ns, int& s, int& t) {
        if (DIR == 0) { s = idx % ns; t = idx / ns; }
        else { t = idx % SW_T; s = idx / SW_T; }
    }
};

template <int DIR, int RECON, typename R>
__global__ void __launch_bounds__(SW_THREADS, 2) k_sweep_tile(Box b, Tabs T, PrimT<R> pr, R ggas, FaceFluxT<R> out) {
    if (b.skip && *b.skip) return;
    extern __shared__ __align__(16) unsigned char sw_raw[];
    R* sm = reinterpret_cast<R*>(sw_raw);
    R* C = sm;                                   // [7][S*T] cell values
    R* D = C + SW_NV * SW_S * SW_T;              // [7][S*T] limited slopes
    R* V = D + SW_NV * SW_S * SW_T;              // [7][S*T] interface values
    R* WL = V + SW_NV * SW_S * SW_T;             // [7][F*T] left states
    R* WR = WL + SW_NV * SW_F * SW_T;            // [7][F*T] right states
    const SweepGeom<DIR> g(b);
    const AxisTabs A = T.ax[DIR];
    const int tid = threadIdx.x;
    constexpr int bt_a = DIR == 0 ? 1 : 0;
    constexpr int bt_b = DIR == 2 ? 1 : 2;
    const R* src[SW_NV] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[bt_a], pr.bc[bt_b]};
    constexpr int SS = SW_S * SW_T;

    // 1. cells f0-2 .. f0+F+2 along DIR (all loads in bounds of the ghosted box)
    for (int idx = tid; idx < SW_NV * SS; idx += SW_THREADS) {
        const int v = idx / SS;
        int s, t;
        SweepGeom<DIR>::decode(idx - v * SS, SW_S, s, t);
        const int c = g.f0 - 2 + s, tt = g.t0 + t;
        R x = R(0);
        if (c <= g.nd + 3 && tt <= g.tmax) x = src[v][g.gidx(b, c, tt)];
        C[v * SS + SweepGeom<DIR>::slot(s, t)] = x;
    }
    __syncthreads();

    if (RECON == 4) {
        // 2. limited slope of cells -1 .. nd+2 (solver/reconstruct.f90:254-280)
        for (int idx = tid; idx < SW_NV * SS; idx += SW_THREADS) {
            const int v = idx / SS;
            int s, t;
            SweepGeom<DIR>::decode(idx - v * SS, SW_S, s, t);
            const int c = g.f0 - 2 + s;
            if (s < 1 || s > SW_S - 2 || c > g.nd + 2) continue;
            const R* Cv = C + v * SS;
            D[v * SS + SweepGeom<DIR>::slot(s, t)] =
                ppm_slope(Cv[SweepGeom<DIR>::slot(s - 1, t)], Cv[SweepGeom<DIR>::slot(s, t)],
                          Cv[SweepGeom<DIR>::slot(s + 1, t)], (R)A.s0[c], (R)A.s1[c]);
        }
        __syncthreads();
        // 3. interface value between cell c and c+1, c = -1 .. nd+1 (:285-286)
        for (int idx = tid; idx < SW_NV * SS; idx += SW_THREADS) {
            const int v = idx / SS;
            int s, t;
            SweepGeom<DIR>::decode(idx - v * SS, SW_S, s, t);
            const int c = g.f0 - 2 + s;
            if (s < 1 || s > SW_S - 3 || c > g.nd + 1) continue;
            const R* Cv = C + v * SS;
            const R* Dv = D + v * SS;
            const int p = SweepGeom<DIR>::slot(s, t), q = SweepGeom<DIR>::slot(s + 1, t);
            V[v * SS + p] = ppm_face(Cv[p], Cv[q], Dv[p], Dv[q], (R)A.a0[c], (R)A.a1[c], (R)A.a2[c], (R)A.a3[c]);
        }
        __syncthreads();
    }
    // 4. extremum fix of cells 0 .. nd+1: vp_out -> left state of face c,
    //    vm_out -> right state of face c-1 (:289-307, solver/spatial.f90:138)
    for (int idx = tid; idx < SW_NV * SS; idx += SW_THREADS) {
        const int v = idx / SS;
        int s, t;
        SweepGeom<DIR>::decode(idx - v * SS, SW_S, s, t);
        const int c = g.f0 - 2 + s;
        if (s < 2 || s > SW_S - 3 || c > g.nd + 1) continue;
        const R* Cv = C + v * SS;
        const int p = SweepGeom<DIR>::slot(s, t);
        R vm, vp;
        if (RECON == 4) {
            const R* Vv = V + v * SS;
            ppm_fix(Cv[p], Vv[SweepGeom<DIR>::slot(s - 1, t)], Vv[p], vm, vp);
        } else {
            const R sl = tvd_slope(Cv[SweepGeom<DIR>::slot(s - 1, t)], Cv[p], Cv[SweepGeom<DIR>::slot(s + 1, t)],
                                   (R)A.tcf[c], (R)A.tcb[c]);
            vp = Cv[p] + R(0.5) * sl;
            vm = Cv[p] - R(0.5) * sl;
        }
        if (s - 2 < SW_F) WL[v * SW_F * SW_T + SweepGeom<DIR>::fslot(s - 2, t)] = vp;
        if (s - 3 >= 0) WR[v * SW_F * SW_T + SweepGeom<DIR>::fslot(s - 3, t)] = vm;
    }
    __syncthreads();

    // 5. HLL at the tile's faces (solver/rsolver.f90:43-130)
    int f, t;
    if (DIR == 0) { f = tid % SW_F; t = tid / SW_F; }
    else { t = tid % SW_T; f = tid / SW_T; }
    const int c = g.f0 + f, tt = g.t0 + t;
    if (c > g.nd || tt > g.tmax) return;
    const int slot[SW_NV] = {IRHO, IVX, IVY, IVZ, ITAU, IBX + bt_a, IBX + bt_b};
    R wl[8], wr[8];
#pragma unroll
    for (int v = 0; v < SW_NV; ++v) {
        wl[slot[v]] = WL[v * SW_F * SW_T + SweepGeom<DIR>::fslot(f, t)];
        wr[slot[v]] = WR[v * SW_F * SW_T + SweepGeom<DIR>::fslot(f, t)];
    }
    const int gi = g.gidx(b, c, tt);
    const R bn = pr.bf[DIR][gi];
    wl[IBX + DIR] = bn;
    wr[IBX + DIR] = bn;
    R fx[7];
    sweep_hll<DIR, R, false>(wl, wr, ggas, fx);
#pragma unroll
    for (int i = 0; i < 7; ++i) out.f[i][gi] = fx[i];
}

template <int DIR>
inline dim3 sweep_grid(const Box& b) {
    if (DIR == 0) return dim3((b.nx + 1 + SW_F - 1) / SW_F, (b.ny + 2 + SW_T - 1) / SW_T, b.nz + 2);
    if (DIR == 1) return dim3((b.nx + 2 + SW_T - 1) / SW_T, (b.ny + 1 + SW_F - 1) / SW_F, b.nz + 2);
    return dim3((b.nx + 2 + SW_T - 1) / SW_T, (b.nz + 1 + SW_F - 1) / SW_F, b.ny + 2);
}

}  // namespace cumc
