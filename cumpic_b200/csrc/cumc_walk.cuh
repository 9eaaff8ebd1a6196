// cumc_walk.cuh — column-walking sweep for the y and z directions
// (GET_FLUXES interpolate + RIEMANN, solver/spatial.f90:209-246, 287-324).
//
// Each thread owns one column (an x position and a position along the third
// axis) and walks along the sweep direction over a segment of faces. A sliding
// window of five values per reconstructed field stays in registers:
//   v(f+1), v(f+2), limited slope of cell f+1, interface value between f and
//   f+1, and vp_out(f).
// Per face the thread loads one new cell per field (coalesced: consecutive
// threads hold consecutive x), forms one limited slope, one interface value
// and one extremum fix, and solves one HLL problem. Every quantity the
// reference evaluates several times per cell (solver/reconstruct.f90:254-307)
// is formed exactly once, with the reference's expression trees, so the fluxes
// are bit-identical to the per-face evaluation. Only the segment prologue
// (three slopes, two interface values, one fix) is repeated per segment.
#pragma once
#include "cumc_kernels.cuh"

namespace cumc {

constexpr int WK_THREADS = 64;

template <int DIR>
struct WalkGeom {
    static_assert(DIR == 1 || DIR == 2, "the walker sweeps along y or z");
    __host__ __device__ static int nd(const Box& b) { return DIR == 1 ? b.ny : b.nz; }
    __host__ __device__ static int n3(const Box& b) { return DIR == 1 ? b.nz : b.ny; }
    __host__ __device__ static int stride(const Box& b) { return DIR == 1 ? b.SX : b.SX * b.SY; }
    // columns: x in 0:nx+1, third in 0:n3+1
    __host__ __device__ static long long ncols(const Box& b) { return (long long)(b.nx + 2) * (n3(b) + 2); }
    __device__ static int idx(const Box& b, int j, int third, int c) {
        return DIR == 1 ? b.idx(j, c, third) : b.idx(j, third, c);
    }
};

// faces per segment: segments of near-equal length close to `target`
inline int walk_segment(int faces, int target, int* nseg) {
    int n = (faces + target - 1) / target;
    if (n < 1) n = 1;
    *nseg = n;
    return (faces + n - 1) / n;
}

template <int DIR, int RECON, typename R>
__global__ void __launch_bounds__(WK_THREADS, 5) k_sweep_walk(Box b, Tabs T, PrimT<R> pr, R ggas, FaceFluxT<R> out,
                                                             int seg) {
    using G = WalkGeom<DIR>;
    const long long col = (long long)blockIdx.x * WK_THREADS + threadIdx.x;
    if (col >= G::ncols(b) || (b.skip && *b.skip)) return;
    const int j = (int)(col % (b.nx + 2));
    const int third = (int)(col / (b.nx + 2));
    const int nd = G::nd(b);
    const int f0 = blockIdx.y * seg;
    if (f0 > nd) return;
    const int f1 = min(f0 + seg, nd + 1);
    const int s = G::stride(b);
    const int base = G::idx(b, j, third, 0);  // cell index 0 along DIR
    const AxisTabs A = T.ax[DIR];
    constexpr int bt_a = 0;                    // tangential cell fields: bx and (bz for y, by for z)
    constexpr int bt_b = DIR == 2 ? 1 : 2;
    const R* src[7] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[bt_a], pr.bc[bt_b]};
    const int slot[7] = {IRHO, IVX, IVY, IVZ, ITAU, IBX + bt_a, IBX + bt_b};
    const R* bn_src = pr.bf[DIR];

    // window (see file comment); v0 = v(f) is carried for TVD only
    R v0[7], v1[7], v2[7], d1[7], Vf[7], vpf[7], nxt[7];
#pragma unroll
    for (int v = 0; v < 7; ++v) {
        const R* q = src[v] + base;
        const R x0 = q[(f0 - 2) * s], x1 = q[(f0 - 1) * s], x2 = q[f0 * s], x3 = q[(f0 + 1) * s],
                x4 = q[(f0 + 2) * s];
        if (RECON == 4) {
            const R dm0 = ppm_slope(x0, x1, x2, (R)A.s0[f0 - 1], (R)A.s1[f0 - 1]);
            const R dmc = ppm_slope(x1, x2, x3, (R)A.s0[f0], (R)A.s1[f0]);
            const R dmp = ppm_slope(x2, x3, x4, (R)A.s0[f0 + 1], (R)A.s1[f0 + 1]);
            const R Vm = ppm_face(x1, x2, dm0, dmc, (R)A.a0[f0 - 1], (R)A.a1[f0 - 1], (R)A.a2[f0 - 1], (R)A.a3[f0 - 1]);
            const R Vp = ppm_face(x2, x3, dmc, dmp, (R)A.a0[f0], (R)A.a1[f0], (R)A.a2[f0], (R)A.a3[f0]);
            R vm, vp;
            ppm_fix(x2, Vm, Vp, vm, vp);
            vpf[v] = vp;
            d1[v] = dmp;
            Vf[v] = Vp;
        } else {
            vpf[v] = x2 + R(0.5) * tvd_slope(x1, x2, x3, (R)A.tcf[f0], (R)A.tcb[f0]);
        }
        v0[v] = x2;
        v1[v] = x3;
        v2[v] = x4;
        nxt[v] = q[(f0 + 3) * s];
    }

    for (int f = f0; f < f1; ++f) {
        R wl[8], wr[8];
        const R bn = bn_src[base + f * s];
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            const R x = nxt[v];
            R vm1, vp1;
            if (RECON == 4) {
                const R d2 = ppm_slope(v1[v], v2[v], x, (R)A.s0[f + 2], (R)A.s1[f + 2]);
                const R Vn = ppm_face(v1[v], v2[v], d1[v], d2, (R)A.a0[f + 1], (R)A.a1[f + 1], (R)A.a2[f + 1],
                                      (R)A.a3[f + 1]);
                ppm_fix(v1[v], Vf[v], Vn, vm1, vp1);
                d1[v] = d2;
                Vf[v] = Vn;
            } else {
                const R sl = tvd_slope(v0[v], v1[v], v2[v], (R)A.tcf[f + 1], (R)A.tcb[f + 1]);
                vm1 = v1[v] - R(0.5) * sl;
                vp1 = v1[v] + R(0.5) * sl;
            }
            wl[slot[v]] = vpf[v];  // vp_out of cell f
            wr[slot[v]] = vm1;     // vm_out of cell f+1
            vpf[v] = vp1;
            v0[v] = v1[v];
            v1[v] = v2[v];
            v2[v] = x;
        }
        // prefetch the next cell (f+4 <= nd+3 while f+1 < f1)
        if (f + 1 < f1) {
#pragma unroll
            for (int v = 0; v < 7; ++v) nxt[v] = src[v][base + (f + 4) * s];
        }
        wl[IBX + DIR] = bn;
        wr[IBX + DIR] = bn;
        R fx[7];
        hll_flux7<DIR>(wl, wr, ggas, fx);
        const int o = base + f * s;
#pragma unroll
        for (int i = 0; i < 7; ++i) out.f[i][o] = fx[i];
    }
}

}  // namespace cumc
