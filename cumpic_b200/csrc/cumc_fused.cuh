// cumc_fused.cuh — directional sweeps with the flux difference fused in
// (GET_FLUXES, solver/spatial.f90:113-380, and the RK stage combine of
// solver/rungekutta.f90:41-51,75-85,109-119 for the hydro variables).
//
// One FP64 stage runs as
//   k_sweep_xacc    x faces; rows staged into shared memory by bulk tensor
//                   copies (TMA); L = 0 - dFx/dx of every interior cell
//   k_walk_acc<1>   y faces; L = L - dFy/dy
//   k_walk_acc<2>   z faces; L = L - dFz/dz + sources, then the RK combine of
//                   rho, rho v, E on (0:n)^3 written straight to the stage's
//                   output state
//   k_emf, k_ct     edge EMFs and the face-field CT update (cumc_kernels.cuh)
//   k_utop_stage    FROMUTORVE, CUSTOM_CHECKRHO, P_to_U, UPDATE's pressure,
//                   and at stage 3 the next step's CFL dt
//   k_boundary
// Only the two tangential-field fluxes of each face (for the edge EMFs) and
// the flux-difference accumulator L (5 values a cell) reach HBM between the
// sweeps; the hydro face fluxes stay in registers. The flux difference of a
// cell needs the fluxes of its two faces along the sweep: a lane-per-cell x
// sweep takes the left face from the neighbouring lane (or, at a chunk's first
// cell, from the previous chunk of the same row), a column walker carries the
// previous face's fluxes from one face to the next.
//
// Every value is formed by the same expressions, in the same order, as the
// unfused kernels (k_sweep_xwarp, k_sweep_walk_sm, k_combine_utop): L starts
// at 0 and takes the x, y and z differences in that order, then the sources.
// The fused stage is bit for bit the unfused one.
#pragma once
#include "cumc_kernels.cuh"
#include "cumc_tma.cuh"
#include "cumc_walk.cuh"

namespace cumc {

// outputs and inputs of the fused stage kernels
struct AccArgs {
    double* L[5];          // flux-difference accumulator of rho, rho v, E (interior cells)
    double* fb[3][2];      // tangential-field fluxes of the x, y, z faces (FaceFlux slots 5 and 6)
    // z sweep only: the stage combine
    const double* u0[5];   // u_old
    const double* uc[5];   // cons entering the combine (stages 2 and 3)
    double* ud[5];         // result (may alias u0 or uc: pointwise)
    double* tape[5];       // when set: a copy of the combine's output
    const double* dt;      // device scalar
    int stage;             // 1, 2, 3
    int model;             // CUMC_MODEL_* of the sources
    int geom_repeat;
    double rho_floor, r_sh;
    unsigned int* err;     // device error word (bit 1: a staged copy never completed)
};

// the stage combine of one value at run-time stage s (rk_point's bits)
__device__ __forceinline__ double rk_stage_point(int s, double u0, double uc, double dt, double L) {
    if (s == 1) return rk_point<1>(u0, 0.0, dt, L);
    if (s == 2) return rk_point<2>(u0, uc, dt, L);
    return rk_point<3>(u0, uc, dt, L);
}

template <int COORD>
__device__ __forceinline__ void sources_rt(const Tabs& T, const Prim& pr, const AccArgs& a, int j, int k, int l, int i,
                                           double* sc) {
    switch (a.model) {
        case CUMC_MODEL_TORUS_SPH: cell_sources<COORD, 2>(T, pr, a.geom_repeat, a.rho_floor, a.r_sh, j, k, l, i, sc); break;
        case CUMC_MODEL_TORUS_CYN: cell_sources<COORD, 3>(T, pr, a.geom_repeat, a.rho_floor, a.r_sh, j, k, l, i, sc); break;
        default: cell_sources<COORD, 1>(T, pr, a.geom_repeat, a.rho_floor, a.r_sh, j, k, l, i, sc); break;
    }
}

// ----------------------------------------------------------------------------
// x sweep with one lane per cell (as k_sweep_xwarp) and the x flux difference.
// A block holds XA_ROWS consecutive rows (y) of one z plane, one warp a row;
// each warp walks its row in chunks of 32 cells that yield 27 faces (lanes
// 2..28), consecutive chunks overlapping by 5 cells. With TMA, one thread
// stages the block's next chunk of all 8 fields (the 7 reconstructed fields
// and the face field Bx) into shared memory as 3-D boxes while the warps work
// on the current one (two buffers, one mbarrier each); without it (rows whose
// pitch is not a multiple of 16 bytes) every lane loads its cells directly.
// The flux difference of cell c takes face c-1 from the next lower lane, and
// at lane 2 from lane 28 of the previous chunk.
// ----------------------------------------------------------------------------
constexpr int XA_ROWS = 6;
constexpr int XA_FACES = 27;
constexpr int XA_BOX = 34;            // staged cells a row and chunk (the 32 of the chunk, start rounded to even)
constexpr int XA_FSTRIDE = 208;       // doubles per staged field box (6 x 34, padded to 128-byte multiples)
constexpr int XA_FIELDS = 8;
constexpr uint32_t XA_BYTES = XA_FIELDS * XA_ROWS * XA_BOX * sizeof(double);  // bytes one chunk lands
// dynamic shared memory: up to 128 bytes to reach a 128-byte boundary, the
// two mbarriers (128 bytes), then the two chunk buffers
constexpr size_t xacc_smem(bool tma) {
    return tma ? 256 + 2 * (size_t)XA_FIELDS * XA_FSTRIDE * sizeof(double) : 0;
}

// tensor maps of the 8 staged fields: rho, vx, vy, vz, p, by, bz (cell) and Bx (face)
struct XaccMaps {
    CUtensorMap m[XA_FIELDS];
};

// rows of the z planes l_lo .. l_lo + gridDim.y - 1
template <int RECON, int COORD, bool TMA>
__global__ void __launch_bounds__(32 * XA_ROWS, 5) k_sweep_xacc(Box b, Tabs T, Prim pr, double ggas, AccArgs a,
                                                               const __grid_constant__ XaccMaps maps, int l_lo) {
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(128) unsigned char xa_raw[];
    if (b.skip && *b.skip) return;
    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
    const int k = blockIdx.x * XA_ROWS + r, l = l_lo + (int)blockIdx.y;
    const bool row_ok = k <= b.ny + 1;
    const bool row_inner = k >= 1 && k <= b.ny && l >= 1 && l <= b.nz;
    const int nw = (b.nx + 1 + XA_FACES - 1) / XA_FACES;  // chunks a row
    const int base = b.idx(0, min(k, b.ny + 1), l);
    const AxisTabs A = T.ax[0];
    const double* src[XA_FIELDS] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[1], pr.bc[2], pr.bf[0]};
    const int slot[7] = {IRHO, IVX, IVY, IVZ, ITAU, IBY, IBZ};

    unsigned char* const al = xa_raw + ((128u - (smem_u32(xa_raw) & 127u)) & 127u);  // bulk copies land on 128 B
    uint64_t* bar = reinterpret_cast<uint64_t*>(al);
    double* stage = reinterpret_cast<double*>(al + 128);
    auto issue = [&](int w) {  // one thread: chunk w of every field into buffer w & 1
        double* dst = stage + (size_t)(w & 1) * XA_FIELDS * XA_FSTRIDE;
        mbar_expect_tx(&bar[w & 1], XA_BYTES);
        const int x0 = (XA_FACES * w) & ~1, y0 = blockIdx.x * XA_ROWS + 2, z0 = l + 2;
#pragma unroll
        for (int v = 0; v < XA_FIELDS; ++v) tma_load_3d(dst + v * XA_FSTRIDE, &maps.m[v], x0, y0, z0, &bar[w & 1]);
    };
    if (TMA) {
        if (threadIdx.x == 0) {
            for (int v = 0; v < XA_FIELDS; ++v) tma_prefetch_map(&maps.m[v]);
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
            mbar_fence_init();
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            issue(0);
            if (nw > 1) issue(1);
        }
    }

    double carry[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // hydro fluxes of lane 28 of the previous chunk
    bool staged_ok = true;
    for (int w = 0; w < nw; ++w) {
        const int c = w * XA_FACES - 2 + lane;  // this lane's cell; its face is c | c+1
        const bool inb = c >= -2 && c <= b.nx + 3;
        const int ct = min(max(c, -2), b.nx + 3);  // table index kept in range for spare lanes
        double x8[XA_FIELDS];
        if (TMA) {
            if (staged_ok) staged_ok = mbar_wait(&bar[w & 1], (w >> 1) & 1, a.err);
            const double* buf = stage + (size_t)(w & 1) * XA_FIELDS * XA_FSTRIDE + r * XA_BOX +
                                lane + ((XA_FACES * w) & 1);
#pragma unroll
            for (int v = 0; v < XA_FIELDS; ++v) x8[v] = staged_ok ? buf[v * XA_FSTRIDE] : 0.0;
        } else {
#pragma unroll
            for (int v = 0; v < XA_FIELDS; ++v) x8[v] = inb ? src[v][base + c] : 0.0;
        }
        double wl[8], wr[8];
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            const double x = x8[v];
            const double xm = __shfl_up_sync(FULL, x, 1), xp = __shfl_down_sync(FULL, x, 1);
            double vm, vp;
            if (RECON == 4) {
                const double d = ppm_slope(xm, x, xp, A.s0[ct], A.s1[ct]);
                const double dp = __shfl_down_sync(FULL, d, 1);
                const double V = ppm_face(x, xp, d, dp, A.a0[ct], A.a1[ct], A.a2[ct], A.a3[ct]);  // c | c+1
                const double Vm = __shfl_up_sync(FULL, V, 1);                                       // c-1 | c
                ppm_fix(x, Vm, V, vm, vp);
            } else {
                const double sl = tvd_slope(xm, x, xp, A.tcf[ct], A.tcb[ct]);
                vm = x - 0.5 * sl;
                vp = x + 0.5 * sl;
            }
            wl[slot[v]] = vp;                             // vp_out of cell c
            wr[slot[v]] = __shfl_down_sync(FULL, vm, 1);  // vm_out of cell c+1
        }
        const bool face = lane >= 2 && lane <= 28 && c >= 0 && c <= b.nx;
        double F[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (face) {
            wl[IBX] = x8[7];
            wr[IBX] = x8[7];
            hll_flux7<0>(wl, wr, ggas, F);
        }
        // the left face of cell c: lane-1, or lane 28 of the previous chunk
        double Fm[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double up = __shfl_up_sync(FULL, F[q], 1);
            Fm[q] = lane == 2 ? carry[q] : up;
            carry[q] = __shfl_sync(FULL, F[q], 28);
        }
        if (TMA) {
            __syncthreads();  // every warp has read buffer w & 1
            if (threadIdx.x == 0 && w + 2 < nw && staged_ok) issue(w + 2);
        }
        if (!face || !row_ok) continue;
        a.fb[0][0][base + c] = F[5];
        a.fb[0][1][base + c] = F[6];
        if (row_inner && c >= 1) {
            double gp, gc, gm;
            geom_flux<COORD, 0>(T, c, k, l, gp, gc, gm);
#pragma unroll
            for (int q = 0; q < 5; ++q) a.L[q][base + c] = 0.0 - (F[q] * gp - Fm[q] * gm) / gc;
        }
    }
}

inline dim3 xacc_grid(const Box& b, int planes) {
    return dim3((unsigned)((b.ny + 2 + XA_ROWS - 1) / XA_ROWS), (unsigned)planes);
}

// ----------------------------------------------------------------------------
// y and z sweeps: the shared-memory-window column walker of k_sweep_walk_sm
// with the flux difference along the walk. Each segment starts one face early
// (except the first), so the face below its first cell is formed there; that
// face's outputs belong to the previous segment and are not stored.
// DIR 1: L = L - dFy/dy on interior cells. DIR 2: L = L - dFz/dz + sources on
// interior cells (0 elsewhere on (0:n)^3), then the RK combine of the hydro
// variables into the stage's output state (and its tape).
// The values a cell's epilogue reads (L; for DIR 2 also u_old and the stage's
// cons) are fetched by asynchronous copies into the thread's own shared-memory
// slots one face ahead, so their latency hides behind the next face's
// reconstruction and HLL solve.
// The columns walked are those whose slow transverse index (z for DIR 1, y
// for DIR 2) lies in c_lo .. c_lo + c_cnt - 1.
// ----------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <int DIR>
constexpr int acc_prefetch() { return DIR == 1 ? 5 : 15; }  // L; L, u_old, cons
template <int DIR>
constexpr size_t acc_smem() {
    return (size_t)(WK_SLOTS * WK_FIELDS + acc_prefetch<DIR>()) * WK_THREADS * sizeof(double);
}

template <int DIR, int RECON, int COORD>
__global__ void __launch_bounds__(WK_THREADS) k_walk_acc(Box b, Tabs T, Prim pr, double ggas, AccArgs a, int seg,
                                                        int c_lo, int c_cnt) {
    static_assert(DIR == 1 || DIR == 2, "y and z sweeps");
    extern __shared__ __align__(16) unsigned char wk_raw[];
    double* const sm = reinterpret_cast<double*>(wk_raw) + threadIdx.x;
    auto at = [&](int slot, int v) -> double& { return sm[(slot * WK_FIELDS + v) * WK_THREADS]; };
    double* const pf = sm + WK_SLOTS * WK_FIELDS * WK_THREADS;  // prefetch slot k at pf[k * WK_THREADS]
    if (b.skip && *b.skip) return;
    using G = WalkGeom<DIR>;
    const long long ncols = (long long)G::wa(b) * c_cnt;
    const long long col = (long long)blockIdx.x * WK_THREADS + threadIdx.x;
    const bool active = col < ncols;
    const long long cc = min(col, ncols - 1);
    const int ca = (int)(cc % G::wa(b)), cb = c_lo + (int)(cc / G::wa(b));  // x, and z (DIR 1) or y (DIR 2)
    const int nd = G::nd(b);
    const int fc = blockIdx.y * seg;  // first face whose outputs this segment stores
    if (fc > nd) return;
    const int f0 = fc > 0 ? fc - 1 : 0;
    const int f1 = min(fc + seg, nd + 1);
    const int s = G::stride(b);
    const int base = G::idx(b, ca, cb, 0);
    constexpr int ta = 0;  // tangential cell fields: (bx, bz) for y, (bx, by) for z
    constexpr int tb = DIR == 1 ? 2 : 1;
    const double* srcv[WK_FIELDS] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[ta], pr.bc[tb]};
    constexpr int slot[WK_FIELDS] = {IRHO, IVX, IVY, IVZ, ITAU, IBX + ta, IBX + tb};
    const double* bnp = pr.bf[DIR] + base;
    const AxisTabs A = T.ax[DIR];
    // the cell's transverse position and whether it can be interior / on (0:n)^3
    const bool t_inner = active && (DIR == 1 ? (ca >= 1 && ca <= b.nx && cb >= 1 && cb <= b.nz)
                                             : (ca >= 1 && ca <= b.nx && cb >= 1 && cb <= b.ny));
    const bool t_box1 = DIR == 2 && active && ca <= b.nx && cb <= b.ny;
    const double dt = DIR == 2 ? *a.dt : 0.0;
    auto inner = [&](int f) { return t_inner && f >= fc && f >= 1 && f <= nd; };
    auto combined = [&](int f) { return t_box1 && f >= fc && f <= nd; };
    // queue the copies of what cell f's epilogue reads
    auto prefetch = [&](int f) {
        const int i = base + f * s;
        if (inner(f)) {
#pragma unroll
            for (int q = 0; q < 5; ++q) cp_async8(pf + q * WK_THREADS, a.L[q] + i);
        }
        if (DIR == 2 && combined(f)) {
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                cp_async8(pf + (5 + q) * WK_THREADS, a.u0[q] + i);
                if (a.stage != 1) cp_async8(pf + (10 + q) * WK_THREADS, a.uc[q] + i);
            }
        }
        cp_async_commit();
    };

    double nxt[WK_FIELDS];
    int r0 = f0 % 3, r1 = (f0 + 1) % 3, r2 = (f0 + 2) % 3;
#pragma unroll
    for (int v = 0; v < WK_FIELDS; ++v) {
        const double* q = srcv[v] + base;
        const double x0 = q[(f0 - 2) * s], x1 = q[(f0 - 1) * s], x2 = q[f0 * s], x3 = q[(f0 + 1) * s],
                     x4 = q[(f0 + 2) * s];
        double vpf, d1, Vf;
        walk_prologue<RECON>(A, f0, x0, x1, x2, x3, x4, vpf, d1, Vf);
        at(r0, v) = x2;
        at(r1, v) = x3;
        at(r2, v) = x4;
        at(3, v) = d1;
        at(4, v) = Vf;
        at(5, v) = vpf;
        nxt[v] = q[(f0 + 3) * s];
    }
    prefetch(f0);

    double carry[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // hydro fluxes of face f-1
    for (int f = f0; f < f1; ++f) {
        double wl[8], wr[8];
        const double bn = bnp[f * s];
#pragma unroll
        for (int v = 0; v < WK_FIELDS; ++v) {
            const double x = nxt[v];
            double d1 = at(3, v), Vf = at(4, v);
            double vm1, vp1;
            walk_step<RECON>(A, f, RECON == 4 ? 0.0 : at(r0, v), at(r1, v), at(r2, v), x, d1, Vf, vm1, vp1);
            wl[slot[v]] = at(5, v);  // vp_out of cell f
            wr[slot[v]] = vm1;       // vm_out of cell f+1
            at(5, v) = vp1;
            if (RECON == 4) {
                at(3, v) = d1;
                at(4, v) = Vf;
            }
            at(r0, v) = x;  // v(f+3) replaces v(f)
        }
        const int rr = r0;
        r0 = r1;
        r1 = r2;
        r2 = rr;
        if (f + 1 < f1) {
#pragma unroll
            for (int v = 0; v < WK_FIELDS; ++v) nxt[v] = srcv[v][base + (f + 4) * s];
        }
        wl[IBX + DIR] = bn;
        wr[IBX + DIR] = bn;
        double F[7];
        hll_flux7<DIR>(wl, wr, ggas, F);
        cp_async_wait_all();  // cell f's epilogue values have landed
        const int i = base + f * s;
        if (active && f >= fc) {
            a.fb[DIR][0][i] = F[5];
            a.fb[DIR][1][i] = F[6];
        }
        // cell f: faces f-1 (carried) and f
        const int j = ca, k = DIR == 1 ? f : cb, l = DIR == 1 ? cb : f;
        if (DIR == 1) {
            if (inner(f)) {
                double gp, gc, gm;
                geom_flux<COORD, 1>(T, j, k, l, gp, gc, gm);
#pragma unroll
                for (int q = 0; q < 5; ++q) a.L[q][i] = pf[q * WK_THREADS] - (F[q] * gp - carry[q] * gm) / gc;
            }
        } else if (combined(f)) {
            double L[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            if (inner(f)) {
                double gp, gc, gm;
                geom_flux<COORD, 2>(T, j, k, l, gp, gc, gm);
#pragma unroll
                for (int q = 0; q < 5; ++q) L[q] = pf[q * WK_THREADS] - (F[q] * gp - carry[q] * gm) / gc;
                double sc[5];
                sources_rt<COORD>(T, pr, a, j, k, l, i, sc);
#pragma unroll
                for (int q = 0; q < 5; ++q) L[q] = L[q] + sc[q];
            }
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double u = rk_stage_point(a.stage, pf[(5 + q) * WK_THREADS],
                                                 a.stage == 1 ? 0.0 : pf[(10 + q) * WK_THREADS], dt, L[q]);
                a.ud[q][i] = u;
                if (a.tape[q]) a.tape[q][i] = u;
            }
        }
        if (f + 1 < f1) prefetch(f + 1);
#pragma unroll
        for (int q = 0; q < 5; ++q) carry[q] = F[q];
    }
    cp_async_wait_all();
}

// ----------------------------------------------------------------------------
// the conversions of a stage whose hydro combine ran in the z sweep: on
// (0:n)^3, bcell from the updated face fields (interior), then FROMUTORVE,
// CUSTOM_CHECKRHO, P_to_U and UPDATE's pressure from the combined cons in
// o.u (utop_point, the expressions of k_combine_utop); at stage 3 with
// o.dtmin set, also the next step's CFL dt (every thread reaches the block
// reduction).
// ----------------------------------------------------------------------------
template <int COORD, int MODEL>
__global__ void __launch_bounds__(256, 8) k_utop_stage(Box b, Tabs T, UtopArgs o) {
    if (b.skip && *b.skip) return;
    int j, k, l, i;
    const bool live = box1_index(b, j, k, l, i);
    const bool fuse_dt = o.dtmin != nullptr;
    if (!live && !fuse_dt) return;
    double dt_cell = 1.0e10;
    if (live) {
        double uh[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) uh[q] = o.u[q][i];
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

}  // namespace cumc
