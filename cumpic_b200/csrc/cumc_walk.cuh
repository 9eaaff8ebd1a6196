// cumc_walk.cuh — column-walking directional sweeps
// (GET_FLUXES interpolate + RIEMANN, solver/spatial.f90:170-324).
//
// Each thread owns one column (a fixed pair of transverse indices) and walks
// along the sweep direction over a segment of faces. A sliding window of
// five values per reconstructed field is carried from face f to face f+1:
//   v(f+1), v(f+2), the limited slope of cell f+1, the interface value
//   between cells f and f+1, and vp_out(f).
// Per face the thread loads one new cell per field, forms one limited slope,
// one interface value and one extremum fix, and solves one HLL problem. Every
// quantity the reference evaluates several times per cell
// (solver/reconstruct.f90:254-307) is formed exactly once, with the
// reference's expression trees, so the fluxes are bit-identical to the
// per-face evaluation. Only the segment prologue (three slopes, two interface
// values, one fix) is repeated per segment.
//
// Two storage forms of the window:
//   k_sweep_walk     window in registers (168 registers a thread in FP64,
//                    which caps residency near 12 warps per SM);
//   k_sweep_walk_sm  window in shared memory, one private slot column per
//                    thread ([slot][field][thread], so a warp's accesses are
//                    conflict-free), which frees about 70 registers a thread.
// Along y and z consecutive threads hold consecutive x, so every load is
// coalesced. Along x consecutive threads hold consecutive y rows; each load
// touches one 32-byte sector per row, which the following three faces reuse
// from L1.
#pragma once
#include "cumc_kernels.cuh"

namespace cumc {

constexpr int WK_THREADS = 64;
// resident blocks per SM the walker and the x sweep are compiled for (the
// register budget a thread gets); build-time tunables
#ifndef CUMC_WALK_MINB
#define CUMC_WALK_MINB 9
#endif
#ifndef CUMC_XWARP_MINB
#define CUMC_XWARP_MINB 8
#endif
constexpr int WK_FIELDS = 7;  // rho, vx, vy, vz, p and the two tangential cell fields

template <int DIR>
struct WalkGeom {
    static_assert(DIR >= 0 && DIR <= 2, "sweep direction");
    __host__ __device__ static int nd(const Box& b) { return DIR == 0 ? b.nx : DIR == 1 ? b.ny : b.nz; }
    // transverse widths: a is the fast column index, c the slow one (each 0:n+1)
    __host__ __device__ static int wa(const Box& b) { return DIR == 0 ? b.ny + 2 : b.nx + 2; }
    __host__ __device__ static int wc(const Box& b) { return DIR == 2 ? b.ny + 2 : b.nz + 2; }
    __host__ __device__ static int stride(const Box& b) { return DIR == 0 ? 1 : DIR == 1 ? b.SX : b.SX * b.SY; }
    __host__ __device__ static long long ncols(const Box& b) { return (long long)wa(b) * wc(b); }
    __device__ static int idx(const Box& b, int a, int c, int f) {
        return DIR == 0 ? b.idx(f, a, c) : DIR == 1 ? b.idx(a, f, c) : b.idx(a, c, f);
    }
};

// faces per segment: segments of near-equal length close to `target`
inline int walk_segment(int faces, int target, int* nseg) {
    int n = (faces + target - 1) / target;
    if (n < 1) n = 1;
    *nseg = n;
    return (faces + n - 1) / n;
}

// segments of a walk along DIR over `ncols` columns: about 64 faces each,
// shorter (down to 8) while the grid would give fewer than 32 warps per SM,
// so that small boxes (a 128^3 adjoint box, the torus) still fill the GPU.
// Each segment repeats the walk's prologue (three slopes, two interface
// values, one fix a field), a few per cent of a face's work at 8 faces.
template <int DIR>
inline int walk_segment_for(const Box& b, long long ncols, int sm_count, int* nseg) {
    const int faces = WalkGeom<DIR>::nd(b) + 1;
    const long long blocks = (ncols + WK_THREADS - 1) / WK_THREADS;
    const long long want = (long long)sm_count * 32 / (WK_THREADS / 32);  // blocks for 32 warps per SM
    int target = 64;
    while (target > 8 && blocks * ((faces + target - 1) / target) < want) target /= 2;
    return walk_segment(faces, target, nseg);
}

// cell index 0 (along DIR) of column `col` of the block's grid, clamped to
// the last column so that the spare threads of the last block stay in bounds
template <int DIR>
__device__ __forceinline__ int walk_base(const Box& b, long long col) {
    using G = WalkGeom<DIR>;
    col = min(col, G::ncols(b) - 1);
    return G::idx(b, (int)(col % G::wa(b)), (int)(col / G::wa(b)), 0);
}

// column set-up shared by both window forms. Every thread of a block stays
// to the end (the x sweep synchronises the block); threads past the last
// column walk a copy of it and store nothing. The columns are those whose
// slow transverse index lies in c_lo .. c_lo + c_cnt - 1 (c_cnt < 0: all).
template <int DIR, typename R>
struct WalkCol {
    int base, s, f0, f1, nd;
    bool active;
    const R* src[WK_FIELDS];
    int slot[WK_FIELDS];
    const R* bn;
    __device__ bool init(const Box& b, const PrimT<R>& pr, int seg, int c_lo = 0, int c_cnt = -1) {
        using G = WalkGeom<DIR>;
        if (b.skip && *b.skip) return false;
        if (c_cnt < 0) c_cnt = G::wc(b);
        const long long ncols = (long long)G::wa(b) * c_cnt;
        const long long col = (long long)blockIdx.x * WK_THREADS + threadIdx.x;
        active = col < ncols;
        nd = G::nd(b);
        f0 = blockIdx.y * seg;
        if (f0 > nd) return false;
        f1 = min(f0 + seg, nd + 1);
        s = G::stride(b);
        const long long cc = min(col, ncols - 1);
        base = G::idx(b, (int)(cc % G::wa(b)), c_lo + (int)(cc / G::wa(b)), 0);
        // tangential cell fields: (by, bz) for x, (bx, bz) for y, (bx, by) for z
        constexpr int ta = DIR == 0 ? 1 : 0;
        constexpr int tb = DIR == 2 ? 1 : 2;
        const R* s7[WK_FIELDS] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[ta], pr.bc[tb]};
        const int q7[WK_FIELDS] = {IRHO, IVX, IVY, IVZ, ITAU, IBX + ta, IBX + tb};
#pragma unroll
        for (int v = 0; v < WK_FIELDS; ++v) {
            src[v] = s7[v] + base;
            slot[v] = q7[v];
        }
        bn = pr.bf[DIR] + base;
        return true;
    }
};

// x-sweep staging. Along x a thread's column is a row of the array, so a
// direct load by a warp touches 32 rows. Instead the block stages its 64
// rows through shared memory in chunks of XS_CELLS = 4 cells (one 32-byte
// sector a row): each warp load then covers 8 rows x 4 consecutive cells.
// A chunk holds cells cb..cb+3 of the 7 reconstructed fields and the normal
// field on faces fc..fc+3; layout [field][row][5] (one pad entry a row keeps
// a warp's 8-byte reads conflict-free).
constexpr int XS_CELLS = 4;
constexpr int XS_PITCH = XS_CELLS + 1;
template <typename R>
constexpr size_t xstage_smem() {
    return (size_t)(WK_FIELDS + 1) * WK_THREADS * XS_PITCH * sizeof(R);
}

//
// The 7 flux components of face f go back into the slots of field 0..6 at
// position (f - fc): by then the thread has consumed its own cells there.
// flush() writes a chunk's fluxes out in the same sector-sized pieces.
template <typename R>
struct XStage {
    R* buf;
    int rowbase[4];  // cell 0 of the rows this thread loads: tid/4 + 16 m
    bool rowok[4];   // the row is a real column (not a spare of the last block)
    const R* fld[WK_FIELDS + 1];
    __device__ void init(const Box& b, const PrimT<R>& pr, R* smem) {
        buf = smem;
        const R* f8[WK_FIELDS + 1] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[1], pr.bc[2], pr.bf[0]};
#pragma unroll
        for (int v = 0; v <= WK_FIELDS; ++v) fld[v] = f8[v];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const long long col = (long long)blockIdx.x * WK_THREADS + (threadIdx.x >> 2) + 16 * m;
            rowbase[m] = walk_base<0>(b, col);
            rowok[m] = col < WalkGeom<0>::ncols(b);
        }
    }
    // fluxes of faces fc..fc+3 (only those < fend)
    __device__ void flush(int fc, int fend, FaceFluxT<R>& out) const {
        const int j = threadIdx.x & 3;
        const int face = fc + j;
        if (face >= fend) return;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            if (!rowok[m]) continue;
            const int row = (threadIdx.x >> 2) + 16 * m;
#pragma unroll
            for (int v = 0; v < WK_FIELDS; ++v) out.f[v][rowbase[m] + face] = buf[(v * WK_THREADS + row) * XS_PITCH + j];
        }
    }
    __device__ void put(int v, int j, R x) { buf[(v * WK_THREADS + threadIdx.x) * XS_PITCH + j] = x; }
    // cells cb..cb+3 (only those <= last, the last ghost cell) and faces
    // fc..fc+3 (only those < fend)
    __device__ void load(int cb, int last, int fc, int fend) {
        const int j = threadIdx.x & 3;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int row = (threadIdx.x >> 2) + 16 * m;
#pragma unroll
            for (int v = 0; v <= WK_FIELDS; ++v) {
                const int cell = (v < WK_FIELDS ? cb : fc) + j;
                const bool ok = v < WK_FIELDS ? cell <= last : cell < fend;
                buf[(v * WK_THREADS + row) * XS_PITCH + j] = ok ? fld[v][rowbase[m] + cell] : R(0);
            }
        }
    }
    __device__ R get(int v, int j) const { return buf[(v * WK_THREADS + threadIdx.x) * XS_PITCH + j]; }
};

// segment prologue for one field: returns vp_out(f0), the slope of cell
// f0+1 and the interface value between f0 and f0+1 (PPM)
template <int RECON, typename R>
__device__ __forceinline__ void walk_prologue(const AxisTabs& A, int f0, R x0, R x1, R x2, R x3, R x4, R& vpf, R& d1,
                                              R& Vf) {
    if (RECON == 4) {
        const R dm0 = ppm_slope(x0, x1, x2, (R)A.s0[f0 - 1], (R)A.s1[f0 - 1]);
        const R dmc = ppm_slope(x1, x2, x3, (R)A.s0[f0], (R)A.s1[f0]);
        const R dmp = ppm_slope(x2, x3, x4, (R)A.s0[f0 + 1], (R)A.s1[f0 + 1]);
        const R Vm = ppm_face(x1, x2, dm0, dmc, (R)A.a0[f0 - 1], (R)A.a1[f0 - 1], (R)A.a2[f0 - 1], (R)A.a3[f0 - 1]);
        const R Vp = ppm_face(x2, x3, dmc, dmp, (R)A.a0[f0], (R)A.a1[f0], (R)A.a2[f0], (R)A.a3[f0]);
        R vm, vp;
        ppm_fix(x2, Vm, Vp, vm, vp);
        vpf = vp;
        d1 = dmp;
        Vf = Vp;
    } else {
        vpf = x2 + R(0.5) * tvd_slope(x1, x2, x3, (R)A.tcf[f0], (R)A.tcb[f0]);
        d1 = R(0);
        Vf = R(0);
    }
}

// one window step for one field at face f: from v(f) (TVD), v(f+1), v(f+2),
// the new cell x = v(f+3), the carried slope d1 and interface Vf, returns
// vm_out(f+1), vp_out(f+1) and updates d1, Vf
template <int RECON, typename R>
__device__ __forceinline__ void walk_step(const AxisTabs& A, int f, R v0, R v1, R v2, R x, R& d1, R& Vf, R& vm1,
                                          R& vp1) {
    if (RECON == 4) {
        const R d2 = ppm_slope(v1, v2, x, (R)A.s0[f + 2], (R)A.s1[f + 2]);
        const R Vn = ppm_face(v1, v2, d1, d2, (R)A.a0[f + 1], (R)A.a1[f + 1], (R)A.a2[f + 1], (R)A.a3[f + 1]);
        ppm_fix(v1, Vf, Vn, vm1, vp1);
        d1 = d2;
        Vf = Vn;
    } else {
        const R sl = tvd_slope(v0, v1, v2, (R)A.tcf[f + 1], (R)A.tcb[f + 1]);
        vm1 = v1 - R(0.5) * sl;
        vp1 = v1 + R(0.5) * sl;
    }
}

// HLL at face f; the x sweep parks the fluxes in the staging slots (j)
template <int DIR, typename R, bool RECIP = false>
__device__ __forceinline__ void walk_flux(const WalkCol<DIR, R>& C, int f, R (&wl)[8], R (&wr)[8], R ggas,
                                          FaceFluxT<R>& out, R bn, XStage<R>& X, int j) {
    wl[IBX + DIR] = bn;
    wr[IBX + DIR] = bn;
    R fx[7];
    sweep_hll<DIR, R, RECIP>(wl, wr, ggas, fx);
    if (DIR == 0) {
#pragma unroll
        for (int i = 0; i < 7; ++i) X.put(i, j, fx[i]);
        return;
    }
    if (!C.active) return;
    const int o = C.base + f * C.s;
#pragma unroll
    for (int i = 0; i < 7; ++i) out.f[i][o] = fx[i];
}

// x sweep, at the first face f of a chunk: write out the previous chunk's
// fluxes, then stage cells f+4..f+7 and faces f..f+3
template <int DIR, typename R>
__device__ __forceinline__ void walk_chunk(const WalkCol<DIR, R>& C, int f, XStage<R>& X, FaceFluxT<R>& out) {
    __syncthreads();
    if (f > C.f0) X.flush(f - XS_CELLS, C.f1, out);
    X.load(f + 4, C.nd + 3, f, C.f1);
    __syncthreads();
}

// x sweep, after the last face: write out the last chunk
template <int DIR, typename R>
__device__ __forceinline__ void walk_last(const WalkCol<DIR, R>& C, XStage<R>& X, FaceFluxT<R>& out) {
    __syncthreads();
    X.flush(C.f0 + ((C.f1 - 1 - C.f0) & ~(XS_CELLS - 1)), C.f1, out);
}

template <int DIR, int RECON, typename R>
__global__ void __launch_bounds__(WK_THREADS, 5) k_sweep_walk(Box b, Tabs T, PrimT<R> pr, R ggas, FaceFluxT<R> out,
                                                             int seg) {
    extern __shared__ __align__(16) unsigned char wk_raw[];
    WalkCol<DIR, R> C;
    if (!C.init(b, pr, seg)) return;
    const AxisTabs A = T.ax[DIR];
    const int s = C.s, f0 = C.f0;
    XStage<R> X;
    if (DIR == 0) X.init(b, pr, reinterpret_cast<R*>(wk_raw));

    R v0[WK_FIELDS], v1[WK_FIELDS], v2[WK_FIELDS], d1[WK_FIELDS], Vf[WK_FIELDS], vpf[WK_FIELDS], nxt[WK_FIELDS];
#pragma unroll
    for (int v = 0; v < WK_FIELDS; ++v) {
        const R* q = C.src[v];
        const R x0 = q[(f0 - 2) * s], x1 = q[(f0 - 1) * s], x2 = q[f0 * s], x3 = q[(f0 + 1) * s],
                x4 = q[(f0 + 2) * s];
        walk_prologue<RECON>(A, f0, x0, x1, x2, x3, x4, vpf[v], d1[v], Vf[v]);
        v0[v] = x2;
        v1[v] = x3;
        v2[v] = x4;
        nxt[v] = q[(f0 + 3) * s];
    }

    for (int f = f0; f < C.f1; ++f) {
        R wl[8], wr[8];
        const int j = (f - f0) & (XS_CELLS - 1);
        if (DIR == 0 && j == 0) walk_chunk(C, f, X, out);
        const R bn = DIR == 0 ? X.get(WK_FIELDS, j) : C.bn[f * s];
#pragma unroll
        for (int v = 0; v < WK_FIELDS; ++v) {
            const R x = nxt[v];
            R vm1, vp1;
            walk_step<RECON>(A, f, v0[v], v1[v], v2[v], x, d1[v], Vf[v], vm1, vp1);
            wl[C.slot[v]] = vpf[v];  // vp_out of cell f
            wr[C.slot[v]] = vm1;     // vm_out of cell f+1
            vpf[v] = vp1;
            v0[v] = v1[v];
            v1[v] = v2[v];
            v2[v] = x;
        }
        // prefetch the next cell (f+4 <= nd+3 while f+1 < f1)
        if (f + 1 < C.f1) {
#pragma unroll
            for (int v = 0; v < WK_FIELDS; ++v) nxt[v] = DIR == 0 ? X.get(v, j) : C.src[v][(f + 4) * s];
        }
        walk_flux<DIR>(C, f, wl, wr, ggas, out, bn, X, j);
    }
    if (DIR == 0) walk_last(C, X, out);
}

// shared-memory window: slots 0..2 are a ring of cell values (v(c) in slot
// c mod 3), 3 the carried slope, 4 the carried interface value, 5 vp_out(f)
constexpr int WK_SLOTS = 6;
template <typename R>
constexpr size_t walk_smem(int dir) {
    return (size_t)WK_SLOTS * WK_FIELDS * WK_THREADS * sizeof(R) + (dir == 0 ? xstage_smem<R>() : 0);
}

// STATES (y and z only): instead of solving HLL, store each face's
// reconstructed states, left in out and right in out_r (field order of the
// sweep, at the face's left cell), for the adjoint's HLL transpose.
// c_lo, c_cnt: the columns walked (WalkCol; c_cnt < 0 for all)
// RECIP: the HLL solve's quotients as products with reciprocals (hll_flux7)
template <int DIR, int RECON, typename R, bool STATES = false, bool RECIP = false>
__global__ void __launch_bounds__(WK_THREADS, CUMC_WALK_MINB) k_sweep_walk_sm(Box b, Tabs T, PrimT<R> pr, R ggas, FaceFluxT<R> out,
                                                             int seg, FaceFluxT<R> out_r, int c_lo, int c_cnt) {
    static_assert(!STATES || DIR != 0, "face states along y and z");
    extern __shared__ __align__(16) unsigned char wk_raw[];
    R* const sm = reinterpret_cast<R*>(wk_raw) + threadIdx.x;
    auto at = [&](int slot, int v) -> R& { return sm[(slot * WK_FIELDS + v) * WK_THREADS]; };
    WalkCol<DIR, R> C;
    if (!C.init(b, pr, seg, c_lo, c_cnt)) return;
    const AxisTabs A = T.ax[DIR];
    const int s = C.s, f0 = C.f0;
    XStage<R> X;
    if (DIR == 0) X.init(b, pr, reinterpret_cast<R*>(wk_raw) + WK_SLOTS * WK_FIELDS * WK_THREADS);

    R nxt[WK_FIELDS];
    // ring positions of v(f), v(f+1), v(f+2) for f = f0
    int r0 = f0 % 3, r1 = (f0 + 1) % 3, r2 = (f0 + 2) % 3;
#pragma unroll
    for (int v = 0; v < WK_FIELDS; ++v) {
        const R* q = C.src[v];
        const R x0 = q[(f0 - 2) * s], x1 = q[(f0 - 1) * s], x2 = q[f0 * s], x3 = q[(f0 + 1) * s],
                x4 = q[(f0 + 2) * s];
        R vpf, d1, Vf;
        walk_prologue<RECON>(A, f0, x0, x1, x2, x3, x4, vpf, d1, Vf);
        at(r0, v) = x2;
        at(r1, v) = x3;
        at(r2, v) = x4;
        at(3, v) = d1;
        at(4, v) = Vf;
        at(5, v) = vpf;
        nxt[v] = q[(f0 + 3) * s];
    }

    for (int f = f0; f < C.f1; ++f) {
        R wl[8], wr[8];
        const int j = (f - f0) & (XS_CELLS - 1);
        if (DIR == 0 && j == 0) walk_chunk(C, f, X, out);
        const R bn = DIR == 0 ? X.get(WK_FIELDS, j) : C.bn[f * s];
#pragma unroll
        for (int v = 0; v < WK_FIELDS; ++v) {
            const R x = nxt[v];
            R d1 = at(3, v), Vf = at(4, v);
            R vm1, vp1;
            walk_step<RECON>(A, f, RECON == 4 ? R(0) : at(r0, v), at(r1, v), at(r2, v), x, d1, Vf, vm1, vp1);
            wl[C.slot[v]] = at(5, v);  // vp_out of cell f
            wr[C.slot[v]] = vm1;       // vm_out of cell f+1
            at(5, v) = vp1;
            if (RECON == 4) {
                at(3, v) = d1;
                at(4, v) = Vf;
            }
            at(r0, v) = x;  // v(f+3) replaces v(f)
        }
        const int r = r0;
        r0 = r1;
        r1 = r2;
        r2 = r;
        if (f + 1 < C.f1) {
#pragma unroll
            for (int v = 0; v < WK_FIELDS; ++v) nxt[v] = DIR == 0 ? X.get(v, j) : C.src[v][(f + 4) * s];
        }
        if (STATES) {
            if (C.active) {
                const int o = C.base + f * s;
#pragma unroll
                for (int v = 0; v < WK_FIELDS; ++v) {
                    out.f[v][o] = wl[C.slot[v]];
                    out_r.f[v][o] = wr[C.slot[v]];
                }
            }
        } else {
            walk_flux<DIR, R, RECIP>(C, f, wl, wr, ggas, out, bn, X, j);
        }
    }
    if (DIR == 0) walk_last(C, X, out);
}

}  // namespace cumc

namespace cumc {

// ---------------------------------------------------------------------------
// x sweep with one lane per cell (GET_FLUXES x sweep, solver/spatial.f90:131-168).
// A warp holds 32 consecutive cells x0 .. x0+31 of one row. Each lane forms
// its own cell's limited slope, the interface value with the next cell and
// the extremum fix once, taking the neighbours' values through warp shuffles
// (the same expressions and operand order as the per-face kernel, so the
// fluxes are bit-identical); lanes 2..28 then solve HLL at their faces. A
// warp yields 27 faces; consecutive warps overlap by 5 cells. Loads and
// stores are one 256-byte row segment per field.
// Eight 128-thread blocks per SM (64 registers, a few spilled to L1): the
// kernel is bound by FP64 dependency latency, and 32 resident warps hide more
// of it than 20 unspilled ones (1.46 -> 1.25 ms at 256^3).
// ---------------------------------------------------------------------------
constexpr int XW_FACES = 27;

// STATES: store each face's reconstructed states (left in out, right in
// out_r, field order of the sweep) instead of solving HLL.
// The rows are those of the z planes l_lo .. l_lo + l_cnt - 1 (l_cnt < 0: all).
template <int RECON, typename R, bool STATES = false, bool RECIP = false>
__global__ void __launch_bounds__(128, CUMC_XWARP_MINB) k_sweep_xwarp(Box b, Tabs T, PrimT<R> pr, R ggas, FaceFluxT<R> out,
                                                        FaceFluxT<R> out_r, int l_lo, int l_cnt) {
    constexpr unsigned FULL = 0xffffffffu;
    const int nw = (b.nx + 1 + XW_FACES - 1) / XW_FACES;  // warps per row
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (l_cnt < 0) l_cnt = b.nz + 2;
    const long long rows = (long long)(b.ny + 2) * l_cnt;
    if (warp >= rows * nw || (b.skip && *b.skip)) return;  // uniform over the warp
    const int w = (int)(warp % nw);
    const long long row = warp / nw;
    const int k = (int)(row % (b.ny + 2)), l = l_lo + (int)(row / (b.ny + 2));
    const int c = w * XW_FACES - 2 + lane;  // this lane's cell; its face is c | c+1
    const bool inb = c >= -2 && c <= b.nx + 3;
    const int ct = min(max(c, -2), b.nx + 3);  // table index kept in range for spare lanes
    const int base = b.idx(0, k, l);
    const AxisTabs A = T.ax[0];
    const R* src[7] = {pr.w[0], pr.w[1], pr.w[2], pr.w[3], pr.w[4], pr.bc[1], pr.bc[2]};
    const int slot[7] = {IRHO, IVX, IVY, IVZ, ITAU, IBY, IBZ};
    R wl[8], wr[8];
#pragma unroll
    for (int v = 0; v < 7; ++v) {
        const R x = inb ? src[v][base + c] : R(0);
        const R xm = __shfl_up_sync(FULL, x, 1), xp = __shfl_down_sync(FULL, x, 1);
        R vm, vp;
        if (RECON == 4) {
            const R d = ppm_slope(xm, x, xp, (R)A.s0[ct], (R)A.s1[ct]);
            const R dp = __shfl_down_sync(FULL, d, 1);
            const R V = ppm_face(x, xp, d, dp, (R)A.a0[ct], (R)A.a1[ct], (R)A.a2[ct], (R)A.a3[ct]);  // c | c+1
            const R Vm = __shfl_up_sync(FULL, V, 1);                                                // c-1 | c
            ppm_fix(x, Vm, V, vm, vp);
        } else {
            const R sl = tvd_slope(xm, x, xp, (R)A.tcf[ct], (R)A.tcb[ct]);
            vm = x - R(0.5) * sl;
            vp = x + R(0.5) * sl;
        }
        wl[slot[v]] = vp;                             // vp_out of cell c
        wr[slot[v]] = __shfl_down_sync(FULL, vm, 1);  // vm_out of cell c+1
    }
    if (lane < 2 || lane > 28 || c < 0 || c > b.nx) return;
    if (STATES) {
#pragma unroll
        for (int v = 0; v < 7; ++v) {
            out.f[v][base + c] = wl[slot[v]];
            out_r.f[v][base + c] = wr[slot[v]];
        }
        return;
    }
    const R bn = pr.bf[0][base + c];
    wl[IBX] = bn;
    wr[IBX] = bn;
    R fx[7];
    sweep_hll<0, R, RECIP>(wl, wr, ggas, fx);
#pragma unroll
    for (int i = 0; i < 7; ++i) out.f[i][base + c] = fx[i];
}

inline long long xwarp_threads(const Box& b, int l_cnt = -1) {
    return (long long)(b.ny + 2) * (l_cnt < 0 ? b.nz + 2 : l_cnt) * ((b.nx + 1 + XW_FACES - 1) / XW_FACES) * 32;
}

}  // namespace cumc
