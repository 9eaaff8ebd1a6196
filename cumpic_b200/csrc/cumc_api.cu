// cumc_api.cu — C-ABI of the B200 CUMC3D hot path (declared in include/cumc.h).
//
// Host side: config validation (solver/setup.f90:121-230), the per-axis
// tables, device allocation, the RK3 stage sequence of
// solver/rungekutta.f90:12-148 and the main-loop driver of
// solver/main.f90:127-143 as a CUDA graph.
#include "../../include/cumc.h"
#include "cumc_kernels.cuh"
#include "cumc_sweep.cuh"
#include "cumc_mixed.h"
#include "cumc_walk.cuh"
#include "cumc_adjoint.cuh"
#include "cumc_fused.cuh"
#include "cumc_emfct.cuh"

#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <type_traits>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace cumc;

namespace {
thread_local std::string g_init_error;

struct ProfEvent {
    int cls;
    cudaEvent_t a, b;
};
}  // namespace

struct cumc_ctx {
    cumc_config cfg{};
    Box box{};
    int coord = 1, model = 1, recon = 4;
    double ggas = 5.0 / 3.0, cfl = 0.4;
    int flag[6]{};
    signed char fac[6][8]{};
    std::string err;
    int device = 0;
    int sm_count = 148;  // multiprocessors of the device (grid sizing)
    cudaStream_t stream = nullptr;

    std::vector<void*> allocs;
    Tabs tabs{};
    double* w[5]{};
    double* bc[3]{};
    double* eps = nullptr;
    double* U[2][8]{};
    double* F[3][7]{};
    double* E[3]{};
    double* L[8]{};      // l_rk (allocated with the FP64 state)
    bool lrk_valid = false;  // L holds cumc_spatial's l_rk (a fused stage reuses L[0..4] as its accumulator)
    double* staging = nullptr;
    double** dsoa = nullptr;   // device array of 8 pointers for the transposes
    double* scal = nullptr;    // dt, t
    unsigned long long* dtmin = nullptr;
    int* ints = nullptr;       // steps, done
    unsigned int* flag_dev = nullptr;
    double* divb_part = nullptr;
    double* host_pinned = nullptr;  // 8 doubles of pinned host scratch
    int cur = 0;
    bool uploaded = false, ready = false;

    bool prof_on = false;
    std::vector<ProfEvent> prof;
    int prof_launches[CUMC_K_COUNT]{};
    double prof_ms[CUMC_K_COUNT]{};
    long long launches = 0;

    cudaGraphExec_t graph_exec = nullptr;
    double graph_t_end = 0.0;
    long long graph_launches_per_step = 0;
    // sweep kernels (environment variable CUMC_SWEEP, for A/B timing; all
    // give the same bits): 0 default (lane-per-cell x, shared-memory-window
    // walker y/z), 1 "simple" (per-face everywhere), 2 "tile" (shared-memory tiles),
    // 3 "walkx" (register walker everywhere, x staged through shared memory),
    // 4 "walksm" (shared-memory-window walker everywhere), 5 "walkreg"
    // (per-face x, register walker y/z), 6 "xwarp" (lane-per-cell x only;
    // y/z one thread per face), 7 "xface" (per-face x, shared-memory-window
    // walker y/z), 8 "fused" (the flux differences fused into the sweeps and
    // the hydro combine into the z sweep, x rows staged by bulk tensor
    // copies), 9 "fused_notma" (the same with the x rows loaded directly)
    int sweep_mode = 0;
    // fused stage (sweep_mode 8): tensor maps of the x sweep's staged fields,
    // one set per state buffer holding the face fields
    XaccMaps xmaps[2]{};
    int xmaps_state = 0;  // 0 not tried, 1 ready, -1 not available (row pitch or driver)
    const char* xmaps_why = "not tried";
    bool mixed = false;         // CUMC_MIXED: state and kernels of cumc_mixed.cu
    bool fast = false;          // CUMC_FP64_FAST: the default sweeps' HLL with reciprocal products
    // the edge EMFs and the CT update in one tiled kernel (k_emf_ct) instead of
    // k_emf + k_ct; environment CUMC_EMF=pair selects the pair (A/B timing)
    bool emf_tiles = true;
    // the hydro combine on cell pairs (k_combine_utop2) when the row stride is
    // even and the arrays are 16-byte aligned; CUMC_COMBINE=scalar selects
    // k_combine_utop (A/B timing)
    bool pair_combine = true;
    MixedBufs mb{};
    MixedParams mp{};
    double* const* tape = nullptr;  // adjoint: 3 x 8 arrays receiving each stage's combine output
    void* adj_slab = nullptr;       // adjoint scratch, kept between runs
    size_t adj_slab_bytes = 0;
    int next_stage = 1;    // cumc_rk_stage: the stage due next
    int part1_stage = 0;   // cumc_rk_stage_part: the stage whose part 1 ran and whose part 2 is due
    bool fuse_dt = false;  // stage 3 also forms the next step's CFL dt (cumc_advance, cumc_rungekutta)
    bool dt_valid = false; // dtmin holds the CFL dt of the current state (set by cumc_rungekutta only)
    int bf_set = 0;        // U[bf_set] holds the current face fields (the last stage's output)
    bool exchange = false;  // a z face is CUMC_BC_EXCHANGE
    unsigned long long* model_max = nullptr;  // cumc_model_torus: the two maxima
    double* snap_dev = nullptr;            // snapshot staging slab (17 state arrays)
    cudaStream_t snap_stream = nullptr;    // device -> host copies of snapshots
    cudaEvent_t snap_taken = nullptr, snap_done = nullptr;
    bool snap_pending = false;

    int fail(int code, const char* fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        err = buf;
        return code;
    }
};

namespace {

int cuda_fail(cumc_ctx* c, cudaError_t e, const char* what) {
    return c->fail(CUMC_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CUMC_CHECK(expr)                                              \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #expr);        \
    } while (0)

template <typename T>
int dalloc(cumc_ctx* c, T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return c->fail(CUMC_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
    }
    c->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return CUMC_OK;
}

template <typename K, typename... Args>
void launch(cumc_ctx* c, int cls, long long nthreads, int block, K kern, Args... args) {
    if (nthreads <= 0) return;
    const unsigned grid = (unsigned)((nthreads + block - 1) / block);
    ProfEvent pe{cls, nullptr, nullptr};
    const bool rec = c->prof_on && cls >= 0;
    if (rec) {
        cudaEventCreate(&pe.a);
        cudaEventCreate(&pe.b);
        cudaEventRecord(pe.a, c->stream);
    }
    kern<<<grid, block, 0, c->stream>>>(args...);
    ++c->launches;
    if (rec) {
        cudaEventRecord(pe.b, c->stream);
        c->prof.push_back(pe);
    }
}

// ---------------------------------------------------------------------------
// per-axis tables
// ---------------------------------------------------------------------------
constexpr int NTAB_AXIS = 11;
constexpr int NTAB_X = 4, NTAB_Y = 4;

void build_axis(const double* fsrc, int n, std::vector<double>& out, size_t off, int stride) {
    // out holds NTAB_AXIS arrays of `stride` entries, entry i+3 for index i
    auto at = [&](int arr, int i) -> double& { return out[off + (size_t)arr * stride + (size_t)(i + 3)]; };
    auto f = [&](int i) { return fsrc[i + 3]; };
    for (int i = -3; i <= n + 3; ++i) {
        at(0, i) = f(i);
        at(1, i) = i > -3 ? f(i) - f(i - 1) : 0.0;                 // COORD_DX
        at(2, i) = i > -3 ? 0.5 * (f(i) + f(i - 1)) : 0.0;         // GET_COORD
    }
    auto d = [&](int i) { return at(1, i); };
    for (int i = -1; i <= n + 2; ++i) {  // PPM slope weights (solver/reconstruct.f90:223-247)
        const double dm1 = d(i - 1), dc = d(i), dp1 = d(i + 1);
        const double cc1 = dc / ((dm1 + dc) + dp1);
        const double cc2 = (2.0 * dm1 + dc) / (dp1 + dc);
        const double cc3 = (dc + 2.0 * dp1) / (dm1 + dc);
        at(3, i) = cc1 * cc2;
        at(4, i) = cc1 * cc3;
    }
    for (int i = -1; i <= n + 1; ++i) {  // PPM interface weights (solver/reconstruct.f90:211-243)
        const double dm1 = d(i - 1), dc = d(i), dp1 = d(i + 1), dp2 = d(i + 2);
        const double a1R = dc / (dc + dp1);
        const double aR = ((2.0 * dp1) * dc) / (dp1 + dc);
        const double deltaXR = ((dm1 + dc) + dp1) + dp2;
        const double z1R = (dm1 + dc) / (2.0 * dc + dp1);
        const double zR = (dp2 + dp1) / (2.0 * dp1 + dc);
        at(5, i) = a1R;
        at(6, i) = (aR * (z1R - zR)) / deltaXR;
        at(7, i) = ((-dc) * z1R) / deltaXR;
        at(8, i) = (dp1 * zR) / deltaXR;
    }
    for (int i = -1; i <= n + 2; ++i) {  // TVD_MM weights (solver/reconstruct.f90:110-111)
        at(9, i) = (d(i) + d(i + 1)) / d(i);
        at(10, i) = (d(i) + d(i - 1)) / d(i);
    }
}

// ---------------------------------------------------------------------------
// stage sequence
// ---------------------------------------------------------------------------
template <typename K, typename... Args>
void launch_grid(cumc_ctx* c, int cls, dim3 grid, int block, size_t smem, K kern, Args... args) {
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return;
    ProfEvent pe{cls, nullptr, nullptr};
    const bool rec = c->prof_on && cls >= 0;
    if (rec) {
        cudaEventCreate(&pe.a);
        cudaEventCreate(&pe.b);
        cudaEventRecord(pe.a, c->stream);
    }
    kern<<<grid, block, smem, c->stream>>>(args...);
    ++c->launches;
    if (rec) {
        cudaEventRecord(pe.b, c->stream);
        c->prof.push_back(pe);
    }
}

// l_lo, l_cnt: the z planes whose x rows (DIR 0) or y columns (DIR 1) the
// default kernels sweep (l_cnt < 0: all); the other forms sweep everything
template <int DIR>
void sweep(cumc_ctx* c, const Box& b, const Prim& pr, int l_lo = 0, int l_cnt = -1) {
    FaceFlux out;
    for (int q = 0; q < 7; ++q) out.f[q] = c->F[DIR][q];
    // default: one lane per cell along x, the shared-memory-window walker
    // along y and z
    // modes 0 and 9 come here only for SPATIAL alone (stage 0) and take the
    // unfused default's kernels
    const int mode = (c->sweep_mode == 9 || c->sweep_mode == 8) ? 0 : c->sweep_mode;
    const bool walk = (DIR > 0 && (mode == 0 || mode == 5 || mode == 7)) || mode == 3 || mode == 4;
    if (walk) {  // column walker
        int nseg;
        const int c_cnt = DIR == 1 && l_cnt >= 0 ? l_cnt : WalkGeom<DIR>::wc(b);
        const int c_lo = DIR == 1 && l_cnt >= 0 ? l_lo : 0;
        const int seg = walk_segment_for<DIR>(b, (long long)WalkGeom<DIR>::wa(b) * c_cnt, c->sm_count, &nseg);
        const dim3 grid((unsigned)(((long long)WalkGeom<DIR>::wa(b) * c_cnt + WK_THREADS - 1) / WK_THREADS),
                        (unsigned)nseg);
        const int cls = CUMC_K_SWEEP_X + DIR;
        if (mode == 4 || mode == 0 || mode == 7) {
            const size_t sm = walk_smem<double>(DIR);
            const bool ppm = c->recon == CUMC_PPMC;
            if (c->fast)
                launch_grid(c, cls, grid, WK_THREADS, sm,
                            ppm ? k_sweep_walk_sm<DIR, 4, double, false, true> : k_sweep_walk_sm<DIR, 1, double, false, true>,
                            b, c->tabs, pr, c->ggas, out, seg, out, c_lo, c_cnt);
            else
                launch_grid(c, cls, grid, WK_THREADS, sm,
                            ppm ? k_sweep_walk_sm<DIR, 4, double> : k_sweep_walk_sm<DIR, 1, double>, b, c->tabs, pr,
                            c->ggas, out, seg, out, c_lo, c_cnt);
        } else {
            const size_t sm = DIR == 0 ? xstage_smem<double>() : 0;
            if (c->recon == CUMC_PPMC)
                launch_grid(c, cls, grid, WK_THREADS, sm, k_sweep_walk<DIR, 4, double>, b, c->tabs, pr, c->ggas, out, seg);
            else
                launch_grid(c, cls, grid, WK_THREADS, sm, k_sweep_walk<DIR, 1, double>, b, c->tabs, pr, c->ggas, out, seg);
        }
        return;
    }
    if (DIR == 0 && (mode == 0 || mode == 6)) {  // x: one lane per cell
        const int cnt = l_cnt >= 0 ? l_cnt : b.nz + 2, lo = l_cnt >= 0 ? l_lo : 0;
        const bool ppm = c->recon == CUMC_PPMC;
        if (c->fast)
            launch(c, CUMC_K_SWEEP_X, xwarp_threads(b, cnt), 128,
                   ppm ? k_sweep_xwarp<4, double, false, true> : k_sweep_xwarp<1, double, false, true>, b, c->tabs, pr,
                   c->ggas, out, out, lo, cnt);
        else
            launch(c, CUMC_K_SWEEP_X, xwarp_threads(b, cnt), 128,
                   ppm ? k_sweep_xwarp<4, double> : k_sweep_xwarp<1, double>, b, c->tabs, pr, c->ggas, out, out, lo,
                   cnt);
        return;
    }
    if (mode != 2) {  // one thread per face
        const long long n = (long long)((DIR == 0 ? b.nx : b.nx + 1) + 1) * ((DIR == 1 ? b.ny : b.ny + 1) + 1) *
                            ((DIR == 2 ? b.nz : b.nz + 1) + 1);
        if (c->recon == CUMC_PPMC)
            launch(c, CUMC_K_SWEEP_X + DIR, n, 128, k_sweep<DIR, 4>, b, c->tabs, pr, c->ggas, out);
        else
            launch(c, CUMC_K_SWEEP_X + DIR, n, 128, k_sweep<DIR, 1>, b, c->tabs, pr, c->ggas, out);
        return;
    }
    const dim3 grid = sweep_grid<DIR>(b);
    if (c->recon == CUMC_PPMC)
        launch_grid(c, CUMC_K_SWEEP_X + DIR, grid, SW_THREADS, sw_smem<double>(), k_sweep_tile<DIR, 4, double>, b, c->tabs, pr, c->ggas, out);
    else
        launch_grid(c, CUMC_K_SWEEP_X + DIR, grid, SW_THREADS, sw_smem<double>(), k_sweep_tile<DIR, 1, double>, b, c->tabs, pr, c->ggas, out);
}

int sweep_attributes(cumc_ctx* c) {
    const void* k[6] = {(const void*)k_sweep_tile<0, 4, double>, (const void*)k_sweep_tile<1, 4, double>,
                        (const void*)k_sweep_tile<2, 4, double>, (const void*)k_sweep_tile<0, 1, double>,
                        (const void*)k_sweep_tile<1, 1, double>, (const void*)k_sweep_tile<2, 1, double>};
    for (const void* f : k) {
        cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw_smem<double>());
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaFuncSetAttribute(sweep smem)");
    }
    return CUMC_OK;
}

// primitive buffers of one state: the context's own, or an adjoint scratch set
struct PrimBufs {
    double* const* w;
    double* const* bc;
    double* eps;
};

UtopArgs utop_args(cumc_ctx* c, double* const* u, const PrimBufs& p);

// k_combine_utop2's conditions: an even row stride and 16-byte alignment of
// every array it reads or writes as pairs
inline bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
template <int STAGE>
bool pairs_aligned(const Box& b, const FaceFlux* ff, const CombineArgs& a, const UtopArgs& o) {
    if (b.SX & 1) return false;
    bool ok = al16(o.eps);
    for (int q = 0; q < 5; ++q) {
        ok = ok && al16(ff[0].f[q]) && al16(ff[1].f[q]) && al16(ff[2].f[q]) && al16(a.u0[q]) && al16(o.u[q]) &&
             al16(o.w[q]) && (!a.tape[q] || al16(a.tape[q]));
        if (STAGE != 1) ok = ok && al16(a.uc[q]);
    }
    for (int q = 0; q < 3; ++q) ok = ok && al16(o.u[IBX + q]) && al16(o.bc[q]);
    return ok;
}

// stage 0: l_rk alone; stages 1-3: face fields, then hydro combine + conversions
template <int COORD, int MODEL, int STAGE>
void combine_stage(cumc_ctx* c, const Box& b, const Prim& pr, const FaceFlux* ff, const CombineArgs& a,
                   const UtopArgs& o) {
    const long long n = (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1);
    if (STAGE == 0) {
        launch(c, CUMC_K_COMBINE, n, 256, k_combine<COORD, MODEL>, b, c->tabs, pr, ff[0], ff[1], ff[2], a);
        return;
    }
    constexpr int S = STAGE == 0 ? 1 : STAGE;
    if (c->emf_tiles) {
        int seg;
        const dim3 g = emf_ct_grid(b, (long long)c->sm_count * CUMC_EC_MINB, &seg);
        launch_grid(c, CUMC_K_CT, g, EC_TX * EC_TY, sizeof(EmfCtSmem), k_emf_ct<COORD, S>, b, c->tabs, pr, ff[0], ff[1],
                    ff[2], a, seg);
    } else {
        launch(c, CUMC_K_CT, n, 256, k_ct<COORD, S>, b, c->tabs, a);
    }
    if (c->pair_combine && pairs_aligned<S>(b, ff, a, o)) {
        const long long np = (long long)((b.nx + 2) / 2) * (b.ny + 1) * (b.nz + 1);
        launch(c, CUMC_K_COMBINE, np, 256, k_combine_utop2<COORD, MODEL, S>, b, c->tabs, pr, ff[0], ff[1], ff[2], a,
               o);
    } else {
        launch(c, CUMC_K_COMBINE, n, 256, k_combine_utop<COORD, MODEL, S>, b, c->tabs, pr, ff[0], ff[1], ff[2], a, o);
    }
}

template <int COORD, int MODEL>
void combine_dispatch(cumc_ctx* c, const Box& b, int stage, const Prim& pr, const FaceFlux* ff, const CombineArgs& a,
                      const UtopArgs& o) {
    switch (stage) {
        case 0: combine_stage<COORD, MODEL, 0>(c, b, pr, ff, a, o); break;
        case 1: combine_stage<COORD, MODEL, 1>(c, b, pr, ff, a, o); break;
        case 2: combine_stage<COORD, MODEL, 2>(c, b, pr, ff, a, o); break;
        default: combine_stage<COORD, MODEL, 3>(c, b, pr, ff, a, o); break;
    }
}

template <int COORD>
void combine_model(cumc_ctx* c, const Box& b, int stage, const Prim& pr, const FaceFlux* ff, const CombineArgs& a,
                   const UtopArgs& o) {
    switch (c->model) {
        case CUMC_MODEL_NONE: combine_dispatch<COORD, 0>(c, b, stage, pr, ff, a, o); break;
        case CUMC_MODEL_RIEMANN: combine_dispatch<COORD, 1>(c, b, stage, pr, ff, a, o); break;
        case CUMC_MODEL_TORUS_SPH: combine_dispatch<COORD, 2>(c, b, stage, pr, ff, a, o); break;
        default: combine_dispatch<COORD, 3>(c, b, stage, pr, ff, a, o); break;
    }
}

UtopArgs utop_args(cumc_ctx* c, double* const* u, const PrimBufs& p) {
    UtopArgs a;
    for (int q = 0; q < 8; ++q) a.u[q] = u[q];
    for (int q = 0; q < 5; ++q) a.w[q] = p.w[q];
    for (int q = 0; q < 3; ++q) a.bc[q] = p.bc[q];
    a.eps = p.eps;
    a.ggas = c->ggas;
    a.rho_floor = c->cfg.rho_floor;
    a.eps_floor = c->cfg.eps_floor;
    a.flag = c->flag_dev;
    return a;
}

void utop_into(cumc_ctx* c, const Box& b, double* const* u, const PrimBufs& p, bool from_cons) {
    const UtopArgs a = utop_args(c, u, p);
    const long long n = (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1);
#define CUMC_UTOP(M)                                                                         \
    if (from_cons) launch(c, CUMC_K_UTOP, n, 256, k_utop<M, true>, b, a);                    \
    else launch(c, CUMC_K_UTOP, n, 256, k_utop<M, false>, b, a);
    switch (c->model) {
        case CUMC_MODEL_NONE: CUMC_UTOP(0) break;
        case CUMC_MODEL_RIEMANN: CUMC_UTOP(1) break;
        case CUMC_MODEL_TORUS_SPH: CUMC_UTOP(2) break;
        default: CUMC_UTOP(3) break;
    }
#undef CUMC_UTOP
}

void utop(cumc_ctx* c, const Box& b, double* const* u, bool from_cons) {
    utop_into(c, b, u, PrimBufs{c->w, c->bc, c->eps}, from_cons);
}

BoundArgs bound_args(cumc_ctx* c, double* const* u, const PrimBufs& p) {
    BoundArgs a;
    for (int q = 0; q < 5; ++q) a.w[q] = p.w[q];
    for (int q = 0; q < 3; ++q) a.bc[q] = p.bc[q];
    a.eps = p.eps;
    for (int q = 0; q < 3; ++q) a.bf[q] = u[IBX + q];
    for (int q = 0; q < 6; ++q) a.flag[q] = c->flag[q];
    a.eps_yout = c->flag[2] == 0 ? 0 : c->flag[3];
    std::memcpy(a.fac, c->fac, sizeof a.fac);
    a.ggas = c->ggas;
    return a;
}

long long ghost_count(const Box& b) { return 6LL * b.SX * b.SY + 6LL * b.SX * b.nz + 6LL * b.ny * b.nz; }

void boundary_into(cumc_ctx* c, const Box& b, double* const* u, const PrimBufs& p) {
    const BoundArgs a = bound_args(c, u, p);
    const long long n = ghost_count(b);
    switch (c->model) {
        case CUMC_MODEL_TORUS_SPH: launch(c, CUMC_K_BOUNDARY, n, 256, k_boundary<2, double>, b, a); break;
        case CUMC_MODEL_TORUS_CYN: launch(c, CUMC_K_BOUNDARY, n, 256, k_boundary<3, double>, b, a); break;
        default: launch(c, CUMC_K_BOUNDARY, n, 256, k_boundary<0, double>, b, a); break;
    }
}

void boundary(cumc_ctx* c, const Box& b, double* const* u) { boundary_into(c, b, u, PrimBufs{c->w, c->bc, c->eps}); }

Prim make_prim(cumc_ctx* c, double* const* u) {
    Prim p;
    for (int q = 0; q < 5; ++q) p.w[q] = c->w[q];
    for (int q = 0; q < 3; ++q) p.bc[q] = c->bc[q];
    for (int q = 0; q < 3; ++q) p.bf[q] = u[IBX + q];
    return p;
}

// launch hooks for the mixed-path kernels: per-kernel events and launch count
void mx_pre(void* u, int cls) {
    auto* c = static_cast<cumc_ctx*>(u);
    if (c->prof_on && cls >= 0) {
        ProfEvent pe{cls, nullptr, nullptr};
        cudaEventCreate(&pe.a);
        cudaEventCreate(&pe.b);
        cudaEventRecord(pe.a, c->stream);
        c->prof.push_back(pe);
    }
}
void mx_post(void* u, int cls) {
    auto* c = static_cast<cumc_ctx*>(u);
    ++c->launches;
    if (c->prof_on && cls >= 0) cudaEventRecord(c->prof.back().b, c->stream);
}
Launcher mx_launcher(cumc_ctx* c) { return Launcher{c->stream, mx_pre, mx_post, c}; }

// One SPATIAL + combine + conversions + boundary (solver/rungekutta.f90:38-66).
// stage 0: SPATIAL only, l_rk stored in c->L.
// an NVTX range for the scope (shown by Nsight tools; a no-op without one)
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

// Tensor maps of the x sweep's staged fields (rho, vx, vy, vz, p, by, bz
// and the face field Bx of either state buffer): 3-D boxes of XA_BOX x
// XA_ROWS x 1 doubles over the ghosted box, zero fill outside it. A map needs
// a row pitch that is a multiple of 16 bytes (nx + 6 even); without one, or
// without the driver entry point, the fused stage loads its rows directly.
int encode_xmaps(cumc_ctx* c) {
    const Box& b = c->box;
    c->xmaps_state = -1;
    if ((b.SX * sizeof(double)) % 16 != 0) {
        c->xmaps_why = "row pitch not a multiple of 16 bytes";
        return CUMC_OK;
    }
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
        cudaGetLastError();
        c->xmaps_why = "no cuTensorMapEncodeTiled entry point";
        return CUMC_OK;
    }
    auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
    const cuuint64_t dims[3] = {(cuuint64_t)b.SX, (cuuint64_t)b.SY, (cuuint64_t)b.SZ};
    const cuuint64_t strides[2] = {(cuuint64_t)b.SX * sizeof(double), (cuuint64_t)b.SX * b.SY * sizeof(double)};
    const cuuint32_t box[3] = {XA_BOX, XA_ROWS, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    for (int set = 0; set < 2; ++set) {
        const double* f[XA_FIELDS] = {c->w[0], c->w[1], c->w[2], c->w[3], c->w[4], c->bc[1], c->bc[2], c->U[set][IBX]};
        for (int v = 0; v < XA_FIELDS; ++v) {
            CUresult r = encode(&c->xmaps[set].m[v], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(f[v]), dims,
                                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) {
                c->xmaps_why = "cuTensorMapEncodeTiled refused a map";
                return CUMC_OK;
            }
        }
    }
    c->xmaps_state = 1;
    c->xmaps_why = "";
    return CUMC_OK;
}

// One RK stage with the flux differences fused into the sweeps and the hydro
// combine into the z sweep (cumc_fused.cuh): sweeps x, y, z; k_emf; k_ct;
// k_utop_stage (conversions, and the next CFL dt at stage 3); k_boundary.
template <int COORD, int RECON>
void fused_xy(cumc_ctx* c, const Box& b, const Prim& pr, const AccArgs& acc, int fset, int l_lo, int l_cnt) {
    const bool tma = c->sweep_mode == 8 && c->xmaps_state == 1;
    const XaccMaps& maps = c->xmaps[fset];
    if (tma)
        launch_grid(c, CUMC_K_SWEEP_X, xacc_grid(b, l_cnt), 32 * XA_ROWS, xacc_smem(true),
                    k_sweep_xacc<RECON, COORD, true>, b, c->tabs, pr, c->ggas, acc, maps, l_lo);
    else
        launch_grid(c, CUMC_K_SWEEP_X, xacc_grid(b, l_cnt), 32 * XA_ROWS, xacc_smem(false),
                    k_sweep_xacc<RECON, COORD, false>, b, c->tabs, pr, c->ggas, acc, maps, l_lo);
    int nseg;
    const int seg = walk_segment_for<1>(b, (long long)WalkGeom<1>::wa(b) * l_cnt, c->sm_count, &nseg);
    const dim3 grid((unsigned)(((long long)WalkGeom<1>::wa(b) * l_cnt + WK_THREADS - 1) / WK_THREADS), (unsigned)nseg);
    launch_grid(c, CUMC_K_SWEEP_Y, grid, WK_THREADS, acc_smem<1>(), k_walk_acc<1, RECON, COORD>, b, c->tabs, pr,
                c->ggas, acc, seg, l_lo, l_cnt);
}

// x and y sweeps of the planes `part` covers (0: all, 1: the active planes
// 1..nz, 2: the ghost planes 0 and nz+1), then with part != 1 the z sweep
template <int COORD, int RECON>
void fused_sweeps(cumc_ctx* c, const Box& b, const Prim& pr, const AccArgs& acc, int fset, int part) {
    if (part == 0) fused_xy<COORD, RECON>(c, b, pr, acc, fset, 0, b.nz + 2);
    if (part == 1) fused_xy<COORD, RECON>(c, b, pr, acc, fset, 1, b.nz);
    if (part == 2) {
        fused_xy<COORD, RECON>(c, b, pr, acc, fset, 0, 1);
        fused_xy<COORD, RECON>(c, b, pr, acc, fset, b.nz + 1, 1);
    }
    if (part == 1) return;
    int nseg;
    const int seg = walk_segment_for<2>(b, WalkGeom<2>::ncols(b), c->sm_count, &nseg);
    const dim3 grid((unsigned)((WalkGeom<2>::ncols(b) + WK_THREADS - 1) / WK_THREADS), (unsigned)nseg);
    launch_grid(c, CUMC_K_SWEEP_Z, grid, WK_THREADS, acc_smem<2>(), k_walk_acc<2, RECON, COORD>, b, c->tabs, pr,
                c->ggas, acc, seg, 0, WalkGeom<2>::wc(b));
}

template <int COORD>
void fused_tail(cumc_ctx* c, const Box& b, int stage, const CombineArgs& a, const UtopArgs& o) {
    const long long n = (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1);
    switch (stage) {
        case 1: launch(c, CUMC_K_CT, n, 256, k_ct<COORD, 1>, b, c->tabs, a); break;
        case 2: launch(c, CUMC_K_CT, n, 256, k_ct<COORD, 2>, b, c->tabs, a); break;
        default: launch(c, CUMC_K_CT, n, 256, k_ct<COORD, 3>, b, c->tabs, a); break;
    }
    switch (c->model) {
        case CUMC_MODEL_NONE: launch(c, CUMC_K_COMBINE, n, 256, k_utop_stage<COORD, 0>, b, c->tabs, o); break;
        case CUMC_MODEL_RIEMANN: launch(c, CUMC_K_COMBINE, n, 256, k_utop_stage<COORD, 1>, b, c->tabs, o); break;
        case CUMC_MODEL_TORUS_SPH: launch(c, CUMC_K_COMBINE, n, 256, k_utop_stage<COORD, 2>, b, c->tabs, o); break;
        default: launch(c, CUMC_K_COMBINE, n, 256, k_utop_stage<COORD, 3>, b, c->tabs, o); break;
    }
}

// part 0: the whole stage; part 1: the x and y sweeps of the active planes
// (they read no ghost plane, so they may run while a halo exchange fills
// them); part 2: the rest of the stage after part 1
void fused_stage(cumc_ctx* c, const Box& b, int stage, const Prim& pr, double* const* Un, double* const* Ua,
                 double* const* dst, int fset, const CombineArgs& a, const UtopArgs& o, int part) {
    AccArgs acc{};
    for (int q = 0; q < 5; ++q) {
        acc.L[q] = c->L[q];
        acc.u0[q] = Un[q];
        acc.uc[q] = Ua[q];
        acc.ud[q] = dst[q];
        acc.tape[q] = a.tape[q];
    }
    for (int d = 0; d < 3; ++d) {
        acc.fb[d][0] = c->F[d][5];
        acc.fb[d][1] = c->F[d][6];
    }
    acc.dt = c->scal;
    acc.stage = stage;
    acc.model = c->model;
    acc.geom_repeat = c->cfg.geom_source_repeat;
    acc.rho_floor = c->cfg.rho_floor;
    acc.r_sh = c->cfg.r_sh;
    acc.err = c->flag_dev;
    const bool ppm = c->recon == CUMC_PPMC;
    switch (c->coord) {
        case CUMC_CARTESIAN:
            ppm ? fused_sweeps<1, 4>(c, b, pr, acc, fset, part) : fused_sweeps<1, 1>(c, b, pr, acc, fset, part);
            break;
        case CUMC_CYLINDRICAL:
            ppm ? fused_sweeps<2, 4>(c, b, pr, acc, fset, part) : fused_sweeps<2, 1>(c, b, pr, acc, fset, part);
            break;
        default:
            ppm ? fused_sweeps<3, 4>(c, b, pr, acc, fset, part) : fused_sweeps<3, 1>(c, b, pr, acc, fset, part);
            break;
    }
    if (part == 1) return;
    FaceFlux ff[3];
    for (int d = 0; d < 3; ++d)
        for (int q = 0; q < 7; ++q) ff[d].f[q] = c->F[d][q];
    EdgeE ee;
    for (int q = 0; q < 3; ++q) ee.e[q] = c->E[q];
    launch(c, CUMC_K_EMF, (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256, k_emf<double>, b, pr, ff[0], ff[1],
           ff[2], ee);
    switch (c->coord) {
        case CUMC_CARTESIAN: fused_tail<1>(c, b, stage, a, o); break;
        case CUMC_CYLINDRICAL: fused_tail<2>(c, b, stage, a, o); break;
        default: fused_tail<3>(c, b, stage, a, o); break;
    }
}

// part (fused stages only): 0 the whole stage, 1 the sweeps that read no
// ghost plane, 2 the rest (see fused_stage); the unfused forms run the whole
// stage at part 0 and 2 and nothing at part 1
void run_stage(cumc_ctx* c, const Box& b, int stage, int part = 0) {
    if (stage > 0) c->lrk_valid = false;
    static const char* const names[4] = {"cumc spatial", "cumc rk stage 1", "cumc rk stage 2", "cumc rk stage 3"};
    const NvtxRange range(names[stage]);
    if (c->mixed) {
        if (stage > 0 && part != 1)
            mixed_stage(mx_launcher(c), b, c->tabs, c->mb, c->mp, stage, stage == 3 && c->fuse_dt ? c->dtmin : nullptr);
        return;
    }
    double* const* Un = c->U[c->cur];
    double* const* Ua = c->U[1 - c->cur];
    double* const* src = (stage <= 1) ? Un : Ua;  // arrays holding prim(ibx:ibz) this stage
    const Prim pr = make_prim(c, src);
    const bool fused = stage > 0 && !c->mixed && (c->sweep_mode == 8 || c->sweep_mode == 9);
    const bool split = c->sweep_mode == 0;  // the default kernels take a plane range
    if (!fused && !split && part == 1) return;
    if (fused) {
        CombineArgs a{};
        double* const* dst = stage == 1 ? Ua : stage == 2 ? Ua : Un;
        for (int q = 0; q < 8; ++q) {
            a.u0[q] = Un[q];
            a.uc[q] = Ua[q];
            a.ud[q] = dst[q];
            a.tape[q] = c->tape ? c->tape[(stage - 1) * 8 + q] : nullptr;
        }
        a.dt = c->scal;
        for (int q = 0; q < 3; ++q) a.ecorn[q] = c->E[q];
        UtopArgs o = utop_args(c, dst, PrimBufs{c->w, c->bc, c->eps});
        if (stage == 3 && c->fuse_dt) {  // the following iteration's finddt, fused (dtmin reset by the caller)
            o.dtmin = c->dtmin;
            o.cfl = c->cfl;
        }
        fused_stage(c, b, stage, pr, Un, Ua, dst, src == c->U[0] ? 0 : 1, a, o, part);
        if (part != 1) boundary(c, b, dst);
        return;
    }
    if (split && part == 1) {  // the x and y sweeps of the active planes: they read no ghost plane
        sweep<0>(c, b, pr, 1, b.nz);
        sweep<1>(c, b, pr, 1, b.nz);
        return;
    }
    if (split && part == 2) {  // the rest: the x and y sweeps of the ghost planes 0 and nz+1 first
        sweep<0>(c, b, pr, 0, 1);
        sweep<0>(c, b, pr, b.nz + 1, 1);
        sweep<1>(c, b, pr, 0, 1);
        sweep<1>(c, b, pr, b.nz + 1, 1);
    } else {
        sweep<0>(c, b, pr);
        sweep<1>(c, b, pr);
    }
    sweep<2>(c, b, pr);
    FaceFlux ff[3];
    for (int d = 0; d < 3; ++d)
        for (int q = 0; q < 7; ++q) ff[d].f[q] = c->F[d][q];
    EdgeE ee;
    for (int q = 0; q < 3; ++q) ee.e[q] = c->E[q];
    // the edge EMFs: k_emf here and k_ct in the combine, or (the default
    // stages) both in k_emf_ct there
    if (stage == 0 || !c->emf_tiles)
        launch(c, CUMC_K_EMF, (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256, k_emf<double>, b, pr, ff[0], ff[1],
               ff[2], ee);

    CombineArgs a{};
    double* const* dst = stage == 1 ? Ua : stage == 2 ? Ua : Un;
    for (int q = 0; q < 8; ++q) {
        a.u0[q] = Un[q];
        a.uc[q] = Ua[q];
        a.ud[q] = dst[q];
        a.lrk[q] = c->L[q];
    }
    a.dt = c->scal;
    for (int q = 0; q < 3; ++q) a.ecorn[q] = c->E[q];
    a.geom_repeat = c->cfg.geom_source_repeat;
    a.rho_floor = c->cfg.rho_floor;
    a.r_sh = c->cfg.r_sh;
    // adjoint recomputation: the combine's output of this stage, on (0:n)^3.
    // Nothing reads the hydro cons outside (0:n)^3, nor a face field outside
    // 0:n along its own axis, and the boundary refills the tangential ones.
    for (int q = 0; q < 8; ++q) a.tape[q] = (c->tape && stage > 0) ? c->tape[(stage - 1) * 8 + q] : nullptr;
    UtopArgs o = utop_args(c, dst, PrimBufs{c->w, c->bc, c->eps});
    if (stage == 3 && c->fuse_dt) {  // the following iteration's finddt, fused (dtmin reset by the caller)
        o.dtmin = c->dtmin;
        o.cfl = c->cfl;
    }
    switch (c->coord) {
        case CUMC_CARTESIAN: combine_model<1>(c, b, stage, pr, ff, a, o); break;
        case CUMC_CYLINDRICAL: combine_model<2>(c, b, stage, pr, ff, a, o); break;
        default: combine_model<3>(c, b, stage, pr, ff, a, o); break;
    }
    if (stage == 0) return;
    boundary(c, b, dst);
}

void rk_step(cumc_ctx* c, const Box& b) {
    run_stage(c, b, 1);
    run_stage(c, b, 2);
    run_stage(c, b, 3);
}

void finddt_launch(cumc_ctx* c, const Box& b) {
    launch(c, -1, 1, 1, k_reset_dtmin, c->dtmin);
    if (c->mixed) {
        mixed_finddt(mx_launcher(c), b, c->tabs, c->mb, c->mp, c->dtmin);
        return;
    }
    const Prim pr = make_prim(c, c->U[c->cur]);
    const long long n = (long long)b.nx * b.ny * b.nz;
    switch (c->coord) {
        case CUMC_CARTESIAN: launch(c, CUMC_K_FINDDT, n, 256, k_finddt<1>, b, c->tabs, pr, c->ggas, c->cfl, c->dtmin); break;
        case CUMC_CYLINDRICAL: launch(c, CUMC_K_FINDDT, n, 256, k_finddt<2>, b, c->tabs, pr, c->ggas, c->cfl, c->dtmin); break;
        default: launch(c, CUMC_K_FINDDT, n, 256, k_finddt<3>, b, c->tabs, pr, c->ggas, c->cfl, c->dtmin); break;
    }
}

Clock make_clock(cumc_ctx* c) {
    Clock k;
    k.dt = c->scal;
    k.t = c->scal + 1;
    k.dtmin = c->dtmin;
    k.steps = c->ints;
    k.done = c->ints + 1;
    return k;
}

// one main-loop iteration with device-resident dt (solver/main.f90:127-143)
// One iteration of the main loop (solver/main.f90:130-142). dt comes from
// the previous iteration's stage 3 (fused finddt, in both forms; the caller
// runs a standalone finddt before the first iteration), so a step reads the
// state once less.
void loop_step(cumc_ctx* c, double t_end) {
    Box b = c->box;
    const Clock k = make_clock(c);
    launch(c, -1, 1, 1, k_check_done, k, t_end);
    b.skip = k.done;
    launch(c, -1, 1, 1, k_clip_dt, k, t_end);
    launch(c, -1, 1, 1, k_reset_dtmin, c->dtmin);
    c->fuse_dt = true;
    rk_step(c, b);
    c->fuse_dt = false;
    launch(c, -1, 1, 1, k_advance_time, k);
}

// ---------------------------------------------------------------------------
// Device-side GET_MODEL of the spherical torus (model/torus_sph/src/model.f90
// :8-284; the same construction as problems.torus on the host), written in
// the upload layout (prim AoS, 8 values a cell, and eps) to the staging
// buffer, so that the rest is cumc_upload_state's path.
// ---------------------------------------------------------------------------
struct TorusK {
    double ggas, r_sh, s_in, q, lkep2, c_const, k_poly, rho_a, rho_max, rho_cut, beta, noise, rho_floor;
    unsigned long long seed;
    int cyl;  // 1: cylindrical torus (model/torus_cyn), 0: spherical (model/torus_sph)
};

// equilibrium of cell (j, k, l) (active): rho, v_phi, p, eps. Spherical:
// potential -1/(r - r_sh), cylindrical radius s = r sin(theta);
// cylindrical: potential -1/(sqrt(R^2 + z^2) - r_sh), s = R
__device__ __forceinline__ void torus_cell(const Tabs& T, const TorusK& m, int j, int k, int l, double& rho, double& vph,
                                           double& p, double& eps) {
    const double r = T.ax[0].c[j];
    double s_eq, schw;
    if (m.cyl) {
        const double z = T.ax[2].c[l];
        s_eq = r;
        schw = -1.0 / (sqrt(r * r + z * z) - m.r_sh);
    } else {
        s_eq = r * T.sinc[k];
        schw = -1.0 / (r - m.r_sh);
    }
    double h = -schw + m.lkep2 * pow(s_eq, 2.0 - 2.0 * m.q) / (2.0 - 2.0 * m.q) + m.c_const;
    h = fmax(h, 0.0);
    const double rho_loc = pow(h * (m.ggas - 1.0) / m.ggas / m.k_poly, 1.0 / (m.ggas - 1.0));
    const bool inside = rho_loc > m.rho_a && s_eq >= m.s_in;
    rho = inside ? rho_loc : m.rho_a;
    vph = inside ? sqrt(m.lkep2) * pow(s_eq, -m.q) * s_eq : 0.0;
    p = m.k_poly * pow(rho, m.ggas);
    eps = m.k_poly * pow(rho, m.ggas - 1.0) / (m.ggas - 1.0);
}

__global__ void __launch_bounds__(256) k_torus_cells(Box b, Tabs T, TorusK m, double* prim, double* eps) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.count()) return;
    const int j = (int)(t % b.SX) - 2, k = (int)((t / b.SX) % b.SY) - 2, l = (int)(t / ((long long)b.SX * b.SY)) - 2;
    double v[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, e = 0.0;
    if (j >= 1 && j <= b.nx && k >= 1 && k <= b.ny && l >= 1 && l <= b.nz)
        torus_cell(T, m, j, k, l, v[IRHO], v[m.cyl ? IVY : IVZ], v[ITAU], e);
#pragma unroll
    for (int q = 0; q < 8; ++q) prim[8 * t + q] = v[q];
    eps[t] = e;
}

// A_phi = max(rho - rho_cut, 0)/rho_max on the active cells (zero elsewhere),
// averaged over (j, j+1) x (l, l+1) at the corner (model.f90:126-146)
__device__ __forceinline__ double torus_corner(const Box& b, const TorusK& m, const double* prim, int j, int k, int l) {
    if (j < 1 || j > b.nx || k < 1 || k > b.ny || l < 1 || l > b.nz) return 0.0;
    auto A = [&](int jj, int ll) -> double {
        if (jj > b.nx || ll > b.nz) return 0.0;
        const double rho = prim[8LL * b.idx(jj, k, ll) + IRHO];
        return rho >= m.rho_cut ? (rho - m.rho_cut) / m.rho_max : 0.0;
    };
    return 0.25 * (((A(j, l) + A(j + 1, l)) + A(j, l + 1)) + A(j + 1, l + 1));
}

// face fields on 0:n, B = curl(A_phi): spherical (model/torus_sph/src/
// model.f90:153-162) B_r, B_theta; cylindrical (model/torus_cyn/src/
// model.f90:149-158) B_R = -dA/dz, B_z = d(R A)/(R dR)
__global__ void __launch_bounds__(256) k_torus_faces(Box b, Tabs T, TorusK m, double* prim) {
    const long long n0 = b.nx + 1, n1 = b.ny + 1, n2 = b.nz + 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n0 * n1 * n2) return;
    const int j = (int)(t % n0), k = (int)((t / n0) % n1), l = (int)(t / (n0 * n1));
    const double a = torus_corner(b, m, prim, j, k, l);
    const double ajm = torus_corner(b, m, prim, j - 1, k, l);
    const double xfj = T.ax[0].f[j], xfjm = T.ax[0].f[j - 1];
    const long long i = b.idx(j, k, l);
    if (m.cyl) {
        const double alm = torus_corner(b, m, prim, j, k, l - 1);
        prim[8 * i + IBX] = -(a - alm) / T.ax[2].d[l];
        prim[8 * i + IBZ] = (xfj * a - xfjm * ajm) / (T.ax[0].c[j] * T.ax[0].d[j]);
    } else {
        const double akm = torus_corner(b, m, prim, j, k - 1, l);
        prim[8 * i + IBX] = (T.sinf[k] * a - T.sinf[k - 1] * akm) / (xfj * T.dcos[k]);
        prim[8 * i + IBY] = -(xfj * a - xfjm * ajm) / (T.ax[0].c[j] * T.ax[0].d[j]);
    }
}

// maxima of p and of the cell magnetic pressure over the active cells
// (model.f90:176-219), as 64-bit patterns of non-negative doubles
__global__ void __launch_bounds__(256) k_torus_max(Box b, TorusK m, const double* prim, unsigned long long* mx) {
    const long long total = (long long)b.nx * b.ny * b.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double pg = 0.0, pm = 0.0;
    if (t < total) {
        const int j = (int)(t % b.nx) + 1, k = (int)((t / b.nx) % b.ny) + 1, l = (int)(t / ((long long)b.nx * b.ny)) + 1;
        const long long i = b.idx(j, k, l);
        const double bcx = 0.5 * (prim[8 * i + IBX] + prim[8LL * b.idx(j - 1, k, l) + IBX]);
        // the second field: B_theta (spherical); B_z averaged over the phi
        // neighbour, as model/torus_cyn/src/model.f90:166 does (cylindrical)
        const int q2 = m.cyl ? IBZ : IBY;
        const double bc2 = 0.5 * (prim[8 * i + q2] + prim[8LL * b.idx(j, k - 1, l) + q2]);
        pg = prim[8 * i + ITAU];
        pm = 0.5 * (bcx * bcx + bc2 * bc2);
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        pg = fmax(pg, __shfl_xor_sync(0xffffffffu, pg, s));
        pm = fmax(pm, __shfl_xor_sync(0xffffffffu, pm, s));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(mx, (unsigned long long)__double_as_longlong(pg));
        atomicMax(mx + 1, (unsigned long long)__double_as_longlong(pm));
    }
}

// normalise the face fields to plasma beta, then the seeded density noise
// (model.f90:256-265): rho (1 + noise (2u - 1)) where rho > rho_floor
__global__ void __launch_bounds__(256) k_torus_finish(Box b, TorusK m, const unsigned long long* mx, double* prim) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.count()) return;
    const int j = (int)(t % b.SX) - 2, k = (int)((t / b.SX) % b.SY) - 2, l = (int)(t / ((long long)b.SX * b.SY)) - 2;
    if (j >= 0 && j <= b.nx && k >= 0 && k <= b.ny && l >= 0 && l <= b.nz) {
        const double pg = __longlong_as_double((long long)mx[0]), pm = __longlong_as_double((long long)mx[1]);
        const double norm = pm > 0.0 ? sqrt((pg / pm) / m.beta) : 0.0;
        prim[8 * t + IBX] *= norm;
        prim[8 * t + (m.cyl ? IBZ : IBY)] *= norm;
    }
    if (j >= 1 && j <= b.nx && k >= 1 && k <= b.ny && l >= 1 && l <= b.nz) {
        const unsigned long long idx =
            (unsigned long long)(j - 1) + (unsigned long long)b.nx * ((unsigned long long)(k - 1) + (unsigned long long)b.ny * (l - 1));
        // splitmix64(seed, idx) -> [0, 1) with 53 bits (problems.uniform01)
        unsigned long long z = m.seed * 0xD1B54A32D192ED03ULL + (idx + 1ULL) * 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z = z ^ (z >> 31);
        const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
        const double d = prim[8 * t + IRHO];
        if (d > m.rho_floor) prim[8 * t + IRHO] = d + d * (u - 0.5) / 0.5 * m.noise;
    }
}

// halo planes of a z face: the 11 arrays a neighbouring slab reads in its
// ghost planes (w, bcell, eps, and the face fields Bx, By), three planes from
// plane l0, each plane whole (x and y ghosts included)
constexpr int HALO_ARRAYS = 11;
struct HaloArgs {
    double* f[HALO_ARRAYS];
};
__global__ void __launch_bounds__(256) k_halo_copy(Box b, HaloArgs a, int l0, double* buf, int to_buf) {
    const long long plane = (long long)b.SX * b.SY;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= HALO_ARRAYS * 3 * plane) return;
    const int q = (int)(t / (3 * plane));
    const long long r = t % (3 * plane);
    const long long at = (long long)(l0 + 2) * plane + r;  // plane l0 + r/plane (Box::idx), cell r%plane
    if (to_buf) buf[t] = a.f[q][at];
    else a.f[q][at] = buf[t];
}

int check_ready(cumc_ctx* c) {
    if (!c) return CUMC_ERR_ARG;
    if (!c->ready) return c->fail(CUMC_ERR_STATE, "cumc_initial_update must run after cumc_upload_state first");
    return CUMC_OK;
}

int sync_status(cumc_ctx* c) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    return CUMC_OK;
}

}  // namespace

extern "C" {

const char* cumc_last_error(const cumc_ctx* c) { return c ? c->err.c_str() : g_init_error.c_str(); }

int cumc_init(const cumc_config* cfg, cumc_ctx** out) {
    g_init_error.clear();
    if (!cfg || !out) { g_init_error = "null argument"; return CUMC_ERR_ARG; }
    *out = nullptr;
    auto bad = [](const char* m) { g_init_error = m; return CUMC_ERR_CONFIG; };
    if (cfg->nx < 3 || cfg->ny < 3 || cfg->nz < 3) return bad("every direction needs at least 3 active cells (3 ghost layers)");
    if ((long long)(cfg->nx + 6) * (cfg->ny + 6) * (cfg->nz + 6) >= (1LL << 31))
        { g_init_error = "grid too large: (nx+6)(ny+6)(nz+6) must stay below 2^31"; return CUMC_ERR_LIMIT; }
    if (!cfg->xf || !cfg->yf || !cfg->zf) { g_init_error = "face coordinate arrays are required"; return CUMC_ERR_ARG; }
    if (cfg->coordinate < 1 || cfg->coordinate > 3) return bad("coordinate must be 1 (cartesian), 2 (cylindrical) or 3 (spherical)");
    if (cfg->recon != CUMC_PPMC && cfg->recon != CUMC_TVDMM) return bad("recon must be CUMC_PPMC or CUMC_TVDMM (the reference implements no other)");
    if (cfg->solver != CUMC_HLL) return bad("solver must be CUMC_HLL (the reference implements no other)");
    if (cfg->precision != CUMC_FP64 && cfg->precision != CUMC_MIXED && cfg->precision != CUMC_FP64_FAST)
        return bad("precision must be CUMC_FP64, CUMC_FP64_FAST or CUMC_MIXED");
    if (cfg->model < 0 || cfg->model > 3) return bad("unknown model id");
    for (int i = 0; i < 6; ++i)
        if ((cfg->boundary_flag[i] < 0 || cfg->boundary_flag[i] > 4) &&
            !(i >= 4 && cfg->boundary_flag[i] == CUMC_BC_EXCHANGE))
            return bad("boundary_flag entries must be 0..4 (z faces: or CUMC_BC_EXCHANGE)");
    if ((cfg->boundary_flag[4] == CUMC_BC_EXCHANGE || cfg->boundary_flag[5] == CUMC_BC_EXCHANGE) &&
        cfg->precision == CUMC_MIXED)
        return bad("CUMC_BC_EXCHANGE faces need CUMC_FP64 or CUMC_FP64_FAST");
    if (cfg->boundary_flag[0] == 4 || cfg->boundary_flag[1] == 4)
        return bad("equatorial symmetry is not allowed for the x-boundary (solver/setup.f90:147-151)");
    if (cfg->boundary_flag[4] == 3 || cfg->boundary_flag[5] == 3)
        return bad("axial symmetry is not allowed for the z-boundary (solver/setup.f90:206-210)");
    if (cfg->boundary_flag[2] != 0 && cfg->boundary_flag[3] == 0)
        return bad("a periodic y-outer face needs a periodic y-inner face (BOUNDARY1D never fills eps there, solver/boundary.f90:211)");
    if (!(cfg->ggas > 1.0)) return bad("ggas must exceed 1");
    if (!(cfg->cfl > 0.0)) return bad("cfl must be positive");
    for (int i = 0; i < 7; ++i)
        if (cfg->reserved[i] != 0) return bad("reserved fields must be zero");

    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_init_error = std::string("no usable CUDA device: ") + cudaGetErrorString(e);
        return CUMC_ERR_CUDA;
    }

    auto* c = new cumc_ctx();
    c->cfg = *cfg;
    if (c->cfg.geom_source_repeat <= 0) c->cfg.geom_source_repeat = 8;
    c->coord = cfg->coordinate;
    c->model = cfg->model;
    c->recon = cfg->recon;
    c->ggas = cfg->ggas;
    c->cfl = cfg->cfl;
    for (int i = 0; i < 6; ++i) c->flag[i] = cfg->boundary_flag[i];
    c->exchange = c->flag[4] == CUMC_BC_EXCHANGE || c->flag[5] == CUMC_BC_EXCHANGE;
    // bfac tables (solver/setup.f90:129-230)
    for (int s = 0; s < 6; ++s)
        for (int q = 0; q < 8; ++q) c->fac[s][q] = 1;
    for (int s = 0; s < 2; ++s) {
        const int f = c->flag[s];
        if (f == 2 || f == 3) { c->fac[s][IVX] = -1; c->fac[s][IBX] = -1; }
        if (f == 3) { c->fac[s][IVZ] = -1; c->fac[s][IBZ] = -1; }
    }
    for (int s = 2; s < 4; ++s) {
        const int f = c->flag[s];
        if (f == 2 || f == 3) { c->fac[s][IVY] = -1; c->fac[s][IBY] = -1; }
        if (f == 3) { c->fac[s][IVZ] = -1; c->fac[s][IBZ] = -1; }
        if (f == 4) { c->fac[s][IVY] = -1; c->fac[s][IBX] = -1; c->fac[s][IBZ] = -1; }
    }
    for (int s = 4; s < 6; ++s) {
        const int f = c->flag[s];
        if (f == 2) { c->fac[s][IVZ] = -1; c->fac[s][IBZ] = -1; }
        if (f == 4) { c->fac[s][IVZ] = -1; c->fac[s][IBX] = -1; c->fac[s][IBY] = -1; }
    }

    Box& b = c->box;
    b.nx = cfg->nx; b.ny = cfg->ny; b.nz = cfg->nz;
    b.SX = b.nx + 6; b.SY = b.ny + 6; b.SZ = b.nz + 6;
    b.skip = nullptr;
    const size_t NT = (size_t)b.count();

    auto fail_init = [&](int code) {
        g_init_error = c->err;
        cumc_free(c);
        return code;
    };
    int rc;
    if ((e = cudaGetDevice(&c->device)) != cudaSuccess) { cuda_fail(c, e, "cudaGetDevice"); return fail_init(CUMC_ERR_CUDA); }
    if ((e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device)) != cudaSuccess) {
        cuda_fail(c, e, "cudaDeviceGetAttribute");
        return fail_init(CUMC_ERR_CUDA);
    }
    {
        const char* sw = getenv("CUMC_SWEEP");
        c->sweep_mode = !sw                              ? 0
                        : std::strcmp(sw, "simple") == 0 ? 1
                        : std::strcmp(sw, "tile") == 0   ? 2
                        : std::strcmp(sw, "walkx") == 0  ? 3
                        : std::strcmp(sw, "walksm") == 0 ? 4
                        : std::strcmp(sw, "walkreg") == 0 ? 5
                        : std::strcmp(sw, "xwarp") == 0   ? 6
                        : std::strcmp(sw, "xface") == 0   ? 7
                        : std::strcmp(sw, "fused") == 0   ? 8
                        : std::strcmp(sw, "fused_notma") == 0 ? 9
                                                          : 0;
    }
    {
        const char* em = getenv("CUMC_EMF");
        c->emf_tiles = !(em && std::strcmp(em, "pair") == 0);
        const char* cm = getenv("CUMC_COMBINE");
        c->pair_combine = !(cm && std::strcmp(cm, "scalar") == 0);
    }
    if ((rc = sweep_attributes(c)) != CUMC_OK) return fail_init(rc);
    c->mixed = cfg->precision == CUMC_MIXED;
    c->fast = cfg->precision == CUMC_FP64_FAST;
    if (c->mixed && (e = mixed_attributes()) != cudaSuccess) {
        cuda_fail(c, e, "cudaFuncSetAttribute(mixed sweep smem)");
        return fail_init(CUMC_ERR_CUDA);
    }
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        cuda_fail(c, e, "cudaStreamCreate");
        return fail_init(CUMC_ERR_CUDA);
    }

    // tables
    const int st[3] = {b.nx + 7, b.ny + 7, b.nz + 7};
    size_t ntab = 0;
    size_t off[3];
    for (int a = 0; a < 3; ++a) { off[a] = ntab; ntab += (size_t)NTAB_AXIS * st[a]; }
    const size_t offx = ntab; ntab += (size_t)NTAB_X * st[0];
    const size_t offy = ntab; ntab += (size_t)NTAB_Y * st[1];
    std::vector<double> h(ntab, 0.0);
    const double* fsrc[3] = {cfg->xf, cfg->yf, cfg->zf};
    const int nn[3] = {b.nx, b.ny, b.nz};
    for (int a = 0; a < 3; ++a) build_axis(fsrc[a], nn[a], h, off[a], st[a]);
    for (int j = -2; j <= b.nx + 3; ++j) {
        const double xp = cfg->xf[j + 3], xm = cfg->xf[j + 2];
        h[offx + 0 * st[0] + j + 3] = xp * xp;
        h[offx + 1 * st[0] + j + 3] = ((xp * xp) * xp - (xm * xm) * xm) / 3.0;
        h[offx + 2 * st[0] + j + 3] = ((2.0 * ((xp * xp) * xp - (xm * xm) * xm)) / 3.0) / (xp * xp - xm * xm);
        h[offx + 3 * st[0] + j + 3] = 0.5 * (xp * xp - xm * xm);
    }
    h[offx + 0 * st[0] + 0] = cfg->xf[0] * cfg->xf[0];
    for (int k = -2; k <= b.ny + 3; ++k) {
        const double yp = cfg->yf[k + 3], ym = cfg->yf[k + 2];
        const double yc = 0.5 * (yp + ym);
        h[offy + 0 * st[1] + k + 3] = std::sin(yp);
        h[offy + 1 * st[1] + k + 3] = std::cos(ym) - std::cos(yp);
        h[offy + 2 * st[1] + k + 3] = std::tan(yc);
        h[offy + 3 * st[1] + k + 3] = std::sin(yc);
    }
    h[offy + 0 * st[1] + 0] = std::sin(cfg->yf[0]);
    double* dtab = nullptr;
    if ((rc = dalloc(c, &dtab, ntab)) != CUMC_OK) return fail_init(rc);
    if ((e = cudaMemcpy(dtab, h.data(), ntab * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess) {
        cuda_fail(c, e, "table upload");
        return fail_init(CUMC_ERR_CUDA);
    }
    for (int a = 0; a < 3; ++a) {
        const double* base = dtab + off[a] + 3;
        AxisTabs& A = c->tabs.ax[a];
        const double** p[NTAB_AXIS] = {&A.f, &A.d, &A.c, &A.s0, &A.s1, &A.a0, &A.a1, &A.a2, &A.a3, &A.tcf, &A.tcb};
        for (int q = 0; q < NTAB_AXIS; ++q) *p[q] = base + (size_t)q * st[a];
    }
    c->tabs.r2 = dtab + offx + 3;
    c->tabs.r3d3 = dtab + offx + st[0] + 3;
    c->tabs.rfac = dtab + offx + 2 * st[0] + 3;
    c->tabs.hr2 = dtab + offx + 3 * st[0] + 3;
    c->tabs.sinf = dtab + offy + 3;
    c->tabs.dcos = dtab + offy + st[1] + 3;
    c->tabs.tanc = dtab + offy + 2 * st[1] + 3;
    c->tabs.sinc = dtab + offy + 3 * st[1] + 3;

    // state
    auto field = [&](double** p) -> int {
        int r = dalloc(c, p, NT);
        if (r != CUMC_OK) return r;
        return cudaMemset(*p, 0, NT * sizeof(double)) == cudaSuccess ? CUMC_OK : CUMC_ERR_CUDA;
    };
    if (!c->mixed) {
        for (int q = 0; q < 5; ++q) if ((rc = field(&c->w[q])) != CUMC_OK) return fail_init(rc);
        for (int q = 0; q < 3; ++q) if ((rc = field(&c->bc[q])) != CUMC_OK) return fail_init(rc);
        if ((rc = field(&c->eps)) != CUMC_OK) return fail_init(rc);
        for (int s = 0; s < 2; ++s)
            for (int q = 0; q < 8; ++q) if ((rc = field(&c->U[s][q])) != CUMC_OK) return fail_init(rc);
        for (int d = 0; d < 3; ++d)
            for (int q = 0; q < 7; ++q) if ((rc = field(&c->F[d][q])) != CUMC_OK) return fail_init(rc);
        for (int q = 0; q < 3; ++q) if ((rc = field(&c->E[q])) != CUMC_OK) return fail_init(rc);
        // l_rk: the fused stage's flux-difference accumulator (0-4) and cumc_spatial's output (0-7)
        for (int q = 0; q < 8; ++q) if ((rc = field(&c->L[q])) != CUMC_OK) return fail_init(rc);
    } else {
        auto ffield = [&](float** p) -> int {
            int r = dalloc(c, p, NT);
            if (r != CUMC_OK) return r;
            return cudaMemset(*p, 0, NT * sizeof(float)) == cudaSuccess ? CUMC_OK : CUMC_ERR_CUDA;
        };
        MixedBufs& m = c->mb;
        for (int q = 0; q < 8; ++q) {
            if (q == ITAU) continue;
            if ((rc = ffield(&m.uh[q])) != CUMC_OK || (rc = ffield(&m.ul[q])) != CUMC_OK) return fail_init(rc);
            if (q < ITAU && (rc = ffield(&m.d[q])) != CUMC_OK) return fail_init(rc);
        }
        for (int q = 0; q < 3; ++q) if ((rc = field(&m.db[q])) != CUMC_OK) return fail_init(rc);
        if ((rc = field(&m.e0)) != CUMC_OK || (rc = field(&m.es)) != CUMC_OK) return fail_init(rc);
        for (int q = 0; q < 5; ++q) if ((rc = ffield(&m.w[q])) != CUMC_OK) return fail_init(rc);
        for (int q = 0; q < 3; ++q)
            if ((rc = ffield(&m.bc[q])) != CUMC_OK || (rc = ffield(&m.bf[q])) != CUMC_OK || (rc = ffield(&m.E[q])) != CUMC_OK)
                return fail_init(rc);
        for (int d = 0; d < 3; ++d)
            for (int q = 0; q < 7; ++q) if ((rc = ffield(&m.F[d][q])) != CUMC_OK) return fail_init(rc);
        MixedParams& mp = c->mp;
        mp.ggas = c->ggas;
        mp.cfl = c->cfl;
        mp.rho_floor = cfg->rho_floor;
        mp.eps_floor = cfg->eps_floor;
        mp.r_sh = cfg->r_sh;
        for (int i = 0; i < 6; ++i) mp.flag[i] = c->flag[i];
        mp.eps_yout = c->flag[2] == 0 ? 0 : c->flag[3];
        std::memcpy(mp.fac, c->fac, sizeof mp.fac);
        mp.model = c->model;
        mp.coord = c->coord;
        mp.recon = c->recon;
        mp.geom_repeat = c->cfg.geom_source_repeat;
        mp.sm_count = c->sm_count;
        const char* ms = getenv("CUMC_MX_STAGE");
        mp.fused = !(ms && std::strcmp(ms, "split") == 0);
        const char* mh = getenv("CUMC_MX_HLL");
        mp.hll_fp32 = mh && std::strcmp(mh, "fp32") == 0;
    }
    if ((rc = dalloc(c, &c->dsoa, 8)) != CUMC_OK) return fail_init(rc);
    if ((rc = dalloc(c, &c->scal, 4)) != CUMC_OK) return fail_init(rc);
    if ((rc = dalloc(c, &c->dtmin, 1)) != CUMC_OK) return fail_init(rc);
    if ((rc = dalloc(c, &c->ints, 4)) != CUMC_OK) return fail_init(rc);
    if ((rc = dalloc(c, &c->flag_dev, 1)) != CUMC_OK) return fail_init(rc);
    c->mb.dt = c->scal;
    c->mb.flag = c->flag_dev;
    cudaMemset(c->scal, 0, 4 * sizeof(double));
    cudaMemset(c->ints, 0, 4 * sizeof(int));
    cudaMemset(c->flag_dev, 0, sizeof(unsigned));
    if ((e = cudaMallocHost(&c->host_pinned, 8 * sizeof(double))) != cudaSuccess) {
        cuda_fail(c, e, "cudaMallocHost");
        return fail_init(CUMC_ERR_NOMEM);
    }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) { cuda_fail(c, e, "init"); return fail_init(CUMC_ERR_CUDA); }
    if (!c->mixed && c->sweep_mode == 8) encode_xmaps(c);  // before any stream capture: host-side driver calls only
    if (getenv("CUMC_VERBOSE") && c->sweep_mode == 8 && c->xmaps_state != 1)
        fprintf(stderr, "cumc: x sweep loads its rows directly: %s\n", c->xmaps_why);
    *out = c;
    return CUMC_OK;
}

int cumc_free(cumc_ctx* c) {
    if (!c) return CUMC_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& pe : c->prof) { cudaEventDestroy(pe.a); cudaEventDestroy(pe.b); }
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    for (void* p : c->allocs) cudaFree(p);
    if (c->adj_slab) cudaFree(c->adj_slab);
    if (c->snap_stream) {
        cudaStreamSynchronize(c->snap_stream);
        cudaStreamDestroy(c->snap_stream);
    }
    if (c->snap_taken) cudaEventDestroy(c->snap_taken);
    if (c->snap_done) cudaEventDestroy(c->snap_done);
    if (c->host_pinned) cudaFreeHost(c->host_pinned);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return CUMC_OK;
}

// staging buffer for the AoS <-> SoA transposes, allocated on first use
static int ensure_staging(cumc_ctx* c) {
    if (c->staging) return CUMC_OK;
    // 8 fields in the reference's AoS layout, plus eps for the mixed upload
    return dalloc(c, &c->staging, 9 * (size_t)c->box.count());
}

static int put_soa(cumc_ctx* c, const double* host, int nv, double* const* dst) {
    const size_t NT = (size_t)c->box.count();
    int rc = ensure_staging(c);
    if (rc != CUMC_OK) return rc;
    CUMC_CHECK(cudaMemcpyAsync(c->dsoa, dst, nv * sizeof(double*), cudaMemcpyHostToDevice, c->stream));
    CUMC_CHECK(cudaMemcpyAsync(c->staging, host, nv * NT * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch(c, -1, (long long)NT, 256, k_aos_to_soa, (long long)NT, nv, (const double*)c->staging, c->dsoa);
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    return sync_status(c);
}

static int get_soa(cumc_ctx* c, double* host, int nv, const double* const* srcp) {
    const size_t NT = (size_t)c->box.count();
    int rc = ensure_staging(c);
    if (rc != CUMC_OK) return rc;
    CUMC_CHECK(cudaMemcpyAsync(c->dsoa, srcp, nv * sizeof(double*), cudaMemcpyHostToDevice, c->stream));
    launch(c, -1, (long long)NT, 256, k_soa_to_aos, (long long)NT, nv, c->staging, (const double* const*)c->dsoa);
    CUMC_CHECK(cudaMemcpyAsync(host, c->staging, nv * NT * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    return sync_status(c);
}

int cumc_upload_state(cumc_ctx* c, const double* prim, const double* eps) {
    if (c) c->dt_valid = false;  // the state changes: the cached CFL dt is stale
    if (!c || !prim || !eps) return c ? c->fail(CUMC_ERR_ARG, "null argument") : CUMC_ERR_ARG;
    if (c->mixed) {  // kept as FP64 AoS until cumc_initial_update converts it
        const size_t NT = (size_t)c->box.count();
        int rc = ensure_staging(c);
        if (rc != CUMC_OK) return rc;
        CUMC_CHECK(cudaMemcpyAsync(c->staging, prim, 8 * NT * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CUMC_CHECK(cudaMemcpyAsync(c->staging + 8 * NT, eps, NT * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CUMC_CHECK(cudaStreamSynchronize(c->stream));
        c->uploaded = true;
        c->ready = false;
        return CUMC_OK;
    }
    double* dst[8] = {c->w[0], c->w[1], c->w[2], c->w[3], c->w[4], c->U[c->cur][IBX], c->U[c->cur][IBY], c->U[c->cur][IBZ]};
    int rc = put_soa(c, prim, 8, dst);
    if (rc != CUMC_OK) return rc;
    double* de[1] = {c->eps};
    rc = put_soa(c, eps, 1, de);
    if (rc != CUMC_OK) return rc;
    c->uploaded = true;
    c->ready = false;
    return CUMC_OK;
}

int cumc_download_state(cumc_ctx* c, double* prim, double* cons, double* eps, double* bcell) {
    if (!c) return CUMC_ERR_ARG;
    int rc;
    if (c->mixed) {
        const size_t NT = (size_t)c->box.count();
        if ((rc = ensure_staging(c)) != CUMC_OK) return rc;
        double* outs[4] = {prim, cons, eps, bcell};
        const int nv[4] = {8, 8, 1, 3};
        for (int w = 0; w < 4; ++w) {
            if (!outs[w]) continue;
            mixed_export(mx_launcher(c), c->box, c->mb, c->mp, w, c->staging);
            CUMC_CHECK(cudaMemcpyAsync(outs[w], c->staging, nv[w] * NT * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            CUMC_CHECK(cudaStreamSynchronize(c->stream));
        }
        return sync_status(c);
    }
    double* const* u = c->U[c->cur];
    if (prim) {
        const double* s[8] = {c->w[0], c->w[1], c->w[2], c->w[3], c->w[4], u[IBX], u[IBY], u[IBZ]};
        if ((rc = get_soa(c, prim, 8, s)) != CUMC_OK) return rc;
    }
    if (cons) {
        const double* s[8] = {u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7]};
        if ((rc = get_soa(c, cons, 8, s)) != CUMC_OK) return rc;
    }
    if (eps) {
        const double* s[1] = {c->eps};
        if ((rc = get_soa(c, eps, 1, s)) != CUMC_OK) return rc;
    }
    if (bcell) {
        const double* s[3] = {c->bc[0], c->bc[1], c->bc[2]};
        if ((rc = get_soa(c, bcell, 3, s)) != CUMC_OK) return rc;
    }
    return CUMC_OK;
}

int cumc_initial_update(cumc_ctx* c) {
    if (c) c->dt_valid = false;  // the state changes: the cached CFL dt is stale
    if (!c) return CUMC_ERR_ARG;
    if (!c->uploaded) return c->fail(CUMC_ERR_STATE, "cumc_upload_state must come first");
    if (c->mixed) {
        const size_t NT = (size_t)c->box.count();
        mixed_initial(mx_launcher(c), c->box, c->tabs, c->mb, c->mp, c->staging, c->staging + 8 * NT);
        c->ready = true;
        return sync_status(c);
    }
    utop(c, c->box, c->U[c->cur], false);
    boundary(c, c->box, c->U[c->cur]);
    c->ready = true;
    c->next_stage = 1;
    c->bf_set = c->cur;
    return sync_status(c);
}

int cumc_finddt(cumc_ctx* c, double* dt) {
    int rc = check_ready(c);
    if (rc != CUMC_OK) return rc;
    if (!dt) return c->fail(CUMC_ERR_ARG, "null dt");
    if (!c->dt_valid) finddt_launch(c, c->box);  // else the last cumc_rungekutta's stage 3 formed it
    CUMC_CHECK(cudaMemcpyAsync(c->host_pinned, c->dtmin, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaMemcpyAsync(c->host_pinned + 1, c->flag_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    if ((rc = sync_status(c)) != CUMC_OK) return rc;
    std::memcpy(dt, c->host_pinned, sizeof(double));
    unsigned fl;
    std::memcpy(&fl, c->host_pinned + 1, sizeof(unsigned));
    if (fl & kTmaTimeoutFlag) return c->fail(CUMC_ERR_CUDA, "a staged bulk tensor copy never completed (wait gave up)");
    if (fl & 1u) return c->fail(CUMC_ERR_NONFINITE, "non-finite density, velocity or pressure in the evolved state");
    return CUMC_OK;
}

int cumc_rungekutta(cumc_ctx* c, double dt) {
    int rc = check_ready(c);
    if (rc != CUMC_OK) return rc;
    if (c->exchange) return c->fail(CUMC_ERR_STATE, "a slab with CUMC_BC_EXCHANGE faces steps by cumc_rk_stage and the halo exchange");
    if (c->next_stage != 1) return c->fail(CUMC_ERR_STATE, "cumc_rk_stage left a step unfinished");
    if (!(dt >= 0.0 && std::isfinite(dt))) return c->fail(CUMC_ERR_ARG, "dt must be finite and non-negative");
    launch(c, -1, 1, 1, k_set_scalar, c->scal, dt);
    // stage 3 forms the next step's CFL dt, which cumc_finddt then returns
    // without a pass over the state (the same expression, so the same bits)
    launch(c, -1, 1, 1, k_reset_dtmin, c->dtmin);
    c->fuse_dt = true;
    rk_step(c, c->box);
    c->fuse_dt = false;
    c->dt_valid = true;
    return sync_status(c);
}

int cumc_rk_stage_part(cumc_ctx* c, int stage, double dt, int part) {
    if (c) c->dt_valid = false;  // the state changes: the cached CFL dt is stale
    int rc = check_ready(c);
    if (rc != CUMC_OK) return rc;
    if (part < 0 || part > 2) return c->fail(CUMC_ERR_ARG, "part must be 0 (whole stage), 1 or 2");
    if (stage != c->next_stage) return c->fail(CUMC_ERR_STATE, "stage %d called where stage %d is due", stage, c->next_stage);
    if (part == 2 && c->part1_stage != stage)
        return c->fail(CUMC_ERR_STATE, "part 2 of stage %d called without its part 1", stage);
    if (part != 2 && c->part1_stage != 0)
        return c->fail(CUMC_ERR_STATE, "stage %d: part 2 is due", c->part1_stage);
    if (part != 2 && stage == 1 && !(dt >= 0.0 && std::isfinite(dt)))
        return c->fail(CUMC_ERR_ARG, "dt must be finite and non-negative");
    if (part != 2 && stage == 1) launch(c, -1, 1, 1, k_set_scalar, c->scal, dt);
    run_stage(c, c->box, stage, part);
    if (part == 1) {
        c->part1_stage = stage;
        return sync_status(c);
    }
    c->part1_stage = 0;
    c->next_stage = stage == 3 ? 1 : stage + 1;
    c->bf_set = stage == 3 ? c->cur : 1 - c->cur;
    return sync_status(c);
}

int cumc_rk_stage(cumc_ctx* c, int stage, double dt) { return cumc_rk_stage_part(c, stage, dt, 0); }

int cumc_halo_doubles(cumc_ctx* c, long long* n) {
    if (!c || !n) return c ? c->fail(CUMC_ERR_ARG, "null argument") : CUMC_ERR_ARG;
    *n = (long long)HALO_ARRAYS * 3 * c->box.SX * c->box.SY;
    return CUMC_OK;
}

static int halo_copy(cumc_ctx* c, int side, double* buf, bool pack) {
    int rc = check_ready(c);
    if (rc != CUMC_OK) return rc;
    if (c->mixed) return c->fail(CUMC_ERR_CONFIG, "the halo exchange covers CUMC_FP64");
    if ((side != 0 && side != 1) || !buf) return c->fail(CUMC_ERR_ARG, "side must be 0 (z-in) or 1 (z-out), buffer non-null");
    const Box& b = c->box;
    HaloArgs a;
    for (int q = 0; q < 5; ++q) a.f[q] = c->w[q];
    for (int q = 0; q < 3; ++q) a.f[5 + q] = c->bc[q];
    a.f[8] = c->eps;
    a.f[9] = c->U[c->bf_set][IBX];
    a.f[10] = c->U[c->bf_set][IBY];
    // pack: the three active planes next to the face; unpack: its three ghost planes
    const int l0 = pack ? (side == 0 ? 1 : b.nz - 2) : (side == 0 ? -2 : b.nz + 1);
    launch(c, -1, (long long)HALO_ARRAYS * 3 * b.SX * b.SY, 256, k_halo_copy, b, a, l0, buf, pack ? 1 : 0);
    return sync_status(c);
}

int cumc_halo_pack(cumc_ctx* c, int side, double* buf) { return halo_copy(c, side, buf, true); }
int cumc_halo_unpack(cumc_ctx* c, int side, const double* buf) {
    if (c) c->dt_valid = false;
    return halo_copy(c, side, const_cast<double*>(buf), false);
}

int cumc_spatial(cumc_ctx* c) {
    if (c) c->dt_valid = false;  // the state changes: the cached CFL dt is stale
    int rc = check_ready(c);
    if (rc != CUMC_OK) return rc;
    if (c->mixed) return c->fail(CUMC_ERR_STATE, "cumc_spatial is available for CUMC_FP64 only");
    run_stage(c, c->box, 0);
    c->lrk_valid = true;
    return sync_status(c);
}

int cumc_download_lrk(cumc_ctx* c, double* lrk) {
    if (!c || !lrk) return c ? c->fail(CUMC_ERR_ARG, "null argument") : CUMC_ERR_ARG;
    if (!c->L[0] || !c->lrk_valid)
        return c->fail(CUMC_ERR_STATE, "no l_rk to download: cumc_spatial has not run since the last stage");
    const double* s[8] = {c->L[0], c->L[1], c->L[2], c->L[3], c->L[4], c->L[5], c->L[6], c->L[7]};
    return get_soa(c, lrk, 8, s);
}

int cumc_divb(cumc_ctx* c, double* maxdb_signed, double* maxabs_norm) {
    int rc = check_ready(c);
    if (rc != CUMC_OK) return rc;
    const Box& b = c->box;
    const long long n = (long long)b.nx * b.ny * b.nz;
    const int nblk = (int)((n + 255) / 256);
    if (!c->divb_part && (rc = dalloc(c, &c->divb_part, 3 * (size_t)nblk)) != CUMC_OK) return rc;
    double* const* u = c->U[c->cur];
    double* fb[3] = {u[IBX], u[IBY], u[IBZ]};
    if (c->mixed) {  // face fields as FP64 (hi + lo) in the staging buffer
        const size_t NT = (size_t)b.count();
        if ((rc = ensure_staging(c)) != CUMC_OK) return rc;
        mixed_export(mx_launcher(c), b, c->mb, c->mp, 4, c->staging);
        for (int q = 0; q < 3; ++q) fb[q] = c->staging + q * NT;
    }
    const double *fx = fb[0], *fy = fb[1], *fz = fb[2];
    switch (c->coord) {
        case CUMC_CARTESIAN: launch(c, -1, n, 256, k_divb<1>, b, c->tabs, fx, fy, fz, c->divb_part); break;
        case CUMC_CYLINDRICAL: launch(c, -1, n, 256, k_divb<2>, b, c->tabs, fx, fy, fz, c->divb_part); break;
        default: launch(c, -1, n, 256, k_divb<3>, b, c->tabs, fx, fy, fz, c->divb_part); break;
    }
    std::vector<double> h(3 * (size_t)nblk);
    CUMC_CHECK(cudaMemcpyAsync(h.data(), c->divb_part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    double smax = 0.0, amax = 0.0, fmx = 0.0;  // the reference starts maxdb at 0 (solver/mhd.f90:41)
    for (int i = 0; i < nblk; ++i) {
        smax = std::fmax(smax, h[3 * i]);
        amax = std::fmax(amax, h[3 * i + 1]);
        fmx = std::fmax(fmx, h[3 * i + 2]);
    }
    if (maxdb_signed) *maxdb_signed = smax;
    if (maxabs_norm) *maxabs_norm = fmx > 0.0 ? amax / fmx : 0.0;
    return sync_status(c);
}

int cumc_advance(cumc_ctx* c, int nsteps, double t_end, double* t_inout, int* steps_done) {
    if (c) c->dt_valid = false;  // the state changes: the cached CFL dt is stale
    int rc = check_ready(c);
    if (rc != CUMC_OK) return rc;
    if (c->exchange) return c->fail(CUMC_ERR_STATE, "a slab with CUMC_BC_EXCHANGE faces steps by cumc_rk_stage and the halo exchange");
    if (c->next_stage != 1) return c->fail(CUMC_ERR_STATE, "cumc_rk_stage left a step unfinished");
    if (nsteps < 0 || !t_inout) return c->fail(CUMC_ERR_ARG, "nsteps must be >= 0 and t_inout non-null");
    launch(c, -1, 1, 1, k_set_scalar, c->scal + 1, *t_inout);
    CUMC_CHECK(cudaMemsetAsync(c->ints, 0, 2 * sizeof(int), c->stream));
    if (nsteps > 0) finddt_launch(c, c->box);  // dt of the first iteration; stage 3 gives the rest
    if (nsteps > 0 && !c->prof_on) {
        if (!c->graph_exec || c->graph_t_end != t_end) {
            if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
            cudaGraph_t g;
            CUMC_CHECK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            const long long before = c->launches;
            loop_step(c, t_end);
            const long long per_step = c->launches - before;
            c->launches = before;
            CUMC_CHECK(cudaStreamEndCapture(c->stream, &g));
            cudaError_t e = cudaGraphInstantiate(&c->graph_exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
            c->graph_t_end = t_end;
            c->graph_launches_per_step = per_step;
        }
    }
    // Steps are issued in chunks; between chunks the host reads t back and
    // stops once it has reached t_end (steps issued after that are no-ops on
    // the device through the done flag, so at most one chunk is wasted).
    constexpr int kChunk = 64;
    int issued = 0;
    while (issued < nsteps) {
        const int m = nsteps - issued < kChunk ? nsteps - issued : kChunk;
        for (int s = 0; s < m; ++s) {
            if (c->prof_on) {
                loop_step(c, t_end);
            } else {
                CUMC_CHECK(cudaGraphLaunch(c->graph_exec, c->stream));
                c->launches += c->graph_launches_per_step;
            }
        }
        issued += m;
        if (issued < nsteps) {
            CUMC_CHECK(cudaMemcpyAsync(c->host_pinned + 3, c->scal + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
            CUMC_CHECK(cudaStreamSynchronize(c->stream));
            double t_now;
            std::memcpy(&t_now, c->host_pinned + 3, sizeof(double));
            if (!(t_now < t_end)) break;
        }
    }
    CUMC_CHECK(cudaMemcpyAsync(c->host_pinned, c->scal + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaMemcpyAsync(c->host_pinned + 1, c->ints, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaMemcpyAsync(c->host_pinned + 2, c->flag_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    if ((rc = sync_status(c)) != CUMC_OK) return rc;
    std::memcpy(t_inout, c->host_pinned, sizeof(double));
    int st;
    std::memcpy(&st, c->host_pinned + 1, sizeof(int));
    if (steps_done) *steps_done = st;
    unsigned fl;
    std::memcpy(&fl, c->host_pinned + 2, sizeof(unsigned));
    if (fl & kTmaTimeoutFlag) return c->fail(CUMC_ERR_CUDA, "a staged bulk tensor copy never completed (wait gave up)");
    if (fl & 1u) return c->fail(CUMC_ERR_NONFINITE, "non-finite density, velocity or pressure in the evolved state");
    return CUMC_OK;
}

int cumc_get_stream(cumc_ctx* c, void** stream) {
    if (!c || !stream) return CUMC_ERR_ARG;
    *stream = (void*)c->stream;
    return CUMC_OK;
}

int cumc_profile(cumc_ctx* c, int enable) {
    if (!c) return CUMC_ERR_ARG;
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    for (auto& pe : c->prof) { cudaEventDestroy(pe.a); cudaEventDestroy(pe.b); }
    c->prof.clear();
    for (int i = 0; i < CUMC_K_COUNT; ++i) { c->prof_launches[i] = 0; c->prof_ms[i] = 0.0; }
    c->prof_on = enable != 0;
    return CUMC_OK;
}

int cumc_profile_read(cumc_ctx* c, int which, int* launches, double* ms) {
    if (!c || which < 0 || which >= CUMC_K_COUNT) return CUMC_ERR_ARG;
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    for (auto& pe : c->prof) {
        float t = 0.f;
        cudaEventElapsedTime(&t, pe.a, pe.b);
        c->prof_launches[pe.cls] += 1;
        c->prof_ms[pe.cls] += t;
        cudaEventDestroy(pe.a);
        cudaEventDestroy(pe.b);
    }
    c->prof.clear();
    if (launches) *launches = c->prof_launches[which];
    if (ms) *ms = c->prof_ms[which];
    return CUMC_OK;
}

int cumc_query(cumc_ctx* c, int what, long long* value) {
    if (!c || !value) return c ? c->fail(CUMC_ERR_ARG, "null argument") : CUMC_ERR_ARG;
    const bool fused = !c->mixed && (c->sweep_mode == 8 || c->sweep_mode == 9);
    switch (what) {
        case CUMC_Q_X_STAGING: *value = !fused ? -1 : (c->sweep_mode == 8 && c->xmaps_state == 1) ? 1 : 0; break;
        case CUMC_Q_FUSED: *value = fused ? 1 : 0; break;
        default: return c->fail(CUMC_ERR_ARG, "unknown query %d", what);
    }
    return CUMC_OK;
}

int cumc_launch_count(cumc_ctx* c, long long* count) {
    if (!c || !count) return CUMC_ERR_ARG;
    *count = c->launches;
    return CUMC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// discrete adjoint (cumc_adjoint_run): checkpointed forward pass, then per
// segment a recomputation that tapes each stage's combine output, then the
// reverse sweep of the kernels in cumc_adjoint.cuh
// ---------------------------------------------------------------------------
namespace {

// device scratch of an adjoint run: bump allocation from the context's
// slab (one cudaMalloc, kept for later runs of the same or smaller size)
struct AdjMem {
    char* base = nullptr;
    size_t cap = 0, off = 0;
};
constexpr size_t ADJ_ALIGN = 256;
size_t adj_round(size_t b) { return (b + ADJ_ALIGN - 1) / ADJ_ALIGN * ADJ_ALIGN; }

int adj_alloc(cumc_ctx* c, AdjMem& m, double** p, size_t n) {
    const size_t b = adj_round(n * sizeof(double));
    if (m.off + b > m.cap) return c->fail(CUMC_ERR_NOMEM, "adjoint: scratch slab too small (internal sizing error)");
    *p = reinterpret_cast<double*>(m.base + m.off);
    m.off += b;
    return CUMC_OK;
}

// one state: conserved U (face fields included) and primitives with ghosts
struct StateSet {
    double* u[8];
    double* w[5];
    double* bc[3];
    double* eps;
    PrimBufs prim() const { return PrimBufs{w, bc, eps}; }
    Prim as_prim() const {
        Prim p;
        for (int q = 0; q < 5; ++q) p.w[q] = w[q];
        for (int q = 0; q < 3; ++q) p.bc[q] = bc[q];
        for (int q = 0; q < 3; ++q) p.bf[q] = u[IBX + q];
        return p;
    }
    double** all(int i) { return i < 8 ? &u[i] : i < 13 ? &w[i - 8] : i < 16 ? &bc[i - 13] : &eps; }
};
constexpr int STATE_ARRAYS = 17;

int adj_state(cumc_ctx* c, AdjMem& m, StateSet& s) {
    for (int i = 0; i < STATE_ARRAYS; ++i) {
        int rc = adj_alloc(c, m, s.all(i), (size_t)c->box.count());
        if (rc != CUMC_OK) return rc;
    }
    return CUMC_OK;
}

StateSet live_state(cumc_ctx* c) {
    StateSet s;
    for (int q = 0; q < 8; ++q) s.u[q] = c->U[c->cur][q];
    for (int q = 0; q < 5; ++q) s.w[q] = c->w[q];
    for (int q = 0; q < 3; ++q) s.bc[q] = c->bc[q];
    s.eps = c->eps;
    return s;
}

void copy_state(cumc_ctx* c, StateSet dst, StateSet src) {
    const size_t bytes = (size_t)c->box.count() * sizeof(double);
    for (int i = 0; i < STATE_ARRAYS; ++i)
        cudaMemcpyAsync(*dst.all(i), *src.all(i), bytes, cudaMemcpyDeviceToDevice, c->stream);
}

// primitives (and boundary-filled face fields) of a taped combine output
void adj_prims_from(cumc_ctx* c, const Box& b, double* const* upre, StateSet& P) {
    const size_t bytes = (size_t)b.count() * sizeof(double);
    for (int q = 0; q < 8; ++q) cudaMemcpyAsync(P.u[q], upre[q], bytes, cudaMemcpyDeviceToDevice, c->stream);
    utop_into(c, b, P.u, P.prim(), true);
    boundary_into(c, b, P.u, P.prim());
}

Arr8 arr8(double* const* p, int n = 8) {
    Arr8 a{};
    for (int q = 0; q < n; ++q) a.a[q] = p[q];
    return a;
}
Arr3 arr3(double* const* p) {
    Arr3 a;
    for (int q = 0; q < 3; ++q) a.a[q] = p[q];
    return a;
}

// reconstruction transpose along y or z: the even segments, then the odd
// ones (k_adj_recon_col)
template <int D, int RECON>
void recon_col(cumc_ctx* c, const Box& b, const Prim& pr, const FaceAdj& fa, const AdjPrim& lp) {
    const int nseg = (WalkGeom<D>::nd(b) + 2 + RC_SEG - 1) / RC_SEG;
    for (int parity = 0; parity < 2; ++parity) {
        const unsigned gz = (unsigned)((nseg - parity + 1) / 2);
        if (gz == 0) continue;
        launch_grid(c, -1, dim3((unsigned)((WalkGeom<D>::ncols(b) + 127) / 128), 7, gz), 128, 0,
                    k_adj_recon_col<D, RECON>, b, c->tabs, pr, fa, lp, parity);
    }
}

template <int COORD, int RECON>
void adj_sweeps(cumc_ctx* c, const Box& b, const Prim& pr, const AdjStage& st, const AdjPrim& lp, double* const* lbf,
                const FaceAdj& fa) {
    const long long fx = (long long)(b.nx + 1) * (b.ny + 2) * (b.nz + 2);
    const long long fy = (long long)(b.nx + 2) * (b.ny + 1) * (b.nz + 2);
    const long long fz = (long long)(b.nx + 2) * (b.ny + 2) * (b.nz + 1);
    // face states of each direction from the forward sweep's STATES form
    FaceFlux sl, sr;
    for (int v = 0; v < 7; ++v) {
        sl.f[v] = fa.l[v];
        sr.f[v] = fa.r[v];
    }
    auto states = [&](auto dir) {
        constexpr int D = decltype(dir)::value;
        int nseg;
        const int seg = walk_segment_for<D>(b, WalkGeom<D>::ncols(b), c->sm_count, &nseg);
        const dim3 grid((unsigned)((WalkGeom<D>::ncols(b) + WK_THREADS - 1) / WK_THREADS), (unsigned)nseg);
        launch_grid(c, -1, grid, WK_THREADS, walk_smem<double>(D), k_sweep_walk_sm<D, RECON, double, true>, b, c->tabs,
                    pr, c->ggas, sl, seg, sr, 0, -1);
    };
    // x: pass A per face, pass B one lane per cell (28 owned cells a warp)
    launch(c, -1, xwarp_threads(b), 128, k_sweep_xwarp<RECON, double, true>, b, c->tabs, pr, c->ggas, sl, sr, 0, -1);
    launch(c, -1, fx, 128, k_adj_hll<COORD, 0, RECON, true>, b, c->tabs, pr, c->ggas, st, fa, lbf[0]);
    const long long xwarps = (long long)(b.ny + 2) * (b.nz + 2) * ((b.nx + 6 + 27) / 28);
    launch(c, -1, xwarps * 32, 128, k_adj_recon_x<RECON>, b, c->tabs, pr, fa, lp);
    // y, z: pass A per face, pass B one thread per (column, field)
    states(std::integral_constant<int, 1>{});
    launch(c, -1, fy, 128, k_adj_hll<COORD, 1, RECON, true>, b, c->tabs, pr, c->ggas, st, fa, lbf[1]);
    recon_col<1, RECON>(c, b, pr, fa, lp);
    states(std::integral_constant<int, 2>{});
    launch(c, -1, fz, 128, k_adj_hll<COORD, 2, RECON, true>, b, c->tabs, pr, c->ggas, st, fa, lbf[2]);
    recon_col<2, RECON>(c, b, pr, fa, lp);
}

// boundary^T: gather onto the sources, then clear the ghosts
void adj_boundary(cumc_ctx* c, const Box& b, const BoundArgs& fw, const AdjPrim& lp, double* const* lbf) {
    launch(c, -1, (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256, k_adj_boundary_gather, b, fw, lp, lbf[0],
           lbf[1], lbf[2]);
    launch(c, -1, ghost_count(b), 256, k_adj_boundary_clear, b, fw, lp, lbf[0], lbf[1], lbf[2]);
}

// SPATIAL^T of one stage: CT^T, ecell^T, GEOM_SOURCE^T (curvilinear grids)
// and the sweeps' transposes, all adding to the adjoints of the stage's
// input primitives (lp) and face fields (lbf)
template <int COORD>
void adj_spatial(cumc_ctx* c, const Box& b, const Prim& pr, const AdjStage& st, const AdjPrim& lp,
                 double* const* lbf, const FaceAdj& fa, double* const* lamE) {
    launch(c, -1, (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256, k_adj_ct<COORD>, b, c->tabs, st, lamE[0],
           lamE[1], lamE[2]);
    launch(c, -1, (long long)(b.nx + 2) * (b.ny + 2) * (b.nz + 2), 256, k_adj_ecell, b, pr, (const double*)lamE[0],
           (const double*)lamE[1], (const double*)lamE[2], lp);
    if (COORD != 1)
        launch(c, -1, (long long)b.nx * b.ny * b.nz, 256, k_adj_source<COORD == 1 ? 2 : COORD>, b, c->tabs, pr, st,
               c->cfg.geom_source_repeat, lp);
    if (c->recon == CUMC_PPMC) adj_sweeps<COORD, 4>(c, b, pr, st, lp, lbf, fa);
    else adj_sweeps<COORD, 1>(c, b, pr, st, lp, lbf, fa);
}

template <bool FROM_CONS>
void adj_utop(cumc_ctx* c, const Box& b, Arr8 u, Arr8 w0, const double* eps0, Arr8 lu, const AdjPrim& lp, Arr8 mu,
              Arr3 lb, double alpha = 0.0, double beta = 0.0, Arr8 lam0 = Arr8{}) {
    const long long n = (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1);
    if (c->model == CUMC_MODEL_RIEMANN)
        launch(c, -1, n, 256, k_adj_utop<1, FROM_CONS>, b, u, w0, eps0, lu, lp, c->ggas, mu, lb, alpha, beta, lam0);
    else
        launch(c, -1, n, 256, k_adj_utop<0, FROM_CONS>, b, u, w0, eps0, lu, lp, c->ggas, mu, lb, alpha, beta, lam0);
}

int adjoint_run(cumc_ctx* c, int N, int K, int obj, const double* weights, const double* dt_in, double* dt_out,
                double* J, double* grad_prim, double* grad_eps) {
    const Box b = c->box;
    const size_t NT = (size_t)b.count();
    const size_t bytes = NT * sizeof(double);
    const int nck = (N + K - 1) / K;
    const size_t arrays = (size_t)nck * STATE_ARRAYS + (size_t)K * 24 + 3 * STATE_ARRAYS + 8 * 3 + 3 * 2 + 9 + 14;
    const long long ncell = (long long)b.nx * b.ny * b.nz;
    const int nblk = (int)((ncell + 255) / 256);
    const size_t need = arrays * adj_round(bytes) + adj_round((size_t)(nblk + 1) * sizeof(double)) +
                        adj_round((size_t)N * sizeof(double));
    if (c->adj_slab_bytes < need) {
        if (c->adj_slab) {
            CUMC_CHECK(cudaStreamSynchronize(c->stream));
            cudaFree(c->adj_slab);
            c->adj_slab = nullptr;
            c->adj_slab_bytes = 0;
        }
        size_t fr = 0, tot = 0;
        CUMC_CHECK(cudaMemGetInfo(&fr, &tot));
        if (need + (256u << 20) > fr)
            return c->fail(CUMC_ERR_NOMEM, "adjoint needs %.2f GB of device memory (%zu arrays), %.2f GB free",
                           need / 1e9, arrays, fr / 1e9);
        if (cudaMalloc(&c->adj_slab, need) != cudaSuccess) {
            cudaGetLastError();
            c->adj_slab = nullptr;
            return c->fail(CUMC_ERR_NOMEM, "adjoint: cudaMalloc of %.2f GB failed", need / 1e9);
        }
        c->adj_slab_bytes = need;
    }
    AdjMem m;
    m.base = static_cast<char*>(c->adj_slab);
    m.cap = c->adj_slab_bytes;
    int rc;
    std::vector<StateSet> ck(nck);
    for (auto& s : ck)
        if ((rc = adj_state(c, m, s)) != CUMC_OK) return rc;
    std::vector<double*> tape((size_t)K * 24);
    for (auto& p : tape)
        if ((rc = adj_alloc(c, m, &p, NT)) != CUMC_OK) return rc;
    StateSet P[2], fin;
    for (StateSet* s : {&P[0], &P[1], &fin})
        if ((rc = adj_state(c, m, *s)) != CUMC_OK) return rc;
    double *lamA[8], *lamB[8], *mu[8], *lb[3], *lamE[3];
    AdjPrim lp;
    for (double** p : {lamA, lamB, mu})
        for (int q = 0; q < 8; ++q)
            if ((rc = adj_alloc(c, m, &p[q], NT)) != CUMC_OK) return rc;
    for (double** p : {lb, lamE})
        for (int q = 0; q < 3; ++q)
            if ((rc = adj_alloc(c, m, &p[q], NT)) != CUMC_OK) return rc;
    for (int q = 0; q < 5; ++q)
        if ((rc = adj_alloc(c, m, &lp.w[q], NT)) != CUMC_OK) return rc;
    for (int q = 0; q < 3; ++q)
        if ((rc = adj_alloc(c, m, &lp.bc[q], NT)) != CUMC_OK) return rc;
    if ((rc = adj_alloc(c, m, &lp.eps, NT)) != CUMC_OK) return rc;
    FaceAdj fa;
    for (int q = 0; q < 7; ++q)
        if ((rc = adj_alloc(c, m, &fa.l[q], NT)) != CUMC_OK || (rc = adj_alloc(c, m, &fa.r[q], NT)) != CUMC_OK)
            return rc;
    double *partial, *ddt;
    if ((rc = adj_alloc(c, m, &partial, (size_t)nblk + 1)) != CUMC_OK) return rc;
    if ((rc = adj_alloc(c, m, &ddt, (size_t)N)) != CUMC_OK) return rc;
    auto zero = [&](double* p) { cudaMemsetAsync(p, 0, bytes, c->stream); };
    for (double** p : {lamA, lamB, mu})
        for (int q = 0; q < 8; ++q) zero(p[q]);
    for (int q = 0; q < 3; ++q) { zero(lb[q]); zero(lamE[q]); }
    auto zero_lp = [&]() {
        for (int q = 0; q < 5; ++q) zero(lp.w[q]);
        for (int q = 0; q < 3; ++q) zero(lp.bc[q]);
        zero(lp.eps);
    };
    zero_lp();

    // ---- forward pass with checkpoints (initial_update, then N steps) ------
    utop(c, b, c->U[c->cur], false);
    boundary(c, b, c->U[c->cur]);
    std::vector<double> dts((size_t)N);
    const int last0 = (nck - 1) * K;  // the last segment is taped now, not recomputed
    for (int n = 0; n < N; ++n) {
        if (n % K == 0) copy_state(c, ck[n / K], live_state(c));
        c->tape = n >= last0 ? &tape[(size_t)(n - last0) * 24] : nullptr;
        double dt;
        if (dt_in) {
            dt = dt_in[n];
        } else {
            finddt_launch(c, b);
            CUMC_CHECK(cudaMemcpyAsync(c->host_pinned, c->dtmin, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
            CUMC_CHECK(cudaStreamSynchronize(c->stream));
            std::memcpy(&dt, c->host_pinned, sizeof(double));
        }
        dts[n] = dt;
        launch(c, -1, 1, 1, k_set_scalar, c->scal, dt);
        rk_step(c, b);
    }
    c->tape = nullptr;
    copy_state(c, fin, live_state(c));
    CUMC_CHECK(cudaMemcpyAsync(c->host_pinned + 1, c->flag_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    if ((rc = sync_status(c)) != CUMC_OK) return rc;
    {
        unsigned fl;
        std::memcpy(&fl, c->host_pinned + 1, sizeof(unsigned));
        if (fl & 1u) return c->fail(CUMC_ERR_NONFINITE, "adjoint: non-finite state in the forward pass");
    }
    CUMC_CHECK(cudaMemcpyAsync(ddt, dts.data(), (size_t)N * sizeof(double), cudaMemcpyHostToDevice, c->stream));

    // ---- objective and seed --------------------------------------------------
    double** lamCur = lamA;  // adjoint of the state at the current stage boundary
    double** lamU0 = lamB;   // adjoint of the step's starting state (accumulated)
    if (obj == CUMC_OBJ_LINEAR) {
        if ((rc = put_soa(c, weights, 8, lamCur)) != CUMC_OK) return rc;
        launch(c, -1, (long long)NT, 256, k_adj_mask_live, b, arr8(lamCur));
    }
    launch(c, -1, ncell, 256, k_adj_objective, b, c->tabs, c->coord, fin.as_prim(), arr8(fin.u), obj, lp, arr8(lamCur), partial);
    launch(c, -1, 256, 256, k_adj_sum, (const double*)partial, nblk, partial + nblk);
    CUMC_CHECK(cudaMemcpyAsync(c->host_pinned, partial + nblk, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    if (J) std::memcpy(J, c->host_pinned, sizeof(double));

    // ---- reverse sweep -----------------------------------------------------
    constexpr double alpha[4] = {0.0, 1.0, 3.0 / 4.0, 1.0 / 3.0};
    constexpr double beta[4] = {0.0, 0.0, 1.0 / 4.0, 2.0 / 3.0};
    constexpr double gam[4] = {0.0, 1.0, 1.0 / 4.0, 2.0 / 3.0};
    int pc = 0;
    bool have_next = false;  // P[pc] holds the primitives after step n
    for (int seg = nck - 1; seg >= 0; --seg) {
        const int a0 = seg * K, a1 = std::min(N, a0 + K);
        if (seg != nck - 1) {  // recompute the segment, taping each stage
            copy_state(c, live_state(c), ck[seg]);
            for (int n = a0; n < a1; ++n) {
                c->tape = &tape[(size_t)(n - a0) * 24];
                launch(c, -1, 1, 1, k_set_scalar, c->scal, dts[n]);
                rk_step(c, b);
            }
            c->tape = nullptr;
        }
        for (int n = a1 - 1; n >= a0; --n) {
            double* const* tp = &tape[(size_t)(n - a0) * 24];
            if (!have_next) adj_prims_from(c, b, tp + 16, P[pc]);
            for (int q = 0; q < 8; ++q) zero(lamU0[q]);
            for (int s = 3; s >= 1; --s) {
                StateSet& Pc = P[pc];
                StateSet& Pp = P[1 - pc];
                if (s >= 2) adj_prims_from(c, b, tp + (s - 2) * 8, Pp);
                else if (n > a0) adj_prims_from(c, b, &tape[(size_t)(n - 1 - a0) * 24 + 16], Pp);
                else copy_state(c, Pp, ck[seg]);
                // boundary^T and utop^T of the stage's output
                adj_boundary(c, b, bound_args(c, Pc.u, Pc.prim()), lp, lamCur + IBX);
                // utop^T and the face-field gather, each with the combine^T of its part
                adj_utop<true>(c, b, arr8(tp + (s - 1) * 8), arr8(Pc.w, 5), nullptr, arr8(lamCur), lp, arr8(mu), arr3(lb),
                               alpha[s], beta[s], arr8(lamU0));
                launch(c, -1, (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256, k_adj_bface, b, arr3(lamCur + IBX),
                       arr3(lb), arr3(mu + IBX), alpha[s], beta[s], arr3(lamU0 + IBX));
                zero_lp();
                // L^T at the stage's input
                AdjStage st;
                for (int q = 0; q < 8; ++q) st.mu[q] = mu[q];
                for (int q = 0; q < 3; ++q) st.lamE[q] = lamE[q];
                st.dt = ddt + n;
                st.gam = gam[s];
                const Prim pr = Pp.as_prim();
                double* const* lbf = s >= 2 ? lamCur + IBX : lamU0 + IBX;
                switch (c->coord) {
                    case CUMC_CARTESIAN: adj_spatial<1>(c, b, pr, st, lp, lbf, fa, lamE); break;
                    case CUMC_CYLINDRICAL: adj_spatial<2>(c, b, pr, st, lp, lbf, fa, lamE); break;
                    default: adj_spatial<3>(c, b, pr, st, lp, lbf, fa, lamE); break;
                }
                pc = 1 - pc;
            }
            std::swap(lamCur, lamU0);  // adjoint of the step's starting state
            have_next = true;
        }
    }
    // ---- initial_update^T: P[pc] and ck[0] hold the state after initial_update
    adj_boundary(c, b, bound_args(c, ck[0].u, ck[0].prim()), lp, lamCur + IBX);
    adj_utop<false>(c, b, arr8(ck[0].u), arr8(ck[0].w, 5), ck[0].eps, arr8(lamCur), lp, arr8(mu), arr3(lb));
    launch(c, -1, (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256, k_adj_bface, b, arr3(lamCur + IBX), arr3(lb),
           arr3(mu + IBX), 0.0, 0.0, Arr3{});
    if ((rc = sync_status(c)) != CUMC_OK) return rc;
    if (grad_prim) {
        const double* s[8] = {mu[0], mu[1], mu[2], mu[3], nullptr, mu[IBX], mu[IBY], mu[IBZ]};
        if ((rc = get_soa(c, grad_prim, 8, s)) != CUMC_OK) return rc;
    }
    if (grad_eps) {
        const double* s[1] = {mu[4]};
        if ((rc = get_soa(c, grad_eps, 1, s)) != CUMC_OK) return rc;
    }
    if (dt_out) std::memcpy(dt_out, dts.data(), (size_t)N * sizeof(double));
    copy_state(c, live_state(c), fin);
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    c->ready = true;
    return sync_status(c);
}

}  // namespace

extern "C" int cumc_adjoint_run(cumc_ctx* c, int nsteps, int checkpoint_every, int objective, const double* weights,
                                const double* dt_in, double* dt_out, double* J, double* grad_prim, double* grad_eps) {
    if (c) c->dt_valid = false;
    if (!c) return CUMC_ERR_ARG;
    if (!c->uploaded) return c->fail(CUMC_ERR_STATE, "cumc_upload_state must come first");
    if (c->mixed || c->fast || c->exchange || (c->model != CUMC_MODEL_NONE && c->model != CUMC_MODEL_RIEMANN))
        return c->fail(CUMC_ERR_CONFIG, "the adjoint covers CUMC_FP64 with model NONE or RIEMANN on one domain");
    if (nsteps < 1 || checkpoint_every < 1) return c->fail(CUMC_ERR_ARG, "nsteps and checkpoint_every must be >= 1");
    if (objective < CUMC_OBJ_MAGNETIC || objective > CUMC_OBJ_LINEAR) return c->fail(CUMC_ERR_ARG, "unknown objective");
    if (objective == CUMC_OBJ_LINEAR && !weights) return c->fail(CUMC_ERR_ARG, "CUMC_OBJ_LINEAR needs weights");
    if (dt_in)
        for (int n = 0; n < nsteps; ++n)
            if (!(dt_in[n] >= 0.0 && std::isfinite(dt_in[n])))
                return c->fail(CUMC_ERR_ARG, "dt_in[%d] must be finite and non-negative", n);
    const int rc = adjoint_run(c, nsteps, std::min(checkpoint_every, nsteps), objective, weights, dt_in, dt_out, J,
                               grad_prim, grad_eps);
    c->tape = nullptr;
    return rc;
}

// ---------------------------------------------------------------------------
// Snapshots and exact restart. The reference writes prim and eps
// (solver/dataio.f90:7-331) and cannot restart; here the whole state (the 17
// arrays a step reads: cons, w, bcell, eps) goes to the host, so that a
// context restored from it continues bit for bit. The copy out overlaps the
// following steps: the state is first copied to a device staging slab on the
// context's stream, then to the host on a stream of its own.
// ---------------------------------------------------------------------------
namespace {
int snapshot_setup(cumc_ctx* c) {
    if (c->snap_dev) return CUMC_OK;
    int rc = dalloc(c, &c->snap_dev, STATE_ARRAYS * (size_t)c->box.count());
    if (rc != CUMC_OK) return rc;
    CUMC_CHECK(cudaStreamCreateWithFlags(&c->snap_stream, cudaStreamNonBlocking));
    CUMC_CHECK(cudaEventCreateWithFlags(&c->snap_taken, cudaEventDisableTiming));
    CUMC_CHECK(cudaEventCreateWithFlags(&c->snap_done, cudaEventDisableTiming));
    return CUMC_OK;
}
}  // namespace

extern "C" int cumc_snapshot_async(cumc_ctx* c, double* host_state) {
    int rc = check_ready(c);
    if (rc != CUMC_OK) return rc;
    if (c->mixed) return c->fail(CUMC_ERR_CONFIG, "snapshots cover CUMC_FP64");
    if (!host_state) return c->fail(CUMC_ERR_ARG, "null host buffer");
    if ((rc = snapshot_setup(c)) != CUMC_OK) return rc;
    const size_t NT = (size_t)c->box.count();
    // the slab is reused: the previous snapshot's copy out must have read it
    if (c->snap_pending) CUMC_CHECK(cudaStreamWaitEvent(c->stream, c->snap_done, 0));
    StateSet s = live_state(c);
    for (int i = 0; i < STATE_ARRAYS; ++i)
        CUMC_CHECK(cudaMemcpyAsync(c->snap_dev + i * NT, *s.all(i), NT * sizeof(double), cudaMemcpyDeviceToDevice,
                                   c->stream));
    CUMC_CHECK(cudaEventRecord(c->snap_taken, c->stream));
    CUMC_CHECK(cudaStreamWaitEvent(c->snap_stream, c->snap_taken, 0));
    CUMC_CHECK(cudaMemcpyAsync(host_state, c->snap_dev, STATE_ARRAYS * NT * sizeof(double), cudaMemcpyDeviceToHost,
                               c->snap_stream));
    CUMC_CHECK(cudaEventRecord(c->snap_done, c->snap_stream));
    c->snap_pending = true;
    return CUMC_OK;
}

extern "C" int cumc_snapshot_wait(cumc_ctx* c) {
    if (!c) return CUMC_ERR_ARG;
    if (c->snap_pending) {
        CUMC_CHECK(cudaEventSynchronize(c->snap_done));
        c->snap_pending = false;
    }
    return CUMC_OK;
}

extern "C" int cumc_restore_state(cumc_ctx* c, const double* host_state) {
    if (c) c->dt_valid = false;  // the state changes: the cached CFL dt is stale
    if (!c || !host_state) return c ? c->fail(CUMC_ERR_ARG, "null argument") : CUMC_ERR_ARG;
    if (c->mixed) return c->fail(CUMC_ERR_CONFIG, "snapshots cover CUMC_FP64");
    int rc = cumc_snapshot_wait(c);  // the staging slab and stream are quiet
    if (rc != CUMC_OK) return rc;
    const size_t NT = (size_t)c->box.count();
    StateSet s = live_state(c);
    for (int i = 0; i < STATE_ARRAYS; ++i)
        CUMC_CHECK(cudaMemcpyAsync(*s.all(i), host_state + i * NT, NT * sizeof(double), cudaMemcpyHostToDevice,
                                   c->stream));
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    c->uploaded = true;
    c->ready = true;
    c->next_stage = 1;
    c->bf_set = c->cur;
    return sync_status(c);
}

// ---------------------------------------------------------------------------
// cumc_model_torus: GET_MODEL of the spherical torus on the device
// ---------------------------------------------------------------------------
extern "C" int cumc_model_torus(cumc_ctx* c, const cumc_torus_model* p) {
    if (c) c->dt_valid = false;  // the state changes: the cached CFL dt is stale
    if (!c || !p) return c ? c->fail(CUMC_ERR_ARG, "null argument") : CUMC_ERR_ARG;
    if (c->coord == CUMC_CARTESIAN)
        return c->fail(CUMC_ERR_CONFIG, "the torus model needs CUMC_SPHERICAL or CUMC_CYLINDRICAL");
    const double g = c->ggas, q = p->q_grad, rsh = p->r_sh;
    const bool cyl = c->coord == CUMC_CYLINDRICAL;
    // the potential on the equator (z = 0 for the cylindrical form)
    auto schw = [&](double r) { return cyl ? -1.0 / (std::sqrt(r * r + 0.0 * 0.0) - rsh) : -1.0 / (r - rsh); };
    TorusK m;
    m.ggas = g;
    m.r_sh = rsh;
    m.s_in = p->s_in;
    m.q = q;
    m.lkep2 = std::pow(p->s_max, 2.0 * q - 1.0) / std::pow(p->s_max - rsh, 2.0);
    m.c_const = schw(p->s_in) - m.lkep2 * std::pow(p->s_in, 2.0 - 2.0 * q) / (2.0 - 2.0 * q);
    const double h_max = -schw(p->s_max) + m.lkep2 * std::pow(p->s_max, 2.0 - 2.0 * q) / (2.0 - 2.0 * q) + m.c_const;
    m.k_poly = h_max * (g - 1.0) / g / std::pow(p->rho_max, g - 1.0);
    if (!(m.k_poly >= 0.0)) return c->fail(CUMC_ERR_CONFIG, "the polytropic constant is negative");
    m.rho_a = p->rho_fac * p->rho_max;
    m.rho_max = p->rho_max;
    m.rho_cut = p->rho_cut;
    m.beta = p->beta;
    m.noise = p->noise;
    m.rho_floor = p->rho_fac * p->rho_max;
    m.seed = p->seed;
    m.cyl = cyl ? 1 : 0;
    int rc = ensure_staging(c);
    if (rc != CUMC_OK) return rc;
    if (!c->model_max && (rc = dalloc(c, &c->model_max, 2)) != CUMC_OK) return rc;
    const Box& b = c->box;
    const size_t NT = (size_t)b.count();
    double* prim = c->staging;
    double* eps = c->staging + 8 * NT;
    launch(c, -1, (long long)NT, 256, k_torus_cells, b, c->tabs, m, prim, eps);
    launch(c, -1, (long long)(b.nx + 1) * (b.ny + 1) * (b.nz + 1), 256, k_torus_faces, b, c->tabs, m, prim);
    CUMC_CHECK(cudaMemsetAsync(c->model_max, 0, 2 * sizeof(unsigned long long), c->stream));
    launch(c, -1, (long long)b.nx * b.ny * b.nz, 256, k_torus_max, b, m, (const double*)prim, c->model_max);
    launch(c, -1, (long long)NT, 256, k_torus_finish, b, m, (const unsigned long long*)c->model_max, prim);
    if (!c->mixed) {  // the FP64 state arrays, as cumc_upload_state fills them
        double* dst[9] = {c->w[0], c->w[1], c->w[2], c->w[3], c->w[4],
                          c->U[c->cur][IBX], c->U[c->cur][IBY], c->U[c->cur][IBZ], c->eps};
        CUMC_CHECK(cudaMemcpyAsync(c->dsoa, dst, 8 * sizeof(double*), cudaMemcpyHostToDevice, c->stream));
        launch(c, -1, (long long)NT, 256, k_aos_to_soa, (long long)NT, 8, (const double*)prim, c->dsoa);
        CUMC_CHECK(cudaMemcpyAsync(c->eps, eps, NT * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    }
    CUMC_CHECK(cudaStreamSynchronize(c->stream));
    c->uploaded = true;
    c->ready = false;
    return sync_status(c);
}
