/*
 * cumc.h — C-ABI of the B200-native CUMC3D hot path.
 *
 * The reference (leon-astrophy/CUMPIC, program CUMC3D) drives its per-step
 * update from solver/main.f90 through argument-free Fortran subroutines that
 * read and write MODULE DEFINITION globals (solver/definition.f90:238-312).
 * This header exports the same steps as plain C functions on an opaque
 * context, so that main.f90 can keep its call sequence through a thin
 * iso_c_binding module with the subroutines' own names, and so that C, C++
 * and Python (ctypes) callers can use the same library.
 *
 * Conventions
 *   - Every function returns an int status: CUMC_OK (0) or a CUMC_ERR_* code.
 *     cumc_last_error() gives a one-line description of the last failure.
 *   - Host arrays use the reference's Fortran layout: prim/cons are
 *     REAL*8 A(1:8, -2:nx+3, -2:ny+3, -2:nz+3) (variable index fastest,
 *     solver/setup.f90:257-260), eps is (-2:nx+3, -2:ny+3, -2:nz+3)
 *     (solver/setup.f90:263), bcell is (6:8, -2:nx+3, ...) (:286).
 *     Variable order irho=1, ivx=2, ivy=3, ivz=4, itau=5, ibx=6, iby=7,
 *     ibz=8 (solver/setup.f90:49-116).  prim(itau) is the gas pressure,
 *     cons(itau) the total energy; prim/cons(ibx) is the face field at xF(j).
 *   - The library owns all device memory; caller buffers are never aliased.
 *   - One host thread per context; calls on a context are serialised on the
 *     context's own CUDA stream.
 *   - There is no CPU fallback: if no CUDA device is usable, cumc_init fails.
 */
#ifndef CUMC_H
#define CUMC_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CUMC_OK              0
#define CUMC_ERR_ARG         1  /* bad pointer or argument value               */
#define CUMC_ERR_CONFIG      2  /* config rejected (reference would STOP)      */
#define CUMC_ERR_CUDA        3  /* CUDA runtime error (message has details)    */
#define CUMC_ERR_NONFINITE   4  /* device flagged NaN/Inf in the evolved state */
#define CUMC_ERR_STATE       5  /* call made in the wrong order                */
#define CUMC_ERR_NOMEM       6  /* device allocation failed                    */
#define CUMC_ERR_LIMIT       7  /* size beyond a documented maximum            */

/* coordinate systems (solver/definition.f90:65-69) */
#define CUMC_CARTESIAN   1
#define CUMC_CYLINDRICAL 2
#define CUMC_SPHERICAL   3

/* reconstruction (solver/definition.f90:158-173); only TVDMM and PPMC are
 * implemented by the reference (solver/reconstruct.f90:36-49) */
#define CUMC_TVDMM 1
#define CUMC_PPMC  4

/* Riemann solver (solver/definition.f90:139-151); the reference implements
 * HLL only (solver/rsolver.f90:26-34) */
#define CUMC_HLL 2

/* arithmetic of the path */
#define CUMC_FP64  0  /* all FP64, bit-compatible with the FP64 restatement  */
#define CUMC_FP64_FAST 2  /* FP64 throughout, but the HLL solve forms its 21
                            quotients a face as products with 5 reciprocals:
                            not bit-compatible, within a few ulp a face
                            (no counterpart in the reference)                */
#define CUMC_MIXED 1  /* FP32 reconstruction/HLL/EMF, compensated FP32 state,
                         FP64 energy and pressure recovery                   */

/* model hooks (model/<m>/src/custom.f90) that sit on the hot path */
#define CUMC_MODEL_NONE      0  /* all hooks empty                                    */
#define CUMC_MODEL_RIEMANN   1  /* CUSTOM_CHECKRHO: eps >= 0 (model/riemann/src/custom.f90:54-76) */
#define CUMC_MODEL_TORUS_SPH 2  /* floors, point-mass gravity, radial no-inflow ghosts
                                   (model/torus_sph/src/custom.f90:47-150)              */
#define CUMC_MODEL_TORUS_CYN 3  /* floors, gravity in (R,z), R and z no-inflow ghosts
                                   (model/torus_cyn/src/custom.f90)                     */

typedef struct cumc_config {
    int nx, ny, nz;          /* active cells per direction (whole domain on one GPU) */
    /* face coordinates, nx+7 (ny+7, nz+7) entries for indices -3..n+3
     * (solver/setup.f90:297-303, filled by GETGRID solver/coords.f90:11-41) */
    const double *xf, *yf, *zf;
    int coordinate;          /* CUMC_CARTESIAN / CUMC_CYLINDRICAL / CUMC_SPHERICAL */
    int boundary_flag[6];    /* x-in, x-out, y-in, y-out, z-in, z-out: 0 periodic,
                                1 outflow, 2 reflect, 3 axis, 4 equatorial
                                (solver/definition.f90:74-87); z faces may also be
                                CUMC_BC_EXCHANGE (a neighbouring slab's face)     */
    double ggas;             /* adiabatic index (model/<m>/src/defs.f90:14)        */
    double cfl;              /* Courant number (solver/definition.f90:116)        */
    int recon;               /* CUMC_PPMC or CUMC_TVDMM                            */
    int solver;              /* CUMC_HLL                                           */
    int precision;           /* CUMC_FP64, CUMC_FP64_FAST or CUMC_MIXED            */
    int model;               /* CUMC_MODEL_*                                       */
    double rho_floor;        /* torus models: atmosphere density floor            */
    double eps_floor;        /* torus models: specific internal energy floor      */
    double r_sh;             /* torus models: potential softening radius          */
    /* GET_SOURCE calls GEOM_SOURCE once per equation index imin..imax, so the
     * geometric source enters 8 times (solver/spatial.f90:86-97).  8 keeps
     * that behaviour (the default); 1 applies it once. Ignored in Cartesian. */
    int geom_source_repeat;
    int reserved[7];         /* must be zero                                      */
} cumc_config;

typedef struct cumc_ctx cumc_ctx;

/* Replaces POPULATE_DEVICE (solver/openacc.f90:28-59, called at
 * solver/main.f90:98-100) plus the bfac tables of SETUP_EQNS
 * (solver/setup.f90:121-230): validates the config, builds the per-axis
 * metric and reconstruction tables and allocates device state. */
int cumc_init(const cumc_config* cfg, cumc_ctx** out);

/* Releases every device allocation of the context. */
int cumc_free(cumc_ctx* ctx);

/* Last error message of this context (ctx may be NULL for cumc_init errors). */
const char* cumc_last_error(const cumc_ctx* ctx);

/* Host -> device copy of the initial model: prim(1:8,...) and eps(...) in the
 * Fortran layout, as GET_MODEL leaves them (solver/initial.f90:93). */
int cumc_upload_state(cumc_ctx* ctx, const double* prim, const double* eps);

/* Device -> host copy replacing "!$ACC UPDATE HOST(prim, eps)"
 * (solver/dataio.f90:24). Any pointer may be NULL. cons and prim cover the
 * whole ghosted array; entries the reference never writes are returned as
 * the library holds them. */
int cumc_download_state(cumc_ctx* ctx, double* prim, double* cons,
                        double* eps, double* bcell);

/* initial_update (solver/initial.f90:83-140):
 * CUSTOM_CHECKRHO -> FROMRVETOU -> BOUNDARY -> UPDATE(0). */
int cumc_initial_update(cumc_ctx* ctx);

/* finddt (solver/rungekutta.f90:161-265): CFL time step as a device
 * min-reduction; the value is returned to the host because main.f90 clips
 * it to total_time (solver/main.f90:133-135). Also reports a non-finite
 * state flagged by the previous steps (CUMC_ERR_NONFINITE). */
int cumc_finddt(cumc_ctx* ctx, double* dt);

/* RUNGEKUTTA (solver/rungekutta.f90:12-148): one full SSP-RK3 step with the
 * given dt, entirely on the device. Returns without a host sync. */
int cumc_rungekutta(cumc_ctx* ctx, double dt);

/* SPATIAL (solver/spatial.f90:11-68) on the current state: fills the
 * library's l_rk without advancing. For unit-level checks. */
int cumc_spatial(cumc_ctx* ctx);

/* Device -> host copy of l_rk(1:8,...) (Fortran layout; entries outside the
 * ranges SPATIAL writes are zero). */
int cumc_download_lrk(cumc_ctx* ctx, double* lrk);

/* find_divb (solver/mhd.f90:15-66): *maxdb_signed is the reference's
 * MAX over cells of the signed, area-weighted divergence; *maxabs_norm is
 * max |div B| * (cell size) / max|B|, the normalised figure used by the
 * tests. Either pointer may be NULL. */
int cumc_divb(cumc_ctx* ctx, double* maxdb_signed, double* maxabs_norm);

/* The time loop of solver/main.f90:127-143 on the device: up to nsteps of
 * (finddt, clip dt so that t does not pass t_end, RUNGEKUTTA), stopping
 * early once t reaches t_end. *t_inout is the start time on entry and the
 * end time on return; *steps_done (may be NULL) gets the steps taken.
 * dt never leaves the device during the loop; one host sync at the end. */
int cumc_advance(cumc_ctx* ctx, int nsteps, double t_end, double* t_inout,
                 int* steps_done);

/* The CUDA stream (cudaStream_t) every call of this context runs on. */
int cumc_get_stream(cumc_ctx* ctx, void** stream);

/* Per-kernel timing with CUDA events on the context stream. enable=1 starts
 * recording (and clears totals); cumc_profile_read returns, for kernel class
 * `which` (CUMC_K_*), the number of launches and their summed milliseconds. */
#define CUMC_K_SWEEP_X  0
#define CUMC_K_SWEEP_Y  1
#define CUMC_K_SWEEP_Z  2
#define CUMC_K_EMF      3
#define CUMC_K_COMBINE  4   /* FP64 stages: hydro combine fused with the conversions */
#define CUMC_K_UTOP     5   /* FP64: initial_update's conversions */
#define CUMC_K_BOUNDARY 6
#define CUMC_K_FINDDT   7
#define CUMC_K_CT       8   /* FP64 stages: face-field (CT) combine */
#define CUMC_K_COUNT    9
int cumc_profile(cumc_ctx* ctx, int enable);
int cumc_profile_read(cumc_ctx* ctx, int which, int* launches, double* ms);

/* Number of kernel launches the library issued since cumc_init. */
int cumc_launch_count(cumc_ctx* ctx, long long* count);

/* Introspection of how the context runs a stage (no counterpart in the
 * reference). CUMC_Q_FUSED: 1 when the FP64 stages run with the flux
 * differences fused into the sweeps (environment CUMC_SWEEP=fused or
 * fused_notma at cumc_init), else 0 (the default: the sweeps write face
 * fluxes and one kernel combines them). CUMC_Q_X_STAGING: for a fused
 * context, 1 when its x sweep stages the rows into shared memory by bulk
 * tensor copies (TMA), 0 when it loads them directly (fused_notma, a row
 * pitch that is not a multiple of 16 bytes, or no tensor-map support in the
 * driver); -1 for other contexts. */
#define CUMC_Q_X_STAGING 1
#define CUMC_Q_FUSED     2
int cumc_query(cumc_ctx* ctx, int what, long long* value);

/* Device-side GET_MODEL of the tori (model/torus_sph/src/model.f90:8-284 on
 * a CUMC_SPHERICAL grid, model/torus_cyn/src/model.f90:8-284 on a
 * CUMC_CYLINDRICAL one), for grids too large to build on the host: a
 * constant-angular-momentum torus, potential -1/(r - r_sh) (spherical) or
 * -1/(sqrt(R^2 + z^2) - r_sh) (cylindrical), polytropic with
 * p = K rho^gamma, density floor rho_fac * rho_max outside;
 * A_phi = max(rho - rho_cut, 0)/rho_max on the cells, averaged to the
 * corners, face fields B = curl A normalised to max p_gas / max p_mag = beta;
 * then density noise rho (1 + noise (2u - 1)) where rho > rho_fac * rho_max,
 * u from splitmix64(seed, linear cell index). Fills the state as
 * cumc_upload_state would (call cumc_initial_update next); the grid is the
 * context's (CUMC_ERR_CONFIG on a Cartesian one). The host generators
 * cumpic_b200.problems.torus and torus_cyl build the same states. */
typedef struct {
    double r_sh, s_in, s_max, q_grad;   /* potential centre, torus inner edge, pressure maximum, l ~ s^(2-q) */
    double rho_max, rho_fac, rho_cut;   /* peak density, floor factor, field threshold */
    double beta, noise;                 /* plasma beta of the maxima, density noise amplitude */
    unsigned long long seed;
} cumc_torus_model;
int cumc_model_torus(cumc_ctx* ctx, const cumc_torus_model* model);

/* z-slab decomposition: the halo exchange between slabs (replaces the MPI
 * path of solver/mpi.f90:255-501, MPI_BOUNDARYP_Z / MPI_BOUNDARY_Z, and the
 * internal faces of solver/boundary.f90:332-336,663-667). A z face whose
 * boundary_flag is CUMC_BC_EXCHANGE is shared with a neighbouring slab: the
 * boundary fill leaves its three ghost planes alone (except the face field
 * Bz on the face itself, which CT computes on both sides) and the caller
 * fills them from the neighbour after cumc_initial_update and after every
 * stage. A slab steps by cumc_rk_stage(ctx, 1..3, dt) (dt read at stage 1;
 * the three stages of RUNGEKUTTA, solver/rungekutta.f90:38-134, each with
 * its conversions and boundary fill); cumc_rungekutta, cumc_advance and
 * cumc_adjoint_run refuse such a context. cumc_halo_pack(ctx, side, buf)
 * copies the three active planes next to face `side` (0: z-in, planes 1..3;
 * 1: z-out, planes nz-2..nz) of w (5), bcell (3), eps and the face fields
 * Bx, By into the device buffer buf (cumc_halo_doubles doubles: 11 arrays
 * x 3 planes x (nx+6)(ny+6)); cumc_halo_unpack(ctx, side, buf) writes a
 * neighbour's packed planes into the ghost planes of face `side` (0: planes
 * -2..0 from the z-in neighbour's side-1 pack; 1: planes nz+1..nz+3 from the
 * z-out neighbour's side-0 pack). Both are enqueued on the context's stream
 * (cumc_get_stream). FP64 only. */
#define CUMC_BC_EXCHANGE (-1)
int cumc_rk_stage(cumc_ctx* ctx, int stage, double dt);
/* One RK stage in two parts, so that the halo exchange of the previous
 * stage's output (the MPI part of the reference's BOUNDARY after each stage,
 * solver/rungekutta.f90:63,97,141) can run beside the next stage's
 * computation: part 1 queues the x and y sweeps of the active planes 1..nz,
 * which read no ghost plane; part 2 queues the rest of the stage and must
 * follow part 1 of the same stage, after the ghost planes are unpacked.
 * part 0 is the whole stage (cumc_rk_stage). dt is read at stage 1, part 1
 * or 0. Forms of the stage without the split (the mixed precision and most
 * CUMC_SWEEP variants) run everything at part 2. */
int cumc_rk_stage_part(cumc_ctx* ctx, int stage, double dt, int part);
int cumc_halo_doubles(cumc_ctx* ctx, long long* n);
int cumc_halo_pack(cumc_ctx* ctx, int side, double* buf);
int cumc_halo_unpack(cumc_ctx* ctx, int side, const double* buf);

/* Snapshot and exact restart of the FP64 state. Replace the reference's
 * output step print_hydroprofile (solver/dataio.f90:7-77, HDF5 prim and eps
 * only, no restart). The state is the 17 arrays a step reads, each
 * (nx+6)(ny+6)(nz+6) doubles in the index order of the prim layout without
 * its field index (x fastest): cons 1-8, prim 1-5 (rho, vx, vy, vz, p),
 * bcell 1-3, eps; CUMC_STATE_ARRAYS of them back to back.
 *
 * cumc_snapshot_async copies the current state (after cumc_initial_update or
 * a step) to a device staging slab on the context's stream, then to
 * host_state on a second stream, and returns at once: the steps issued next
 * overlap the copy out and do not change what it delivers. host_state should
 * be pinned for the copy to be asynchronous, and must stay untouched until
 * cumc_snapshot_wait returns. A second snapshot waits (on the device) for the
 * first one's copy out. The staging slab is allocated on the first call.
 * cumc_restore_state uploads such a state; the context then continues
 * exactly as the one that took it (no cumc_initial_update needed). Both
 * return CUMC_ERR_CONFIG for CUMC_MIXED. */
#define CUMC_STATE_ARRAYS 17
int cumc_snapshot_async(cumc_ctx* ctx, double* host_state);
int cumc_snapshot_wait(cumc_ctx* ctx);
int cumc_restore_state(cumc_ctx* ctx, const double* host_state);

/* Discrete adjoint of the FP64 path. No counterpart in the reference, which
 * has no derivatives; it is the new entry point cumc_adjoint_run of the hot
 * path's drop-in boundary.
 *
 * Starting from the state last given to cumc_upload_state, runs
 * initial_update and nsteps RUNGEKUTTA steps, evaluates the objective J on
 * the final state and returns dJ/d(uploaded state) by the transpose of every
 * kernel of the step (reconstruction limiters, extremum fixes and HLL wave
 * choices frozen as the forward pass took them; HLL, CT, boundaries and the
 * conversions differentiated exactly). The dt sequence is frozen: taken from
 * dt_in[0..nsteps) when given, else from finddt each step, and returned in
 * dt_out (may be NULL). Memory is traded for recomputation: the forward state
 * is checkpointed every checkpoint_every steps and each segment is recomputed
 * once during the reverse sweep; this needs
 *   (ceil(nsteps/checkpoint_every) * 17 + checkpoint_every * 24 + 107)
 * arrays of (nx+6)(ny+6)(nz+6) doubles of device memory (CUMC_ERR_NOMEM if
 * absent).
 *
 * objective: CUMC_OBJ_MAGNETIC  J = 1/2 sum |bcell|^2 dV over the active cells
 *            CUMC_OBJ_KINETIC   J = 1/2 sum rho |v|^2 dV
 *            CUMC_OBJ_LINEAR    J = sum weights . cons over the entries the
 *                               step defines (active cells; face fields at
 *                               index 0:n along their axis, 1:n across);
 *                               weights in the cons layout.
 * grad_prim (prim layout, may be NULL): dJ/d(rho, vx, vy, vz) in slots 1-4,
 *            0 in slot 5 (initial_update takes the pressure from eps), and
 *            dJ/d(face Bx, By, Bz) in slots 6-8; grad_eps (eps layout, may be
 *            NULL): dJ/d(eps). Ghost entries, which initial_update
 *            overwrites, get 0.
 * dV is the cell volume: dx dy dz (Cartesian), R dR dphi dz (cylindrical),
 * (r^3)/3 d(-cos theta) dphi over the cell (spherical).
 * On return the context holds the final state, as after cumc_initial_update
 * and nsteps cumc_rungekutta calls. Supported: CUMC_FP64 on every coordinate
 * system (the geometric flux, CT and source terms included), models NONE
 * and RIEMANN (CUMC_ERR_CONFIG otherwise). */
#define CUMC_OBJ_MAGNETIC 1
#define CUMC_OBJ_KINETIC  2
#define CUMC_OBJ_LINEAR   3
int cumc_adjoint_run(cumc_ctx* ctx, int nsteps, int checkpoint_every, int objective,
                     const double* weights, const double* dt_in, double* dt_out,
                     double* J, double* grad_prim, double* grad_eps);

/* CFL time step over caller-owned device arrays, allocating nothing.
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory when they need a time step, such as a code capturing
 * its time loop into a CUDA graph (cudaMalloc is not allowed during capture)
 * or a host program whose device memory is owned by another runtime (an
 * OpenACC data region, a framework's caching allocator, a fixed pool).
 *
 * Inputs are device arrays in the library's layout: one FP64 array per field
 * over the ghosted box (-2:n+3)^3, x fastest (rho, vx, vy, vz, p, and the
 * cell-centred field bcx, bcy, bcz), and per-axis cell widths dx, dy, dz with
 * nx+7 (ny+7, nz+7) entries for indices -3..n+3. Cylindrical and spherical
 * grids also need the cell-centre radius xc (nx+7 entries) and, spherical,
 * sin of the polar cell centre sin_yc (ny+7 entries); both may be NULL for
 * CUMC_CARTESIAN. The result is written to the device double *dt_out; the
 * work is queued on `stream` (NULL: the default stream) and the call returns
 * without synchronising.
 *
 * Its only scratch, the per-block partial minima, is a fixed device array of
 * the library (512 KiB per device, held until the process exits), which
 * limits a call to CUMC_STATIC_MAX_CELLS active cells; larger grids get
 * CUMC_ERR_LIMIT. The first call on each device looks up that array's device
 * address (cudaGetSymbolAddress), so make a first call on each device before
 * any stream capture. Nothing in the array needs to start at zero: each call
 * writes every entry it later reads. Every call on a device shares the
 * array, so calls that overlap on the GPU race; order them on one stream or
 * synchronise between them. cumc_cfl_dt_static_error() describes the last
 * failure of the calling thread. */
#define CUMC_STATIC_MAX_CELLS (256 * 256 * 256)
int cumc_cfl_dt_static(int nx, int ny, int nz,
                       const double* rho, const double* vx, const double* vy,
                       const double* vz, const double* p,
                       const double* bcx, const double* bcy, const double* bcz,
                       const double* dx, const double* dy, const double* dz,
                       int coordinate, const double* xc, const double* sin_yc,
                       double ggas, double cfl, double* dt_out, void* stream);
const char* cumc_cfl_dt_static_error(void);

#ifdef __cplusplus
}
#endif
#endif /* CUMC_H */
