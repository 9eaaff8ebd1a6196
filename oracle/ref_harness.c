/* ref_harness.c — TEST INFRASTRUCTURE: drives the mechanical C translation
 * of the reference's own Fortran sources (generated by oracle/f2c_ref.py into
 * oracle/_ref/) with the same orc_* entry points as the hand-written oracle,
 * so the two can be compared on identical inputs.
 *
 * The call sequence follows solver/main.f90:57-143 without MPI: SETUP_EQNS,
 * starts/stops (:69-74), BUILD_HYDRO (solver/setup.f90:249), the face
 * coordinates (GETGRID or CUSTOM_GRID; supplied by the caller), the initial
 * model (GET_MODEL; supplied by the caller), initial_update, then finddt and
 * RUNGEKUTTA. The translated code keeps the reference's module globals, so
 * one process holds one configuration at a time.
 */
#include REF_TRANSLATION
#include "../include/cumc.h"

static size_t g_nt = 0;
static int g_live = 0;

void* orc_create(const cumc_config* c, char* err, int errlen) {
    f2c_novr = 0;
    f2c_set_override("nxtot", 0, c->nx);
    f2c_set_override("nytot", 0, c->ny);
    f2c_set_override("nztot", 0, c->nz);
    f2c_set_override("coordinate", 0, c->coordinate);
    for (int i = 0; i < 6; ++i) f2c_set_override("boundary_flag", i, c->boundary_flag[i]);
    f2c_set_override("cfl", 0, c->cfl);
    f2c_set_override("recon", 0, c->recon);
    f2c_set_override("solver", 0, c->solver);
    f2c_set_override("ggas", 0, c->ggas);
#ifdef REF_MODEL_TORUS
    f2c_set_override("r_sh", 0, c->r_sh);
#endif
    if (c->geom_source_repeat != 8 && c->coordinate != CUMC_CARTESIAN) {
        snprintf(err, errlen, "the reference applies the geometric source 8 times; other repeats are not available");
        return NULL;
    }
    f2c_init_params();
    fs_setup_eqns();
    for (int i = 0; i < 3; ++i) f_starts.d[i] = 0;
    f_stops.d[0] = f_nx;
    f_stops.d[1] = f_ny;
    f_stops.d[2] = f_nz;
    fs_build_hydro();
    for (int i = 0; i < f_nx + 7; ++i) f_xf.d[i] = c->xf[i];
    for (int i = 0; i < f_ny + 7; ++i) f_yf.d[i] = c->yf[i];
    for (int i = 0; i < f_nz + 7; ++i) f_zf.d[i] = c->zf[i];
#ifdef REF_MODEL_TORUS
    f_rho_floor = c->rho_floor;
    f_eps_floor = c->eps_floor;
#endif
    g_nt = (size_t)(f_nx + 6) * (size_t)(f_ny + 6) * (size_t)(f_nz + 6);
    g_live = 1;
    (void)errlen;
    return &g_live;
}

void orc_free(void* h) { (void)h; g_live = 0; }
void orc_set_threads(int n) { (void)n; }
int orc_get_threads(void) { return 1; }

int orc_upload(void* h, const double* prim, const double* eps) {
    (void)h;
    memcpy(f_prim.d, prim, sizeof(double) * 8 * g_nt);
    memcpy(f_eps.d, eps, sizeof(double) * g_nt);
    return 0;
}
int orc_initial_update(void* h) { (void)h; fs_initial_update(); return 0; }
int orc_finddt(void* h, double* dt) { (void)h; fs_finddt(); *dt = f_dt; return 0; }
int orc_rungekutta(void* h, double dt) { (void)h; f_dt = dt; fs_rungekutta(); return 0; }
int orc_spatial(void* h) { (void)h; fs_spatial(); return 0; }
int orc_divb(void* h, double* maxdb) { (void)h; *maxdb = 0.0; return 1; }
int orc_download(void* h, double* prim, double* cons, double* eps, double* bcell, double* lrk) {
    (void)h;
    if (prim) memcpy(prim, f_prim.d, sizeof(double) * 8 * g_nt);
    if (cons) memcpy(cons, f_cons.d, sizeof(double) * 8 * g_nt);
    if (eps) memcpy(eps, f_eps.d, sizeof(double) * g_nt);
    if (bcell) memcpy(bcell, f_bcell.d, sizeof(double) * 3 * g_nt);
    if (lrk) memcpy(lrk, f_l_rk.d, sizeof(double) * 8 * g_nt);
    return 0;
}
