/*
 * cumc_main.c — a C program that drives the library through its C-ABI with
 * the call sequence of the reference's main program (solver/main.f90:57-171),
 * the way a Fortran main.f90 calls it through an iso_c_binding module:
 *
 *   SETUP / GETGRID          the configuration and the face coordinates
 *                            (solver/main.f90:69-88, solver/coords.f90:24-32)
 *   GET_MODEL                the Brio-Wu shock tube along x
 *                            (model/riemann/src/riemann1d.f90:54-89)
 *   POPULATE_DEVICE          cumc_init + cumc_upload_state      (main.f90:98-100)
 *   initial_update           cumc_initial_update                (main.f90:105)
 *   DO WHILE (global_time < total_time)                         (main.f90:127-143)
 *     finddt; clip dt to total_time; RUNGEKUTTA; advance time
 *   find_divb                cumc_divb                          (main.f90:159,171)
 *   print_hydroprofile       cumc_download_state                (solver/dataio.f90:24)
 *
 * Usage: cumc_main NX NY NZ T_END OUT [advance]
 *   Brio-Wu along x on NX x NY x NZ cells (x in [0,1], the same cell size
 *   across, outflow along x and periodic across), gamma = 2, CFL 0.4, PPM/HLL,
 *   run to T_END with the host loop above (or, with "advance", the loop on the
 *   device: cumc_advance). OUT receives the final state as raw doubles: a
 *   header of 8 doubles (nx, ny, nz, steps, time, signed max div B, normalised
 *   max |div B|, 0) then prim (8 a cell), cons (8), eps (1) and bcell (3) in
 *   the reference's layout. Exit status 0 on success, 1 on a library error
 *   (its message on stderr), 2 on bad arguments.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/cumc.h"

#define CHECK(call)                                                                       \
    do {                                                                                  \
        int rc_ = (call);                                                                 \
        if (rc_ != CUMC_OK) {                                                             \
            fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, cumc_last_error(ctx));    \
            cumc_free(ctx);                                                               \
            return 1;                                                                     \
        }                                                                                 \
    } while (0)

/* GETGRID: x_F(j) = start + j (end - start)/n, j = -3..n+3 */
static void uniform_faces(double* f, double start, double end, int n) {
    const double d = (end - start) / (double)n;
    for (int j = -3; j <= n + 3; ++j) f[j + 3] = start + (double)j * d;
}

int main(int argc, char** argv) {
    if (argc < 6) {
        fprintf(stderr, "usage: %s NX NY NZ T_END OUT [advance]\n", argv[0]);
        return 2;
    }
    const int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]);
    const double total_time = atof(argv[4]);
    const char* out_path = argv[5];
    const int device_loop = argc > 6 && strcmp(argv[6], "advance") == 0;
    if (nx < 1 || ny < 1 || nz < 1 || !(total_time >= 0.0)) {
        fprintf(stderr, "bad arguments\n");
        return 2;
    }
    const double ggas = 2.0;
    cumc_ctx* ctx = NULL;

    /* SETUP and GETGRID: unit tube along x, the same cell size across */
    double* xf = malloc(sizeof(double) * (size_t)(nx + 7));
    double* yf = malloc(sizeof(double) * (size_t)(ny + 7));
    double* zf = malloc(sizeof(double) * (size_t)(nz + 7));
    const size_t nt = (size_t)(nx + 6) * (size_t)(ny + 6) * (size_t)(nz + 6);
    double* prim = calloc(8 * nt, sizeof(double));
    double* cons = calloc(8 * nt, sizeof(double));
    double* eps = calloc(nt, sizeof(double));
    double* bcell = calloc(3 * nt, sizeof(double));
    if (!xf || !yf || !zf || !prim || !cons || !eps || !bcell) {
        fprintf(stderr, "host allocation failed\n");
        return 1;
    }
    const double cell = 1.0 / (double)nx;
    uniform_faces(xf, 0.0, 1.0, nx);
    uniform_faces(yf, 0.0, ny * cell, ny);
    uniform_faces(zf, 0.0, nz * cell, nz);

    /* GET_MODEL: the Brio-Wu states split at x = 0.5 on cells 0:n (the
     * cell-centre test of riemann1d.f90), face Bx = 0.75, By = +-1 */
    for (int l = 0; l <= nz; ++l)
        for (int k = 0; k <= ny; ++k)
            for (int j = 0; j <= nx; ++j) {
                const size_t i = (size_t)(j + 2) + (size_t)(nx + 6) * ((size_t)(k + 2) + (size_t)(ny + 6) * (size_t)(l + 2));
                const double x = 0.5 * (xf[j + 3] + xf[j + 2]);
                const int left = x <= 0.5;
                const double rho = left ? 1.0 : 0.125, p = left ? 1.0 : 0.1;
                double* w = prim + 8 * i;
                w[0] = rho;
                w[4] = p;
                w[5] = 0.75;
                w[6] = left ? 1.0 : -1.0;
                eps[i] = p / rho / (ggas - 1.0);
            }

    /* POPULATE_DEVICE */
    cumc_config cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.nx = nx;
    cfg.ny = ny;
    cfg.nz = nz;
    cfg.xf = xf;
    cfg.yf = yf;
    cfg.zf = zf;
    cfg.coordinate = CUMC_CARTESIAN;
    cfg.boundary_flag[0] = 1;
    cfg.boundary_flag[1] = 1;
    cfg.ggas = ggas;
    cfg.cfl = 0.4;
    cfg.recon = CUMC_PPMC;
    cfg.solver = CUMC_HLL;
    cfg.precision = CUMC_FP64;
    cfg.model = CUMC_MODEL_RIEMANN;
    cfg.geom_source_repeat = 8;
    CHECK(cumc_init(&cfg, &ctx));
    CHECK(cumc_upload_state(ctx, prim, eps));
    CHECK(cumc_initial_update(ctx));

    /* the main loop */
    double global_time = 0.0;
    int n_step = 0;
    if (device_loop) {
        CHECK(cumc_advance(ctx, 1000000000, total_time, &global_time, &n_step));
    } else {
        while (global_time < total_time) {
            double dt;
            CHECK(cumc_finddt(ctx, &dt));
            if (global_time + dt > total_time) dt = total_time - global_time;
            CHECK(cumc_rungekutta(ctx, dt));
            global_time = global_time + dt;
            n_step = n_step + 1;
        }
    }
    double divb_signed = 0.0, divb_norm = 0.0;
    CHECK(cumc_divb(ctx, &divb_signed, &divb_norm));
    CHECK(cumc_download_state(ctx, prim, cons, eps, bcell));
    CHECK(cumc_free(ctx));
    ctx = NULL;
    printf("Brio-Wu %dx%dx%d: %d steps to t = %.17g, max div B %.3e (normalised %.3e)\n", nx, ny, nz, n_step,
           global_time, divb_signed, divb_norm);

    FILE* f = fopen(out_path, "wb");
    if (!f) {
        fprintf(stderr, "cannot open %s\n", out_path);
        return 1;
    }
    const double head[8] = {nx, ny, nz, n_step, global_time, divb_signed, divb_norm, 0.0};
    int ok = fwrite(head, sizeof(double), 8, f) == 8;
    ok = ok && fwrite(prim, sizeof(double), 8 * nt, f) == 8 * nt;
    ok = ok && fwrite(cons, sizeof(double), 8 * nt, f) == 8 * nt;
    ok = ok && fwrite(eps, sizeof(double), nt, f) == nt;
    ok = ok && fwrite(bcell, sizeof(double), 3 * nt, f) == 3 * nt;
    ok = fclose(f) == 0 && ok;
    free(xf);
    free(yf);
    free(zf);
    free(prim);
    free(cons);
    free(eps);
    free(bcell);
    if (!ok) {
        fprintf(stderr, "writing %s failed\n", out_path);
        return 1;
    }
    return 0;
}
