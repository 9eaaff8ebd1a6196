// cumc_mixed.h — host interface of the mixed-precision path (cumc_mixed.cu).
//
// State of the mixed form, per cell:
//   U^n  : rho, rho v, B as hi/lo FP32 pairs (compensated), total energy FP64
//   d_s  : stage increment U_s - U^n as FP32 for rho, rho v; FP64 for B (the
//          CT curl of the FP32 EMFs is formed in FP64 so that the face-field
//          update keeps div B at round-off); stage energy FP64
//   prims: rho, v, p, bcell and the current face field as FP32 (with ghosts)
// Reconstruction, HLL and EMFs run in FP32; the pressure recovery
// E - rho v^2/2 - B^2/2 and the energy combine run in FP64.
#pragma once
#include <cuda_runtime.h>

#include "cumc_device.cuh"

namespace cumc {

struct MixedBufs {
    float* uh[8];   // U^n high parts (index 4 unused: energy is e0)
    float* ul[8];   // U^n low parts
    double* e0;     // U^n total energy
    float* d[8];    // stage increment of rho, rho v (indices 0-3; 4-7 unused)
    double* db[3];  // stage increment of the face fields (FP64: keeps the CT
                    // update divergence-free to round-off)
    double* es;     // stage total energy
    float* w[5];    // rho, vx, vy, vz, p
    float* bc[3];   // bcell
    float* bf[3];   // current face field
    float* F[3][7]; // face fluxes per direction
    float* E[3];    // edge EMFs
    const double* dt;
    unsigned int* flag;
};

struct MixedParams {
    double ggas, cfl, rho_floor, eps_floor, r_sh;
    int flag[6];
    int eps_yout;
    signed char fac[6][8];
    int model, coord, recon, geom_repeat;
    int sm_count;  // multiprocessors of the device (grid sizing)
    int fused = 1; // the stage's tiled EMF + CT and fused combine + conversion kernels
                   // (0: k_emf, k_combine_mx, k_utop_mx)
    int hll_fp32 = 0;  // the HLL solve all in FP32 (reciprocal form) instead of
                       // the hydro components in FP64 (hll_flux7_mixed)
};

// How the mixed kernels are launched: the caller's stream, and hooks that
// record per-kernel timing and count launches.
struct Launcher {
    cudaStream_t stream;
    void (*pre)(void* user, int cls);
    void (*post)(void* user, int cls);
    void* user;
};

cudaError_t mixed_attributes();
// stage 3 with dtmin non-null also forms the next step's CFL dt (atomicMin
// into dtmin, which the caller has reset)
void mixed_stage(const Launcher& L, const Box& b, const Tabs& T, const MixedBufs& m, const MixedParams& p, int stage,
                 unsigned long long* dtmin = nullptr);
void mixed_initial(const Launcher& L, const Box& b, const Tabs& T, const MixedBufs& m, const MixedParams& p,
                   const double* prim_aos, const double* eps_aos);
void mixed_finddt(const Launcher& L, const Box& b, const Tabs& T, const MixedBufs& m, const MixedParams& p,
                  unsigned long long* dtmin);
// what: 0 prim (8 fields), 1 cons (8), 2 eps (1), 3 bcell (3) as AoS doubles;
//       4 the three face fields as SoA doubles (3 arrays of the box size)
void mixed_export(const Launcher& L, const Box& b, const MixedBufs& m, const MixedParams& p, int what, double* aos);

}  // namespace cumc
