// cumc_static.cu — CFL time step over caller-owned device arrays, with no
// memory allocation at all (cumc_cfl_dt_static in include/cumc.h).
//
// Why it exists: some callers cannot allocate device memory at the moment
// they need a time step. A code that records its time loop into a CUDA graph
// cannot call cudaMalloc while the stream is being captured; a host program
// whose device memory belongs to another runtime (an OpenACC data region, a
// framework's caching allocator, a pre-sized pool in a long-running service)
// must not take memory behind that runtime's back. This entry point works on
// the arrays the caller already has and keeps its only scratch, the
// per-block partial minima of the reduction, in a fixed file-scope device
// array that exists as soon as the library is loaded.
//
// The per-cell formula is the one of finddt (solver/rungekutta.f90:213-247):
// cfl_cell_dt and cfl_lengths of cumc_device.cuh, the functions the library's
// own finddt kernel calls, so both give the same double.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/cumc.h"
#include "cumc_device.cuh"

namespace {

constexpr int kThreads = 256;
// One partial minimum per block of 256 cells: at most CUMC_STATIC_MAX_CELLS
// active cells (256^3) per call.
constexpr int kMaxBlocks = CUMC_STATIC_MAX_CELLS / kThreads;

// Scratch shared by every call on a device (65536 doubles, 512 KiB per
// device, held until the process exits). No entry needs to start at zero: k_cfl_partial writes
// partial[0..nblocks) before k_cfl_final reads exactly those entries, on the
// same stream. Two calls that overlap on the GPU (different streams, no
// ordering) race on it. Host code must not take this symbol's address
// directly: on the host it names a stand-in, not device memory.
static __device__ __align__(256) double g_cfl_partial[kMaxBlocks];

constexpr int kMaxDevices = 64;
double* g_partial_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

__global__ void __launch_bounds__(kThreads) k_cfl_partial(int nx, int ny, int nz, const double* rho, const double* vx,
                                                        const double* vy, const double* vz, const double* p,
                                                        const double* bcx, const double* bcy, const double* bcz,
                                                        const double* dxw, const double* dyw, const double* dzw,
                                                        int coordinate, const double* xc, const double* sinyc,
                                                        double ggas, double cfl, double* partial) {
    const int SX = nx + 6, SY = ny + 6;
    const long long total = (long long)nx * ny * nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dt_out = 1.0e10;
    if (t < total) {
        const int j = (int)(t % nx) + 1;
        const int k = (int)((t / nx) % ny) + 1;
        const int l = (int)(t / ((long long)nx * ny)) + 1;
        const int i = (j + 2) + SX * ((k + 2) + SY * (l + 2));
        double dyl = dyw[k + 3], dzl = dzw[l + 3];
        if (coordinate != CUMC_CARTESIAN)
            cumc::cfl_lengths(coordinate, xc[j + 3], coordinate == CUMC_SPHERICAL ? sinyc[k + 3] : 0.0, dyl, dzl);
        dt_out = cumc::cfl_cell_dt(rho[i], p[i], vx[i], vy[i], vz[i], bcx[i], bcy[i], bcz[i], dxw[j + 3], dyl, dzl,
                                   ggas, cfl);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dt_out = fmin(dt_out, __shfl_xor_sync(0xffffffffu, dt_out, o));
    __shared__ double red[kThreads / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dt_out;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = red[0];
        for (int w = 1; w < kThreads / 32; ++w) v = fmin(v, red[w]);
        partial[blockIdx.x] = v;
    }
}

__global__ void __launch_bounds__(1024) k_cfl_final(const double* partial, int nblocks, double* dt_out) {
    double v = 1.0e10;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v = fmin(v, partial[b]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmin(m, red[w]);
        *dt_out = m;
    }
}

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached.
cudaError_t partial_address(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partial_ptr[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_cfl_partial);
        if (e != cudaSuccess) return e;
        g_partial_ptr[dev] = p;
    }
    *out = g_partial_ptr[dev];
    return cudaSuccess;
}

thread_local char g_static_error[256];

int fail(int code, const char* msg) {
    snprintf(g_static_error, sizeof g_static_error, "%s", msg);
    return code;
}

}  // namespace

extern "C" {

int cumc_cfl_dt_static(int nx, int ny, int nz, const double* rho, const double* vx, const double* vy,
                       const double* vz, const double* p, const double* bcx, const double* bcy, const double* bcz,
                       const double* dx, const double* dy, const double* dz, int coordinate, const double* xc,
                       const double* sin_yc, double ggas, double cfl, double* dt_out, void* stream) {
    g_static_error[0] = '\0';
    // an error left pending by earlier, unrelated work belongs to its caller:
    // report it without clearing it, and launch nothing
    cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        snprintf(g_static_error, sizeof g_static_error, "a CUDA error from earlier work is pending (left uncleared): %s",
                 cudaGetErrorString(pending));
        return CUMC_ERR_CUDA;
    }
    if (nx < 1 || ny < 1 || nz < 1) return fail(CUMC_ERR_ARG, "cell counts must be positive");
    const long long cells = (long long)nx * ny * nz;
    if (cells > CUMC_STATIC_MAX_CELLS)
        return fail(CUMC_ERR_LIMIT, "cumc_cfl_dt_static handles at most CUMC_STATIC_MAX_CELLS (256^3) active cells");
    if (!rho || !vx || !vy || !vz || !p || !bcx || !bcy || !bcz || !dx || !dy || !dz || !dt_out)
        return fail(CUMC_ERR_ARG, "null array");
    if (coordinate != CUMC_CARTESIAN && coordinate != CUMC_CYLINDRICAL && coordinate != CUMC_SPHERICAL)
        return fail(CUMC_ERR_ARG, "coordinate must be CUMC_CARTESIAN, CUMC_CYLINDRICAL or CUMC_SPHERICAL");
    if (coordinate != CUMC_CARTESIAN && (!xc || (coordinate == CUMC_SPHERICAL && !sin_yc)))
        return fail(CUMC_ERR_ARG, "curvilinear grids need the cell-centre radius (and sin of the polar centre)");
    double* partial = nullptr;
    cudaError_t e = partial_address(&partial);
    if (e != cudaSuccess) return fail(CUMC_ERR_CUDA, cudaGetErrorString(e));
    const int nblocks = (int)((cells + kThreads - 1) / kThreads);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_cfl_partial<<<nblocks, kThreads, 0, s>>>(nx, ny, nz, rho, vx, vy, vz, p, bcx, bcy, bcz, dx, dy, dz, coordinate,
                                              xc, sin_yc, ggas, cfl, partial);
    k_cfl_final<<<1, 1024, 0, s>>>(partial, nblocks, dt_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CUMC_ERR_CUDA, cudaGetErrorString(e));
    return CUMC_OK;
}

const char* cumc_cfl_dt_static_error(void) { return g_static_error; }

}  // extern "C"
