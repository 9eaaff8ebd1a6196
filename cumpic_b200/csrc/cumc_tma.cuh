// cumc_tma.cuh — bulk tensor copies (TMA) from global into shared memory for
// the sweep kernels, with mbarrier completion, for sm_100a.
//
// A copy is issued by one thread: cp.async.bulk.tensor of a box of a field
// (x fastest) into a shared-memory buffer, completing on an mbarrier that
// counts the bytes (arrive.expect_tx). Consumers wait on the barrier's phase
// with a bounded spin: if a copy never lands, the wait gives up after
// kSpinLimit polls, sets bit 1 of the kernel's error word and the kernel
// stops using the buffer, so a fault in the copy engine turns into an error
// status on the host instead of a hung GPU.
//
// Rules kept by every caller: the box's x start is a multiple of 2 doubles
// (16 bytes); tensor maps cover only this GPU's own memory; there is no
// multicast. Boxes that reach past the array are filled with zeros by the
// copy engine.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cumc {

constexpr unsigned kTmaTimeoutFlag = 2u;  // bit of the device error word: a staged copy never completed
constexpr long long kSpinLimit = 1LL << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the barrier initialisation visible to the copy engine
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// wait for phase `phase` of the barrier; false (and bit 1 of *err set) when
// the copy did not land within the spin limit
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, unsigned int* err) {
    for (long long it = 0; it < kSpinLimit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    atomicOr(err, kTmaTimeoutFlag);
    return false;
}

// 3-D box load of a tensor map at element coordinates (x, y, z) into dst,
// completing on bar
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace cumc
