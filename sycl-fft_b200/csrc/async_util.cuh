// Shared-memory barrier, bulk-copy and proxy-fence helpers (inline PTX) used by the
// copy-engine-pipelined and tensor-core kernels. Every wait on an mbarrier in this
// project is a bounded poll of mbar_try_wait: at most the plan's wait limit (kSpinLimit
// polls by default), and kSpinLimit for the drain of a copy still in flight after a wait
// gave up.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace sfb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

constexpr long long kSpinLimit = 1ll << 26;

// Bounded wait for phase `parity` of `bar`: true once it completed, false after `polls`
// polls (0 polls gives up at once).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long polls) {
    for (long long spin = 0; spin < polls; ++spin)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Records a bounded wait that gave up in the plan's status word. The word lives in
// page-locked host memory mapped into the device, so this is a plain system-scope store
// (no atomic over the bus); the host reads it once the launch has completed.
__device__ __forceinline__ void report_status(int* status, int code) {
    if (!status) return;
    *reinterpret_cast<volatile int*>(status) = code;
    __threadfence_system();
}
}  // namespace sfb
