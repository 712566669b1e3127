// Tensor-memory-accelerator (TMA) bulk copies of mesh boxes into shared memory.
//
// One thread issues `cp.async.bulk.tensor.3d` for a whole box and arms an mbarrier
// with the box's byte count; every thread of the CTA waits on the barrier's phase.
// The copies read this GPU's own memory only and use no cluster multicast.
// Waits are bounded (about one second of SM clock); a wait that runs out reports it
// to the caller, which sets the device error word instead of spinning forever.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace djb {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return unsigned(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the asynchronous proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses (made visible to
// it by a CTA barrier) before its subsequent asynchronous-proxy writes.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Box at global element coordinates (x, y, z) of `map` into shared memory at `dst`
// (16-byte aligned); completion is signalled on `bar` as transaction bytes.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Waits for the barrier phase with the given parity; false when about 2^31 SM clock
// cycles (about a second) pass without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const long long t0 = clock64();
    for (unsigned it = 0;; ++it) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((it & 255u) == 255u && clock64() - t0 > (1LL << 31)) return false;
    }
}

}  // namespace djb
