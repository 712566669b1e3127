// Tensor-memory-accelerator (TMA) bulk copies between mesh boxes and shared memory.
//
// Loads: one thread issues `cp.async.bulk.tensor.3d` for a whole box and arms an
// mbarrier with the box's byte count; every thread of the CTA waits on the barrier's
// phase. Reductions: one thread issues `cp.reduce.async.bulk.tensor.3d ... .add` of a
// whole box and waits for its source reads (bulk group). The copies touch this GPU's
// own memory only and use no cluster multicast.
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

// Element-wise float add of the shared-memory box at `src` (16-byte aligned, laid out
// as the map's box) into global memory at box coordinates (x, y, z) of `map`; the
// coordinates are non-negative and the box lies inside the tensor.
__device__ __forceinline__ void tma_reduce_add_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
        : "memory");
}

// Commits this thread's bulk operations and waits until their shared-memory sources
// have been read (the shared memory may then be overwritten or released).
__device__ __forceinline__ void bulk_commit_and_wait_read() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Vector float reduction of four consecutive floats at a 16-byte aligned address.
__device__ __forceinline__ void red_add_v4(float* dst, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(dst), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

// Waits for the barrier phase with the given parity; false when `limit` SM clock cycles
// pass without completion (by default 2^31, about a second).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long limit = (1LL << 31)) {
    const long long t0 = clock64();
    for (unsigned it = 0;; ++it) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((it & 255u) == 255u && clock64() - t0 > limit) return false;
    }
}

}  // namespace djb
