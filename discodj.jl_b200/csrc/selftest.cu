// Self-test of the bounded waits that every bulk-copy kernel of the library uses.
//
// k_wait_selftest waits, with the same mbar_wait, on an mbarrier of its own: with
// `arrive` set, the CTA's threads arrive first and the wait completes; without it,
// nothing ever arrives, the wait gives up after `limit` SM cycles, and the kernel sets
// bit 8 of the error word (as the brick and z-pass kernels do) and returns. No copy is
// in flight in either case, so the kernel ends normally and the context stays usable.
#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"
#include "tma.cuh"

namespace {

__global__ void k_wait_selftest(int arrive, long long limit, int* err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) djb::mbar_init(&bar, blockDim.x);
    __syncthreads();
    if (arrive) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(djb::smem_u32(&bar)) : "memory");
    const bool ok = djb::mbar_wait(&bar, 0, limit);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(err, 8);
}

}  // namespace

extern "C" int djb_selftest_bounded_wait(int32_t device, int32_t arrive, int64_t limit_cycles, int32_t* err_word) {
    djb::clear_error();
    if (!err_word) return djb::fail(DJB_ERR_INVALID, "null argument");
    if (limit_cycles < 0 || limit_cycles > (int64_t(1) << 31))
        return djb::fail(DJB_ERR_INVALID, "limit_cycles must be in [0, 2^31]");
    int prev = -1;
    cudaGetDevice(&prev);
    int rc = DJB_OK;
    int* d_err = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d_err), sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d_err, 0, sizeof(int));
    if (e == cudaSuccess) {
        k_wait_selftest<<<1, 64>>>(arrive ? 1 : 0, static_cast<long long>(limit_cycles), d_err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(err_word, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = djb::fail(DJB_ERR_CUDA, "bounded-wait self-test failed: %s", cudaGetErrorString(e));
    if (d_err) cudaFree(d_err);
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}
