// 3³ periodic convolution as an implicit GEMM on the fifth-generation tensor cores
// (tcgen05.mma, accumulator in tensor memory), for the force-correction network.
//
// Output tile: 8 (x) × 16 (y) voxels of one z plane = the 128 rows of one M = 128 MMA.
// A CTA walks a column of such tiles along z. Its input planes are staged in shared
// memory with a one-voxel halo (10 × 18 positions per plane, periodic wrap), as
// [plane slot][8-channel chunk][position][8 channels]: in every chunk the 16-byte rows
// of consecutive positions are contiguous. That is the no-swizzle K-major operand
// layout with 8-row groups 160 bytes apart (one staged y row), so the A operand of a
// tap (dx, dy, dz) is the same staged block read from a start address shifted by
// (dy·10 + dx) rows: the 27 taps need no copies (no im2col).
// Per tile: 27 taps × (K / 16) MMAs of 128 × N × 16 (bf16 operands, float32
// accumulation), committed to an mbarrier. Two accumulators in tensor memory let the
// epilogue of one tile (tcgen05.ld → bias, ReLU → bf16 rows) run while the MMAs of the
// next are in flight; the next plane is copied in (cp.async) at the same time.
// The weights of the layer, [tap][chunk][n][8] (K-major B operand), stay in shared
// memory for the CTA's whole run.
// Waits are bounded: a wait that runs out sets the error word, and the CTA drains its
// copies, frees its tensor memory and returns.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "tma.cuh"

namespace djb {
namespace conv {

constexpr int kTX = 8, kTY = 16;                       // tile: 8 × 16 voxels = 128 MMA rows
constexpr int kBX = kTX + 2, kBY = kTY + 2;            // staged plane with its halo
constexpr int kPlane = kBX * kBY;                      // 180 positions
constexpr int kRing = 4;                               // planes z−1, z, z+1 and the next
constexpr int kThreads = 128;                          // four warps: tensor-memory lanes 0-127

struct Args {
    const __nv_bfloat16* X;   // [nvox][cin] input activations (cin = 8·CC)
    const __nv_bfloat16* W;   // [27][cin][cout] weights (tap = kz·9 + ky·3 + kx)
    const float* bias;        // [cout]
    __nv_bfloat16* Y;         // hidden layers: [nvox][cout] bf16, relu(acc + bias)
    float* Yf;                // last layer: [nout][nvox] float32, acc + bias
    int res, cin, cout, nout;
    int ntx, nty, nzs, zlen;  // tiles along x, y; z segments of zlen planes
    int* err;                 // set to 1 when a wait runs out
};

template <int KC, int N>
constexpr int smem_bytes() {
    return 27 * KC * N * 16 + kRing * KC * kPlane * 16 + 32;
}

// Shared-memory matrix descriptor, no swizzle: start, leading (K-chunk) and stride
// (8-row group) byte offsets in 16-byte units, descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: bf16 A and B (K-major), float32 D, M = 128.
template <int N>
__device__ __forceinline__ uint32_t idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(dtmem),
        "l"(a), "l"(b), "r"(id), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive float32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* f) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) f[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ int wrap(int v, int res) {
    v %= res;
    return v < 0 ? v + res : v;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Copies input plane z (any integer, wrapped) of the tile column at (x0, y0) into `slot`.
template <int CC, int KC>
__device__ __forceinline__ void stage_plane(const Args& a, uint32_t ring, int slot, int z, int x0, int y0) {
    const int gz = wrap(z, a.res);
    for (int e = threadIdx.x; e < CC * kPlane; e += kThreads) {
        const int pos = e / CC, kc = e - pos * CC;
        const int by = pos / kBX, bx = pos - by * kBX;
        const int gy = wrap(y0 - 1 + by, a.res), gx = wrap(x0 - 1 + bx, a.res);
        const __nv_bfloat16* src = a.X + ((int64_t(gz) * a.res + gy) * a.res + gx) * (CC * 8) + kc * 8;
        cp_async16(ring + uint32_t(((slot * KC + kc) * kPlane + pos) * 16), src);
    }
}

template <int CC, int N, bool LAST>
__global__ void __launch_bounds__(kThreads, 2) k_conv3_tc(Args a) {
    constexpr int KC = (CC + 1) / 2 * 2;          // K chunks staged (K a multiple of 16)
    constexpr uint32_t kCols = N * 2 < 32 ? 32 : N * 2;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* ws = smem;
    uint8_t* ringp = smem + 27 * KC * N * 16;
    uint64_t* bar = reinterpret_cast<uint64_t*>(ringp + kRing * KC * kPlane * 16);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t ws_u = smem_u32(ws), ring = smem_u32(ringp);

    // weights → [tap][chunk][n][8 k], zeros beyond cin and cout
    for (int i = tid; i < 27 * KC * N; i += kThreads) {
        const int n = i % N, kc = (i / N) % KC, tap = i / (N * KC);
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float f[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int k = kc * 8 + 2 * j + u;
                f[u] = (k < a.cin && n < a.cout) ? __bfloat162float(a.W[(int64_t(tap) * a.cin + k) * a.cout + n]) : 0.0f;
            }
            w[j] = pack_bf16(f[0], f[1]);
        }
        *reinterpret_cast<uint4*>(ws + size_t(i) * 16) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    // K-padding chunks of every slot are zero for good
    if constexpr (KC > CC) {
        for (int i = tid; i < kRing * (KC - CC) * kPlane; i += kThreads) {
            const int pos = i % kPlane, r = i / kPlane, kc = CC + r % (KC - CC), slot = r / (KC - CC);
            *reinterpret_cast<uint4*>(ringp + size_t((slot * KC + kc) * kPlane + pos) * 16) = make_uint4(0, 0, 0, 0);
        }
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_proxy_async_smem();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t lane_base = uint32_t(warp * 32) << 16;
    const uint32_t id = idesc<N>();
    const int64_t nvox = int64_t(a.res) * a.res * a.res;

    uint32_t ph[2] = {0u, 0u};
    int t = 0;        // tiles committed by this CTA; accumulator t & 1
    bool ok = true;

    auto epilogue = [&](int x0, int y0, int z, int buf) {
        float f[N];
#pragma unroll
        for (int q = 0; q < N / 16; ++q) tmem_ld16(tmem + lane_base + uint32_t(buf * N + q * 16), f + q * 16);
        const int x = x0 + (tid & 7), y = y0 + (tid >> 3);
        if (x >= a.res || y >= a.res) return;
        const int64_t v = (int64_t(z) * a.res + y) * a.res + x;
        if constexpr (LAST) {
#pragma unroll
            for (int c = 0; c < N; ++c)
                if (c < a.nout) a.Yf[int64_t(c) * nvox + v] = f[c] + __ldg(a.bias + c);
        } else {
            uint4* dst = reinterpret_cast<uint4*>(a.Y + v * a.cout);
#pragma unroll
            for (int c8 = 0; c8 < N / 8; ++c8) {
                if (c8 * 8 >= a.cout) break;
                uint32_t w[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = c8 * 8 + 2 * j;
                    w[j] = pack_bf16(fmaxf(f[c] + __ldg(a.bias + c), 0.0f), fmaxf(f[c + 1] + __ldg(a.bias + c + 1), 0.0f));
                }
                dst[c8] = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
    };

    const int items = a.ntx * a.nty * a.nzs;
    for (int item = blockIdx.x; item < items && ok; item += gridDim.x) {
        const int tx = item % a.ntx, rr = item / a.ntx, ty = rr % a.nty, zs = rr / a.nty;
        const int x0 = tx * kTX, y0 = ty * kTY, z0 = zs * a.zlen;
        const int nt = min(a.zlen, a.res - z0);
        // planes z0 − 1 + j live in slot j % kRing; tile i reads j = i, i + 1, i + 2
        stage_plane<CC, KC>(a, ring, 0, z0 - 1, x0, y0);
        stage_plane<CC, KC>(a, ring, 1, z0, x0, y0);
        stage_plane<CC, KC>(a, ring, 2, z0 + 1, x0, y0);
        cp_async_commit();
        for (int i = 0; i < nt; ++i) {
            cp_async_wait_all();       // plane i + 2 (the newest group)
            fence_proxy_async_smem();  // the copies are read by the tensor cores
            tc_before_sync();
            __syncthreads();
            tc_after_sync();
            const int buf = t & 1;
            if (tid == 0) {
                const uint32_t d = tmem + uint32_t(buf * N);
#pragma unroll 1
                for (int dz = 0; dz < 3; ++dz) {
                    const uint32_t plane = ring + uint32_t(((i + dz) % kRing) * KC * kPlane * 16);
#pragma unroll
                    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                        for (int dx = 0; dx < 3; ++dx) {
                            const int tap = dz * 9 + dy * 3 + dx;
                            const uint32_t a0 = plane + uint32_t((dy * kBX + dx) * 16);
                            const uint32_t b0 = ws_u + uint32_t(tap * KC * N * 16);
#pragma unroll
                            for (int s = 0; s < KC / 2; ++s)
                                mma_bf16(d, sdesc(a0 + uint32_t(2 * s * kPlane * 16), kPlane * 16, kBX * 16),
                                         sdesc(b0 + uint32_t(2 * s * N * 16), N * 16, 128), id,
                                         (tap | s) != 0 ? 1u : 0u);
                        }
                }
                mma_commit(&bar[buf]);
            }
            if (i > 0) {
                const bool w = mbar_wait(&bar[buf ^ 1], ph[buf ^ 1]);
                ph[buf ^ 1] ^= 1u;
                if (!__syncthreads_and(w)) {
                    ok = false;
                    ++t;
                    break;
                }
                tc_after_sync();
            }
            // plane i + 3 into the slot of plane i − 1 (its last reader, tile i − 1, is done)
            if (i + 3 <= nt + 1) stage_plane<CC, KC>(a, ring, (i + 3) % kRing, z0 + i + 2, x0, y0);
            cp_async_commit();
            if (i > 0) epilogue(x0, y0, z0 + i - 1, buf ^ 1);
            ++t;
        }
        if (!ok) break;
        // the column's last tile
        const int lb = (t - 1) & 1;
        const bool w = mbar_wait(&bar[lb], ph[lb]);
        ph[lb] ^= 1u;
        if (!__syncthreads_and(w)) {
            ok = false;
            break;
        }
        tc_after_sync();
        epilogue(x0, y0, z0 + nt - 1, lb);
        tc_before_sync();
        __syncthreads();   // slots and accumulators are free for the next column
    }
    cp_async_wait_all();
    if (!ok) {
        if (tid == 0) atomicExch(a.err, 1);
        // let the MMAs this CTA committed finish before the tensor memory is released
        for (int b = 0; b < 2; ++b) mbar_wait(&bar[b], ph[b]);
    }
    tc_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

}  // namespace conv
}  // namespace djb
