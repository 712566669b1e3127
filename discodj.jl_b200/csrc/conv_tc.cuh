// 3³ periodic convolution as an implicit GEMM on the fifth-generation tensor cores
// (tcgen05.mma, accumulator in tensor memory), for the force-correction network.
//
// Output tile: 8 (x) × 16 (y) voxels of one z plane = the 128 rows of one M = 128 MMA.
// A CTA walks columns of such tiles along z, in segments of up to kMaxSegment tiles.
// Its input planes are staged in shared memory with a one-voxel halo (10 × 18
// positions per plane, periodic wrap), as [plane slot][8-channel chunk][position][8
// channels]: in every chunk the 16-byte rows of consecutive positions are contiguous.
// That is the no-swizzle K-major operand layout with 8-row groups 160 bytes apart (one
// staged y row), so the A operand of a tap (dx, dy) is the staged plane read from a
// start address shifted by (dy·10 + dx) rows: the taps need no copies (no im2col).
// A staged plane is the kz = 0, 1, 2 input of the tiles z + 1, z, z − 1, whose
// accumulators are adjacent in tensor memory: one MMA of N = 3 × (output channels) per
// (dy, dx, K step) serves all three, so each plane is read once per shift.
// Warp roles (persistent CTAs, producer/consumer mbarriers):
//   loader (warp 8): planes into a ring of kRing slots (128-byte aligned), one bulk
//     tensor copy per plane (5-D map over [z][chunk][y][x][8 channels]) where the halo
//     does not wrap, else 16-byte cp.async with the periodic wrap; completion on the
//     slot's `full` barrier.
//   MMA (warp 9, converged; one elected lane issues): per plane, tcgen05.mma of
//     128 × N·(tiles it feeds) × 16 (bf16 operands, float32 accumulation) per
//     (dy, dx, K step); commits to the `empty` barrier of the plane and to the `accf`
//     barrier of the tile the plane completes.
//   epilogue (warps 0-7, two groups of four on alternate tiles; warp w reads tensor-
//     memory lanes 32·(w % 4) .. +31): tcgen05.ld of the accumulator, `acce` arrive,
//     then bias + ReLU → bf16 rows (hidden layers), bias → float32 channel-major mesh
//     (last layer), or the ReLU mask of the layer below → bf16 (data gradient: the
//     convolution with the flipped, transposed weights). bf16 tiles leave by one bulk
//     tensor store each from double-buffered shared-memory staging.
// The weights of the layer, [dy·3 + dx][chunk][kz·N + n][8] (K-major B operand), stay
// in shared memory for the CTA's whole run. The x-pair form of the first layer and the
// weight-gradient kernel are described where they are defined below.
// Waits are bounded: a wait that runs out sets the error word and the CTA's abort
// flag; every role then stops, the MMAs and copies in flight are waited for (bounded),
// and the tensor memory is freed.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

#include "tma.cuh"

namespace djb {
namespace conv {

constexpr int kTX = 8, kTY = 16;                       // tile: 8 × 16 voxels = 128 MMA rows
constexpr int kBX = kTX + 2, kBY = kTY + 2;            // staged plane with its halo
constexpr int kPlane = kBX * kBY;                      // 180 positions
#ifndef DJB_CONV_RING
#define DJB_CONV_RING 8
#endif
#ifndef DJB_CONV_CTAS
#define DJB_CONV_CTAS 1
#endif
constexpr int kRing = DJB_CONV_RING;                   // staged planes
constexpr int kAccTiles = 16;                          // tile accumulators in tensor memory
constexpr int kMaxSegment = kAccTiles;                 // z segment length (tiles) at most
constexpr int kOneCtaSmem = 116 * 1024;                // more than half an SM: one CTA per SM
#ifndef DJB_CONV_EPI
#define DJB_CONV_EPI 2
#endif
constexpr int kEpiGroups = DJB_CONV_EPI;               // epilogue groups of four warps, alternate tiles
#ifndef DJB_CONV_OSTAGES
#define DJB_CONV_OSTAGES 4
#endif
constexpr int kOutStages = DJB_CONV_OSTAGES;           // output staging buffers per epilogue group
constexpr int kLoaderWarp = 4 * kEpiGroups, kMmaWarp = kLoaderWarp + 1;
constexpr int kThreads = 32 * (kMmaWarp + 1);

enum Mode { kHidden = 0, kLast = 1, kBackData = 2 };

struct Args {
    const __nv_bfloat16* X;   // [nvox][cin] input (cin = 8·CC)
    const __nv_bfloat16* W;   // flip = 0: [27][cin][cout]; flip = 1: [27][cout][cin] of the forward layer
    const float* bias;        // [cout] (kHidden, kLast)
    const __nv_bfloat16* M;   // kBackData: [nvox][cout], output kept where M > 0
    __nv_bfloat16* Y;         // kHidden, kBackData: [nvox][cout] bf16
    float* Yf;                // kLast: [nout][nvox] float32
    int res, cin, cout, nout, flip;
    int ntx, nty, nzs, zlen;  // tiles along x, y; z segments of zlen planes
    int use_tma;              // the map covers X: interior planes by bulk tensor copy
    int use_ostore;           // kHidden / kBackData with cout == N: tiles leave by bulk tensor stores
    int* err;                 // set to 1 when a wait runs out
};

// Bytes per staged plane: KC chunks of kPlane 16-byte positions, rounded up to 128 bytes
// (the alignment of a bulk tensor copy's shared-memory destination; one chunk alone is
// 2880 bytes, an odd multiple of 64).
template <int KC>
__host__ __device__ constexpr uint32_t slot_bytes() {
    return (uint32_t(KC * kPlane * 16) + 127u) / 128u * 128u;
}

// Shared memory of k_conv3_tc: weights (27 taps × KC chunks × N rows of 16 bytes, the
// same for the x-pair form's 3 dy × 2 chunks × 3N), the plane ring, barriers.
template <int KC, int N, bool PAIR = false>
constexpr int smem_bytes() {
    const int w = PAIR ? 3 * 2 * 3 * N * 16 : 27 * KC * N * 16;
    const int stage = kEpiGroups * kOutStages * 128 * N * 2;   // output staging per epilogue group
    const int b = w + kRing * int(slot_bytes<KC>()) + stage + (2 * kRing + (kEpiGroups + 1) * kAccTiles + 1) * 8 + 16;
    return b < kOneCtaSmem ? kOneCtaSmem : b;   // the CTA's tensor memory may be all 512 columns
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

// The same with the descriptors as (low, high) words: the start address lives in the
// low word, so per-tap offsets are 32-bit adds.
__device__ __forceinline__ void mma_bf16_w(uint32_t dtmem, uint32_t alo, uint32_t ahi, uint32_t blo, uint32_t bhi,
                                           uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n .reg .b64 da, db;\n setp.ne.b32 p, %6, 0;\n"
        " mov.b64 da, {%1, %2};\n mov.b64 db, {%3, %4};\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], da, db, %5, p;\n}" ::"r"(dtmem),
        "r"(alo), "r"(ahi), "r"(blo), "r"(bhi), "r"(id), "r"(acc)
        : "memory");
}

// The same, executed by the whole converged warp: one lane, chosen by elect.sync inside
// the instruction sequence, issues it; the operands stay warp-uniform.
__device__ __forceinline__ void mma_bf16_warp(uint32_t dtmem, uint32_t alo, uint32_t ahi, uint32_t blo, uint32_t bhi,
                                              uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p, e;\n .reg .b64 da, db;\n setp.ne.b32 p, %6, 0;\n"
        " mov.b64 da, {%1, %2};\n mov.b64 db, {%3, %4};\n elect.sync _|e, 0xffffffff;\n"
        " @e tcgen05.mma.cta_group::1.kind::f16 [%0], da, db, %5, p;\n}" ::"r"(dtmem),
        "r"(alo), "r"(ahi), "r"(blo), "r"(bhi), "r"(id), "r"(acc)
        : "memory");
}

// tcgen05.commit by one elected lane of the converged warp.
__device__ __forceinline__ void mma_commit_warp(uint64_t* bar) {
    asm volatile(
        "{\n .reg .pred e;\n elect.sync _|e, 0xffffffff;\n"
        " @e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n}" ::"r"(smem_u32(bar))
        : "memory");
}

// One lane of the (converged) warp.
__device__ __forceinline__ bool elect_one() {
    uint32_t e;
    asm volatile("{\n .reg .pred p;\n elect.sync _|p, 0xffffffff;\n selp.u32 %0, 1, 0, p;\n}" : "=r"(e));
    return e != 0;
}

// Arrives on `bar` once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive float32 columns of this thread's tensor-memory lane (no wait).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Arrives on `bar` when this thread's earlier cp.async copies have landed (the barrier's
// expected count includes this arrival).
__device__ __forceinline__ void cp_async_arrive(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            int c4, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

// Tile from shared memory to global memory at (c0, c1, c2, c3) of `map` (a bulk group).
__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, int c0, int c1, int c2, int c3, uint32_t src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(src)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Waits until at most kOutStages − 1 of this thread's bulk groups still read shared memory.
__device__ __forceinline__ void bulk_wait_read_stages() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(kOutStages - 1) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Barrier `id` of the 128 threads of one epilogue group; returns whether any passed true.
__device__ __forceinline__ bool group_bar_or(int id, bool v) {
    uint32_t r;
    asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 q, %2, 0;\n bar.red.or.pred p, %1, 128, q;\n"
                 " selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(r)
                 : "r"(id), "r"(v ? 1u : 0u)
                 : "memory");
    return r != 0;
}
__device__ __forceinline__ void group_bar(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

__device__ __forceinline__ int wrap(int v, int res) {
    v %= res;
    return v < 0 ? v + res : v;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Bounded barrier wait of one role; false (and the CTA's abort flag set) when it ran
// out or another role has aborted.
__device__ __forceinline__ bool role_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
    if (*abort_flag) return false;
    if (mbar_wait(bar, parity)) return true;
    *abort_flag = 1;
    return false;
}

struct Item {
    int x0, y0, z0, nt;
};

template <class A>
__device__ __forceinline__ Item item_of(const A& a, int item) {
    const int tx = item % a.ntx, rr = item / a.ntx, ty = rr % a.nty, zs = rr / a.nty;
    Item it;
    it.x0 = tx * kTX;
    it.y0 = ty * kTY;
    it.z0 = zs * a.zlen;
    it.nt = min(a.zlen, a.res - it.z0);
    return it;
}

// PAIR: the first layer with at most 4 input channels, staged from the x-pair layout
// [v][8] = (4 channels of v, 4 channels of v + x̂): one K = 16 step reads the pairs at
// x − 1 and x + 1 (K chunks 32 bytes apart) and so covers dx = −1, 0, 1 (and a zero
// weight for dx = 2): three MMAs per plane instead of nine.
template <int CC, int N, int MODE, bool PAIR = false>
__global__ void __launch_bounds__(kThreads, 1)
    k_conv3_tc(const __grid_constant__ Args a, const __grid_constant__ CUtensorMap tmap,
               const __grid_constant__ CUtensorMap omap) {
    static_assert(!PAIR || CC == 1, "the x-pair layout has one 16-byte chunk per position");
    constexpr int KC = PAIR ? 1 : (CC + 1) / 2 * 2;   // chunks staged per position
    constexpr int NSH = PAIR ? 3 : 9;                  // weight shifts: dy (PAIR) or (dy, dx)
    constexpr int KW = PAIR ? 2 : KC;                  // weight K chunks per shift
    constexpr uint32_t kCols = kAccTiles * N;     // 512 (N = 32) or 256 (N = 16)
    constexpr uint32_t kSlot = slot_bytes<KC>();        // 128-byte aligned plane slots
    static_assert((NSH * KW * 3 * N * 16) % 128 == 0, "the plane ring starts 128-byte aligned");
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* ws = smem;
    uint8_t* ringp = smem + NSH * KW * 3 * N * 16;
    uint8_t* ostage = ringp + kRing * kSlot;                     // [group][kOutStages][128 rows][N bf16]
    uint64_t* full = reinterpret_cast<uint64_t*>(ostage + kEpiGroups * kOutStages * 128 * N * 2);
    uint64_t* empty = full + kRing;
    uint64_t* accf = empty + kRing;                  // [group][accumulator]
    uint64_t* acce = accf + kEpiGroups * kAccTiles;
    uint64_t* fin = acce + kAccTiles;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ws_u = smem_u32(ws), ring = smem_u32(ringp);

    // weights → [shift][chunk][n = kz·N + o][8 k], zeros beyond cin and cout; PAIR:
    // shift = dy, k = chunk·8 + half·4 + channel with dx = chunk·2 + half − 1
    for (int i = tid; i < NSH * KW * 3 * N; i += kThreads) {
        const int n3 = i % (3 * N), kc = (i / (3 * N)) % KW, shift = i / (3 * N * KW);
        const int n = n3 % N, kz = n3 / N;
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float f[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int e = 2 * j + u;
                float v = 0.0f;
                if constexpr (PAIR) {
                    const int dx = kc * 2 + e / 4 - 1, ch = e % 4;
                    if (dx <= 1 && n < a.cout)
                        v = __bfloat162float(a.W[(int64_t(kz * 9 + shift * 3 + dx + 1) * a.cin + ch) * a.cout + n]);
                } else {
                    const int k = kc * 8 + e, tap = kz * 9 + shift;
                    if (k < a.cin && n < a.cout)
                        v = __bfloat162float(a.flip ? a.W[(int64_t(26 - tap) * a.cout + n) * a.cin + k]
                                                    : a.W[(int64_t(tap) * a.cin + k) * a.cout + n]);
                }
                f[u] = v;
            }
            w[j] = pack_bf16(f[0], f[1]);
        }
        *reinterpret_cast<uint4*>(ws + size_t(i) * 16) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    // K-padding chunks of every slot are zero for good
    if constexpr (KC > CC) {
        for (int i = tid; i < kRing * (KC - CC) * kPlane; i += kThreads) {
            const int pos = i % kPlane, r = i / kPlane, kc = CC + r % (KC - CC), slot = r / (KC - CC);
            *reinterpret_cast<uint4*>(ringp + size_t(slot) * kSlot + size_t(kc * kPlane + pos) * 16) =
                make_uint4(0, 0, 0, 0);
        }
    }
    if (tid == 0) {
        for (int i = 0; i < kRing; ++i) {
            mbar_init(&full[i], 32);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < kEpiGroups * kAccTiles; ++i) mbar_init(&accf[i], 1);
        for (int i = 0; i < kAccTiles; ++i) mbar_init(&acce[i], 4);
        mbar_init(fin, 1);
        *abort_flag = 0;
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
    const int items = a.ntx * a.nty * a.nzs;
    // accumulator of the column segment's tile t (t < zlen ≤ kAccTiles): adjacent tiles
    // sit in adjacent accumulators, tile t + 1 just below tile t
    auto acc_of = [&](int t) { return a.zlen - 1 - t; };

    if (warp == kLoaderWarp) {
        // ── loader ──────────────────────────────────────────────────────────────
        uint32_t k = 0;   // planes issued by this CTA; plane k in slot k % kRing
        bool ok = true;
        for (int item = blockIdx.x; item < items && ok; item += gridDim.x) {
            const Item it = item_of(a, item);
            const bool interior = a.use_tma && it.x0 >= 1 && it.x0 - 1 + kBX <= a.res && it.y0 >= 1 &&
                                  it.y0 - 1 + kBY <= a.res;
            for (int j = 0; j < it.nt + 2; ++j, ++k) {
                const int slot = int(k % kRing);
                if (!role_wait(&empty[slot], ((k / kRing) & 1u) ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                const int gz = wrap(it.z0 - 1 + j, a.res);
                const uint32_t dst = ring + uint32_t(slot) * kSlot;
                if (interior) {
                    if (lane == 0) {
                        mbar_arrive_expect_tx(&full[slot], uint32_t(CC * kPlane * 16));
                        tma_load_5d(dst, &tmap, 0, it.x0 - 1, it.y0 - 1, 0, gz, &full[slot]);
                    } else {
                        mbar_arrive(&full[slot]);
                    }
                } else {
                    for (int e = lane; e < CC * kPlane; e += 32) {
                        const int pos = e / CC, kc = e - pos * CC;
                        const int by = pos / kBX, bx = pos - by * kBX;
                        const int gy = wrap(it.y0 - 1 + by, a.res), gx = wrap(it.x0 - 1 + bx, a.res);
                        const __nv_bfloat16* src =
                            a.X + ((int64_t(gz) * a.res + gy) * a.res + gx) * (CC * 8) + kc * 8;
                        cp_async16(dst + uint32_t((kc * kPlane + pos) * 16), src);
                    }
                    cp_async_arrive(&full[slot]);
                }
            }
        }
        cp_async_wait_all();
        if (!ok) {
            // bulk copies still in flight land before the CTA ends
            const uint32_t n = k < uint32_t(kRing) ? k : uint32_t(kRing);
            for (uint32_t q = k - n; q < k; ++q) mbar_wait(&full[q % kRing], (q / kRing) & 1u);
        }
    } else if (warp == kMmaWarp) {
        // ── MMA issue: per staged plane u (z0 − 1 .. z0 + L), one MMA per (shift, K step)
        // of N · (tiles it feeds): the plane is the kz = 0, 1, 2 input of tiles u + 1, u,
        // u − 1, whose accumulators are adjacent; the warp runs the loop, one lane issues.
        const uint32_t id0 = idesc<0>();   // N field filled in per MMA: (n >> 3) << 17
        // A: K chunks kPlane positions apart, or (PAIR) the pair two positions on
        const uint64_t adesc0 = sdesc(ring, PAIR ? 32 : kPlane * 16, kBX * 16);
        const uint64_t bdesc0 = sdesc(ws_u, 3 * N * 16, 128);
        const uint32_t alo0 = uint32_t(adesc0), ahi = uint32_t(adesc0 >> 32);
        const uint32_t blo0 = uint32_t(bdesc0), bhi = uint32_t(bdesc0 >> 32);
        uint32_t live[kAccTiles], waited[kAccTiles];   // accf commits / acce completions seen
        for (int i = 0; i < kAccTiles; ++i) live[i] = waited[i] = 0;
        uint32_t kp = 0, done = 0;   // planes issued; tiles completed (tile n goes to group n % kEpiGroups)
        bool ok = true;
        for (int item = blockIdx.x; item < items && ok; item += gridDim.x) {
            const Item it = item_of(a, item);
            const int L = it.nt;
            const uint32_t base = kp;
            for (int u = -1; u <= L; ++u) {
                const uint32_t p = base + uint32_t(u + 1);
                const int lo = max(u - 1, 0), hi = min(u + 1, L - 1), nv = hi - lo + 1;
                const bool first = u + 1 <= L - 1;     // tile u + 1 starts here
                bool w = role_wait(&full[p % kRing], (p / kRing) & 1u, abort_flag);
                if (w && first) {
                    const int c = acc_of(u + 1);
                    if (waited[c] < live[c]) {          // its last tile's epilogue has read it
                        w = role_wait(&acce[c], waited[c] & 1u, abort_flag);
                        ++waited[c];
                    }
                }
                ok = __all_sync(0xffffffffu, w);
                if (!ok) break;
                tc_after_sync();
                const uint32_t d0 = tmem + uint32_t(acc_of(hi) * N);
                const int b0 = u + 1 - hi;               // weight block (kz) of tile hi
                const uint32_t alo = alo0 + (((p % kRing) * kSlot) >> 4);
                const uint32_t idv = id0 | (uint32_t(nv * N / 8) << 17);
#pragma unroll
                for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                    for (int dx = 0; dx < (PAIR ? 1 : 3); ++dx)
#pragma unroll
                        for (int s = 0; s < (PAIR ? 1 : KC / 2); ++s) {
                            const int sh = PAIR ? dy : dy * 3 + dx;
                            const uint32_t av = alo + uint32_t(((2 * s * kPlane + dy * kBX + dx) * 16) >> 4);
                            const uint32_t bv =
                                blo0 + uint32_t((((sh * KW + 2 * s) * 3 * N) * 16) >> 4) + uint32_t(b0 * N);
                            if (sh == 0 && s == 0 && first) {
                                mma_bf16_warp(d0, av, ahi, bv, bhi, id0 | (uint32_t(N / 8) << 17), 0u);
                                if (nv > 1)
                                    mma_bf16_warp(d0 + N, av, ahi, bv + N, bhi, id0 | (uint32_t((nv - 1) * N / 8) << 17),
                                                  1u);
                            } else {
                                mma_bf16_warp(d0, av, ahi, bv, bhi, idv, 1u);
                            }
                        }
                mma_commit_warp(&empty[p % kRing]);
                if (u >= 1)   // tile u − 1 is complete
                    mma_commit_warp(&accf[(done % kEpiGroups) * kAccTiles + acc_of(u - 1)]);
                __syncwarp();
                if (u >= 1) {
                    ++live[acc_of(u - 1)];
                    ++done;
                }
            }
            if (!ok) break;
            kp = base + uint32_t(L + 2);
        }
        // every MMA has completed before the tensor memory is released
        if (elect_one()) mma_commit(fin);
        __syncwarp();
        mbar_wait(fin, 0);
    } else {
        // ── epilogue: group g = warp / 4 takes the CTA's tiles n ≡ g (mod kEpiGroups);
        // warp w reads tensor-memory lanes 32·(w % 4) .. +31 ──────────────────────────
        const int g = warp >> 2, row = tid & 127;
        const uint32_t lane_base = uint32_t((warp & 3) * 32) << 16;
        const int64_t nvox = int64_t(a.res) * a.res * a.res;
        float bias[N];
#pragma unroll
        for (int cc = 0; cc < N; ++cc)
            bias[cc] = (MODE != kBackData && cc < (MODE == kLast ? a.nout : a.cout)) ? __ldg(a.bias + cc) : 0.0f;
        uint32_t uses[kAccTiles];   // this group's earlier tiles per accumulator
        for (int i = 0; i < kAccTiles; ++i) uses[i] = 0;
        uint32_t n = 0;             // the CTA's tiles so far
        uint32_t kst = 0;           // this group's tiles so far (staging buffer kst % kOutStages)
        const bool ostore = MODE != kLast && a.use_ostore;
        const uint32_t stage0 = smem_u32(ostage) + uint32_t(g * kOutStages * 128 * N * 2);
        bool ok = true;
        for (int item = blockIdx.x; item < items && ok; item += gridDim.x) {
            const Item it = item_of(a, item);
            const int x = it.x0 + (row & 7), y = it.y0 + (row >> 3);
            const bool valid = x < a.res && y < a.res;
            for (int i = 0; i < it.nt; ++i, ++n) {
                if (int(n % kEpiGroups) != g) continue;
                const int c = acc_of(i);
                bool bad = !role_wait(&accf[g * kAccTiles + c], uses[c] & 1u, abort_flag);
                if (ostore) bad = group_bar_or(1 + g, bad);   // the group's barriers stay matched
                if (bad) {
                    ok = false;
                    break;
                }
                ++uses[c];
                tc_after_sync();
                uint32_t r[N];
#pragma unroll
                for (int q = 0; q < N / 16; ++q)
                    tmem_ld16(tmem + lane_base + uint32_t(c * N + q * 16), r + q * 16);
                tmem_wait_ld();
                tc_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acce[c]);
                if (!valid && !ostore) continue;
                const int64_t v = (int64_t(it.z0 + i) * a.res + y) * a.res + x;
                if constexpr (MODE == kLast) {
#pragma unroll
                    for (int cc = 0; cc < N; ++cc)
                        if (cc < a.nout) a.Yf[int64_t(cc) * nvox + v] = __uint_as_float(r[cc]) + bias[cc];
                } else {
                    uint4 out[N / 8];
#pragma unroll
                    for (int c8 = 0; c8 < N / 8; ++c8) {
                        uint32_t w[4];
                        if constexpr (MODE == kBackData) {
                            const uint4 m4 = (valid && c8 * 8 < a.cout)
                                                 ? __ldg(reinterpret_cast<const uint4*>(a.M + v * a.cout) + c8)
                                                 : make_uint4(0u, 0u, 0u, 0u);
                            const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const __nv_bfloat162 m2 = *reinterpret_cast<const __nv_bfloat162*>(&mw[j]);
                                const float g0 = __bfloat162float(m2.x) > 0.0f ? __uint_as_float(r[c8 * 8 + 2 * j]) : 0.0f;
                                const float g1 =
                                    __bfloat162float(m2.y) > 0.0f ? __uint_as_float(r[c8 * 8 + 2 * j + 1]) : 0.0f;
                                w[j] = pack_bf16(g0, g1);
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const int cc = c8 * 8 + 2 * j;
                                w[j] = pack_bf16(fmaxf(__uint_as_float(r[cc]) + bias[cc], 0.0f),
                                                 fmaxf(__uint_as_float(r[cc + 1]) + bias[cc + 1], 0.0f));
                            }
                        }
                        out[c8] = make_uint4(w[0], w[1], w[2], w[3]);
                    }
                    if (ostore) {
                        // the bulk store that last read this buffer (kOutStages tiles ago) is done
                        if (row == 0) bulk_wait_read_stages();
                        group_bar(1 + g);
                        const uint32_t buf =
                            stage0 + (kst % kOutStages) * uint32_t(128 * N * 2) + uint32_t(row * N * 2);
#pragma unroll
                        for (int c8 = 0; c8 < N / 8; ++c8)
                            asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(buf + c8 * 16),
                                         "r"(out[c8].x), "r"(out[c8].y), "r"(out[c8].z), "r"(out[c8].w)
                                         : "memory");
                        fence_proxy_async_smem();   // the rows are read by the bulk store
                        group_bar(1 + g);
                        if (row == 0)   // rows outside the mesh are clipped by the store
                            tma_store_4d(&omap, 0, it.x0, it.y0, it.z0 + i,
                                         stage0 + (kst % kOutStages) * uint32_t(128 * N * 2));
                        ++kst;
                    } else {
                        uint4* dst = reinterpret_cast<uint4*>(a.Y + v * a.cout);
#pragma unroll
                        for (int c8 = 0; c8 < N / 8; ++c8)
                            if (c8 * 8 < a.cout) dst[c8] = out[c8];
                    }
                }
            }
        }
        if (ostore && row == 0) bulk_wait_all();   // the last stores have landed
    }
    tc_before_sync();
    __syncthreads();
    if (tid == 0 && *abort_flag) atomicExch(a.err, 1);
    if (warp == 0) {
        tc_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

// ── weight gradient ─────────────────────────────────────────────────────────────
// dW[tap][c][o] = Σ_v X[v + offset(tap)][c] · dY[v][o] for 32 input channels.
// The operand trick: in the staged layout [slot][chunk][position][8] the 8-channel
// groups of consecutive slots are evenly spaced (slot stride = 4 × chunk stride), so
// one MN-major A operand of 128 rows = (4 slots, 32 channels) covers four consecutive
// planes, with K = the 16 voxels of two tile rows read at a (dy, dx) position shift.
// B = the dY tile, [chunk][voxel][8] (MN-major). The ring holds kWRing planes and
// repeats its first three slots after its end (a plane landing in slot s < 3 is also
// copied to slot kWRing + s), so the window starting at the slot of plane z − 1 is
// always contiguous: rows of window slot q accumulate the tap dz = q − 1 (q = 3, the
// plane after, is discarded and may still be landing). One accumulator per (dy, dx):
// 9 × N columns of tensor memory, one pass over the mesh. At the end every row (tap,
// channel) is added to dW with float atomics (one per entry and CTA).

constexpr int kWRing = 8;                  // planes in the ring
constexpr int kWMirror = 3;                // slots repeated after the ring's end
constexpr int kWY = 4;                     // dY tile buffers

struct WArgs {
    const __nv_bfloat16* X;   // [nvox][32]
    const __nv_bfloat16* dY;  // [nvox][cout] (cout = 8·CCO)
    float* dW;                // [27][cin_w][cout], accumulated with atomics
    int res, cout;
    int cin_w;                // input-channel rows of dW (<= 32: the input may be zero-widened)
    int ntx, nty, nzs, zlen;
    int use_tma;              // plane map (X) and tile map (dY) accepted
    int* err;
};

template <int N>
constexpr int wg_smem_bytes() {
    return (kWRing + kWMirror) * 4 * kPlane * 16 + kWY * N * 128 * 2 + (2 * kWRing + 2 * kWY + 2) * 8 + 16;
}

template <int N>
__device__ __forceinline__ uint32_t idesc_mn() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | (uint32_t(N >> 3) << 17) |
           (uint32_t(128 >> 4) << 24);
}

template <int CCO, int N>
__global__ void __launch_bounds__(kThreads, 1)
    k_conv3_wgrad(const __grid_constant__ WArgs a, const __grid_constant__ CUtensorMap xmap,
                  const __grid_constant__ CUtensorMap ymap) {
    constexpr int CC = 4;
    constexpr uint32_t kSlot = CC * kPlane * 16;            // 11520 = 4 × the chunk stride
    static_assert(kSlot % 128 == 0 && kSlot == slot_bytes<CC>(), "slots 128-byte aligned, no padding");
    constexpr uint32_t kYBuf = N * 128 * 2;                 // [N/8][128 voxels][8]
    constexpr uint32_t kCols = 9 * N <= 256 ? 256 : 512;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* ringp = smem;
    uint8_t* ybufp = ringp + (kWRing + kWMirror) * kSlot;
    uint64_t* fullx = reinterpret_cast<uint64_t*>(ybufp + kWY * kYBuf);
    uint64_t* emptyx = fullx + kWRing;
    uint64_t* fully = emptyx + kWRing;
    uint64_t* emptyy = fully + kWY;
    uint64_t* accf = emptyy + kWY;
    uint64_t* fin = accf + 1;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ring = smem_u32(ringp), ybuf = smem_u32(ybufp);

    // dY channel padding (chunks CCO .. N/8 − 1) is zero for good
    if constexpr (N / 8 > CCO) {
        for (int i = tid; i < kWY * (N / 8 - CCO) * 128; i += kThreads) {
            const int v = i % 128, r = i / 128, kc = CCO + r % (N / 8 - CCO), b = r / (N / 8 - CCO);
            *reinterpret_cast<uint4*>(ybufp + size_t(b) * kYBuf + size_t(kc * 128 + v) * 16) = make_uint4(0, 0, 0, 0);
        }
    }
    if (tid == 0) {
        for (int i = 0; i < kWRing; ++i) {
            mbar_init(&fullx[i], 32);
            mbar_init(&emptyx[i], 1);
        }
        for (int i = 0; i < kWY; ++i) {
            mbar_init(&fully[i], 32);
            mbar_init(&emptyy[i], 1);
        }
        mbar_init(accf, 1);
        mbar_init(fin, 1);
        *abort_flag = 0;
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
    const int items = a.ntx * a.nty * a.nzs;

    if (warp == kLoaderWarp) {
        uint32_t kx = 0, ky = 0;
        bool ok = true;
        auto load_plane = [&](const Item& it, int j, bool interior) -> bool {
            const int slot = int(kx % kWRing);
            if (!role_wait(&emptyx[slot], ((kx / kWRing) & 1u) ^ 1u, abort_flag)) return false;
            const int gz = wrap(it.z0 - 1 + j, a.res);
            const bool mirror = slot < kWMirror;
            const uint32_t dst = ring + uint32_t(slot) * kSlot;
            const uint32_t dst2 = ring + uint32_t(kWRing + slot) * kSlot;
            if (interior) {
                if (lane == 0) {
                    mbar_arrive_expect_tx(&fullx[slot], mirror ? 2 * kSlot : kSlot);
                    tma_load_5d(dst, &xmap, 0, it.x0 - 1, it.y0 - 1, 0, gz, &fullx[slot]);
                    if (mirror) tma_load_5d(dst2, &xmap, 0, it.x0 - 1, it.y0 - 1, 0, gz, &fullx[slot]);
                } else {
                    mbar_arrive(&fullx[slot]);
                }
            } else {
                for (int e = lane; e < CC * kPlane; e += 32) {
                    const int pos = e / CC, kc = e - pos * CC;
                    const int by = pos / kBX, bx = pos - by * kBX;
                    const int gy = wrap(it.y0 - 1 + by, a.res), gx = wrap(it.x0 - 1 + bx, a.res);
                    const __nv_bfloat16* src = a.X + ((int64_t(gz) * a.res + gy) * a.res + gx) * (CC * 8) + kc * 8;
                    const uint32_t off = uint32_t((kc * kPlane + pos) * 16);
                    cp_async16(dst + off, src);
                    if (mirror) cp_async16(dst2 + off, src);
                }
                cp_async_arrive(&fullx[slot]);
            }
            ++kx;
            return true;
        };
        auto load_dy = [&](const Item& it, int i) -> bool {
            const int b = int(ky % kWY);
            if (!role_wait(&emptyy[b], ((ky / kWY) & 1u) ^ 1u, abort_flag)) return false;
            const uint32_t dst = ybuf + uint32_t(b) * kYBuf;
            const int z = it.z0 + i;
            if (a.use_tma) {
                if (lane == 0) {
                    mbar_arrive_expect_tx(&fully[b], uint32_t(CCO * 128 * 16));
                    tma_load_5d(dst, &ymap, 0, it.x0, it.y0, 0, z, &fully[b]);
                } else {
                    mbar_arrive(&fully[b]);
                }
            } else {
                // voxels outside the mesh contribute nothing: zero rows
                for (int e = lane; e < CCO * 128; e += 32) {
                    const int v = e / CCO, kc = e - v * CCO;
                    const int x = it.x0 + (v & 7), y = it.y0 + (v >> 3);
                    const uint32_t d = dst + uint32_t((kc * 128 + v) * 16);
                    if (x < a.res && y < a.res)
                        cp_async16(d, a.dY + ((int64_t(z) * a.res + y) * a.res + x) * (CCO * 8) + kc * 8);
                    else
                        asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(d), "r"(0) : "memory");
                }
                fence_proxy_async_smem();
                cp_async_arrive(&fully[b]);
            }
            ++ky;
            return true;
        };
        for (int item = blockIdx.x; item < items && ok; item += gridDim.x) {
            const Item it = item_of(a, item);
            const bool interior = a.use_tma && it.x0 >= 1 && it.x0 - 1 + kBX <= a.res && it.y0 >= 1 &&
                                  it.y0 - 1 + kBY <= a.res;
            for (int i = 0; i < it.nt && ok; ++i) {
                if (i == 0) ok = load_plane(it, 0, interior) && load_plane(it, 1, interior);
                ok = ok && load_plane(it, i + 2, interior) && load_dy(it, i);
            }
        }
        cp_async_wait_all();
        if (!ok) {
            for (uint32_t q = kx > kWRing ? kx - kWRing : 0; q < kx; ++q) mbar_wait(&fullx[q % kWRing], (q / kWRing) & 1u);
            for (uint32_t q = ky > kWY ? ky - kWY : 0; q < ky; ++q) mbar_wait(&fully[q % kWY], (q / kWY) & 1u);
        }
    } else if (warp == kMmaWarp) {
        const uint32_t id = idesc_mn<N>();
        // A: M groups (slot, chunk) every 2880 bytes, K groups (tile rows) every 160
        const uint64_t ad0 = sdesc(ring, kBX * 16, kPlane * 16);
        // B: N groups every 128 voxels, K groups every 8 voxels
        const uint64_t bd0 = sdesc(ybuf, 128, 128 * 16);
        const uint32_t alo0 = uint32_t(ad0), ahi = uint32_t(ad0 >> 32);
        const uint32_t blo0 = uint32_t(bd0), bhi = uint32_t(bd0 >> 32);
        uint32_t kx = 0, ky = 0;
        bool ok = true, first = true;
        for (int item = blockIdx.x; item < items && ok; item += gridDim.x) {
            const Item it = item_of(a, item);
            const uint32_t base = kx;
            for (int i = 0; i < it.nt; ++i, ++ky) {
                bool w = role_wait(&fully[ky % kWY], (ky / kWY) & 1u, abort_flag);
                for (int j = (i == 0 ? 0 : i + 2); w && j <= i + 2; ++j) {
                    const uint32_t p = base + uint32_t(j);
                    w = role_wait(&fullx[p % kWRing], (p / kWRing) & 1u, abort_flag);
                }
                ok = __all_sync(0xffffffffu, w);
                if (!ok) break;
                tc_after_sync();
                // window: the slot of plane i (z − 1) and the three after it
                const uint32_t aw = alo0 + ((((base + i) % kWRing) * kSlot) >> 4);
                const uint32_t yb = blo0 + (((ky % kWY) * kYBuf) >> 4);
                if (elect_one()) {
#pragma unroll
                    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                        for (int dx = 0; dx < 3; ++dx) {
                            const uint32_t d = tmem + uint32_t((dy * 3 + dx) * N);
#pragma unroll
                            for (int s = 0; s < 8; ++s)
                                mma_bf16_w(d, aw + uint32_t((((dy + 2 * s) * kBX + dx) * 16) >> 4), ahi,
                                           yb + uint32_t((s * 256) >> 4), bhi, id, (!first || s > 0) ? 1u : 0u);
                        }
                    mma_commit(&emptyx[(base + i) % kWRing]);   // tile i is the last reader of plane i
                    mma_commit(&emptyy[ky % kWY]);
                }
                __syncwarp();
                first = false;
            }
            if (!ok) break;
            if (elect_one()) {
                mma_commit(&emptyx[(base + it.nt) % kWRing]);
                mma_commit(&emptyx[(base + it.nt + 1) % kWRing]);
            }
            __syncwarp();
            kx = base + it.nt + 2;
        }
        if (elect_one()) {
            if (ok) mma_commit(accf);
            mma_commit(fin);
        }
        __syncwarp();
        mbar_wait(fin, 0);
    } else if (warp < 4) {
        // ── epilogue: warps 0-3, row tid = (window slot q, channel); q = 3 is discarded ──
        const uint32_t lane_base = uint32_t(warp * 32) << 16;
        const int q = tid >> 5, c = tid & 31;
        // one wait for the whole run: bounded in rounds of about a second each, ended early
        // when another role aborts
        bool w = false;
        for (int k = 0; k < 120 && !w && !*abort_flag; ++k) w = mbar_wait(accf, 0);
        if (!w) *abort_flag = 1;
        if (w) {
            tc_after_sync();
            for (int tap9 = 0; tap9 < 9; ++tap9) {   // (dy, dx)
                uint32_t v[N];
#pragma unroll
                for (int h = 0; h < N / 16; ++h) tmem_ld16(tmem + lane_base + uint32_t(tap9 * N + h * 16), v + h * 16);
                tmem_wait_ld();
                if (q < 3 && c < a.cin_w) {
                    float* dst = a.dW + (size_t(q * 9 + tap9) * a.cin_w + c) * a.cout;
#pragma unroll
                    for (int o = 0; o < N; ++o)
                        if (o < a.cout) atomicAdd(dst + o, __uint_as_float(v[o]));
                }
            }
        }
    }
    tc_before_sync();
    __syncthreads();
    if (tid == 0 && *abort_flag) atomicExch(a.err, 1);
    if (warp == 0) {
        tc_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

}  // namespace conv
}  // namespace djb
