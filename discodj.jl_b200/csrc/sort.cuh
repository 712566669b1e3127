// Eulerian binning of the particles: an index sort by brick.
//
// Every force evaluation ranks the particles by the B^3-cell brick (linear brick
// index) that holds the base node of their position, with a counting sort: histogram
// with atomics (k_bin, which also applies the step's first drift and writes the
// drifted displacements back), exclusive scan (k_scan_block, k_scan_sums) and
// placement (k_place). The particle state stays in the reference's Lagrangian order;
// the brick kernels (brick.cuh) read it through `perm`.
#pragma once

#include <cstdint>

#include "pm_kernels.cuh"

namespace djb {

constexpr int kScanThreads = 1024;
constexpr int kScanPerThread = 4;
constexpr int kScanBlock = kScanThreads * kScanPerThread;  // entries per scan block

struct SortGeom {
    int res;
    int brick;   // cells per brick side (power of two)
    int lgb;     // log2(brick)
    int nb;      // bricks per axis
    int hb;      // sub-blocks of 2 cells per brick side (brick / 2, at least 1)
};

// Sort key of the cell floor(g) (the shift-0 cell; the brick kernels' boxes cover the
// base nodes of the interlacing shifts and odd-order rounding around it): the linear
// brick index, then the 2^3-cell sub-block inside the brick, so that particles of one
// cell are consecutive in the sorted order.
__device__ __forceinline__ uint32_t brick_key(const float X[3], float L, float resf, const SortGeom& sg, int* err) {
    int bc[3], sc[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float g = grid_coord(X[a], L, resf, err);
        // g lies in [0, res]: g == res (mod(X, L) rounded up to L) is the node 0 image
        int c = __float2int_rd(g);
        c = c >= sg.res ? c - sg.res : (c < 0 ? 0 : c);
        bc[a] = c >> sg.lgb;
        sc[a] = (sg.hb > 1) ? ((c & (sg.brick - 1)) >> 1) : 0;
    }
    const uint32_t brick = uint32_t((bc[2] * sg.nb + bc[1]) * sg.nb + bc[0]);
    return brick * uint32_t(sg.hb * sg.hb * sg.hb) + uint32_t((sc[2] * sg.hb + sc[1]) * sg.hb + sc[0]);
}

// Applies the first drift Ψ <- Ψ + dd1·Mom when `mom` is given (written back), then
// bins the particle at X = q + Ψ: key and rank within the key.
__global__ void __launch_bounds__(256) k_bin(float* __restrict__ psi, const float* __restrict__ mom,
                                             float dd1, const float* __restrict__ q1, int n, int64_t np,
                                             float L, SortGeom sg, unsigned* __restrict__ count,
                                             uint2* __restrict__ keyrank, int* err) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= np) return;
    LatticeDiv ld;
    ld.init(n);
    int i, j, k;
    ld.ijk(p, i, j, k);
    float X[3] = {psi[p], psi[p + np], psi[p + 2 * np]};
    if (mom) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            X[c] = X[c] + dd1 * mom[p + c * np];
            psi[p + c * np] = X[c];
        }
    }
    X[0] = X[0] + q1[i];
    X[1] = X[1] + q1[j];
    X[2] = X[2] + q1[k];
    const uint32_t key = brick_key(X, L, float(sg.res), sg, err);
    const unsigned r = atomicAdd(count + key, 1u);
    keyrank[p] = make_uint2(key, r);
}

// Block-local exclusive scan of `count` (kScanBlock entries per block) into `offset`;
// the block totals go to `bsum`.
__global__ void __launch_bounds__(kScanThreads) k_scan_block(const unsigned* __restrict__ count, int64_t nbins,
                                                              unsigned* __restrict__ offset,
                                                              unsigned* __restrict__ bsum) {
    __shared__ unsigned s_warp[kScanThreads / 32];
    const int64_t base = int64_t(blockIdx.x) * kScanBlock + int64_t(threadIdx.x) * kScanPerThread;
    unsigned v[kScanPerThread];
    unsigned local = 0;
#pragma unroll
    for (int e = 0; e < kScanPerThread; ++e) {
        v[e] = (base + e < nbins) ? count[base + e] : 0u;
        local += v[e];
    }
    // warp inclusive scan of the per-thread totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned w = (lane < kScanThreads / 32) ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;  // inclusive warp prefix
    }
    __syncthreads();
    unsigned run = incl - local + (warp > 0 ? s_warp[warp - 1] : 0u);
#pragma unroll
    for (int e = 0; e < kScanPerThread; ++e) {
        if (base + e < nbins) offset[base + e] = run;
        run += v[e];
    }
    if (threadIdx.x == kScanThreads - 1) bsum[blockIdx.x] = run;
}

// Exclusive scan of the block totals, in place (one CTA; nblocks <= kScanThreads * 64).
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(unsigned* __restrict__ bsum, int nblocks) {
    __shared__ unsigned s_warp[kScanThreads / 32];
    constexpr int per = 64;
    const int base = threadIdx.x * per;
    unsigned local = 0;
    for (int e = 0; e < per; ++e)
        if (base + e < nblocks) local += bsum[base + e];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        unsigned w = (lane < kScanThreads / 32) ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    unsigned run = incl - local + (warp > 0 ? s_warp[warp - 1] : 0u);
    for (int e = 0; e < per; ++e) {
        if (base + e < nblocks) {
            const unsigned t = bsum[base + e];
            bsum[base + e] = run;
            run += t;
        }
    }
}

// perm[sorted slot] = particle; slot = block-local offset + block total + rank.
__global__ void __launch_bounds__(256) k_place(const uint2* __restrict__ keyrank, int64_t np,
                                               const unsigned* __restrict__ offset,
                                               const unsigned* __restrict__ bsum, int* __restrict__ perm) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const uint2 kr = keyrank[p];
    const unsigned slot = offset[kr.x] + bsum[kr.x / kScanBlock] + kr.y;
    perm[slot] = int(p);
}

}  // namespace djb
