// Device kernels of the particle-mesh step (sm_100a).
//
// Mesh layout in HBM: a real mesh is stored [iz][iy][ix] with x fastest and each
// x row padded to res+2 floats, so cuFFT's in-place R2C halves the x axis and
// the spectrum is [kz][ky][kx], kx in [0, res/2]. The reference halves z
// (`rfft(x, [3,1,2])`, pm.jl:16-17); every multiplier of the PM force is even in
// each k component and zeroes every Nyquist the same way on every axis
// (pm.jl:125-183), so the choice of halved axis changes only round-off.
//
// Particle layout: Julia (n,n,n,3) column-major = three component blocks of n^3
// floats, x fastest (pm.jl:15-17). Particle p = i + n*(j + n*k).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace djb {

// Julia `mod(x::Float32, y::Float32)` for y > 0 (rem, then add y when the sign differs).
// Positions lie within one box length of [0, y), where the remainder is exact and
// needs no fmodf: x itself, x - y (exact for y <= x < 2y), or x + y for -y <= x < 0
// (the remainder x, then + y as below).
__device__ __forceinline__ float jmodf(float x, float y) {
    if (x >= 0.0f && x < y) return x;
    if (x >= y && x < 2.0f * y) return x - y;
    if (x < 0.0f && x >= -y) return x + y;
    float r = fmodf(x, y);
    if (r < 0.0f) r += y;
    return r;
}

__device__ __forceinline__ int wrapi(int i, int res) {
    i = (i >= res) ? i - res : i;
    return (i < 0) ? i + res : i;
}

// Lowest stencil offset per assignment order (pm.jl:53-55): CIC [0,1], TSC [-1,1], PCS [-1,2].
template <int W>
struct WLo {
    static constexpr int v = (W == 2) ? 0 : -1;
};

// pm.jl:52 — even orders floor, odd orders round half to even.
template <int W>
__device__ __forceinline__ int wbase(float g) {
    return (W % 2 == 0) ? __float2int_rd(g) : __float2int_rn(g);
}

// pm.jl:49-51 — CIC, TSC and PCS (cubic B-spline) kernels of the distance d >= 0.
template <int W>
__device__ __forceinline__ float wk(float d) {
    if (W == 2) return d > 1.0f ? 0.0f : 1.0f - d;
    if (W == 3) {
        if (d > 1.5f) return 0.0f;
        if (d > 0.5f) {
            const float t = 1.5f - d;
            return 0.5f * (t * t);
        }
        return 0.75f - d * d;
    }
    if (d > 2.0f) return 0.0f;
    if (d > 1.0f) {
        const float t = 2.0f - d;
        return (t * t * t) / 6.0f;
    }
    return (4.0f - 6.0f * (d * d) + 3.0f * (d * d * d)) / 6.0f;
}

// Grid coordinate of one component: mod(X, L)/L*res (pm.jl:61). A non-finite
// position is reported through `err` and mapped to 0 so no index leaves the mesh.
__device__ __forceinline__ float grid_coord(float x, float L, float resf, int* err) {
    float g = jmodf(x, L) / L * resf;
    if (!(g >= 0.0f && g <= resf)) {
        if (err) atomicOr(err, 1);
        g = 0.0f;
    }
    return g;
}

// Lattice indices (i, j, k) of particle p = i + n (j + n k) by 64-bit multiply-high with
// m = ceil(2^64 / n): exact for p < 2^64 / n, i.e. for every particle (n >= 2).
struct LatticeDiv {
    uint64_t m;
    unsigned n;
    __device__ __forceinline__ void init(int nn) {
        n = unsigned(nn);
        m = ~0ull / n + 1ull;
    }
    __device__ __forceinline__ void ijk(int64_t p, int& i, int& j, int& k) const {
        const uint64_t q = __umul64hi(uint64_t(p), m);
        const uint64_t r = __umul64hi(q, m);
        i = int(uint64_t(p) - q * n);
        j = int(q - r * n);
        k = int(r);
    }
};

// Weights and wrapped node indices along one axis.
template <int W>
__device__ __forceinline__ void axis_weights(float g, int res, float* w, int* idx) {
    const int b = wbase<W>(g);
#pragma unroll
    for (int o = 0; o < W; ++o) {
        const int node = b + WLo<W>::v + o;
        w[o] = wk<W>(fabsf(g - float(node)));
        idx[o] = wrapi(node, res);
    }
}

}  // namespace djb
