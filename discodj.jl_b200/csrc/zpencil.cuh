// Fused z pass of the Poisson solve on a 1024^3 mesh: forward DFT along z, the
// multiplier Kφ, inverse DFT along z, in place on the half spectrum.
//
// The 3-D R2C / C2R transforms of the force calculation are split into a batched 2-D
// transform of the z planes (cuFFT) and this kernel, which does both z transforms of
// one (ky, kx) pencil around the multiplication while the pencil is on chip. That
// replaces three passes over the spectrum (the z stage of the forward transform, the
// k-space multiplication and the z stage of the inverse transform) by one.
//
// Layout: spectrum f[(kz * res + ky) * nh + kx], nh = res/2 + 1 (the 2-D R2C halves x).
// A CTA owns 8 consecutive kx of one ky: 8 pencils x 32 threads, thread (q, t) at
// threadIdx.x = q + 8 t, so that a warp reads 4 kz rows of 8 consecutive kx (64 bytes
// each) per load. res = 1024 = 32 x 32 (Cooley-Tukey with n = n2 + 32 n1 and
// k = k1 + 32 k2):
//   A  thread n2 loads x[n2 + 32 n1], DFT over n1 (radix-2 DIF in registers),
//      multiplies by W^(n2 k1) (W = exp(-2 pi i / 1024)), writes to shared memory;
//   B  thread k1 reads its row, DFT over n2 -> X[k1 + 32 k2]; X *= Kφ(kx, ky, kz);
//   A' inverse DFT over k2 (radix-2 DIT on the bit-reversed registers), multiplies by
//      W^-(n2 k1), writes back transposed;
//   B' thread n2 reads its column, inverse DFT over k1 (DIF) -> x[n2 + 32 n1], stores.
// Both transforms are unnormalised, as cuFFT's, so Kφ keeps its 1/res^3 factor.
// Twiddles: W_32^j from a constant table (uniform across the warp), W^(n2 k1) from a
// float table of the 1024 roots computed in float64 on the host.
#pragma once

#include <cstdint>

namespace djb {

#ifndef DJB_ZPASS_BLOCKS
#define DJB_ZPASS_BLOCKS 2
#endif
#ifndef DJB_ZPASS_KTABLE
#define DJB_ZPASS_KTABLE 0
#endif

constexpr int kZRes = 1024;
#ifndef DJB_ZPASS_PENCILS
#define DJB_ZPASS_PENCILS 8
#endif
constexpr int kZPencils = DJB_ZPASS_PENCILS;  // kx per CTA
constexpr int kZThreads = kZPencils * 32;
constexpr int kZRow = 33;              // shared row pitch (float2), breaks bank alignment
constexpr int kZPlane = 32 * kZRow + 2;  // per-pencil block (float2)
constexpr int kZKRow = kZRes + 4;        // Kφ row pitch (floats): the 8 pencils on different banks
constexpr int kZSmem = kZPencils * kZPlane * 8 + (DJB_ZPASS_KTABLE ? kZPencils * kZKRow * 4 : 0);  // dynamic shared bytes

__constant__ float2 c_w32[16];  // exp(-2 pi i j / 32), j < 16

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

__host__ __device__ constexpr int brev5(int i) {
    return ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
}

// One radix-2 stage on blocks of LEN points (LEN a template constant, so every register
// index below is a compile-time constant and the pencil stays in registers).
template <int LEN>
__device__ __forceinline__ void dif_stage(float2 (&a)[32]) {
    constexpr int half = LEN / 2;
#pragma unroll
    for (int s = 0; s < 32; s += LEN) {
#pragma unroll
        for (int j = 0; j < half; ++j) {
            const float2 u = a[s + j], v = a[s + j + half];
            a[s + j] = make_float2(u.x + v.x, u.y + v.y);
            const float2 d = make_float2(u.x - v.x, u.y - v.y);
            a[s + j + half] = (j == 0) ? d : cmul(d, c_w32[j * (32 / LEN)]);
        }
    }
}

template <int LEN>
__device__ __forceinline__ void dit_stage(float2 (&a)[32]) {
    constexpr int half = LEN / 2;
#pragma unroll
    for (int s = 0; s < 32; s += LEN) {
#pragma unroll
        for (int j = 0; j < half; ++j) {
            const float2 u = a[s + j];
            const float2 v = (j == 0) ? a[s + j + half] : cmul(a[s + j + half], c_w32[j * (32 / LEN)]);
            a[s + j] = make_float2(u.x + v.x, u.y + v.y);
            a[s + j + half] = make_float2(u.x - v.x, u.y - v.y);
        }
    }
}

// Radix-2 decimation in frequency, natural order in, bit-reversed order out (forward).
__device__ __forceinline__ void dft32_dif(float2 (&a)[32]) {
    dif_stage<32>(a);
    dif_stage<16>(a);
    dif_stage<8>(a);
    dif_stage<4>(a);
    dif_stage<2>(a);
}

// Radix-2 decimation in time, bit-reversed order in, natural order out (forward).
__device__ __forceinline__ void dft32_dit(float2 (&a)[32]) {
    dit_stage<2>(a);
    dit_stage<4>(a);
    dit_stage<8>(a);
    dit_stage<16>(a);
    dit_stage<32>(a);
}

// kphi(kx, ky, kz): the multiplier. One CTA per (ky, 8 kx) tile. By default Kφ is
// evaluated in step B with float64 sums and products and one float division
// (KPhiFn::fast, within 1.5 ulp of the float64 quotient); DJB_ZPASS_KTABLE = 1 evaluates
// the float64 quotient for the tile into shared memory before the pencils are loaded
// (measured 9% slower on the 1024^3 step).
template <class KPhi>
__global__ void __launch_bounds__(kZThreads, DJB_ZPASS_BLOCKS) k_zpencil_kphi(float2* __restrict__ f, int nh,
                                                                             const float2* __restrict__ wN,
                                                                             KPhi kphi) {
    extern __shared__ __align__(16) float2 s[];  // kZPencils transpose blocks (then Kφ rows)
    const int q = threadIdx.x & (kZPencils - 1);
    const int t = threadIdx.x / kZPencils;  // n2 (steps A, B'), k1 (steps B, A')
    const int ky = blockIdx.y;
    const int kx = blockIdx.x * kZPencils + q;
    const bool active = kx < nh;
#if DJB_ZPASS_KTABLE
    float* const sK = reinterpret_cast<float*>(s + kZPencils * kZPlane);
    for (int e = threadIdx.x; e < kZPencils * kZRes; e += kZThreads) {
        const int qq = e / kZRes, kz = e - qq * kZRes;
        const int kxx = blockIdx.x * kZPencils + qq;
        sK[qq * kZKRow + kz] = (kxx < nh) ? kphi(kxx, ky, kz) : 0.0f;
    }
#endif
    const int64_t zstride = int64_t(kZRes) * nh;
    float2* __restrict__ col = f + int64_t(ky) * nh + (active ? kx : 0);
    float2* const sq = s + q * kZPlane;
    float2 a[32];
    // A: x[t + 32 n1], n1 = 0..31
#pragma unroll
    for (int n1 = 0; n1 < 32; ++n1)
        a[n1] = active ? __ldcs(col + int64_t(t + 32 * n1) * zstride) : make_float2(0.f, 0.f);
    dft32_dif(a);  // a[i] = Y[k1 = brev(i)]
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const int k1 = brev5(i);
        sq[k1 * kZRow + t] = (k1 == 0) ? a[i] : cmul(a[i], __ldg(wN + ((t * k1) & (kZRes - 1))));
    }
    __syncthreads();  // transpose block (and Kφ rows) complete
    // B: thread k1 = t: DFT over n2
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2) a[n2] = sq[t * kZRow + n2];
    dft32_dif(a);  // a[i] = X[t + 32 brev(i)]
#pragma unroll
    for (int i = 0; i < 32; ++i) {
#if DJB_ZPASS_KTABLE
        const float K = sK[q * kZKRow + t + 32 * brev5(i)];
#else
        const float K = kphi.fast(kx, ky, t + 32 * brev5(i));
#endif
        a[i] = make_float2(a[i].x * K, -(a[i].y * K));  // conjugated for the inverse below
    }
    // A': inverse DFT over k2 (input bit-reversed) -> Z[k1 = t][n2], n2 natural; row t of
    // the transpose block is read and written by this thread only
    dft32_dit(a);
#pragma unroll
    for (int n2 = 0; n2 < 32; ++n2) {
        const float2 z = conjf2(a[n2]);
        sq[t * kZRow + n2] = (t == 0 || n2 == 0) ? z : cmul(z, conjf2(__ldg(wN + ((n2 * t) & (kZRes - 1)))));
    }
    __syncthreads();
    // B': thread n2 = t: inverse DFT over k1 -> x[t + 32 n1]
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) a[k1] = conjf2(sq[k1 * kZRow + t]);
    dft32_dif(a);  // a[i] = conj(x[t + 32 brev(i)])
    if (active) {
#pragma unroll
        for (int i = 0; i < 32; ++i) __stcs(col + int64_t(t + 32 * brev5(i)) * zstride, conjf2(a[i]));
    }
}

// ── pencil transforms on thread pairs ───────────────────────────────────────
// The same transform with each 32-point DFT split over two threads (lanes 8 apart):
// thread h of the pair holds points 16h .. 16h + 15. The radix-2 stage of length 32
// pairs point j with j + 16, i.e. the two threads, and exchanges them with one
// shuffle per point; the stages of length 16 .. 2 stay inside each thread. Half the
// registers per thread (16 points) let twice as many warps share an SM, which the pass
// needs to keep enough loads in flight (it is bound by load latency).
#ifndef DJB_ZPASS_PAIR
#define DJB_ZPASS_PAIR 1
#endif
constexpr int kZPairThreads = kZPencils * 64;

template <int LEN>
__device__ __forceinline__ void dif_stage16(float2 (&b)[16]) {
    constexpr int half = LEN / 2;
#pragma unroll
    for (int s = 0; s < 16; s += LEN) {
#pragma unroll
        for (int j = 0; j < half; ++j) {
            const float2 u = b[s + j], v = b[s + j + half];
            b[s + j] = make_float2(u.x + v.x, u.y + v.y);
            const float2 d = make_float2(u.x - v.x, u.y - v.y);
            b[s + j + half] = (j == 0) ? d : cmul(d, c_w32[j * (32 / LEN)]);
        }
    }
}

template <int LEN>
__device__ __forceinline__ void dit_stage16(float2 (&b)[16]) {
    constexpr int half = LEN / 2;
#pragma unroll
    for (int s = 0; s < 16; s += LEN) {
#pragma unroll
        for (int j = 0; j < half; ++j) {
            const float2 u = b[s + j];
            const float2 v = (j == 0) ? b[s + j + half] : cmul(b[s + j + half], c_w32[j * (32 / LEN)]);
            b[s + j] = make_float2(u.x + v.x, u.y + v.y);
            b[s + j + half] = make_float2(u.x - v.x, u.y - v.y);
        }
    }
}

// The partner of the pair is `P` lanes away (P pencils per CTA, P = 8 or 16).
template <int P>
__device__ __forceinline__ float2 shfl_pair(float2 v) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, P), __shfl_xor_sync(0xffffffffu, v.y, P));
}

// Forward DIF over the pair: natural order in, bit-reversed order out (position 16h + i).
template <int P>
__device__ __forceinline__ void dft32_dif_pair(float2 (&b)[16], int h) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const float2 o = shfl_pair<P>(b[j]);
        if (h == 0) {
            b[j] = make_float2(b[j].x + o.x, b[j].y + o.y);
        } else {
            const float2 d = make_float2(o.x - b[j].x, o.y - b[j].y);
            b[j] = (j == 0) ? d : cmul(d, c_w32[j]);
        }
    }
    dif_stage16<16>(b);
    dif_stage16<8>(b);
    dif_stage16<4>(b);
    dif_stage16<2>(b);
}

// Forward DIT over the pair: bit-reversed order in, natural order out.
template <int P>
__device__ __forceinline__ void dft32_dit_pair(float2 (&b)[16], int h) {
    dit_stage16<2>(b);
    dit_stage16<4>(b);
    dit_stage16<8>(b);
    dit_stage16<16>(b);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const float2 m = (h == 1 && j > 0) ? cmul(b[j], c_w32[j]) : b[j];
        const float2 o = shfl_pair<P>(m);
        b[j] = (h == 0) ? make_float2(m.x + o.x, m.y + o.y) : make_float2(o.x - m.x, o.y - m.y);
    }
}

// P pencils per CTA of 64·P threads. Thread (q, h, t) at threadIdx.x = q + P h + 2P t:
// pencil q, half h, and t = n2 (steps A, B') or k1 (steps B, A'); a warp reads 32/P kz
// row pairs of P consecutive kx (8·P bytes each) per load.
template <class KPhi, int P = 8>
__global__ void __launch_bounds__(64 * P, P == 8 ? 2 : 1) k_zpencil_pair(float2* __restrict__ f, int nh,
                                                                         const float2* __restrict__ wN, KPhi kphi) {
    extern __shared__ __align__(16) float2 s[];  // P transpose blocks
    const int q = threadIdx.x & (P - 1);
    const int h = (threadIdx.x / P) & 1;
    const int t = threadIdx.x / (2 * P);
    const int ky = blockIdx.y;
    const int kx = blockIdx.x * P + q;
    const bool active = kx < nh;
    const int64_t zstride = int64_t(kZRes) * nh;
    float2* __restrict__ col = f + int64_t(ky) * nh + (active ? kx : 0);
    float2* const sq = s + q * kZPlane;
    float2 b[16];
    // A: x[t + 32 n1], n1 = 16 h + i
#pragma unroll
    for (int i = 0; i < 16; ++i)
        b[i] = active ? __ldcs(col + int64_t(t + 32 * (16 * h + i)) * zstride) : make_float2(0.f, 0.f);
    dft32_dif_pair<P>(b, h);  // b[i] = Y[k1 = brev(16h + i)]
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int k1 = brev5(16 * h + i);
        sq[k1 * kZRow + t] = (k1 == 0) ? b[i] : cmul(b[i], __ldg(wN + ((t * k1) & (kZRes - 1))));
    }
    __syncthreads();
    // B: thread pair k1 = t: DFT over n2 (this thread: n2 = 16 h + i)
#pragma unroll
    for (int i = 0; i < 16; ++i) b[i] = sq[t * kZRow + 16 * h + i];
    dft32_dif_pair<P>(b, h);  // b[i] = X[t + 32 brev(16h + i)]
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const float K = kphi.fast(kx, ky, t + 32 * brev5(16 * h + i));
        b[i] = make_float2(b[i].x * K, -(b[i].y * K));  // conjugated for the inverse below
    }
    // A': inverse DFT over k2 -> Z[k1 = t][n2 = 16 h + i]; this thread reads and writes
    // only its half of row t
    dft32_dit_pair<P>(b, h);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int n2 = 16 * h + i;
        const float2 z = conjf2(b[i]);
        sq[t * kZRow + n2] = (t == 0 || n2 == 0) ? z : cmul(z, conjf2(__ldg(wN + ((n2 * t) & (kZRes - 1)))));
    }
    __syncthreads();
    // B': thread pair n2 = t: inverse DFT over k1 (this thread: k1 = 16 h + i)
#pragma unroll
    for (int i = 0; i < 16; ++i) b[i] = conjf2(sq[(16 * h + i) * kZRow + t]);
    dft32_dif_pair<P>(b, h);  // b[i] = conj(x[t + 32 brev(16h + i)])
    if (active) {
#pragma unroll
        for (int i = 0; i < 16; ++i) __stcs(col + int64_t(t + 32 * brev5(16 * h + i)) * zstride, conjf2(b[i]));
    }
}

}  // namespace djb
