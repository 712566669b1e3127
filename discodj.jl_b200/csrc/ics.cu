// Second- and third-order LPT initial conditions on the GPU: white noise -> phi(k) ->
// psi_1, psi_2 (, psi_3) -> (Psi, Pi) at growth factor D, with cuFFT transforms and fused
// k-space / real-space kernels.
//
// Restates, for n_order = 2 and 3 (EdS growth, as the reference's `compute_core`):
//   src/ics/grf.jl:118-144   phi(k) = rfft(w) * (-sqrt(P(|k|) (n/L)^3) / k^2), 0 at k = 0, with
//                            P linearly interpolated in a host table (clamped at its ends);
//   src/lpt/nlpt_core.jl     psi_1 = -D phi (D_a = i k_a, the Nyquist entries zeroed);
//                            the second-order source mu2 = sum_{a<b} (psi_aa psi_bb - psi_ab^2),
//                            psi_ab = D_b psi_a, evaluated on the 3/2-padded grid (ext = 3n/2:
//                            spectra embedded with the Nyquist planes dropped, scaled by
//                            (ext/n)^3; products in real space; cropped back, scaled by
//                            (n/ext)^3); psi_2 = -1/k^2 (DC: -1) * D (-3/7 mu2);
//                            third order (nlpt_core.jl:223-280, i = 3): the longitudinal source
//                            -5/9 mu2(psi_1, psi_2) - 1/3 mu3(psi_1, psi_1, psi_1) and the
//                            transverse source 1/3 C(psi_1, psi_2), products of the padded
//                            derivative fields in real space with the reference's index and
//                            sign tables; psi_3 = il (D fL - D x C) (the curl form of
//                            nlpt_core.jl:267-280);
//   src/nbody/run_nbody.jl:180-208   Psi = sum_m D^m psi_m, Pi = dPsi/dD = sum_m m D^(m-1) psi_m.
//
// Layout: real fields of n^3 floats with x fastest ([k][j][i], the library's particle
// component blocks); cuFFT's R2C then halves x, so spectra are [kz][ky][kx], kx in
// [0, n/2]. Every multiplier here treats the three axes alike (the Nyquist zeroed on each),
// so halving x instead of z changes only round-off. Transforms are unnormalised; the
// inverse ones are scaled by 1/N in the kernels that follow them.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.h"

using djb::fail;

namespace {

#define ICS_CUDA(expr)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (expr);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            rc = fail(DJB_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));         \
            goto done;                                                                       \
        }                                                                                    \
    } while (0)
#define ICS_FFT(expr)                                                                        \
    do {                                                                                     \
        cufftResult r_ = (expr);                                                             \
        if (r_ != CUFFT_SUCCESS) {                                                           \
            rc = fail(DJB_ERR_CUFFT, "%s failed (%d)", #expr, int(r_));                      \
            goto done;                                                                       \
        }                                                                                    \
    } while (0)

constexpr int kT = 256;

inline int grid_of(int64_t n) { return int(std::min<int64_t>((n + kT - 1) / kT, int64_t(148) * 32)); }

// Signed mode index of a full axis; the Nyquist index n/2 is kept positive.
__device__ __forceinline__ int mode_full(int i, int n) { return i <= n / 2 ? i : i - n; }

// The derivative multiplier's real factor k_a (i k_a), zeroed at the Nyquist index.
__device__ __forceinline__ float dk_full(int i, int n, float dk) { return i == n / 2 ? 0.0f : float(mode_full(i, n)) * dk; }
__device__ __forceinline__ float dk_half(int i, int n, float dk) { return i == n / 2 ? 0.0f : float(i) * dk; }

// spec *= -sqrt(P(|k|) (n/L)^3) / k^2 (0 at k = 0); P by linear interpolation in (kt, pt).
__global__ void k_fphi(float2* __restrict__ spec, int n, double dk, double amp, const double* __restrict__ kt,
                       const double* __restrict__ pt, int npk) {
    const int nh = n / 2 + 1;
    const int64_t total = int64_t(n) * n * nh;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int kx = int(t % nh);
        const int64_t r = t / nh;
        const int ky = int(r % n), kz = int(r / n);
        const double mx = kx, my = mode_full(ky, n), mz = mode_full(kz, n);
        const double k2 = (mx * mx + my * my + mz * mz) * dk * dk;
        double s = 0.0;
        if (k2 > 0.0) {
            const double k = sqrt(k2);
            double P;
            if (k <= kt[0]) {
                P = pt[0];
            } else if (k >= kt[npk - 1]) {
                P = pt[npk - 1];
            } else {
                int lo = 0, hi = npk - 1;  // kt[lo] < k <= kt[hi]
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (kt[mid] < k) lo = mid;
                    else hi = mid;
                }
                const double f = (k - kt[lo]) / (kt[hi] - kt[lo]);
                P = pt[lo] + f * (pt[hi] - pt[lo]);
            }
            s = -sqrt(P * amp) / k2;
        }
        const float2 v = spec[t];
        spec[t] = make_float2(float(v.x * s), float(v.y * s));
    }
}

// The ext-grid spectrum of psi_ab = D_b psi_a = (i k_b)(-(i k_a) phi) = k_a k_b phi
// (Nyquist-zeroed factors), embedded from the n grid (index h = n/2 dropped on every axis,
// the upper half of the full axes moved to the top of the ext axes) and scaled by
// (ext/n)^3 / ext^3 = 1/n^3, the inverse transform's normalisation folded in.
__global__ void k_pad_deriv(const float2* __restrict__ phi, int n, int ext, float dk, int a, int b,
                            float2* __restrict__ out) {
    const int eh = ext / 2 + 1, h = n / 2;
    const int64_t total = int64_t(ext) * ext * eh;
    const float scale = 1.0f / (float(n) * float(n) * float(n));
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int ex = int(t % eh);
        const int64_t r = t / eh;
        const int ey = int(r % ext), ez = int(r / ext);
        // source indices on the n grid (or none)
        const int sx = ex < h ? ex : -1;
        const int sy = ey < h ? ey : (ey > ext - h ? ey - ext + n : -1);
        const int sz = ez < h ? ez : (ez > ext - h ? ez - ext + n : -1);
        float2 v = make_float2(0.0f, 0.0f);
        if (sx >= 0 && sy >= 0 && sz >= 0) {
            const float2 p = phi[(int64_t(sz) * n + sy) * (h + 1) + sx];
            // the derivative factors of the source mode: the ext grid's own factors agree with the
            // n grid's on the embedded modes (the dropped Nyquist planes carry the only zeros)
            const float k3[3] = {dk_half(sx, n, dk), dk_full(sy, n, dk), dk_full(sz, n, dk)};
            const float f = k3[a] * k3[b] * scale;
            v = make_float2(p.x * f, p.y * f);
        }
        out[t] = v;
    }
}

// mu2 = a b + a c + b c (ext grid, real).
__global__ void k_mu2_diag(const float* __restrict__ a, const float* __restrict__ b, const float* __restrict__ c,
                           int64_t m, float* __restrict__ mu) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m; t += int64_t(gridDim.x) * blockDim.x) {
        const float x = a[t], y = b[t], z = c[t];
        mu[t] = x * y + x * z + y * z;
    }
}

// mu2 -= d^2.
__global__ void k_mu2_sub(const float* __restrict__ d, int64_t m, float* __restrict__ mu) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m; t += int64_t(gridDim.x) * blockDim.x) {
        const float x = d[t];
        mu[t] -= x * x;
    }
}

// psi_2 component a (n grid spectrum): the cropped source (n/ext)^3 mu2(K), times
// -3/7, times i k_a, times -1/k^2 (-1 at k = 0); the 1/n^3 of the inverse transform folded
// in. psi_1 component a: -(i k_a) phi / n^3. Both written as spectra for C2R.
__global__ void k_crop_assemble(const float2* __restrict__ mu, const float2* __restrict__ phi, int n, int ext,
                                float dk, int a, float2* __restrict__ psi1, float2* __restrict__ psi2) {
    const int nh = n / 2 + 1, eh = ext / 2 + 1, h = n / 2;
    const int64_t total = int64_t(n) * n * nh;
    const float inv_n3 = 1.0f / (float(n) * float(n) * float(n));
    const float crop = float(double(n) * n * n / (double(ext) * ext * ext));
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int kx = int(t % nh);
        const int64_t r = t / nh;
        const int ky = int(r % n), kz = int(r / n);
        const float k3[3] = {dk_half(kx, n, dk), dk_full(ky, n, dk), dk_full(kz, n, dk)};
        // -(i k_a) phi
        const float2 p = phi[t];
        psi1[t] = make_float2(k3[a] * p.y * inv_n3, -k3[a] * p.x * inv_n3);
        float2 q = make_float2(0.0f, 0.0f);
        if (kx != h && ky != h && kz != h) {
            const int ey = ky < h ? ky : ky - n + ext, ez = kz < h ? kz : kz - n + ext;
            const float2 m = mu[(int64_t(ez) * ext + ey) * eh + kx];
            const float fl = -3.0f / 7.0f * crop;
            const float mx = float(kx), my = float(mode_full(ky, n)), mz = float(mode_full(kz, n));
            const float k2 = (mx * mx + my * my + mz * mz) * dk * dk;
            const float il = (kx == 0 && ky == 0 && kz == 0) ? -1.0f : -1.0f / k2;
            // il * (i k_a) * fl * m
            const float g = il * k3[a] * fl * inv_n3;
            q = make_float2(-g * m.y, g * m.x);
        }
        psi2[t] = q;
    }
}

// Psi = D psi1 + D^2 psi2, Pi = psi1 + 2 D psi2 (component block c of 3).
__global__ void k_lpt_combine(const float* __restrict__ p1, const float* __restrict__ p2, int64_t m, float D,
                              float* __restrict__ psi, float* __restrict__ pi) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m; t += int64_t(gridDim.x) * blockDim.x) {
        const float a = p1[t], b = p2[t];
        psi[t] = D * a + (D * D) * b;
        pi[t] = a + (2.0f * D) * b;
    }
}

// Symmetric 3x3 index (a, b in 0..2) -> storage slot: diagonal 0..2, then (0,1), (0,2), (1,2).
__device__ __forceinline__ int sym3(int a, int b) {
    if (a == b) return a;
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    return lo == 0 ? (hi == 1 ? 3 : 4) : 5;
}

// Ext-grid spectrum of D_b psi_2,a (psi_2 = il D fL2, fL2 = fl * mu2(k) the cropped source):
// (i k_b)(i k_a) il fl mu2_ext(k_e) on the embedded modes (0 elsewhere), scaled by 1/n^3:
// the pad factor (ext/n)^3 and the inverse transform's 1/ext^3.
__global__ void k_q_deriv(const float2* __restrict__ mu, int n, int ext, float dk, float fl, int a, int b,
                          float2* __restrict__ out) {
    const int eh = ext / 2 + 1, h = n / 2;
    const int64_t total = int64_t(ext) * ext * eh;
    const float scale = 1.0f / (float(n) * float(n) * float(n));
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int ex = int(t % eh);
        const int64_t r = t / eh;
        const int ey = int(r % ext), ez = int(r / ext);
        const int sx = ex < h ? ex : -1;
        const int sy = ey < h ? ey : (ey > ext - h ? ey - ext + n : -1);
        const int sz = ez < h ? ez : (ez > ext - h ? ez - ext + n : -1);
        float2 v = make_float2(0.0f, 0.0f);
        if (sx >= 0 && sy >= 0 && sz >= 0) {
            const float k3[3] = {dk_half(sx, n, dk), dk_full(sy, n, dk), dk_full(sz, n, dk)};
            const float mx = float(sx), my = float(mode_full(sy, n)), mz = float(mode_full(sz, n));
            const float k2 = (mx * mx + my * my + mz * mz) * dk * dk;
            const float il = (sx == 0 && sy == 0 && sz == 0) ? -1.0f : -1.0f / k2;
            const float f = -k3[a] * k3[b] * il * fl * scale;
            const float2 m = mu[t];
            v = make_float2(m.x * f, m.y * f);
        }
        out[t] = v;
    }
}

// The third-order sources at every ext-grid point, from P_ab = D_b psi_1,a and
// Q_ab = D_b psi_2,a (symmetric, six slots each; P and Q point at six fields of E floats):
//   fL3 = -5/9 mu2(psi_1, psi_2) - 1/3 mu3(psi_1, psi_1, psi_1),   C3_c = 1/3 C_c(psi_1, psi_2),
// with mu2, C and mu3 the sums of nlpt_core.jl:223-263 (1-based index tables as there).
// Written in place of Q's first four slots (each thread reads its point's inputs first).
__global__ void k_lpt3_source(const float* __restrict__ P, float* __restrict__ Q, int64_t E) {
    constexpr int MI[12] = {1, 1, 2, 3, 2, 2, 3, 1, 3, 3, 1, 2}, MJ[12] = {2, 3, 1, 1, 3, 1, 2, 2, 1, 2, 3, 3};
    constexpr int MK[12] = {1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3}, ML[12] = {2, 3, 2, 3, 3, 1, 3, 1, 1, 2, 1, 2};
    constexpr float MS[12] = {1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1};
    constexpr int CI[6] = {1, 1, 2, 2, 3, 3}, CK[6] = {2, 3, 2, 3, 2, 3}, CL[6] = {3, 2, 3, 2, 3, 2};
    constexpr float CS[6] = {1, -1, 1, -1, 1, -1};
    constexpr int UK[6] = {1, 1, 2, 2, 3, 3}, UL[6] = {2, 3, 3, 1, 1, 2}, UM[6] = {3, 2, 1, 3, 2, 1};
    constexpr float US[6] = {1, -1, 1, -1, 1, -1};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < E; t += int64_t(gridDim.x) * blockDim.x) {
        float p[6], q[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            p[i] = P[i * E + t];
            q[i] = Q[i * E + t];
        }
        auto pa = [&](int m, int ax) { return p[sym3(m - 1, ax - 1)]; };
        auto qa = [&](int m, int ax) { return q[sym3(m - 1, ax - 1)]; };
        float mu2 = 0.0f;
#pragma unroll
        for (int i = 0; i < 12; ++i) mu2 += MS[i] * (pa(MI[i], MK[i]) * qa(MJ[i], ML[i]));
        float c3[3];
#pragma unroll
        for (int sh = 0; sh < 3; ++sh) {
            float acc = 0.0f;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const int ci = (CI[i] - 1 + sh) % 3 + 1, ck = (CK[i] - 1 + sh) % 3 + 1, cl = (CL[i] - 1 + sh) % 3 + 1;
                acc += CS[i] * (pa(ci, ck) * qa(ci, cl));
            }
            c3[sh] = acc;
        }
        float mu3 = 0.0f;
#pragma unroll
        for (int i = 0; i < 6; ++i) mu3 += US[i] * (pa(1, UK[i]) * (pa(2, UL[i]) * pa(3, UM[i])));
        Q[t] = (-5.0f / 9.0f) * mu2 - (1.0f / 3.0f) * mu3;
#pragma unroll
        for (int c = 0; c < 3; ++c) Q[(c + 1) * E + t] = (1.0f / 3.0f) * c3[c];
    }
}

// psi_3 component a (n grid spectrum, 1/n^3 folded in): il (i k_a FL - (i k_b C_c - i k_c C_b)),
// (a, b, c) cyclic, FL and C_c the cropped ext spectra src[0] and src[1 + c] (each Es modes).
__global__ void k_crop_assemble3(const float2* __restrict__ src, int64_t Es, int n, int ext, float dk, int a,
                                 float2* __restrict__ psi3) {
    const int nh = n / 2 + 1, eh = ext / 2 + 1, h = n / 2;
    const int64_t total = int64_t(n) * n * nh;
    const float inv_n3 = 1.0f / (float(n) * float(n) * float(n));
    const float crop = float(double(n) * n * n / (double(ext) * ext * ext));
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int kx = int(t % nh);
        const int64_t r = t / nh;
        const int ky = int(r % n), kz = int(r / n);
        float2 q = make_float2(0.0f, 0.0f);
        if (kx != h && ky != h && kz != h) {
            const int ey = ky < h ? ky : ky - n + ext, ez = kz < h ? kz : kz - n + ext;
            const int64_t e = (int64_t(ez) * ext + ey) * eh + kx;
            const float k3[3] = {dk_half(kx, n, dk), dk_full(ky, n, dk), dk_full(kz, n, dk)};
            const float2 fl = src[e], cb = src[(1 + b) * Es + e], cc = src[(1 + c) * Es + e];
            const float mx = float(kx), my = float(mode_full(ky, n)), mz = float(mode_full(kz, n));
            const float k2 = (mx * mx + my * my + mz * mz) * dk * dk;
            const float il = (kx == 0 && ky == 0 && kz == 0) ? -1.0f : -1.0f / k2;
            // w = k_a FL - (k_b C_c - k_c C_b); psi3 = il * i * w * crop / n^3
            const float wx = k3[a] * fl.x - (k3[b] * cc.x - k3[c] * cb.x);
            const float wy = k3[a] * fl.y - (k3[b] * cc.y - k3[c] * cb.y);
            const float g = il * crop * inv_n3;
            q = make_float2(-g * wy, g * wx);
        }
        psi3[t] = q;
    }
}

// Psi += D^3 psi3, Pi += 3 D^2 psi3.
__global__ void k_lpt_combine3(const float* __restrict__ p3, int64_t m, float D, float* __restrict__ psi,
                               float* __restrict__ pi) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m; t += int64_t(gridDim.x) * blockDim.x) {
        const float c = p3[t];
        psi[t] += (D * D * D) * c;
        pi[t] += (3.0f * D * D) * c;
    }
}

// cuFFT plans kept per (device, size, kind) for the life of the library: creating a 768^3
// plan takes longer than the whole 512^3 computation.
std::mutex g_plan_mu;
std::map<std::tuple<int, int, int>, cufftHandle> g_plans;

cufftResult cached_plan(int device, int size, cufftType kind, cufftHandle* out) {
    std::lock_guard<std::mutex> lock(g_plan_mu);
    const auto key = std::make_tuple(device, size, int(kind));
    auto it = g_plans.find(key);
    if (it != g_plans.end()) {
        *out = it->second;
        return CUFFT_SUCCESS;
    }
    cufftHandle h = 0;
    const cufftResult r = cufftPlan3d(&h, size, size, size, kind);
    if (r != CUFFT_SUCCESS) return r;
    g_plans[key] = h;
    *out = h;
    return CUFFT_SUCCESS;
}

}  // namespace

namespace {

// Work area of one call, carved from one block: byte offsets of phi, the two n-grid
// spectra, the ext spectrum of mu2, P, mu2, Q, the second ext spectrum, the two n-grid
// real fields and the P(k) table (each 256-byte aligned).
struct IcsLayout {
    enum { kPhi, kSpec, kEspec, kP, kMu, kQ, kEspec2, kF, kKt, kPt, kCount };
    int64_t off[kCount];
    int64_t total;
};

IcsLayout ics_layout(int n, int order, int npk) {
    const int ext = 3 * n / 2;
    const int64_t N = int64_t(n) * n * n, Ns = int64_t(n) * n * (n / 2 + 1);
    const int64_t E = int64_t(ext) * ext * ext, Es = int64_t(ext) * ext * (ext / 2 + 1);
    const bool third = order == 3;
    const int64_t bytes[IcsLayout::kCount] = {8 * Ns,        16 * Ns,       8 * Es,      4 * E * (third ? 6 : 4),
                                              4 * E,         third ? 24 * E : 0,       third ? 8 * Es : 0,
                                              8 * N,         8 * int64_t(npk),         8 * int64_t(npk)};
    IcsLayout l;
    int64_t at = 0;
    for (int i = 0; i < IcsLayout::kCount; ++i) {
        l.off[i] = at;
        at += (bytes[i] + 255) / 256 * 256;
    }
    l.total = at;
    return l;
}

int lpt_ics(const float* white, int32_t n, double boxsize, const double* k_tab, const double* p_tab, int32_t npk,
            int32_t order, double D, float* psi, float* pi, void* work, int64_t work_bytes, int32_t device,
            void* stream) {
    djb::clear_error();
    if (!white || !k_tab || !p_tab || !psi || !pi) return fail(DJB_ERR_INVALID, "null argument");
    if (order != 2 && order != 3) return fail(DJB_ERR_INVALID, "n_order must be 2 or 3");
    if (n < 4 || (n & 1) || (3 * n) % 2 != 0 || ((3 * n / 2) & 1))
        return fail(DJB_ERR_INVALID, "n must be a multiple of 4 (n and the 3/2-padded 3n/2 even)");
    if (npk < 2) return fail(DJB_ERR_INVALID, "the P(k) table needs at least 2 points");
    if (!(boxsize > 0)) return fail(DJB_ERR_INVALID, "boxsize must be positive");
    int prev = -1;
    cudaGetDevice(&prev);
    int rc = DJB_OK;
    const int ext = 3 * n / 2;
    const int nh = n / 2 + 1, eh = ext / 2 + 1;
    const int64_t N = int64_t(n) * n * n, Ns = int64_t(n) * n * nh;
    const int64_t E = int64_t(ext) * ext * ext, Es = int64_t(ext) * ext * eh;
    const double dk = 2 * M_PI / boxsize;
    const bool third = order == 3;
    const IcsLayout lay = ics_layout(n, order, npk);
    const float crop = float(double(n) * n * n / (double(E)));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cufftHandle r2c_n = 0, c2r_n = 0, r2c_e = 0, c2r_e = 0;
    float2 *phi = nullptr, *spec = nullptr, *espec = nullptr, *espec2 = nullptr, *s1 = nullptr, *s2 = nullptr;
    float *P = nullptr, *Q = nullptr, *emu = nullptr, *f1 = nullptr, *f2 = nullptr;
    double *dkt = nullptr, *dpt = nullptr;
    float2* src3 = nullptr;   // third order: the four source spectra, over P
    uint8_t* owned = nullptr;
    uint8_t* base = static_cast<uint8_t*>(work);
    if (work && work_bytes < lay.total)
        return fail(DJB_ERR_INVALID, "work area of %lld bytes, %lld needed", (long long)work_bytes,
                    (long long)lay.total);
    ICS_CUDA(cudaSetDevice(device));
    if (!base) {
        ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&owned), size_t(lay.total), st));
        base = owned;
    }
    phi = reinterpret_cast<float2*>(base + lay.off[IcsLayout::kPhi]);
    spec = reinterpret_cast<float2*>(base + lay.off[IcsLayout::kSpec]);
    espec = reinterpret_cast<float2*>(base + lay.off[IcsLayout::kEspec]);
    P = reinterpret_cast<float*>(base + lay.off[IcsLayout::kP]);
    emu = reinterpret_cast<float*>(base + lay.off[IcsLayout::kMu]);
    if (third) {
        Q = reinterpret_cast<float*>(base + lay.off[IcsLayout::kQ]);
        espec2 = reinterpret_cast<float2*>(base + lay.off[IcsLayout::kEspec2]);
    }
    f1 = reinterpret_cast<float*>(base + lay.off[IcsLayout::kF]);
    dkt = reinterpret_cast<double*>(base + lay.off[IcsLayout::kKt]);
    dpt = reinterpret_cast<double*>(base + lay.off[IcsLayout::kPt]);
    s1 = spec;
    s2 = spec + Ns;
    f2 = f1 + N;
    ICS_CUDA(cudaMemcpyAsync(dkt, k_tab, sizeof(double) * npk, cudaMemcpyHostToDevice, st));
    ICS_CUDA(cudaMemcpyAsync(dpt, p_tab, sizeof(double) * npk, cudaMemcpyHostToDevice, st));
    ICS_FFT(cached_plan(device, n, CUFFT_R2C, &r2c_n));
    ICS_FFT(cached_plan(device, n, CUFFT_C2R, &c2r_n));
    ICS_FFT(cached_plan(device, ext, CUFFT_R2C, &r2c_e));
    ICS_FFT(cached_plan(device, ext, CUFFT_C2R, &c2r_e));
    ICS_FFT(cufftSetStream(r2c_n, st));
    ICS_FFT(cufftSetStream(c2r_n, st));
    ICS_FFT(cufftSetStream(r2c_e, st));
    ICS_FFT(cufftSetStream(c2r_e, st));
    // phi(k)
    ICS_FFT(cufftExecR2C(r2c_n, const_cast<float*>(white), reinterpret_cast<cufftComplex*>(phi)));
    k_fphi<<<grid_of(Ns), kT, 0, st>>>(phi, n, dk, std::pow(double(n) / boxsize, 3), dkt, dpt, npk);
    ICS_CUDA(cudaGetLastError());
    // mu2 on the ext grid: the three diagonal second derivatives, then the off-diagonal squares
    for (int a = 0; a < 3; ++a) {
        k_pad_deriv<<<grid_of(Es), kT, 0, st>>>(phi, n, ext, float(dk), a, a, espec);
        ICS_FFT(cufftExecC2R(c2r_e, reinterpret_cast<cufftComplex*>(espec), P + a * E));
    }
    k_mu2_diag<<<grid_of(E), kT, 0, st>>>(P, P + E, P + 2 * E, E, emu);
    for (int p = 0; p < 3; ++p) {
        const int a = p == 2 ? 1 : 0, b = p == 0 ? 1 : 2;   // (0,1), (0,2), (1,2): slots 3, 4, 5
        float* off = P + (third ? 3 + p : 3) * E;
        k_pad_deriv<<<grid_of(Es), kT, 0, st>>>(phi, n, ext, float(dk), a, b, espec);
        ICS_FFT(cufftExecC2R(c2r_e, reinterpret_cast<cufftComplex*>(espec), off));
        k_mu2_sub<<<grid_of(E), kT, 0, st>>>(off, E, emu);
    }
    ICS_CUDA(cudaGetLastError());
    ICS_FFT(cufftExecR2C(r2c_e, emu, reinterpret_cast<cufftComplex*>(espec)));
    src3 = reinterpret_cast<float2*>(P);
    if (third) {
        // Q_ab = D_b psi_2,a on the ext grid from the mu2 spectrum
        const float fl = -3.0f / 7.0f * crop;
        for (int slot = 0; slot < 6; ++slot) {
            const int a = slot < 3 ? slot : (slot == 5 ? 1 : 0);
            const int b = slot < 3 ? slot : (slot == 3 ? 1 : 2);
            k_q_deriv<<<grid_of(Es), kT, 0, st>>>(espec, n, ext, float(dk), fl, a, b, espec2);
            ICS_FFT(cufftExecC2R(c2r_e, reinterpret_cast<cufftComplex*>(espec2), Q + slot * E));
        }
        k_lpt3_source<<<grid_of(E), kT, 0, st>>>(P, Q, E);
        ICS_CUDA(cudaGetLastError());
        for (int f = 0; f < 4; ++f)
            ICS_FFT(cufftExecR2C(r2c_e, Q + f * E, reinterpret_cast<cufftComplex*>(src3 + f * Es)));
    }
    // psi_1, psi_2 (, psi_3) per component, then Psi and Pi
    for (int a = 0; a < 3; ++a) {
        k_crop_assemble<<<grid_of(Ns), kT, 0, st>>>(espec, phi, n, ext, float(dk), a, s1, s2);
        ICS_FFT(cufftExecC2R(c2r_n, reinterpret_cast<cufftComplex*>(s1), f1));
        ICS_FFT(cufftExecC2R(c2r_n, reinterpret_cast<cufftComplex*>(s2), f2));
        k_lpt_combine<<<grid_of(N), kT, 0, st>>>(f1, f2, N, float(D), psi + a * N, pi + a * N);
        if (third) {
            k_crop_assemble3<<<grid_of(Ns), kT, 0, st>>>(src3, Es, n, ext, float(dk), a, s1);
            ICS_FFT(cufftExecC2R(c2r_n, reinterpret_cast<cufftComplex*>(s1), f1));
            k_lpt_combine3<<<grid_of(N), kT, 0, st>>>(f1, N, float(D), psi + a * N, pi + a * N);
        }
    }
    ICS_CUDA(cudaGetLastError());
    ICS_CUDA(cudaStreamSynchronize(st));
done:
    if (owned) cudaFreeAsync(owned, st);
    cudaStreamSynchronize(st);
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

}  // namespace

extern "C" int djb_lpt2_ics(const float* white, int32_t n, double boxsize, const double* k_tab, const double* p_tab,
                            int32_t npk, double D, float* psi, float* pi, int32_t device, void* stream) {
    return lpt_ics(white, n, boxsize, k_tab, p_tab, npk, 2, D, psi, pi, nullptr, 0, device, stream);
}

extern "C" int djb_lpt_ics_work_bytes(int32_t n, int32_t n_order, int32_t npk, int64_t* bytes) {
    djb::clear_error();
    if (!bytes) return fail(DJB_ERR_INVALID, "null argument");
    if (n_order != 2 && n_order != 3) return fail(DJB_ERR_INVALID, "n_order must be 2 or 3");
    if (n < 4 || (n & 3)) return fail(DJB_ERR_INVALID, "n must be a multiple of 4 (n and the 3/2-padded 3n/2 even)");
    if (npk < 2) return fail(DJB_ERR_INVALID, "the P(k) table needs at least 2 points");
    *bytes = ics_layout(n, n_order, npk).total;
    return DJB_OK;
}

extern "C" int djb_lpt_ics(const float* white, int32_t n, double boxsize, const double* k_tab, const double* p_tab,
                           int32_t npk, int32_t n_order, double D, float* psi, float* pi, void* work,
                           int64_t work_bytes, int32_t device, void* stream) {
    return lpt_ics(white, n, boxsize, k_tab, p_tab, npk, n_order, D, psi, pi, work, work_bytes, device, stream);
}
