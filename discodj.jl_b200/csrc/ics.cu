// Second-order LPT initial conditions on the GPU: white noise -> phi(k) -> psi_1, psi_2 ->
// (Psi, Pi) at growth factor D, with cuFFT transforms and fused k-space / real-space
// kernels.
//
// Restates, for n_order = 2:
//   src/ics/grf.jl:118-144   phi(k) = rfft(w) * (-sqrt(P(|k|) (n/L)^3) / k^2), 0 at k = 0, with
//                            P linearly interpolated in a host table (clamped at its ends);
//   src/lpt/nlpt_core.jl     psi_1 = -D phi (D_a = i k_a, the Nyquist entries zeroed);
//                            the second-order source mu2 = sum_{a<b} (psi_aa psi_bb - psi_ab^2),
//                            psi_ab = D_b psi_a, evaluated on the 3/2-padded grid (ext = 3n/2:
//                            spectra embedded with the Nyquist planes dropped, scaled by
//                            (ext/n)^3; products in real space; cropped back, scaled by
//                            (n/ext)^3); psi_2 = -1/k^2 (DC: -1) * D (-3/7 mu2);
//   src/nbody/run_nbody.jl:180-208   Psi = D psi_1 + D^2 psi_2, Pi = dPsi/dD = psi_1 + 2 D psi_2.
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

extern "C" int djb_lpt2_ics(const float* white, int32_t n, double boxsize, const double* k_tab, const double* p_tab,
                            int32_t npk, double D, float* psi, float* pi, int32_t device, void* stream) {
    djb::clear_error();
    if (!white || !k_tab || !p_tab || !psi || !pi) return fail(DJB_ERR_INVALID, "null argument");
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
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cufftHandle r2c_n = 0, c2r_n = 0, r2c_e = 0, c2r_e = 0;
    float2 *phi = nullptr, *spec = nullptr, *espec = nullptr, *s1 = nullptr, *s2 = nullptr;
    float *ediag = nullptr, *emu = nullptr, *eoff = nullptr, *f1 = nullptr, *f2 = nullptr;
    double *dkt = nullptr, *dpt = nullptr;
    ICS_CUDA(cudaSetDevice(device));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&phi), sizeof(float2) * Ns, st));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&spec), sizeof(float2) * Ns * 2, st));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&espec), sizeof(float2) * Es, st));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ediag), sizeof(float) * E * 3, st));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&emu), sizeof(float) * E, st));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&eoff), sizeof(float) * E, st));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&f1), sizeof(float) * N * 2, st));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dkt), sizeof(double) * npk, st));
    ICS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dpt), sizeof(double) * npk, st));
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
        ICS_FFT(cufftExecC2R(c2r_e, reinterpret_cast<cufftComplex*>(espec), ediag + a * E));
    }
    k_mu2_diag<<<grid_of(E), kT, 0, st>>>(ediag, ediag + E, ediag + 2 * E, E, emu);
    for (int p = 0; p < 3; ++p) {
        const int a = p == 2 ? 1 : 0, b = p == 0 ? 1 : 2;   // (0,1), (0,2), (1,2)
        k_pad_deriv<<<grid_of(Es), kT, 0, st>>>(phi, n, ext, float(dk), a, b, espec);
        ICS_FFT(cufftExecC2R(c2r_e, reinterpret_cast<cufftComplex*>(espec), eoff));
        k_mu2_sub<<<grid_of(E), kT, 0, st>>>(eoff, E, emu);
    }
    ICS_CUDA(cudaGetLastError());
    ICS_FFT(cufftExecR2C(r2c_e, emu, reinterpret_cast<cufftComplex*>(espec)));
    // psi_1, psi_2 per component, then Psi and Pi
    for (int a = 0; a < 3; ++a) {
        k_crop_assemble<<<grid_of(Ns), kT, 0, st>>>(espec, phi, n, ext, float(dk), a, s1, s2);
        ICS_FFT(cufftExecC2R(c2r_n, reinterpret_cast<cufftComplex*>(s1), f1));
        ICS_FFT(cufftExecC2R(c2r_n, reinterpret_cast<cufftComplex*>(s2), f2));
        k_lpt_combine<<<grid_of(N), kT, 0, st>>>(f1, f2, N, float(D), psi + a * N, pi + a * N);
    }
    ICS_CUDA(cudaGetLastError());
    ICS_CUDA(cudaStreamSynchronize(st));
done:
    for (void* q : {static_cast<void*>(phi), static_cast<void*>(spec), static_cast<void*>(espec),
                    static_cast<void*>(ediag), static_cast<void*>(emu), static_cast<void*>(eoff),
                    static_cast<void*>(f1), static_cast<void*>(dkt), static_cast<void*>(dpt)})
        if (q) cudaFreeAsync(q, st);
    cudaStreamSynchronize(st);
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}
