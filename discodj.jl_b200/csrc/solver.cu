// libdjb200 PM solver: device state, cuFFT plans, and the orchestration of one
// force evaluation / one drift-kick-drift step (the hot path of DiscoDJNative's
// `run_nbody`, native/DiscoDJNative/src/nbody/pm.jl:466-521 and run_nbody.jl:155-163).
//
// One step, for each group of interlacing shifts (up to kMaxGroup meshes live):
//   k_scatter      drift Psi += dd1*Mom (first group only), X = q + Psi + shift,
//                  W-order mass assignment into the group's meshes
//   [resampling]   extra particle sets from the Lagrangian sheet (pm.jl:443-464)
//   cuFFT R2C      in place, per mesh
//   k_kspace_*     x Kφ (Green's function, deconvolution, 1/(ρ̄ n_sets N)), and for
//                  grad_order 0 the ik gradient into three spectra
//   cuFFT C2R      in place (unnormalised; 1/N folded into Kφ)
//   k_gather_*     force interpolation; finite-difference gradients are applied to
//                  the potential inside the gather; the last group finishes the
//                  mean over shifts, the kick Mom = a*Mom + b*acc and the drift
//                  Psi += dd2*Mom
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <new>
#include <string>
#include <vector>

#include "common.h"
#include "pm_kernels.cuh"
#include "snapshot.h"

using djb::fail;

namespace {

constexpr int kMaxGroup = 2;  // interlacing meshes processed per particle pass
constexpr int kThreads = 256;

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(DJB_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));      \
    } while (0)

#define CUFFT_TRY(expr)                                                                     \
    do {                                                                                    \
        cufftResult r_ = (expr);                                                            \
        if (r_ != CUFFT_SUCCESS) return fail(DJB_ERR_CUFFT, "%s failed: cufft status %d", #expr, int(r_)); \
    } while (0)

// Shift list of the `dealias` decorator (pm.jl:237-246), in the same order.
std::vector<double> aa_shifts(int aa, double dh) {
    std::vector<double> s;
    auto push = [&](double a, double b, double c) {
        s.push_back(a);
        s.push_back(b);
        s.push_back(c);
    };
    if (aa == 0) {
        push(0, 0, 0);
    } else if (aa == -1) {
        push(dh, dh, dh);
    } else if (aa == 1) {
        push(0, 0, 0);
        push(dh, dh, dh);
    } else {
        const double v[2] = {0.0, dh};
        for (double a : v)
            for (double b : v)
                for (double c : v) push(a, b, c);
        if (aa == 3) {
            const double q = dh / 2, u[2] = {-q, q};
            for (double a : u)
                for (double b : u)
                    for (double c : u) push(a, b, c);
        }
    }
    return s;
}

// pm.jl:233-234: offsets (0..nr-1)/nr per axis, last axis fastest, zero offset dropped.
std::vector<double> resample_shifts(int nr) {
    std::vector<double> s;
    for (int a = 0; a < nr; ++a)
        for (int b = 0; b < nr; ++b)
            for (int c = 0; c < nr; ++c) {
                if (a == 0 && b == 0 && c == 0) continue;
                s.push_back(double(a) / nr);
                s.push_back(double(b) / nr);
                s.push_back(double(c) / nr);
            }
    return s;
}

struct Shift3 {
    float x, y, z;
};

struct GroupShifts {
    Shift3 s[kMaxGroup];
};

}  // namespace

// ─────────────────────────────────────────────────────────────────────────────
// kernels
// ─────────────────────────────────────────────────────────────────────────────
namespace djb {

// Mass assignment of NS shifted copies of the particles (pm.jl:57-74; interlacing
// copies as in pm.jl:515-517). When `mom` is non-null the first drift of the
// step is applied first and written back: Psi <- Psi + dd1*Mom (run_nbody.jl:156).
// `perm` (optional): thread t takes particle perm[t].
template <int W, int NS>
__global__ void __launch_bounds__(kThreads) k_scatter(
    float* __restrict__ psi, const float* __restrict__ mom, float dd1, const float* __restrict__ q1,
    int n, int64_t np, float L, int res, int pitch, GroupShifts sh, float* __restrict__ mesh0,
    float* __restrict__ mesh1, int* err, const int* __restrict__ perm = nullptr) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int64_t p = perm ? int64_t(perm[t]) : t;   // perm: visit in brick order (local atomics)
    const int i = int(p % n);
    const int j = int((p / n) % n);
    const int k = int(p / (int64_t(n) * n));
    float ps[3] = {psi[p], psi[p + np], psi[p + 2 * np]};
    if (mom) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ps[c] = ps[c] + dd1 * mom[p + c * np];
            psi[p + c * np] = ps[c];
        }
    }
    const float X[3] = {ps[0] + q1[i], ps[1] + q1[j], ps[2] + q1[k]};
    const float resf = float(res);
#pragma unroll
    for (int g = 0; g < NS; ++g) {
        float* mesh = (g == 0) ? mesh0 : mesh1;
        const float gx = grid_coord(X[0] + sh.s[g].x, L, resf, err);
        const float gy = grid_coord(X[1] + sh.s[g].y, L, resf, err);
        const float gz = grid_coord(X[2] + sh.s[g].z, L, resf, err);
        float wx[W], wy[W], wz[W];
        int ix[W], iy[W], iz[W];
        axis_weights<W>(gx, res, wx, ix);
        axis_weights<W>(gy, res, wy, iy);
        axis_weights<W>(gz, res, wz, iz);
#pragma unroll
        for (int c = 0; c < W; ++c) {
#pragma unroll
            for (int b = 0; b < W; ++b) {
                float* row = mesh + (int64_t(iz[c]) * res + iy[b]) * pitch;
#pragma unroll
                for (int a = 0; a < W; ++a) atomicAdd(row + ix[a], wx[a] * wy[b] * wz[c]);
            }
        }
    }
}

// Deposit of externally placed positions (resampled sheet particles): X given per
// component in `xr` (3 blocks of `count` floats). pm.jl:477,481.
template <int W>
__global__ void __launch_bounds__(kThreads) k_scatter_positions(
    const float* __restrict__ xr, int64_t count, int64_t cstride, float L, int res, int pitch,
    float* __restrict__ mesh, int* err) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= count) return;
    const float resf = float(res);
    const float gx = grid_coord(xr[p], L, resf, err);
    const float gy = grid_coord(xr[p + cstride], L, resf, err);
    const float gz = grid_coord(xr[p + 2 * cstride], L, resf, err);
    float wx[W], wy[W], wz[W];
    int ix[W], iy[W], iz[W];
    axis_weights<W>(gx, res, wx, ix);
    axis_weights<W>(gy, res, wy, iy);
    axis_weights<W>(gz, res, wz, iz);
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
        for (int b = 0; b < W; ++b) {
            float* row = mesh + (int64_t(iz[c]) * res + iy[b]) * pitch;
#pragma unroll
            for (int a = 0; a < W; ++a) atomicAdd(row + ix[a], wx[a] * wy[b] * wz[c]);
        }
}

// Combined Fourier multiplier Kφ (pm.jl:389-391) evaluated per mode from 1-D
// float64 tables: Kφ = s0 * mak / (T[kx] + T[ky] + T[kz]), DC = 0. T = -k² for
// lap_order 0 (so 1/T = -1/k², pm.jl:166-170) or the finite-difference terms
// (pm.jl:140-147,171-176); mak = Π sinc^(-2W) (pm.jl:150-151) or 1.
__device__ __forceinline__ float kphi(const double* __restrict__ T, const double* __restrict__ M,
                                      double s0, int kx, int ky, int kz) {
    if ((kx | ky | kz) == 0) return 0.0f;
    double v = s0 / (T[kx] + T[ky] + T[kz]);
    if (M) v *= M[kx] * M[ky] * M[kz];
    return float(v);
}

// fd <- Kφ·fd in place on a half spectrum [kz][ky][kx], kx in [0, res/2] (pm.jl:317-320,632).
// Grid (ceil(res / kSpecRows), res): a block takes kSpecRows rows of one kz plane as one
// flat run of kSpecRows·nh modes, so the row index is a 32-bit multiply-high division
// (exact: e·nh < 2^32).
constexpr int kSpecRows = 8;
__global__ void __launch_bounds__(kThreads) k_kspace_mul(float2* __restrict__ f, int res,
                                                          const double* __restrict__ T,
                                                          const double* __restrict__ M, double s0) {
    const int nh = res / 2 + 1;
    const int kz = blockIdx.y;
    const int ky0 = blockIdx.x * kSpecRows;
    const int nrow = min(kSpecRows, res - ky0);
    const int cnt = nrow * nh;
    const unsigned inv = 0xffffffffu / unsigned(nh) + 1u;
    float2* __restrict__ run = f + (int64_t(kz) * res + ky0) * nh;
    for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
        const int rl = int(__umulhi(unsigned(e), inv));
        const int kx = e - rl * nh;
        const float K = kphi(T, M, s0, kx, ky0 + rl, kz);
        float2 v = run[e];
        v.x *= K;
        v.y *= K;
        run[e] = v;
    }
}

// ik gradient (grad_order 0): out_ax = -(i g_ax Kφ fd) for the three axes
// (pm.jl:322-328,487-492). gh: halved-axis k with Nyquist zeroed; gf: full-axis k
// with Nyquist zeroed (pm.jl:125-130).
__global__ void __launch_bounds__(kThreads) k_kspace_ik(const float2* __restrict__ f, int res,
                                                         const double* __restrict__ T,
                                                         const double* __restrict__ M, double s0,
                                                         const float* __restrict__ gh,
                                                         const float* __restrict__ gf,
                                                         float2* __restrict__ ox,
                                                         float2* __restrict__ oy,
                                                         float2* __restrict__ oz) {
    const int nh = res / 2 + 1;
    const int64_t total = int64_t(res) * res * nh;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int kx = int(t % nh);
        const int ky = int((t / nh) % res);
        const int kz = int(t / (int64_t(nh) * res));
        const float K = kphi(T, M, s0, kx, ky, kz);
        const float2 v = f[t];
        const float g[3] = {gh[kx], gf[ky], gf[kz]};
        float2* o[3] = {ox, oy, oz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float tk = g[c] * K;  // (i g)·K·(a + i b) = (-g K b) + i (g K a); negated
            o[c][t] = make_float2(tk * v.y, -(tk * v.x));
        }
    }
}

// Σ over the W³ nodes of w · F_c, with F_c = -D_c φ the order-2R central
// difference (pm.jl:330-342,419-424) applied to the potential on the fly.
// Written as one pass over the cross-shaped union of the three stencils: for each
// axis the weights are convolved with the antisymmetric difference stencil, so
// each potential value is loaded once per particle.
template <int W, int R>
__device__ __forceinline__ void gather_fd(const float* __restrict__ phi, int res, int pitch, float gx,
                                          float gy, float gz, float c1, float c2, float c3,
                                          float& Sx, float& Sy, float& Sz) {
    constexpr int E = W + 2 * R;
    float wx[W], wy[W], wz[W];
    int cx[W], cy[W], cz[W];
    axis_weights<W>(gx, res, wx, cx);
    axis_weights<W>(gy, res, wy, cy);
    axis_weights<W>(gz, res, wz, cz);
    const int bx = wbase<W>(gx) + WLo<W>::v, by = wbase<W>(gy) + WLo<W>::v,
              bz = wbase<W>(gz) + WLo<W>::v;
    const float cc[4] = {0.0f, c1, c2, c3};
    // kappa(t) = coefficient of φ(node + t) in F(node): -c_t for t > 0, +c_|t| for t < 0.
    float ux[E], uy[E], uz[E];
    int ex[E];
    int64_t ey[E], ez[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        float sx = 0.0f, sy = 0.0f, sz = 0.0f;
#pragma unroll
        for (int a = 0; a < W; ++a) {
            const int t = e - R - a;
            const float kap = (t > 0 && t <= R) ? -cc[t > 0 ? t : 0] : ((t < 0 && -t <= R) ? cc[t < 0 ? -t : 0] : 0.0f);
            sx += wx[a] * kap;
            sy += wy[a] * kap;
            sz += wz[a] * kap;
        }
        ux[e] = sx;
        uy[e] = sy;
        uz[e] = sz;
        ex[e] = wrapi(bx - R + e, res);
        ey[e] = int64_t(wrapi(by - R + e, res)) * pitch;
        ez[e] = int64_t(wrapi(bz - R + e, res)) * res * pitch;
    }
    (void)cx;
    (void)cy;
    (void)cz;
    float sX = 0.0f, sY = 0.0f, sZ = 0.0f;
    // core rows: y and z inside the W-node stencil, x over the extended range
#pragma unroll
    for (int c = 0; c < W; ++c) {
#pragma unroll
        for (int b = 0; b < W; ++b) {
            const float* row = phi + ez[c + R] + ey[b + R];
            float rx = 0.0f, rc = 0.0f;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const float v = __ldg(row + ex[e]);
                rx += ux[e] * v;
                if (e >= R && e < R + W) rc += wx[e - R] * v;
            }
            sX += (wy[b] * wz[c]) * rx;
            sY += (uy[b + R] * wz[c]) * rc;
            sZ += (uz[c + R] * wy[b]) * rc;
        }
    }
    // y halo rows (for the y derivative) and z halo rows (for the z derivative)
#pragma unroll
    for (int c = 0; c < W; ++c) {
#pragma unroll
        for (int h = 0; h < 2 * R; ++h) {
            const int e = (h < R) ? h : h + W;
            const float* row = phi + ez[c + R] + ey[e];
            float rc = 0.0f;
#pragma unroll
            for (int a = 0; a < W; ++a) rc += wx[a] * __ldg(row + ex[a + R]);
            sY += (uy[e] * wz[c]) * rc;
        }
    }
#pragma unroll
    for (int h = 0; h < 2 * R; ++h) {
        const int e = (h < R) ? h : h + W;
#pragma unroll
        for (int b = 0; b < W; ++b) {
            const float* row = phi + ez[e] + ey[b + R];
            float rc = 0.0f;
#pragma unroll
            for (int a = 0; a < W; ++a) rc += wx[a] * __ldg(row + ex[a + R]);
            sZ += (uz[e] * wy[b]) * rc;
        }
    }
    Sx = sX;
    Sy = sY;
    Sz = sZ;
}

// Σ over the W³ nodes of w·F_c for three precomputed force meshes (ik gradient;
// pm.jl:344-364).
template <int W>
__device__ __forceinline__ void gather_f3(const float* __restrict__ fx, const float* __restrict__ fy,
                                          const float* __restrict__ fz, int res, int pitch, float gx,
                                          float gy, float gz, float& Sx, float& Sy, float& Sz) {
    float wx[W], wy[W], wz[W];
    int ix[W], iy[W], iz[W];
    axis_weights<W>(gx, res, wx, ix);
    axis_weights<W>(gy, res, wy, iy);
    axis_weights<W>(gz, res, wz, iz);
    float s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
        for (int b = 0; b < W; ++b) {
            const int64_t r = (int64_t(iz[c]) * res + iy[b]) * pitch;
#pragma unroll
            for (int a = 0; a < W; ++a) {
                const float w = wx[a] * wy[b] * wz[c];
                s1 += __ldg(fx + r + ix[a]) * w;
                s2 += __ldg(fy + r + ix[a]) * w;
                s3 += __ldg(fz + r + ix[a]) * w;
            }
        }
    Sx = s1;
    Sy = s2;
    Sz = s3;
}

struct GatherArgs {
    float* psi;         // displacements (read; written by the fused final drift)
    float* mom;         // momenta (read/written by the fused kick) or null
    float* acc;         // running acceleration sums (partial groups) / output
    const float* q1;    // lattice coordinates q_i = i*L/n
    const float* mesh[kMaxGroup];      // potentials (FD) or x-force meshes (ik)
    const float* meshy[kMaxGroup];     // ik: y-force meshes
    const float* meshz[kMaxGroup];     // ik: z-force meshes
    GroupShifts sh;
    int n;
    int64_t np;
    float L;
    int res, pitch;
    float c1, c2, c3;
    int first;          // 1: start the sums at zero; 0: continue from acc
    int last;           // 1: finish (mean over shifts, then write acc or kick-drift)
    float nshift_f;     // number of interlacing shifts (divisor when > 1)
    int divide;
    int step;           // 1: kick + drift after the last group; 0: write acc
    float alpha, beta, dd2;
    int* err;
    const int* perm;    // brick-sorted particle order for the tiled kernels (null: Lagrangian tiles)
    const float* extra; // (3 blocks of np) added to the final acceleration, or null (network correction)
    float* part;        // brick interpolation: partial sums and Ψ in sorted order (6 blocks of np), or null
};

template <int W, int R, int NS>
__global__ void __launch_bounds__(kThreads) k_gather(GatherArgs A) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= A.np) return;
    const int64_t np = A.np;
    const int n = A.n;
    const int i = int(p % n);
    const int j = int((p / n) % n);
    const int k = int(p / (int64_t(n) * n));
    const float ps[3] = {A.psi[p], A.psi[p + np], A.psi[p + 2 * np]};
    const float X[3] = {ps[0] + A.q1[i], ps[1] + A.q1[j], ps[2] + A.q1[k]};
    float acc[3];
    if (A.first) {
        acc[0] = acc[1] = acc[2] = 0.0f;
    } else {
        acc[0] = A.acc[p];
        acc[1] = A.acc[p + np];
        acc[2] = A.acc[p + 2 * np];
    }
    const float resf = float(A.res);
#pragma unroll
    for (int g = 0; g < NS; ++g) {
        const float gx = grid_coord(X[0] + A.sh.s[g].x, A.L, resf, A.err);
        const float gy = grid_coord(X[1] + A.sh.s[g].y, A.L, resf, A.err);
        const float gz = grid_coord(X[2] + A.sh.s[g].z, A.L, resf, A.err);
        float s1, s2, s3;
        if (R == 0)
            gather_f3<W>(A.mesh[g], A.meshy[g], A.meshz[g], A.res, A.pitch, gx, gy, gz, s1, s2, s3);
        else
            gather_fd<W, (R == 0 ? 1 : R)>(A.mesh[g], A.res, A.pitch, gx, gy, gz, A.c1, A.c2, A.c3,
                                           s1, s2, s3);
        acc[0] += s1;
        acc[1] += s2;
        acc[2] += s3;
    }
    if (A.last && A.divide) {  // acc ./= length(shifts) (pm.jl:519)
        acc[0] = acc[0] / A.nshift_f;
        acc[1] = acc[1] / A.nshift_f;
        acc[2] = acc[2] / A.nshift_f;
    }
    if (A.last && A.extra) {
        acc[0] += A.extra[p];
        acc[1] += A.extra[p + np];
        acc[2] += A.extra[p + 2 * np];
    }
    if (A.last && A.step) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float m = A.alpha * A.mom[p + c * np] + A.beta * acc[c];
            A.mom[p + c * np] = m;
            A.psi[p + c * np] = ps[c] + A.dd2 * m;
        }
    } else {
        A.acc[p] = acc[0];
        A.acc[p + np] = acc[1];
        A.acc[p + 2 * np] = acc[2];
    }
}

// ── mesh <-> particle transfers of three-component fields (force correction) ──
// out_c(p) = Σ_n W(X_p − n) f_c(n) over the W-order stencil of X_p = q + Ψ_p, for three
// dense res³ meshes f_c = f + c·res³ ([z][y][x]); the interpolation of pm.jl:344-364
// applied to given node values, without shifts.
// perm (or null): the particles are visited in that order (the brick sort: neighbouring
// threads then read neighbouring nodes).
template <int W>
__global__ void __launch_bounds__(kThreads) k_interp3(const float* __restrict__ psi, const float* __restrict__ q1,
                                                      int n, int64_t np, float L, int res,
                                                      const float* __restrict__ f, float scale,
                                                      float* __restrict__ out, int* err,
                                                      const int* __restrict__ perm = nullptr) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int64_t p = perm ? int64_t(perm[t]) : t;
    LatticeDiv ld;
    ld.init(n);
    int i, j, k;
    ld.ijk(p, i, j, k);
    const float resf = float(res);
    float wx[W], wy[W], wz[W];
    int ix[W], iy[W], iz[W];
    axis_weights<W>(grid_coord(psi[p] + q1[i], L, resf, err), res, wx, ix);
    axis_weights<W>(grid_coord(psi[p + np] + q1[j], L, resf, err), res, wy, iy);
    axis_weights<W>(grid_coord(psi[p + 2 * np] + q1[k], L, resf, err), res, wz, iz);
    const int64_t cells = int64_t(res) * res * res;
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
        for (int b = 0; b < W; ++b) {
            const int64_t row = (int64_t(iz[c]) * res + iy[b]) * res;
            const float wyz = wy[b] * wz[c];
#pragma unroll
            for (int a = 0; a < W; ++a) {
                const int64_t o = row + ix[a];
                const float w = wx[a] * wyz;
                s0 += w * __ldg(f + o);
                s1 += w * __ldg(f + cells + o);
                s2 += w * __ldg(f + 2 * cells + o);
            }
        }
    out[p] = scale * s0;
    out[p + np] = scale * s1;
    out[p + 2 * np] = scale * s2;
}

// The transpose of k_interp3: f_c(n) += Σ_p W(X_p − n) v_c(p) (float atomics).
template <int W>
__global__ void __launch_bounds__(kThreads) k_deposit3(const float* __restrict__ psi, const float* __restrict__ q1,
                                                       int n, int64_t np, float L, int res,
                                                       const float* __restrict__ v, float* __restrict__ f, int* err) {
    const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= np) return;
    LatticeDiv ld;
    ld.init(n);
    int i, j, k;
    ld.ijk(p, i, j, k);
    const float resf = float(res);
    float wx[W], wy[W], wz[W];
    int ix[W], iy[W], iz[W];
    axis_weights<W>(grid_coord(psi[p] + q1[i], L, resf, err), res, wx, ix);
    axis_weights<W>(grid_coord(psi[p + np] + q1[j], L, resf, err), res, wy, iy);
    axis_weights<W>(grid_coord(psi[p + 2 * np] + q1[k], L, resf, err), res, wz, iz);
    const int64_t cells = int64_t(res) * res * res;
    const float v0 = v[p], v1 = v[p + np], v2 = v[p + 2 * np];
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
        for (int b = 0; b < W; ++b) {
            const int64_t row = (int64_t(iz[c]) * res + iy[b]) * res;
            const float wyz = wy[b] * wz[c];
#pragma unroll
            for (int a = 0; a < W; ++a) {
                const int64_t o = row + ix[a];
                const float w = wx[a] * wyz;
                atomicAdd(f + o, w * v0);
                atomicAdd(f + cells + o, w * v1);
                atomicAdd(f + 2 * cells + o, w * v2);
            }
        }
}

// out[c][cell] = in[c][cell] · scale[c] for `nc` channels of `cells` floats.
__global__ void k_scale_channels(const float* __restrict__ in, float* __restrict__ out, int64_t cells, int nc,
                                 float s0, float s1, float s2, float s3) {
    const int64_t total = cells * nc;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(t / cells);
        const float s = c == 0 ? s0 : c == 1 ? s1 : c == 2 ? s2 : s3;
        out[t] = in[t] * s;
    }
}

// ── elementwise kernels ───────────────────────────────────────────────────────
__global__ void k_drift(float* __restrict__ psi, const float* __restrict__ mom, float dd, int64_t m) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m;
         t += int64_t(gridDim.x) * blockDim.x)
        psi[t] = psi[t] + dd * mom[t];
}

__global__ void k_kick_drift(float* __restrict__ psi, float* __restrict__ mom,
                             const float* __restrict__ acc, float alpha, float beta, float dd2,
                             int64_t m) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m;
         t += int64_t(gridDim.x) * blockDim.x) {
        const float v = alpha * mom[t] + beta * acc[t];
        mom[t] = v;
        psi[t] = psi[t] + dd2 * v;
    }
}

__global__ void k_set_mom(float* __restrict__ dst, const float* __restrict__ src, double scale,
                          int64_t m) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m;
         t += int64_t(gridDim.x) * blockDim.x)
        dst[t] = float(double(src[t]) * scale);
}

// run_nbody.jl:148-149,164: X = mod(q + Psi + L, L) (or Psi), P = float((Mom/div)*mul).
__global__ void k_output(const float* __restrict__ psi, const float* __restrict__ mom,
                         const float* __restrict__ q1, int n, int64_t np, float L, int wrap,
                         double pdiv, double pmul, float* __restrict__ xo, float* __restrict__ po) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < 3 * np;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(t / np);
        const int64_t p = t - c * np;
        if (xo) {
            float x = psi[t];
            if (wrap) {
                const int ii = (c == 0) ? int(p % n) : (c == 1) ? int((p / n) % n) : int(p / (int64_t(n) * n));
                x = x + q1[ii];
                if (wrap == 1) x = jmodf(x + L, L);
            }
            xo[t] = x;
        }
        if (po) po[t] = float((double(mom[t]) / pdiv) * pmul);
    }
}

// ── sheet resampling (pm.jl:186-234,426-464) ──────────────────────────────────
// ψ_c = mod(X_c + s_c - q_c + L/2, L) - L/2 with X = q + Psi, written transposed to
// [i][j][k] (k fastest, row padded to n+2) so that the in-place R2C halves the z
// axis as the reference's rfft does (pm.jl:430-433).
__global__ void k_wrap_psi(const float* __restrict__ psi, const float* __restrict__ q1, int n,
                           int64_t np, float L, Shift3 s, int c, float* __restrict__ out,
                           int padded) {
    const int pitch = padded ? n + 2 : n;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < np;
         t += int64_t(gridDim.x) * blockDim.x) {
        // t enumerates the output in [i][j][k] order (k fastest)
        const int kk = int(t % n);
        const int jj = int((t / n) % n);
        const int ii = int(t / (int64_t(n) * n));
        const int64_t p = ii + int64_t(n) * (jj + int64_t(n) * kk);  // input index, x fastest
        const float sc = (c == 0) ? s.x : (c == 1) ? s.y : s.z;
        const int qi = (c == 0) ? ii : (c == 1) ? jj : kk;
        const float X = (psi[p + c * np] + q1[qi]) + sc;
        const float v = jmodf((X - q1[qi]) + L / 2.0f, L) - L / 2.0f;
        out[(int64_t(ii) * n + jj) * pitch + kk] = v;
    }
}

// Phase shift of ψ̂ for a Lagrangian offset d (pm.jl:434-437,451-458): out =
// ψ̂·px[i]·py[j]·pz[k]/n³ on the (n, n, n/2+1) spectrum [i][j][kz]. The kz = 0 and
// kz = n/2 planes are made Hermitian ((H(k) + conj H(-k))/2), which is the value
// a C2R that ignores the imaginary part of those planes after the full-axis
// transforms produces from the raw product; it makes the result independent of
// the C2R implementation.
__global__ void k_phase(const float2* __restrict__ in, float2* __restrict__ out, int n,
                        const float2* __restrict__ px, const float2* __restrict__ py,
                        const float2* __restrict__ pz, float scale) {
    const int nh = n / 2 + 1;
    const int64_t total = int64_t(n) * n * nh;
    auto cmul = [](float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int kz = int(t % nh);
        const int j = int((t / nh) % n);
        const int i = int(t / (int64_t(nh) * n));
        float2 f = cmul(px[i], py[j]);
        f = cmul(f, pz[kz]);
        f.x *= scale;
        f.y *= scale;
        float2 h = cmul(in[t], f);
        if (kz == 0 || kz == nh - 1) {
            const int im = (n - i) % n, jm = (n - j) % n;
            const int64_t tm = (int64_t(im) * n + jm) * nh + kz;
            float2 fm = cmul(px[im], py[jm]);
            fm = cmul(fm, pz[kz]);
            fm.x *= scale;
            fm.y *= scale;
            const float2 hm = cmul(in[tm], fm);
            h = make_float2(0.5f * (h.x + hm.x), 0.5f * (h.y - hm.y));
        }
        out[t] = h;
    }
}

// Resampled positions X' = mod(q + ψ' + d·L/n + L, L) for the Fourier method
// (pm.jl:438-441), ψ' in [i][j][k] padded layout, written to xr (3 blocks of n³,
// same [i][j][k] order).
__global__ void k_place(const float* __restrict__ rb, const float* __restrict__ q1, int n,
                        int64_t np, float L, float shiftc, int c, float* __restrict__ xr) {
    const int pitch = n + 2;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < np;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int kk = int(t % n);
        const int jj = int((t / n) % n);
        const int ii = int(t / (int64_t(n) * n));
        const int qi = (c == 0) ? ii : (c == 1) ? jj : kk;
        const float v = rb[(int64_t(ii) * n + jj) * pitch + kk];
        xr[t + c * np] = jmodf(((q1[qi] + v) + shiftc) + L, L);
    }
}

// Periodic trilinear resampling (pm.jl:207-212,220-231): ψ (x-fastest, 3 blocks)
// interpolated at (i+dx, j+dy, k+dz), placed at q + ψ' + d·L/n, wrapped.
__global__ void k_place_linear(const float* __restrict__ w, const float* __restrict__ q1, int n,
                               int64_t np, float L, float dx, float dy, float dz, float sx,
                               float sy, float sz, float* __restrict__ xr) {
    for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < np;
         p += int64_t(gridDim.x) * blockDim.x) {
        const int i = int(p % n);
        const int j = int((p / n) % n);
        const int k = int(p / (int64_t(n) * n));
        const int i1 = (i + 1) % n, j1 = (j + 1) % n, k1 = (k + 1) % n;
        auto at = [&](int a, int b, int cc) { return int64_t(a) + int64_t(n) * (b + int64_t(n) * cc); };
        const float shifts[3] = {sx, sy, sz};
        const int qi[3] = {i, j, k};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float* f = w + c * np;
            const float v = f[at(i, j, k)] * (1 - dx) * (1 - dy) * (1 - dz) +
                            f[at(i1, j, k)] * dx * (1 - dy) * (1 - dz) +
                            f[at(i, j1, k)] * (1 - dx) * dy * (1 - dz) +
                            f[at(i, j, k1)] * (1 - dx) * (1 - dy) * dz +
                            f[at(i1, j1, k)] * dx * dy * (1 - dz) +
                            f[at(i1, j, k1)] * dx * (1 - dy) * dz +
                            f[at(i, j1, k1)] * (1 - dx) * dy * dz +
                            f[at(i1, j1, k1)] * dx * dy * dz;
            xr[p + c * np] = jmodf(((q1[qi[c]] + v) + shifts[c]) + L, L);
        }
    }
}

// ψ = mod(X + s - q + L/2, L) - L/2 in the particle layout (x fastest), 3 blocks.
__global__ void k_wrap_psi_lin(const float* __restrict__ psi, const float* __restrict__ q1, int n,
                               int64_t np, float L, Shift3 s, float* __restrict__ out) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < 3 * np;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(t / np);
        const int64_t p = t - c * np;
        const int qi = (c == 0) ? int(p % n) : (c == 1) ? int((p / n) % n) : int(p / (int64_t(n) * n));
        const float sc = (c == 0) ? s.x : (c == 1) ? s.y : s.z;
        const float X = (psi[t] + q1[qi]) + sc;
        out[t] = jmodf((X - q1[qi]) + L / 2.0f, L) - L / 2.0f;
    }
}

}  // namespace djb

#include "brick.cuh"
#include "zpencil.cuh"
#include "adjoint.cuh"

namespace djb {
// Kφ as a functor for the fused z pass.
struct KPhiFn {
    const double* T;
    const double* M;
    double s0;
    __device__ __forceinline__ float operator()(int kx, int ky, int kz) const { return kphi(T, M, s0, kx, ky, kz); }
    // float64 sums and products, one float division (within 1.5 ulp of the above)
    __device__ __forceinline__ float fast(int kx, int ky, int kz) const {
        if ((kx | ky | kz) == 0) return 0.0f;
        double num = s0;
        if (M) num *= M[kx] * M[ky] * M[kz];
        return float(num) / float(T[kx] + T[ky] + T[kz]);
    }
};
}  // namespace djb

// ─────────────────────────────────────────────────────────────────────────────
// solver object
// ─────────────────────────────────────────────────────────────────────────────
namespace {

// Shared-memory budgets of the tiled kernels: 24 K 32-bit cells (96 KB) for the mass
// assignment, 24 K floats (96 KB) for the interpolation: 2 CTAs/SM each.
#ifndef DJB_SCATTER_BUDGET
#define DJB_SCATTER_BUDGET (24 * 1024)
#endif
#ifndef DJB_GATHER_BUDGET
#define DJB_GATHER_BUDGET (24 * 1024)
#endif
constexpr int kScatterBudget = DJB_SCATTER_BUDGET;
constexpr int kGatherBudget = DJB_GATHER_BUDGET;

// Phases of a force evaluation, timed with CUDA events on the solver's stream.
enum Phase { PH_CLEAR = 0, PH_SCATTER, PH_RESAMPLE, PH_R2C, PH_KSPACE, PH_C2R, PH_GATHER, PH_SORT, PH_NN, PH_COUNT };

// Launch counts of this library's kernels (always on) and, when enabled, per-phase
// device time from event pairs recorded around each phase.
struct Profiler {
    bool on = false;
    struct Rec {
        int phase;
        cudaEvent_t a, b;
    };
    std::vector<cudaEvent_t> pool;
    std::vector<Rec> recs;
    size_t next = 0;
    cudaEvent_t cur = nullptr;
    int64_t launches[PH_COUNT] = {};
    int64_t calls[PH_COUNT] = {};

    cudaEvent_t take() {
        if (next == pool.size()) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            pool.push_back(e);
        }
        return pool[next++];
    }
    void begin(cudaStream_t st, int ph) {
        (void)ph;
        if (!on) return;
        cur = take();
        if (cur) cudaEventRecord(cur, st);
    }
    void end(cudaStream_t st, int ph, int nlaunch) {
        launches[ph] += nlaunch;
        calls[ph] += 1;
        if (!on || !cur) return;
        cudaEvent_t b = take();
        if (!b) return;
        cudaEventRecord(b, st);
        recs.push_back({ph, cur, b});
        cur = nullptr;
    }
    void reset() {
        recs.clear();
        next = 0;
        for (int i = 0; i < PH_COUNT; ++i) launches[i] = calls[i] = 0;
    }
    void destroy() {
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
        pool.clear();
        recs.clear();
        next = 0;
    }
};

}  // namespace

struct djb_solver {
    Profiler prof;
    djb_pm_config cfg{};
    int n = 0, res = 0, pitch = 0, W = 2, R = 0;
    int64_t np = 0;          // particles
    int64_t mesh_floats = 0; // res*res*(res+2)
    double L = 0;
    float Lf = 0;
    int nshift = 1, group = 1;
    std::vector<double> shifts;     // 3 per shift
    std::vector<double> rshifts;    // resampling offsets, 3 per offset
    float c1 = 0, c2 = 0, c3 = 0;   // FD coefficients (pm.jl:419-424)
    double s0 = 0;                  // Kφ scale

    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    cufftHandle r2c = 0, c2r = 0, r2c_n = 0, c2r_n = 0, r2c_d = 0, c2r_d = 0;
    bool have_r2c = false, have_c2r = false, have_r2c_n = false, have_c2r_n = false, have_r2c_d = false,
         have_c2r_d = false;

    float* psi = nullptr;
    float* mom = nullptr;
    float* acc = nullptr;
    float* q1 = nullptr;
    float* mesh[kMaxGroup] = {nullptr, nullptr};
    // dense [res]^3 meshes (finite-difference gradients, res % 4 == 0, not lean): the
    // mass assignment writes the density here, an out-of-place R2C takes it to the
    // spectrum in `mesh`, and an out-of-place C2R brings the potential back. The brick
    // kernels add their boxes to them and fetch their boxes from them with bulk tensor
    // copies described by `tmap_s` (mass-assignment boxes) and `tmap` (interpolation).
    float* phi[kMaxGroup] = {nullptr, nullptr};
    CUtensorMap tmap[kMaxGroup];
    CUtensorMap tmap_s[kMaxGroup];
    CUtensorMap tmap_adj[3];     // the VJP work meshes, deposit-box boxes (dense meshes only)
    CUtensorMap tmap_rho;        // the first dense mesh, deposit-box boxes (the VJP's rho-bar gather)
    bool have_tmap_adj = false;
    bool tma = false;
    // res == 1024: the dense transforms are batched 2-D transforms of the z planes and
    // the z stages run fused with Kφ in k_zpencil_pair (zpencil.cuh); wN = exp(-2πi j/res)
    bool zpass = false;
    float2* wN = nullptr;
    float* adj[3] = {nullptr, nullptr, nullptr};  // VJP work meshes (allocated on first use)
    float* scr[10] = {};    // staging and work buffers of the adjoint entry points, kept between calls
    size_t scr_n[10] = {};
    int nsm = 148;  // SMs of the device (persistent grids)
    // brick boxes (brick.cuh): width along x, extent along y and z, first node relative
    // to the brick's first cell; g = interpolation, s = mass assignment
    int gsx = 0, gS = 0, gfirst = 0;
    int ssx = 0, sS = 0, sfirst = 0;
    float* fmesh[kMaxGroup][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    double* lapT = nullptr;
    double* makT = nullptr;
    float* gh = nullptr;
    float* gf = nullptr;
    // resampling work areas
    float2* psihat = nullptr;   // 3 spectra (n, n, n/2+1)
    float2* cb = nullptr;       // one spectrum
    float* rb = nullptr;        // real n*n*(n+2) (in-place C2R)
    float* xr = nullptr;        // 3*np resampled positions
    float2* phase = nullptr;    // px, py, pz tables (n + n + n/2+1)
    // brick sort of the particles (sort.cuh)
    bool sorted = true;
    bool fd_scalar = false;  // stencil kernels with 4-byte copies only (DJB_FD_SCALAR=1; the 16-byte path is the default)
    djb::SortGeom sg{};
    int64_t nbins = 0;
    int nscan = 0;
    unsigned* count = nullptr;
    unsigned* offset = nullptr;
    unsigned* bsum = nullptr;
    uint2* keyrank = nullptr;
    int* perm = nullptr;
    float* part = nullptr;  // brick interpolation's partial sums and Ψ in sorted order (6 np floats), or null
    const int* cur_perm = nullptr;  // order used by the tiled kernels of the current force call
    int* err = nullptr;
    bool have_state = false;
    bool tiled = true;  // shared-memory tiled scatter/gather (DJB_KERNELS=simple selects the per-particle ones)
    // force correction (djb_solver_attach_nn): network inputs [δ, F_x, F_y, F_z] scaled by
    // nn_in (δ) and nn_fin (F), its output scaled by nn_out, interpolated to the particles
    djb_nn* nn = nullptr;
    float nn_in = 1.0f, nn_fin = 1.0f, nn_out = 1.0f;
    float* nnf = nullptr;    // 4 res³ meshes (network input)
    float* nnd = nullptr;    // 3 res³ meshes (network output)
    float* nnacc = nullptr;  // 3·np particle corrections
    int nn_every = 1;        // network schedule (djb_solver_nn_schedule): from step nn_start on,
    int nn_start = 0;        //   on every nn_every-th step
    int64_t nn_steps = 0;    // steps taken since the state or the network was set
    bool nn_valid = false;   // nnacc holds a correction of the current particles
    int64_t bytes = 0;
    std::vector<void*> allocs;
};

// Work buffer `slot` of at least `count` floats, kept by the solver between calls (a
// per-call allocation and release of gigabytes made the adjoint's time vary by 3x).
int scratch(djb_solver* s, int slot, size_t count, float** out) {
    if (s->scr_n[slot] < count) {
        if (s->scr[slot]) {
            CUDA_TRY(cudaStreamSynchronize(s->stream));
            cudaFree(s->scr[slot]);
            s->scr[slot] = nullptr;
            s->scr_n[slot] = 0;
        }
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&s->scr[slot]), count * sizeof(float));
        if (e != cudaSuccess) {
            cudaGetLastError();
            s->scr[slot] = nullptr;
            return fail(DJB_ERR_ALLOC, "work buffer allocation of %zu floats failed: %s", count, cudaGetErrorString(e));
        }
        s->scr_n[slot] = count;
    }
    *out = s->scr[slot];
    return DJB_OK;
}

namespace {

int dmalloc(djb_solver* s, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DJB_ERR_ALLOC, "cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    s->allocs.push_back(*p);
    s->bytes += int64_t(bytes);
    return DJB_OK;
}

#define TRY(expr)                 \
    do {                          \
        int rc_ = (expr);         \
        if (rc_ != DJB_OK) return rc_; \
    } while (0)

int validate(const djb_pm_config& c) {
    if (c.worder < 2 || c.worder > 4) return fail(DJB_ERR_INVALID, "worder must be 2, 3 or 4");
    if (!(c.grad_order == 0 || c.grad_order == 2 || c.grad_order == 4 || c.grad_order == 6))
        return fail(DJB_ERR_INVALID, "grad_order must be 0, 2, 4 or 6");
    if (!(c.lap_order == 0 || c.lap_order == 2 || c.lap_order == 4 || c.lap_order == 6))
        return fail(DJB_ERR_INVALID, "lap_order must be 0, 2, 4 or 6");
    if (c.antialias < -1 || c.antialias > 3)
        return fail(DJB_ERR_INVALID, "antialias must be -1, 0, 1, 2 or 3");
    if (c.resampling != DJB_RESAMPLE_FOURIER && c.resampling != DJB_RESAMPLE_LINEAR)
        return fail(DJB_ERR_INVALID, "resampling must be :fourier or :linear");
    if (c.res_pm < 8 || (c.res_pm & 1))
        return fail(DJB_ERR_INVALID, "res_pm must be even and >= 8 (got %d)", c.res_pm);
    if (c.n_part < 2) return fail(DJB_ERR_INVALID, "n_part must be >= 2 (got %d)", c.n_part);
    if (c.n_resample < 1) return fail(DJB_ERR_INVALID, "n_resample must be >= 1");
    if (c.n_resample > 1 && c.resampling == DJB_RESAMPLE_FOURIER && (c.n_part & 1))
        return fail(DJB_ERR_INVALID, "Fourier resampling needs an even n_part");
    if (!(c.boxsize > 0.0)) return fail(DJB_ERR_INVALID, "boxsize must be positive");
    if (c.lean && !(c.antialias == 0 && c.n_resample == 1 && c.grad_order != 0))
        return fail(DJB_ERR_INVALID,
                    "PMSolverLean supports antialias = 0, n_resample = 1 and finite-difference gradients (2/4/6)");
    return DJB_OK;
}

int make_plan(cufftHandle* h, bool* have, int n, cufftType type, cudaStream_t st, size_t* work) {
    CUFFT_TRY(cufftCreate(h));
    *have = true;
    long long dims[3] = {n, n, n};
    long long rembed[3] = {n, n, 2 * (n / 2 + 1)};
    long long cembed[3] = {n, n, n / 2 + 1};
    const bool fwd = (type == CUFFT_R2C);
    long long* inembed = fwd ? rembed : cembed;
    long long* onembed = fwd ? cembed : rembed;
    long long idist = inembed[0] * inembed[1] * inembed[2];
    long long odist = onembed[0] * onembed[1] * onembed[2];
    CUFFT_TRY(cufftMakePlanMany64(*h, 3, dims, inembed, 1, idist, onembed, 1, odist, type, 1, work));
    CUFFT_TRY(cufftSetStream(*h, st));
    return DJB_OK;
}

int grid_for(int64_t count) {
    int64_t b = (count + kThreads - 1) / kThreads;
    return int(std::min<int64_t>(b, 148LL * 64));
}

inline int blocks(int64_t count) { return int((count + kThreads - 1) / kThreads); }

GroupShifts group_shifts(const djb_solver* s, int first, int ns) {
    GroupShifts g{};
    for (int i = 0; i < ns; ++i) {
        g.s[i].x = float(s->shifts[3 * (first + i) + 0]);
        g.s[i].y = float(s->shifts[3 * (first + i) + 1]);
        g.s[i].z = float(s->shifts[3 * (first + i) + 2]);
    }
    return g;
}

dim3 tile_grid(int n) {
    return dim3((n + djb::kTX - 1) / djb::kTX, (n + djb::kTY - 1) / djb::kTY, (n + djb::kTZ - 1) / djb::kTZ);
}

djb::BrickList brick_list(const djb_solver* s) {
    const int hb = s->sg.hb;
    return djb::BrickList{s->offset, s->bsum, s->perm, s->sg.nb, s->sg.brick, hb * hb * hb, s->nbins,
                          unsigned(s->np), s->gsx, s->gS, s->gfirst, s->ssx, s->sS, s->sfirst};
}

// Range [lo, hi] of a particle's base node relative to the cell floor(g) that bins it,
// over the configuration's shifts (grid units). Shift 0 reproduces the binning's own
// coordinate, so the base is the cell (even orders) or the cell or the next node (odd
// orders round to nearest). Other shifts: the floor (or round-to-nearest) over
// [c + s, c + 1 + s), widened by 0.01 cells for the round-off of mod(X + s, L) and, for
// round-to-nearest, by one node below for ties rounded to even.
void base_range(const djb_solver* s, int& lo, int& hi) {
    const bool odd = (s->W % 2) != 0;
    const double d = odd ? 0.5 : 0.0, eps = 0.01;
    lo = 0;
    hi = 0;
    for (size_t i = 0; i < s->shifts.size(); ++i) {
        const double sg = s->shifts[i] * s->res / s->L;
        int l, h;
        if (sg == 0.0) {
            l = 0;
            h = odd ? 1 : 0;
        } else {
            l = int(std::floor(sg + d - eps)) - (odd ? 1 : 0);
            h = int(std::floor(sg + d + 1.0 + eps));
        }
        lo = (i == 0) ? l : std::min(lo, l);
        hi = (i == 0) ? h : std::max(hi, h);
    }
}

// Width along x of a box of S nodes whose first node lies `first` nodes from a brick
// origin: rounded down to a 16-byte group the box starts up to 3 nodes earlier (exactly
// first & 3 when bricks are multiples of 4 cells); rounded up to a multiple of 4, and to
// 4 mod 8, which keeps the rows of one plane on different shared-memory banks.
int box_sx(int brick, int S, int first) {
    const int off = (brick % 4 == 0) ? (first & 3) : 3;
    int sx = (S + off + 3) & ~3;
    if (sx % 8 == 0) sx += 4;
    return sx;
}

// Brick box geometry for bricks of `brick` cells (mass assignment and interpolation).
void brick_boxes(djb_solver* s, int brick) {
    int lo, hi;
    base_range(s, lo, hi);
    const int lw = (s->W == 2) ? 0 : -1;  // lowest stencil offset (pm.jl:53-55)
    s->sS = brick + (hi - lo) + s->W - 1;
    s->sfirst = lo + lw;
    s->ssx = box_sx(brick, s->sS, s->sfirst);
    s->gS = s->sS + 2 * s->R;
    s->gfirst = s->sfirst - s->R;
    s->gsx = box_sx(brick, s->gS, s->gfirst);
}

// Per shift of a group: one box, rounded up to 128 bytes (djb::box_stride).
size_t scatter_smem(const djb_solver* s) {
    return size_t(djb::box_stride(s->ssx * s->sS * s->sS)) * 4;
}

// The density mesh of group member m (dense when the solver has dense meshes) and its pitch.
float* rho_mesh(const djb_solver* s, int m) { return s->phi[m] ? s->phi[m] : s->mesh[m]; }
int rho_pitch(const djb_solver* s) { return s->phi[0] ? s->res : s->pitch; }

size_t gather_smem(const djb_solver* s) { return size_t(s->gsx) * s->gS * s->gS * 4; }

// Dynamic shared memory of a brick kernel, 2 CTAs per SM: 228 KB of shared memory
// less 1 KB per CTA reserved by the runtime and the kernel's static barrier.
constexpr int kBrickSmemMax = 113 * 1024;

// Tensor map of a dense [res]^3 float mesh with boxes of sx x S x S elements.
int make_tmap(CUtensorMap* m, const float* base, int res, int sx, int S) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) return fail(DJB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[3] = {cuuint64_t(res), cuuint64_t(res), cuuint64_t(res)};
    const cuuint64_t strides[2] = {cuuint64_t(res) * 4, cuuint64_t(res) * res * 4};
    const cuuint32_t box[3] = {cuuint32_t(sx), cuuint32_t(S), cuuint32_t(S)};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(DJB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", int(r));
    return DJB_OK;
}

// Mass assignment into m0 (and m1) of row pitch `pitch`; `dense`: m0/m1 are the
// solver's dense meshes (bulk tensor reductions allowed).
template <int W, int NS>
void launch_scatter_t(djb_solver* s, const float* mom, float dd1, const GroupShifts& g, float* m0, float* m1,
                      int pitch, bool dense) {
    if (s->tiled && s->cur_perm) {  // brick-owned: the drift was applied by the binning pass
        const unsigned nbricks = unsigned(s->sg.nb) * s->sg.nb * s->sg.nb;
        const int tma = (dense && s->tma) ? 1 : 0;
        djb::k_scatter_brick<W, NS><<<nbricks, djb::kTileThreads, std::min(NS, djb::kScatterBoxes) * scatter_smem(s), s->stream>>>(
            s->psi, s->q1, s->n, s->np, s->Lf, s->res, pitch, g, m0, m1, s->err, brick_list(s), s->tmap_s[0],
            s->tmap_s[NS > 1 ? 1 : 0], tma);
        return;
    }
    if (s->tiled) {
        const dim3 grid = s->cur_perm ? dim3(unsigned((s->np + djb::kTileThreads - 1) / djb::kTileThreads))
                                      : tile_grid(s->n);
        djb::k_scatter_tiled<W, NS><<<grid, djb::kTileThreads, kScatterBudget * sizeof(unsigned int), s->stream>>>(
            s->psi, mom, dd1, s->q1, s->n, s->np, s->Lf, s->res, pitch, g, m0, m1, s->err, kScatterBudget,
            s->cur_perm);
        return;
    }
    djb::k_scatter<W, NS><<<blocks(s->np), kThreads, 0, s->stream>>>(
        s->psi, mom, dd1, s->q1, s->n, s->np, s->Lf, s->res, pitch, g, m0, m1, s->err);
}

void launch_scatter(djb_solver* s, const float* mom, float dd1, const GroupShifts& g, int ns) {
    float* m0 = rho_mesh(s, 0);
    float* m1 = rho_mesh(s, 1);
    const int pitch = rho_pitch(s);
    const bool dense = s->phi[0] != nullptr;
#define DJB_SC(W_)                                                                 \
    if (s->W == W_) {                                                               \
        if (ns == 1) launch_scatter_t<W_, 1>(s, mom, dd1, g, m0, m1, pitch, dense);  \
        else launch_scatter_t<W_, 2>(s, mom, dd1, g, m0, m1, pitch, dense);          \
    }
    DJB_SC(2) DJB_SC(3) DJB_SC(4)
#undef DJB_SC
}

void launch_scatter_positions(djb_solver* s, const float* xr, int64_t count, float* mesh, int pitch) {
    const int b = blocks(count);
    if (s->W == 2) djb::k_scatter_positions<2><<<b, kThreads, 0, s->stream>>>(xr, count, count, s->Lf, s->res, pitch, mesh, s->err);
    if (s->W == 3) djb::k_scatter_positions<3><<<b, kThreads, 0, s->stream>>>(xr, count, count, s->Lf, s->res, pitch, mesh, s->err);
    if (s->W == 4) djb::k_scatter_positions<4><<<b, kThreads, 0, s->stream>>>(xr, count, count, s->Lf, s->res, pitch, mesh, s->err);
}

template <int W, int R>
void launch_gather_wr(djb_solver* s, const djb::GatherArgs& a, int ns) {
    if (R > 0 && s->tiled && a.perm) {
        constexpr int RR = R > 0 ? R : 1;
        const size_t smem = gather_smem(s);
        const unsigned nbricks = unsigned(s->sg.nb) * s->sg.nb * s->sg.nb;
        const int tma = (s->tma && a.mesh[0] == s->phi[0]) ? 1 : 0;
        djb::GatherArgs ag = a;
        ag.part = (a.perm == s->perm) ? s->part : nullptr;
        if (ns == 1)
            djb::k_gather_brick<W, RR, 1><<<nbricks, djb::kTileThreads, smem, s->stream>>>(
                ag, brick_list(s), s->tmap[0], s->tmap[0], tma);
        else
            djb::k_gather_brick<W, RR, 2><<<nbricks, djb::kTileThreads, smem, s->stream>>>(
                ag, brick_list(s), s->tmap[0], s->tmap[1], tma);
        return;
    }
    if (R > 0 && s->tiled) {
        constexpr int RR = R > 0 ? R : 1;
        const size_t smem = kGatherBudget * sizeof(float);
        const dim3 grid = a.perm ? dim3(unsigned((s->np + djb::kTileThreads - 1) / djb::kTileThreads))
                                 : tile_grid(s->n);
        if (ns == 1)
            djb::k_gather_tiled<W, RR, 1><<<grid, djb::kTileThreads, smem, s->stream>>>(a, kGatherBudget);
        else
            djb::k_gather_tiled<W, RR, 2><<<grid, djb::kTileThreads, smem, s->stream>>>(a, kGatherBudget);
        return;
    }
    if (ns == 1) djb::k_gather<W, R, 1><<<blocks(s->np), kThreads, 0, s->stream>>>(a);
    else djb::k_gather<W, R, 2><<<blocks(s->np), kThreads, 0, s->stream>>>(a);
}

// Opt the tiled interpolation kernels in to their shared-memory budget (> 48 KB).
template <int W, int R>
int tiled_attrs_wr() {
    const int smem = kGatherBudget * int(sizeof(float));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_gather_tiled<W, R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_gather_tiled<W, R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_gather_brick<W, R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kBrickSmemMax));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_gather_brick<W, R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kBrickSmemMax));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_gather_brick<W, R, 1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  int(cudaSharedmemCarveoutMaxShared)));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_gather_brick<W, R, 2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  int(cudaSharedmemCarveoutMaxShared)));
    return DJB_OK;
}

template <int W>
int scatter_attrs_w() {
    const int smem = kScatterBudget * int(sizeof(unsigned int));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_scatter_tiled<W, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_scatter_tiled<W, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_scatter_brick<W, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kBrickSmemMax));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_scatter_brick<W, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kBrickSmemMax));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_scatter_weighted_brick<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kBrickSmemMax));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_gather_grad_brick<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kBrickSmemMax));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_interp3_brick<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kBrickSmemMax));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_scatter_brick<W, 1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  int(cudaSharedmemCarveoutMaxShared)));
    CUDA_TRY(cudaFuncSetAttribute(djb::k_scatter_brick<W, 2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  int(cudaSharedmemCarveoutMaxShared)));
    return DJB_OK;
}

int tiled_attrs(int W, int R) {
    // the CIC deposit of djb_state_power_spectrum uses the W = 2 kernels
    TRY(scatter_attrs_w<2>());
    if (W == 3) TRY(scatter_attrs_w<3>());
    if (W == 4) TRY(scatter_attrs_w<4>());
    if (R == 0) return DJB_OK;
#define DJB_TA(W_, R_) \
    if (W == W_ && R == R_) return tiled_attrs_wr<W_, R_>();
    DJB_TA(2, 1) DJB_TA(2, 2) DJB_TA(2, 3) DJB_TA(3, 1) DJB_TA(3, 2) DJB_TA(3, 3)
    DJB_TA(4, 1) DJB_TA(4, 2) DJB_TA(4, 3)
#undef DJB_TA
    return DJB_OK;
}

template <int W>
void launch_gather_w(djb_solver* s, const djb::GatherArgs& a, int ns) {
    switch (s->R) {
        case 0: launch_gather_wr<W, 0>(s, a, ns); break;
        case 1: launch_gather_wr<W, 1>(s, a, ns); break;
        case 2: launch_gather_wr<W, 2>(s, a, ns); break;
        default: launch_gather_wr<W, 3>(s, a, ns); break;
    }
}

void launch_gather(djb_solver* s, const djb::GatherArgs& a, int ns) {
    if (s->W == 2) launch_gather_w<2>(s, a, ns);
    else if (s->W == 3) launch_gather_w<3>(s, a, ns);
    else launch_gather_w<4>(s, a, ns);
}

// Extra particle sets of the Lagrangian sheet for shift `si`, deposited into `mesh`
// (pm.jl:471-484).
int resample_deposit(djb_solver* s, int si, float* mesh) {
    const int n = s->n;
    const int64_t np = s->np;
    const Shift3 sh{float(s->shifts[3 * si]), float(s->shifts[3 * si + 1]), float(s->shifts[3 * si + 2])};
    const int nh = n / 2 + 1;
    const int64_t nspec = int64_t(n) * n * nh;
    const int64_t nreal = int64_t(n) * n * (n + 2);
    const int nof = int(s->rshifts.size() / 3);
    if (s->cfg.resampling == DJB_RESAMPLE_FOURIER) {
        for (int c = 0; c < 3; ++c) {
            djb::k_wrap_psi<<<grid_for(np), kThreads, 0, s->stream>>>(s->psi, s->q1, n, np, s->Lf, sh, c, s->rb, 1);
            CUFFT_TRY(cufftExecR2C(s->r2c_n, s->rb, reinterpret_cast<cufftComplex*>(s->psihat + c * nspec)));
        }
        for (int o = 0; o < nof; ++o) {
            const double d[3] = {s->rshifts[3 * o], s->rshifts[3 * o + 1], s->rshifts[3 * o + 2]};
            const float2* px = s->phase + int64_t(o) * (2 * n + nh);
            for (int c = 0; c < 3; ++c) {
                djb::k_phase<<<grid_for(nspec), kThreads, 0, s->stream>>>(
                    s->psihat + c * nspec, s->cb, n, px, px + n, px + 2 * n, float(1.0 / (double(n) * n * n)));
                CUFFT_TRY(cufftExecC2R(s->c2r_n, reinterpret_cast<cufftComplex*>(s->cb), s->rb));
                djb::k_place<<<grid_for(np), kThreads, 0, s->stream>>>(
                    s->rb, s->q1, n, np, s->Lf, float(d[c] * s->cfg.boxsize / n), c, s->xr);
            }
            launch_scatter_positions(s, s->xr, np, mesh, rho_pitch(s));
        }
        (void)nreal;
    } else {
        djb::k_wrap_psi_lin<<<grid_for(3 * np), kThreads, 0, s->stream>>>(s->psi, s->q1, n, np, s->Lf, sh, s->rb);
        for (int o = 0; o < nof; ++o) {
            const double* d = &s->rshifts[3 * o];
            djb::k_place_linear<<<grid_for(np), kThreads, 0, s->stream>>>(
                s->rb, s->q1, n, np, s->Lf, float(d[0]), float(d[1]), float(d[2]),
                float(d[0] * s->cfg.boxsize / n), float(d[1] * s->cfg.boxsize / n),
                float(d[2] * s->cfg.boxsize / n), s->xr);
            launch_scatter_positions(s, s->xr, np, mesh, rho_pitch(s));
        }
    }
    return DJB_OK;
}

// Force evaluation for all shifts; if `step`, fused with the drift/kick/drift.
// Reads s->psi (and s->mom). Output: s->acc (step == 0) or updated psi/mom.
// The fused z pass of the 1024³ Poisson solve on the half spectrum in `mesh`.
void launch_zpass(djb_solver* s, float* mesh, int nh) {
    const dim3 grid(unsigned((nh + djb::kZPencils - 1) / djb::kZPencils), unsigned(s->res));
    const djb::KPhiFn kp{s->lapT, s->makT, s->s0};
    if (DJB_ZPASS_PAIR)
        djb::k_zpencil_pair<<<grid, djb::kZPairThreads, djb::kZSmem, s->stream>>>(reinterpret_cast<float2*>(mesh), nh,
                                                                                  s->wN, kp);
    else
        djb::k_zpencil_kphi<<<grid, djb::kZThreads, djb::kZSmem, s->stream>>>(reinterpret_cast<float2*>(mesh), nh,
                                                                              s->wN, kp);
}

// Brick sort of the particles at X = q + Ψ (+ dd1·Mom when `mom`): perm (sort.cuh).
int sort_particles(djb_solver* s, const float* mom, float dd1) {
    s->prof.begin(s->stream, PH_SORT);
    CUDA_TRY(cudaMemsetAsync(s->count, 0, size_t(s->nbins) * sizeof(unsigned), s->stream));
    djb::k_bin<<<blocks(s->np), 256, 0, s->stream>>>(s->psi, mom, dd1, s->q1, s->n, s->np, s->Lf, s->sg, s->count,
                                                      s->keyrank, s->err);
    djb::k_scan_block<<<s->nscan, djb::kScanThreads, 0, s->stream>>>(s->count, s->nbins, s->offset, s->bsum);
    djb::k_scan_sums<<<1, djb::kScanThreads, 0, s->stream>>>(s->bsum, s->nscan);
    djb::k_place<<<blocks(s->np), 256, 0, s->stream>>>(s->keyrank, s->np, s->offset, s->bsum, s->perm);
    s->prof.end(s->stream, PH_SORT, 4);
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

dim3 fd_grid(int res);
int fd_vec(const djb_solver* s, int res, int pitch, std::initializer_list<const void*> meshes);
int nn_correction(djb_solver* s);

int force(djb_solver* s, bool step, double dd1, double alpha, double beta, double dd2) {
    const int nh = s->res / 2 + 1;
    const int64_t nspec = int64_t(s->res) * s->res * nh;
    const bool ik = (s->cfg.grad_order == 0);
    const bool resample = (s->cfg.n_resample > 1);
    // the network runs from step nn_start on, on every nn_every-th step (and on every
    // force outside a step); between its evaluations each particle keeps the correction it
    // was last given; before nn_start the force is uncorrected
    const bool nn_active = s->nn && (!step || s->nn_steps >= s->nn_start);
    const bool nn_eval =
        nn_active && (!step || !s->nn_valid || (s->nn_steps - s->nn_start) % s->nn_every == 0);
    if (s->nn && step) ++s->nn_steps;
    if (nn_eval) s->nn_valid = true;
    s->cur_perm = nullptr;
    // the first drift is applied by the binning pass (or the first deposit without the
    // sort), before the network correction reads the positions
    if (s->tiled && s->sorted) {
        TRY(sort_particles(s, (step && dd1 != 0.0) ? s->mom : nullptr, float(dd1)));
        s->cur_perm = s->perm;
    }
    for (int first = 0; first < s->nshift; first += s->group) {
        const int ns = std::min(s->group, s->nshift - first);
        const GroupShifts g = group_shifts(s, first, ns);
        s->prof.begin(s->stream, PH_CLEAR);
        const size_t rho_floats = s->phi[0] ? size_t(s->res) * s->res * s->res : size_t(s->mesh_floats);
        for (int m = 0; m < ns; ++m)
            CUDA_TRY(cudaMemsetAsync(rho_mesh(s, m), 0, rho_floats * sizeof(float), s->stream));
        s->prof.end(s->stream, PH_CLEAR, 0);
        // with the brick sort the binning pass has applied the first drift already
        const bool drift_here = step && first == 0 && !s->cur_perm && dd1 != 0.0;
        s->prof.begin(s->stream, PH_SCATTER);
        launch_scatter(s, drift_here ? s->mom : nullptr, float(dd1), g, ns);
        s->prof.end(s->stream, PH_SCATTER, 1);
        if (resample) {
            s->prof.begin(s->stream, PH_RESAMPLE);
            TRY(resample_deposit(s, first, rho_mesh(s, 0)));
            s->prof.end(s->stream, PH_RESAMPLE, 0);
        }
        for (int m = 0; m < ns; ++m) {
            float* mesh = s->mesh[m];
            cufftComplex* spec = reinterpret_cast<cufftComplex*>(mesh);
            s->prof.begin(s->stream, PH_R2C);
            if (s->phi[m]) CUFFT_TRY(cufftExecR2C(s->r2c_d, s->phi[m], spec));
            else CUFFT_TRY(cufftExecR2C(s->r2c, mesh, spec));
            s->prof.end(s->stream, PH_R2C, 0);
            // network input, δ: the unshifted density is still in phi[0] after the R2C
            const bool nn_here = nn_eval && first == 0 && m == 0;
            if (nn_here) {
                const float f = float(double(s->res) * s->res * s->res / double(s->np));
                djb::k_mesh_affine<<<grid_for(int64_t(s->res) * s->res * s->res), 256, 0, s->stream>>>(
                    s->phi[0], s->res, s->res, f * s->nn_in, s->nn_in, s->nnf);
            }
            if (s->zpass) {
                s->prof.begin(s->stream, PH_KSPACE);
                const int nh = s->res / 2 + 1;
                launch_zpass(s, mesh, nh);
                s->prof.end(s->stream, PH_KSPACE, 1);
                s->prof.begin(s->stream, PH_C2R);
                CUFFT_TRY(cufftExecC2R(s->c2r_d, spec, s->phi[m]));
                s->prof.end(s->stream, PH_C2R, 0);
            } else if (!ik) {
                s->prof.begin(s->stream, PH_KSPACE);
                djb::k_kspace_mul<<<dim3(unsigned((s->res + djb::kSpecRows - 1) / djb::kSpecRows), unsigned(s->res)),
                                    kThreads, 0, s->stream>>>(
                    reinterpret_cast<float2*>(mesh), s->res, s->lapT, s->makT, s->s0);
                s->prof.end(s->stream, PH_KSPACE, 1);
                s->prof.begin(s->stream, PH_C2R);
                if (s->phi[m]) CUFFT_TRY(cufftExecC2R(s->c2r_d, spec, s->phi[m]));
                else CUFFT_TRY(cufftExecC2R(s->c2r, spec, mesh));
                s->prof.end(s->stream, PH_C2R, 0);
            } else {
                s->prof.begin(s->stream, PH_KSPACE);
                djb::k_kspace_ik<<<grid_for(nspec), kThreads, 0, s->stream>>>(
                    reinterpret_cast<const float2*>(mesh), s->res, s->lapT, s->makT, s->s0, s->gh, s->gf,
                    reinterpret_cast<float2*>(s->fmesh[m][0]), reinterpret_cast<float2*>(s->fmesh[m][1]),
                    reinterpret_cast<float2*>(s->fmesh[m][2]));
                s->prof.end(s->stream, PH_KSPACE, 1);
                s->prof.begin(s->stream, PH_C2R);
                for (int c = 0; c < 3; ++c)
                    CUFFT_TRY(cufftExecC2R(s->c2r, reinterpret_cast<cufftComplex*>(s->fmesh[m][c]),
                                           s->fmesh[m][c]));
                s->prof.end(s->stream, PH_C2R, 0);
            }
            if (nn_here) {
                // network input, F = −Dφ of the unshifted potential; then the network and
                // the interpolation of its output to the particles
                const int64_t cells = int64_t(s->res) * s->res * s->res;
                s->prof.begin(s->stream, PH_NN);
                djb::k_fd_grad3<<<fd_grid(s->res), djb::kFdThreads, 0, s->stream>>>(
                    s->phi[0], s->res, s->res, s->c1 * s->nn_fin, s->c2 * s->nn_fin, s->c3 * s->nn_fin,
                    s->nnf + cells, s->nnf + 2 * cells, s->nnf + 3 * cells,
                    fd_vec(s, s->res, s->res, {s->phi[0], s->nnf + cells, s->nnf + 2 * cells, s->nnf + 3 * cells}));
                TRY(nn_correction(s));
                s->prof.end(s->stream, PH_NN, 3);
            }
        }
        djb::GatherArgs a{};
        a.psi = s->psi;
        a.mom = s->mom;
        a.acc = s->acc;
        a.q1 = s->q1;
        for (int m = 0; m < ns; ++m) {
            a.mesh[m] = ik ? s->fmesh[m][0] : (s->phi[m] ? s->phi[m] : s->mesh[m]);
            a.meshy[m] = ik ? s->fmesh[m][1] : nullptr;
            a.meshz[m] = ik ? s->fmesh[m][2] : nullptr;
        }
        a.sh = g;
        a.n = s->n;
        a.np = s->np;
        a.L = s->Lf;
        a.res = s->res;
        a.pitch = (!ik && s->phi[0]) ? s->res : s->pitch;
        a.c1 = s->c1;
        a.c2 = s->c2;
        a.c3 = s->c3;
        a.first = (first == 0);
        a.last = (first + ns >= s->nshift);
        a.divide = (s->nshift > 1);
        a.nshift_f = float(s->nshift);
        a.step = step ? 1 : 0;
        a.alpha = float(alpha);
        a.beta = float(beta);
        a.dd2 = float(dd2);
        a.err = s->err;
        a.perm = s->cur_perm;
        a.extra = nn_active ? s->nnacc : nullptr;
        s->prof.begin(s->stream, PH_GATHER);
        launch_gather(s, a, ns);
        s->prof.end(s->stream, PH_GATHER, 1);
    }
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

// Potential of the density in rho_mesh(s, m), left in the same mesh: R2C, Kφ, C2R with the
// force's transforms (finite-difference configurations).
int poisson(djb_solver* s, int m) {
    float* mesh = s->mesh[m];
    cufftComplex* spec = reinterpret_cast<cufftComplex*>(mesh);
    if (s->phi[m]) CUFFT_TRY(cufftExecR2C(s->r2c_d, s->phi[m], spec));
    else CUFFT_TRY(cufftExecR2C(s->r2c, mesh, spec));
    const int nh = s->res / 2 + 1;
    if (s->zpass) {
        launch_zpass(s, mesh, nh);
        CUFFT_TRY(cufftExecC2R(s->c2r_d, spec, s->phi[m]));
    } else {
        djb::k_kspace_mul<<<dim3(unsigned((s->res + djb::kSpecRows - 1) / djb::kSpecRows), unsigned(s->res)), kThreads,
                            0, s->stream>>>(reinterpret_cast<float2*>(mesh), s->res, s->lapT, s->makT, s->s0);
        if (s->phi[m]) CUFFT_TRY(cufftExecC2R(s->c2r_d, spec, s->phi[m]));
        else CUFFT_TRY(cufftExecC2R(s->c2r, spec, mesh));
    }
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

// Grid of the column-sweep stencil kernels for a res^3 mesh.
dim3 fd_grid(int res) {
    return dim3(unsigned((res + djb::kFdTX - 1) / djb::kFdTX), unsigned((res + djb::kFdTY - 1) / djb::kFdTY),
                unsigned((res + djb::kFdZ - 1) / djb::kFdZ));
}

// 1 when the stencil kernels may stage with 16-byte copies: rows and the mesh width are
// multiples of 4 floats and every mesh is 16-byte aligned.
int fd_vec(const djb_solver* s, int res, int pitch, std::initializer_list<const void*> meshes) {
    if (s->fd_scalar || (res & 3) || (pitch & 3)) return 0;
    for (const void* m : meshes)
        if (reinterpret_cast<uintptr_t>(m) & 15u) return 0;
    return 1;
}

// The attached network on its scaled inputs in s->nnf (filled by the force pipeline),
// then its output, times nn_out, interpolated to the particles at s->psi into s->nnacc.
int nn_correction(djb_solver* s) {
    TRY(djb_nn_set_stream(s->nn, s->stream));
    TRY(djb_nn_apply(s->nn, s->nnf, s->res, s->nnd, DJB_MEM_DEVICE));
    // brick-owned form when the particles are in brick order and the three fields' deposit
    // boxes fit two CTAs per SM
    const int sxI = (s->sS + ((s->sg.brick % 4 == 0) ? (s->sfirst & 3) : 3) + 3) & ~3;
    const size_t smem = 3 * size_t(djb::box_stride(sxI * s->sS * s->sS)) * 4;
    if (s->cur_perm && s->tiled && smem <= size_t(kBrickSmemMax)) {
        const int64_t cells = int64_t(s->res) * s->res * s->res;
        CUtensorMap tm[3];
        int tma = 0;
        if (s->tma && s->phi[0] && sxI <= s->res) {
            for (int c = 0; c < 3; ++c) TRY(make_tmap(&tm[c], s->nnd + c * cells, s->res, sxI, s->sS));
            tma = 1;
        } else {
            for (int c = 0; c < 3; ++c) tm[c] = s->tmap_s[0];
        }
        const unsigned nbricks = unsigned(s->sg.nb) * s->sg.nb * s->sg.nb;
#define DJB_INTERPB(W_)                                                                                        \
    if (s->W == W_)                                                                                            \
        djb::k_interp3_brick<W_><<<nbricks, djb::kTileThreads, smem, s->stream>>>(                             \
            s->psi, s->q1, s->n, s->np, s->Lf, s->res, s->nnd, s->nn_out, s->nnacc, s->err, brick_list(s), sxI,  \
            tm[0], tm[1], tm[2], tma);
        DJB_INTERPB(2)
        DJB_INTERPB(3)
        DJB_INTERPB(4)
#undef DJB_INTERPB
        CUDA_TRY(cudaGetLastError());
        return DJB_OK;
    }
#define DJB_INTERP(W_)                                                                                          \
    if (s->W == W_)                                                                                             \
        djb::k_interp3<W_><<<blocks(s->np), kThreads, 0, s->stream>>>(s->psi, s->q1, s->n, s->np, s->Lf, s->res, \
                                                                      s->nnd, s->nn_out, s->nnacc, s->err,   \
                                                                      s->cur_perm);
    DJB_INTERP(2)
    DJB_INTERP(3)
    DJB_INTERP(4)
#undef DJB_INTERP
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

// perm != null: psi, abar and psibar are in brick order (gathered through perm).
template <int W>
void launch_vjp_kernels(djb_solver* s, int stage, const float* psi, const float* abar, float* psibar,
                        const Shift3& sh, float scale, const int* perm) {
    float* rho = rho_mesh(s, 0);
    const int pitch = rho_pitch(s);
    const int b = blocks(s->np);
    if (perm) {   // brick-owned forms: boxes in shared memory, one CTA per brick
        const unsigned nbricks = unsigned(s->sg.nb) * s->sg.nb * s->sg.nb;
        const size_t smem = scatter_smem(s);
        const djb::BrickList bl = brick_list(s);
        const int tma = s->have_tmap_adj ? 1 : 0;
        if (stage == 0)
            djb::k_gather_grad_brick<W><<<nbricks, djb::kTileThreads, smem, s->stream>>>(
                psi, s->q1, s->n, s->np, s->Lf, s->res, pitch, sh.x, sh.y, sh.z, s->adj[0], s->adj[1], s->adj[2],
                abar, scale, psibar, s->err, bl, 1, s->tmap_adj[0], s->tmap_adj[1], s->tmap_adj[2], tma);
        else if (stage == 1)
            djb::k_scatter_weighted_brick<W><<<nbricks, djb::kTileThreads, smem, s->stream>>>(
                psi, s->q1, s->n, s->np, s->Lf, s->res, pitch, sh.x, sh.y, sh.z, abar, scale, s->adj[0], s->adj[1],
                s->adj[2], s->err, bl, 1, s->tmap_adj[0], s->tmap_adj[1], s->tmap_adj[2], tma);
        else
            djb::k_gather_grad_brick<W><<<nbricks, djb::kTileThreads, smem, s->stream>>>(
                psi, s->q1, s->n, s->np, s->Lf, s->res, pitch, sh.x, sh.y, sh.z, rho, nullptr, nullptr, nullptr,
                scale, psibar, s->err, bl, 1, s->tmap_rho, s->tmap_rho, s->tmap_rho, tma);
        return;
    }
    if (stage == 0)
        djb::k_gather_grad<W><<<b, 256, 0, s->stream>>>(psi, s->q1, s->n, s->np, s->Lf, s->res, pitch, sh.x, sh.y,
                                                         sh.z, s->adj[0], s->adj[1], s->adj[2], abar, scale, psibar,
                                                         s->err, perm);
    else if (stage == 1)
        djb::k_scatter_weighted<W><<<b, 256, 0, s->stream>>>(psi, s->q1, s->n, s->np, s->Lf, s->res, pitch, sh.x,
                                                              sh.y, sh.z, abar, scale, s->adj[0], s->adj[1],
                                                              s->adj[2], s->err, perm);
    else
        djb::k_gather_grad<W><<<b, 256, 0, s->stream>>>(psi, s->q1, s->n, s->np, s->Lf, s->res, pitch, sh.x, sh.y,
                                                         sh.z, rho, nullptr, nullptr, nullptr, scale, psibar, s->err,
                                                         perm);
}

void vjp_kernels(djb_solver* s, int stage, const float* psi, const float* abar, float* psibar, const Shift3& sh,
                 float scale, const int* perm) {
    if (s->W == 2) launch_vjp_kernels<2>(s, stage, psi, abar, psibar, sh, scale, perm);
    else if (s->W == 3) launch_vjp_kernels<3>(s, stage, psi, abar, psibar, sh, scale, perm);
    else launch_vjp_kernels<4>(s, stage, psi, abar, psibar, sh, scale, perm);
}

// psibar += (∂acc/∂Ψ)ᵀ abar at the displacements psi (device arrays, Lagrangian order).
int force_vjp(djb_solver* s, float* psi, const float* abar, float* psibar) {
    if (s->cfg.grad_order == 0 || s->cfg.n_resample > 1)
        return fail(DJB_ERR_INVALID, "the force VJP covers finite-difference gradients (2/4/6) without resampling");
    const size_t rho_floats = s->phi[0] ? size_t(s->res) * s->res * s->res : size_t(s->mesh_floats);
    for (int c = 0; c < 3; ++c)
        if (!s->adj[c]) TRY(dmalloc(s, (void**)&s->adj[c], rho_floats * sizeof(float)));
    if (s->tma && s->phi[0] && !s->have_tmap_adj) {   // dense meshes: bulk reductions of the cotangent deposit
        for (int c = 0; c < 3; ++c) TRY(make_tmap(&s->tmap_adj[c], s->adj[c], s->res, s->ssx, s->sS));
        TRY(make_tmap(&s->tmap_rho, rho_mesh(s, 0), s->res, s->ssx, s->sS));
        s->have_tmap_adj = true;
    }
    float* rho = rho_mesh(s, 0);
    const int pitch = rho_pitch(s);
    const float inv_ns = 1.0f / float(s->nshift);
    // visit the particles in brick order (the forward's counting sort on these positions):
    // the gathers and float atomics below then stay within L2-resident neighbourhoods
    const int* perm = nullptr;
    if (s->tiled && s->sorted) {
        CUDA_TRY(cudaMemsetAsync(s->count, 0, size_t(s->nbins) * sizeof(unsigned), s->stream));
        djb::k_bin<<<blocks(s->np), 256, 0, s->stream>>>(psi, nullptr, 0.0f, s->q1, s->n, s->np, s->Lf, s->sg,
                                                          s->count, s->keyrank, s->err);
        djb::k_scan_block<<<s->nscan, djb::kScanThreads, 0, s->stream>>>(s->count, s->nbins, s->offset, s->bsum);
        djb::k_scan_sums<<<1, djb::kScanThreads, 0, s->stream>>>(s->bsum, s->nscan);
        djb::k_place<<<blocks(s->np), 256, 0, s->stream>>>(s->keyrank, s->np, s->offset, s->bsum, s->perm);
        perm = s->perm;
    }
    // the brick kernels read positions and cotangents in brick order (coalesced) and
    // accumulate Ψ̄ there; it goes back to the Lagrangian order once at the end
    const size_t pcount = size_t(3 * s->np);
    float *psi_s = nullptr, *abar_s = nullptr, *pb_s = nullptr;
    if (perm) {
        TRY(scratch(s, 7, pcount, &psi_s));
        TRY(scratch(s, 8, pcount, &abar_s));
        TRY(scratch(s, 9, pcount, &pb_s));
        djb::k_gather_sorted3<<<blocks(s->np), 256, 0, s->stream>>>(psi, perm, s->np, psi_s);
        djb::k_gather_sorted3<<<blocks(s->np), 256, 0, s->stream>>>(abar, perm, s->np, abar_s);
        CUDA_TRY(cudaMemsetAsync(pb_s, 0, pcount * sizeof(float), s->stream));
    }
    const float* kpsi = perm ? psi_s : psi;
    const float* kabar = perm ? abar_s : abar;
    float* kpb = perm ? pb_s : psibar;
    for (int si = 0; si < s->nshift; ++si) {
        const GroupShifts g = group_shifts(s, si, 1);
        const Shift3 sh = g.s[0];
        CUDA_TRY(cudaMemsetAsync(rho, 0, rho_floats * sizeof(float), s->stream));
        if (perm) {   // the forward's brick-owned deposit on these positions
            const unsigned nbricks = unsigned(s->sg.nb) * s->sg.nb * s->sg.nb;
            const int tma = (s->phi[0] != nullptr && s->tma) ? 1 : 0;
#define DJB_VS(W_)                                                                                             \
    if (s->W == W_)                                                                                            \
        djb::k_scatter_brick<W_, 1><<<nbricks, djb::kTileThreads, scatter_smem(s), s->stream>>>(                \
            psi, s->q1, s->n, s->np, s->Lf, s->res, pitch, g, rho, nullptr, s->err, brick_list(s), s->tmap_s[0], \
            s->tmap_s[0], tma);
            DJB_VS(2) DJB_VS(3) DJB_VS(4)
#undef DJB_VS
        } else {
            if (s->W == 2) djb::k_scatter<2, 1><<<blocks(s->np), kThreads, 0, s->stream>>>(
                psi, nullptr, 0.0f, s->q1, s->n, s->np, s->Lf, s->res, pitch, g, rho, nullptr, s->err);
            if (s->W == 3) djb::k_scatter<3, 1><<<blocks(s->np), kThreads, 0, s->stream>>>(
                psi, nullptr, 0.0f, s->q1, s->n, s->np, s->Lf, s->res, pitch, g, rho, nullptr, s->err);
            if (s->W == 4) djb::k_scatter<4, 1><<<blocks(s->np), kThreads, 0, s->stream>>>(
                psi, nullptr, 0.0f, s->q1, s->n, s->np, s->Lf, s->res, pitch, g, rho, nullptr, s->err);
        }
        TRY(poisson(s, 0));  // φ
        djb::k_fd_grad3<<<fd_grid(s->res), djb::kFdThreads, 0, s->stream>>>(
            rho, s->res, pitch, s->c1, s->c2, s->c3, s->adj[0], s->adj[1], s->adj[2],
            fd_vec(s, s->res, pitch, {rho, s->adj[0], s->adj[1], s->adj[2]}));
        vjp_kernels(s, 0, kpsi, kabar, kpb, sh, inv_ns, perm);  // interpolation weights
        for (int c = 0; c < 3; ++c) CUDA_TRY(cudaMemsetAsync(s->adj[c], 0, rho_floats * sizeof(float), s->stream));
        vjp_kernels(s, 1, kpsi, kabar, kpb, sh, inv_ns, perm);  // Ḡ
        djb::k_fd_div3<<<fd_grid(s->res), djb::kFdThreads, 0, s->stream>>>(
            s->adj[0], s->adj[1], s->adj[2], s->res, pitch, s->c1, s->c2, s->c3, rho,
            fd_vec(s, s->res, pitch, {rho, s->adj[0], s->adj[1], s->adj[2]}));  // φ̄
        TRY(poisson(s, 0));                                    // ρ̄
        vjp_kernels(s, 2, kpsi, kabar, kpb, sh, 1.0f, perm);  // deposit weights
    }
    if (perm) djb::k_scatter_add_sorted3<<<blocks(s->np), 256, 0, s->stream>>>(pb_s, perm, s->np, psibar);
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

int check_err(djb_solver* s) {
    int h = 0;
    CUDA_TRY(cudaMemcpyAsync(&h, s->err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (h) {
        CUDA_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->stream));
        return fail(DJB_ERR_DEVICE, "non-finite particle position encountered (device error word %d)", h);
    }
    return DJB_OK;
}

int copy_in(djb_solver* s, float* dst, const float* src, size_t count, int mem) {
    CUDA_TRY(cudaMemcpyAsync(dst, src, count * sizeof(float),
                             mem == DJB_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                             s->stream));
    return DJB_OK;
}

int copy_out(djb_solver* s, float* dst, const float* src, size_t count, int mem) {
    CUDA_TRY(cudaMemcpyAsync(dst, src, count * sizeof(float),
                             mem == DJB_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                             s->stream));
    return DJB_OK;
}

void release(djb_solver* s) {
    if (!s) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->cfg.device);
    s->prof.destroy();
    if (s->have_r2c) cufftDestroy(s->r2c);
    if (s->have_c2r) cufftDestroy(s->c2r);
    if (s->have_r2c_n) cufftDestroy(s->r2c_n);
    if (s->have_c2r_n) cufftDestroy(s->c2r_n);
    if (s->have_c2r_d) cufftDestroy(s->c2r_d);
    if (s->have_r2c_d) cufftDestroy(s->r2c_d);
    for (void* p : s->allocs) cudaFree(p);
    for (float* p : s->scr)
        if (p) cudaFree(p);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
    if (prev >= 0) cudaSetDevice(prev);
    delete s;
}

int create(const djb_pm_config* cfg, djb_solver** out) {
    TRY(validate(*cfg));
    djb_solver* s = new (std::nothrow) djb_solver();
    if (!s) return fail(DJB_ERR_ALLOC, "host allocation failed");
    *out = s;
    s->cfg = *cfg;
    CUDA_TRY(cudaSetDevice(cfg->device));
    s->n = cfg->n_part;
    s->res = cfg->res_pm;
    s->pitch = s->res + 2;
    s->np = int64_t(s->n) * s->n * s->n;
    s->mesh_floats = int64_t(s->res) * s->res * s->pitch;
    s->L = cfg->boxsize;
    s->Lf = float(cfg->boxsize);
    s->W = cfg->worder;
    s->R = cfg->grad_order / 2;
    {
        const char* kind = std::getenv("DJB_KERNELS");
        s->tiled = !(kind && std::strcmp(kind, "simple") == 0);
    }
    if (s->tiled) TRY(tiled_attrs(s->W, s->R));
    {
        const char* fs = std::getenv("DJB_FD_SCALAR");
        s->fd_scalar = fs && std::strcmp(fs, "1") == 0;
    }
    {
        const char* srt = std::getenv("DJB_SORT");
        s->sorted = s->tiled && !(srt && std::strcmp(srt, "0") == 0);
    }
    s->shifts = aa_shifts(cfg->antialias, 0.5 * s->L / s->res);
    s->nshift = int(s->shifts.size() / 3);
    const bool resample = cfg->n_resample > 1;
    const bool ik = cfg->grad_order == 0;
    s->group = resample ? 1 : std::min(kMaxGroup, s->nshift);
    if (resample) s->rshifts = resample_shifts(cfg->n_resample);
    if (!ik) {
        // pm.jl:419-424 in float64, rounded to float like T.(...)
        const double h = s->L / s->res;
        double d1 = 0, d2 = 0, d3 = 0;
        if (cfg->grad_order == 2) d1 = 1 / (2 * h);
        if (cfg->grad_order == 4) { d1 = 8 / (12 * h); d2 = -1 / (12 * h); }
        if (cfg->grad_order == 6) { d1 = 45 / (60 * h); d2 = -9 / (60 * h); d3 = 1 / (60 * h); }
        s->c1 = float(d1);
        s->c2 = float(d2);
        s->c3 = float(d3);
    }
    CUDA_TRY(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, cfg->device));
    s->stream = s->own_stream;

    // 1-D tables (float64): lap terms, deconvolution, ik gradient
    const int res = s->res;
    std::vector<double> T(res), M(res);
    const double dk = 2 * M_PI / s->L;
    const double mm = (res / 2) * dk / M_PI;  // maximum(abs.(k))/π = res/L
    for (int i = 0; i < res; ++i) {
        const double k = (i < res / 2 ? i : i - res) * 2 * M_PI / s->L;
        if (cfg->lap_order == 0) {
            T[i] = -(k * k);
        } else {
            const double c1 = std::cos(k / mm), c2 = std::cos(2 * k / mm), c3 = std::cos(3 * k / mm);
            if (cfg->lap_order == 2) T[i] = -2 * (1 - c1) * mm * mm;
            if (cfg->lap_order == 4) T[i] = -(c2 - 16 * c1 + 15) / 6 * (mm * mm);
            if (cfg->lap_order == 6) T[i] = -(-2 * c3 + 27 * c2 - 270 * c1 + 245) / 90 * (mm * mm);
        }
        const double x = k / (2 * M_PI) / mm;
        const double sinc = (x == 0) ? 1.0 : std::sin(M_PI * x) / (M_PI * x);
        M[i] = std::pow(sinc, -2.0 * cfg->worder);
    }
    // The 1-D tables serve the halved axis too: every term is even in k.
    const double rhomean = double(s->np) / (double(res) * res * res);
    const double nsets = double(cfg->n_resample) * cfg->n_resample * cfg->n_resample;
    s->s0 = 1.0 / rhomean / nsets / (double(res) * res * res);
    TRY(dmalloc(s, (void**)&s->lapT, sizeof(double) * res));
    CUDA_TRY(cudaMemcpy(s->lapT, T.data(), sizeof(double) * res, cudaMemcpyHostToDevice));
    if (cfg->deconvolve) {
        TRY(dmalloc(s, (void**)&s->makT, sizeof(double) * res));
        CUDA_TRY(cudaMemcpy(s->makT, M.data(), sizeof(double) * res, cudaMemcpyHostToDevice));
    }
    if (ik) {
        std::vector<float> gh(res / 2 + 1), gf(res);
        for (int m = 0; m <= res / 2; ++m) gh[m] = (m == res / 2) ? 0.0f : float(m * 2 * M_PI / s->L);
        for (int m = 0; m < res; ++m) gf[m] = (m == res / 2) ? 0.0f : float((m < res / 2 ? m : m - res) * 2 * M_PI / s->L);
        TRY(dmalloc(s, (void**)&s->gh, sizeof(float) * gh.size()));
        TRY(dmalloc(s, (void**)&s->gf, sizeof(float) * gf.size()));
        CUDA_TRY(cudaMemcpy(s->gh, gh.data(), sizeof(float) * gh.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(s->gf, gf.data(), sizeof(float) * gf.size(), cudaMemcpyHostToDevice));
    }
    // lattice coordinates (pm.jl:186): float(i * (L/n))
    std::vector<float> q(s->n);
    for (int i = 0; i < s->n; ++i) q[i] = float(i * (s->L / s->n));
    TRY(dmalloc(s, (void**)&s->q1, sizeof(float) * s->n));
    CUDA_TRY(cudaMemcpy(s->q1, q.data(), sizeof(float) * s->n, cudaMemcpyHostToDevice));

    const size_t pbytes = size_t(3 * s->np) * sizeof(float);
    TRY(dmalloc(s, (void**)&s->psi, pbytes));
    TRY(dmalloc(s, (void**)&s->mom, pbytes));
    TRY(dmalloc(s, (void**)&s->acc, pbytes));
    for (int m = 0; m < s->group; ++m) {
        TRY(dmalloc(s, (void**)&s->mesh[m], size_t(s->mesh_floats) * sizeof(float)));
        if (ik)
            for (int c = 0; c < 3; ++c)
                TRY(dmalloc(s, (void**)&s->fmesh[m][c], size_t(s->mesh_floats) * sizeof(float)));
    }
    TRY(dmalloc(s, (void**)&s->err, sizeof(int)));
    if (s->sorted) {
        // bricks of 16^3 cells; smaller when a box would not stay well inside the periodic
        // mesh (box_rel needs res > box width + 4)
        int brick = 16, lgb = 4;
        brick_boxes(s, brick);
        while (brick > 2 && (brick > s->res / 2 || s->gsx + 4 >= s->res)) {
            brick /= 2;
            --lgb;
            brick_boxes(s, brick);
        }
        const int nb = (s->res + brick - 1) / brick;
        const int hb = brick > 2 ? brick / 2 : 1;
        s->sg = djb::SortGeom{s->res, brick, lgb, nb, hb};
        s->nbins = int64_t(nb) * nb * nb * hb * hb * hb;  // keys: bricks x 2^3-cell sub-blocks
        if (s->nbins > int64_t(djb::kScanBlock) * djb::kScanThreads * 64)
            return fail(DJB_ERR_INVALID, "mesh too large for the particle sort (%lld keys)", (long long)s->nbins);
        if (gather_smem(s) > size_t(kBrickSmemMax) || s->group * scatter_smem(s) > size_t(kBrickSmemMax))
            return fail(DJB_ERR_INVALID, "brick box exceeds the shared-memory budget");
        s->nscan = int((s->nbins + djb::kScanBlock - 1) / djb::kScanBlock);
        TRY(dmalloc(s, (void**)&s->count, sizeof(unsigned) * size_t(s->nbins)));
        TRY(dmalloc(s, (void**)&s->offset, sizeof(unsigned) * size_t(s->nbins)));
        TRY(dmalloc(s, (void**)&s->bsum, sizeof(unsigned) * size_t(s->nscan)));
        TRY(dmalloc(s, (void**)&s->keyrank, sizeof(uint2) * size_t(s->np)));
        TRY(dmalloc(s, (void**)&s->perm, sizeof(int) * size_t(s->np)));
        // sorted-order partial sums of the brick interpolation (several shifts);
        // DJB_GATHER_PART=0: through the acceleration array in particle order
        const char* gp = std::getenv("DJB_GATHER_PART");
        if (s->R > 0 && s->nshift > 1 && !(gp && std::strcmp(gp, "0") == 0))
            TRY(dmalloc(s, (void**)&s->part, 6 * sizeof(float) * size_t(s->np)));
    }
    CUDA_TRY(cudaMemset(s->err, 0, sizeof(int)));
    size_t work = 0;
    TRY(make_plan(&s->r2c, &s->have_r2c, res, CUFFT_R2C, s->stream, &work));
    s->bytes += int64_t(work);
    TRY(make_plan(&s->c2r, &s->have_c2r, res, CUFFT_C2R, s->stream, &work));
    s->bytes += int64_t(work);
    if (!ik && !cfg->lean && res % 4 == 0) {
        // dense potentials written by an out-of-place C2R from the (padded) spectrum
        for (int m = 0; m < s->group; ++m)
            TRY(dmalloc(s, (void**)&s->phi[m], sizeof(float) * size_t(res) * res * res));
        {
            const char* zp = std::getenv("DJB_ZPASS");
            s->zpass = (res == djb::kZRes) && !(zp && std::strcmp(zp, "0") == 0);
        }
        // 3-D transforms, or with the fused z pass 2-D transforms batched over the z planes
        const int rank = s->zpass ? 2 : 3;
        const long long batch = s->zpass ? res : 1;
        long long dims[3] = {res, res, res};
        long long cembed[3] = {res, res, res / 2 + 1};
        long long dembed[3] = {res, res, res};
        long long* cd = s->zpass ? cembed + 1 : cembed;
        long long* dd = s->zpass ? dembed + 1 : dembed;
        const long long cdist = s->zpass ? cembed[1] * cembed[2] : cembed[0] * cembed[1] * cembed[2];
        const long long ddist = s->zpass ? dembed[1] * dembed[2] : dembed[0] * dembed[1] * dembed[2];
        CUFFT_TRY(cufftCreate(&s->c2r_d));
        s->have_c2r_d = true;
        CUFFT_TRY(cufftMakePlanMany64(s->c2r_d, rank, s->zpass ? dims + 1 : dims, cd, 1, cdist, dd, 1, ddist,
                                      CUFFT_C2R, batch, &work));
        CUFFT_TRY(cufftSetStream(s->c2r_d, s->stream));
        s->bytes += int64_t(work);
        CUFFT_TRY(cufftCreate(&s->r2c_d));
        s->have_r2c_d = true;
        CUFFT_TRY(cufftMakePlanMany64(s->r2c_d, rank, s->zpass ? dims + 1 : dims, dd, 1, ddist, cd, 1, cdist,
                                      CUFFT_R2C, batch, &work));
        CUFFT_TRY(cufftSetStream(s->r2c_d, s->stream));
        s->bytes += int64_t(work);
        if (s->zpass) {
            std::vector<float2> w(res);
            for (int j = 0; j < res; ++j)
                w[j] = make_float2(float(std::cos(2 * M_PI * j / res)), float(-std::sin(2 * M_PI * j / res)));
            TRY(dmalloc(s, (void**)&s->wN, sizeof(float2) * res));
            CUDA_TRY(cudaMemcpy(s->wN, w.data(), sizeof(float2) * res, cudaMemcpyHostToDevice));
            float2 w32[16];
            for (int j = 0; j < 16; ++j)
                w32[j] = make_float2(float(std::cos(2 * M_PI * j / 32)), float(-std::sin(2 * M_PI * j / 32)));
            CUDA_TRY(cudaMemcpyToSymbol(djb::c_w32, w32, sizeof(w32)));
            CUDA_TRY(cudaFuncSetAttribute(djb::k_zpencil_kphi<djb::KPhiFn>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, djb::kZSmem));
            CUDA_TRY(cudaFuncSetAttribute(djb::k_zpencil_pair<djb::KPhiFn>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, djb::kZSmem));
        }
        const char* tm = std::getenv("DJB_TMA");   // DJB_TMA=0: boxes by asynchronous copies only
        if (s->sorted && s->gsx <= res && !(tm && std::strcmp(tm, "0") == 0)) {
            for (int m = 0; m < s->group; ++m) {
                TRY(make_tmap(&s->tmap[m], s->phi[m], res, s->gsx, s->gS));
                TRY(make_tmap(&s->tmap_s[m], s->phi[m], res, s->ssx, s->sS));
            }
            for (int m = s->group; m < kMaxGroup; ++m) {
                s->tmap[m] = s->tmap[0];
                s->tmap_s[m] = s->tmap_s[0];
            }
            s->tma = true;
        }
    }
    if (resample) {
        const int n = s->n, nh = n / 2 + 1;
        const int64_t nspec = int64_t(n) * n * nh;
        TRY(dmalloc(s, (void**)&s->rb, sizeof(float) * std::max<int64_t>(int64_t(n) * n * (n + 2), 3 * s->np)));
        TRY(dmalloc(s, (void**)&s->xr, pbytes));
        if (cfg->resampling == DJB_RESAMPLE_FOURIER) {
            TRY(dmalloc(s, (void**)&s->psihat, sizeof(float2) * 3 * nspec));
            TRY(dmalloc(s, (void**)&s->cb, sizeof(float2) * nspec));
            // phase tables exp(2πi m d/n) per offset (pm.jl:453-456); full axes hold
            // -n/2 at index n/2, the halved axis m/n for m = 0..n/2
            const int nof = int(s->rshifts.size() / 3);
            std::vector<float2> h(size_t(nof) * (2 * n + nh));
            for (int o = 0; o < nof; ++o) {
                const double* d = &s->rshifts[3 * o];
                float2* t = &h[size_t(o) * (2 * n + nh)];
                for (int m = 0; m < n; ++m) {
                    const double mf = double(m < n / 2 ? m : m - n) / n;
                    t[m] = make_float2(float(std::cos(2 * M_PI * mf * d[0])), float(std::sin(2 * M_PI * mf * d[0])));
                    t[n + m] = make_float2(float(std::cos(2 * M_PI * mf * d[1])), float(std::sin(2 * M_PI * mf * d[1])));
                }
                for (int m = 0; m < nh; ++m) {
                    const double mh = double(m) / n;
                    t[2 * n + m] = make_float2(float(std::cos(2 * M_PI * mh * d[2])), float(std::sin(2 * M_PI * mh * d[2])));
                }
            }
            TRY(dmalloc(s, (void**)&s->phase, sizeof(float2) * h.size()));
            CUDA_TRY(cudaMemcpy(s->phase, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice));
            TRY(make_plan(&s->r2c_n, &s->have_r2c_n, n, CUFFT_R2C, s->stream, &work));
            s->bytes += int64_t(work);
            TRY(make_plan(&s->c2r_n, &s->have_c2r_n, n, CUFFT_C2R, s->stream, &work));
            s->bytes += int64_t(work);
        }
    }
    return DJB_OK;
}

}  // namespace

extern "C" {

const char* djb_version(void) { return "djb200 0.1 (sm_100a)"; }

int djb_solver_create(const djb_pm_config* cfg, djb_solver** out) {
    djb::clear_error();
    if (!cfg || !out) return fail(DJB_ERR_INVALID, "djb_solver_create: null argument");
    *out = nullptr;
    djb_solver* s = nullptr;
    int rc = create(cfg, &s);
    if (rc != DJB_OK) {
        std::string msg = djb_last_error();
        release(s);
        return fail(rc, "%s", msg.c_str());
    }
    *out = s;
    return DJB_OK;
}

int djb_solver_destroy(djb_solver* s) {
    release(s);
    return DJB_OK;
}

int djb_solver_set_stream(djb_solver* s, void* stream) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    s->stream = stream ? static_cast<cudaStream_t>(stream) : s->own_stream;
    if (s->have_r2c) CUFFT_TRY(cufftSetStream(s->r2c, s->stream));
    if (s->have_c2r) CUFFT_TRY(cufftSetStream(s->c2r, s->stream));
    if (s->have_r2c_n) CUFFT_TRY(cufftSetStream(s->r2c_n, s->stream));
    if (s->have_c2r_n) CUFFT_TRY(cufftSetStream(s->c2r_n, s->stream));
    if (s->have_c2r_d) CUFFT_TRY(cufftSetStream(s->c2r_d, s->stream));
    if (s->have_r2c_d) CUFFT_TRY(cufftSetStream(s->r2c_d, s->stream));
    return DJB_OK;
}

int djb_solver_device_bytes(const djb_solver* s, int64_t* bytes) {
    if (!s || !bytes) return fail(DJB_ERR_INVALID, "null argument");
    *bytes = s->bytes;
    return DJB_OK;
}

// Device staging of `count` floats: the caller's device array itself, or a stream-ordered
// copy of a host array (`copy` = 1) or zero-filled work area (`copy` = 0).
struct Stage {
    float* p = nullptr;
    bool owned = false;
};

// Device inputs are used in place; host inputs are copied (or work buffers zeroed) into
// the solver's work buffer `slot`.
int stage_in(djb_solver* s, Stage& st, const float* src, size_t count, int mem, bool copy, int slot) {
    if (mem == DJB_MEM_DEVICE && src) {
        st.p = const_cast<float*>(src);
        return DJB_OK;
    }
    TRY(scratch(s, slot, count, &st.p));
    if (copy && src) return copy_in(s, st.p, src, count, mem);
    CUDA_TRY(cudaMemsetAsync(st.p, 0, count * sizeof(float), s->stream));
    return DJB_OK;
}

void stage_free(djb_solver*, Stage& st) { st = Stage{}; }

int djb_pm_acceleration_vjp(djb_solver* s, const float* psi, const float* acc_bar, float* psi_bar, int32_t mem) {
    djb::clear_error();
    if (!s || !psi || !acc_bar || !psi_bar) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    const size_t count = size_t(3 * s->np);
    Stage sp, sa, sb;
    int rc = stage_in(s, sp, psi, count, mem, true, 0);
    if (rc == DJB_OK) rc = stage_in(s, sa, acc_bar, count, mem, true, 1);
    if (rc == DJB_OK) rc = stage_in(s, sb, mem == DJB_MEM_DEVICE ? nullptr : psi_bar, count, mem, false, 2);
    float* pb = (mem == DJB_MEM_DEVICE) ? psi_bar : sb.p;
    if (rc == DJB_OK && mem == DJB_MEM_DEVICE) {
        cudaError_t e = cudaMemsetAsync(pb, 0, count * sizeof(float), s->stream);
        if (e != cudaSuccess) rc = fail(DJB_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    }
    if (rc == DJB_OK) rc = force_vjp(s, sp.p, sa.p, pb);
    if (rc == DJB_OK && mem == DJB_MEM_HOST) rc = copy_out(s, psi_bar, pb, count, DJB_MEM_HOST);
    stage_free(s, sp);
    stage_free(s, sa);
    stage_free(s, sb);
    if (rc != DJB_OK) return rc;
    return check_err(s);
}

int djb_step_vjp(djb_solver* s, double dd1, double alpha, double beta, double dd2, const float* psi0,
                 const float* mom0, float* psi_bar, float* mom_bar, int32_t mem) {
    djb::clear_error();
    if (!s || !psi0 || !mom0 || !psi_bar || !mom_bar) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    const size_t count = size_t(3 * s->np);
    const int64_t m = int64_t(count);
    Stage sp, sm, sb, smb, s1, sa;
    int rc = stage_in(s, sp, psi0, count, mem, true, 0);
    if (rc == DJB_OK) rc = stage_in(s, sm, mom0, count, mem, true, 1);
    if (rc == DJB_OK) rc = stage_in(s, sb, psi_bar, count, mem, true, 2);
    if (rc == DJB_OK) rc = stage_in(s, smb, mom_bar, count, mem, true, 3);
    if (rc == DJB_OK) rc = stage_in(s, s1, nullptr, count, DJB_MEM_HOST, false, 4);
    if (rc == DJB_OK) rc = stage_in(s, sa, nullptr, count, DJB_MEM_HOST, false, 5);
    if (rc == DJB_OK) {
        djb::k_drifted<<<grid_for(m), kThreads, 0, s->stream>>>(sp.p, sm.p, float(dd1), s1.p, m);
        djb::k_step_vjp_pre<<<grid_for(m), kThreads, 0, s->stream>>>(sb.p, smb.p, float(dd2), float(beta), sa.p, m);
        rc = force_vjp(s, s1.p, sa.p, sb.p);
    }
    if (rc == DJB_OK) {
        djb::k_step_vjp_post<<<grid_for(m), kThreads, 0, s->stream>>>(sb.p, smb.p, float(alpha), float(dd1), m);
        if (cudaGetLastError() != cudaSuccess) rc = fail(DJB_ERR_CUDA, "step VJP kernel launch failed");
    }
    if (rc == DJB_OK && mem == DJB_MEM_HOST) {
        rc = copy_out(s, psi_bar, sb.p, count, DJB_MEM_HOST);
        if (rc == DJB_OK) rc = copy_out(s, mom_bar, smb.p, count, DJB_MEM_HOST);
    }
    stage_free(s, sp);
    stage_free(s, sm);
    stage_free(s, sb);
    stage_free(s, smb);
    stage_free(s, s1);
    stage_free(s, sa);
    if (rc != DJB_OK) return rc;
    return check_err(s);
}

int djb_mesh_fields(djb_solver* s, const float* psi, float* out, int32_t mem) {
    djb::clear_error();
    if (!s || !psi || !out) return fail(DJB_ERR_INVALID, "null argument");
    if (s->cfg.grad_order == 0 || s->cfg.n_resample > 1)
        return fail(DJB_ERR_INVALID, "mesh fields need a finite-difference gradient (2/4/6) without resampling");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    const size_t count = size_t(3 * s->np);
    const int res = s->res;
    const int64_t cells = int64_t(res) * res * res;
    const size_t rho_floats = s->phi[0] ? size_t(cells) : size_t(s->mesh_floats);
    for (int c = 0; c < 3; ++c)
        if (!s->adj[c]) TRY(dmalloc(s, (void**)&s->adj[c], rho_floats * sizeof(float)));
    Stage sp, so;
    int rc = stage_in(s, sp, psi, count, mem, true, 0);
    if (rc == DJB_OK && mem == DJB_MEM_HOST) rc = stage_in(s, so, nullptr, size_t(4 * cells), DJB_MEM_HOST, false, 1);
    float* o = (mem == DJB_MEM_HOST) ? so.p : out;
    if (rc == DJB_OK) {
        float* rho = rho_mesh(s, 0);
        const int pitch = rho_pitch(s);
        GroupShifts g{};
        CUDA_TRY(cudaMemsetAsync(rho, 0, rho_floats * sizeof(float), s->stream));
        if (s->W == 2) djb::k_scatter<2, 1><<<blocks(s->np), kThreads, 0, s->stream>>>(
            sp.p, nullptr, 0.0f, s->q1, s->n, s->np, s->Lf, res, pitch, g, rho, nullptr, s->err);
        if (s->W == 3) djb::k_scatter<3, 1><<<blocks(s->np), kThreads, 0, s->stream>>>(
            sp.p, nullptr, 0.0f, s->q1, s->n, s->np, s->Lf, res, pitch, g, rho, nullptr, s->err);
        if (s->W == 4) djb::k_scatter<4, 1><<<blocks(s->np), kThreads, 0, s->stream>>>(
            sp.p, nullptr, 0.0f, s->q1, s->n, s->np, s->Lf, res, pitch, g, rho, nullptr, s->err);
        const int cb = grid_for(cells);
        const float f = float(double(cells) / double(s->np));
        djb::k_mesh_affine<<<cb, 256, 0, s->stream>>>(rho, res, pitch, f, 1.0f, o);  // δ
        rc = poisson(s, 0);
        if (rc == DJB_OK) {
            djb::k_fd_grad3<<<fd_grid(s->res), djb::kFdThreads, 0, s->stream>>>(
                rho, res, pitch, s->c1, s->c2, s->c3, s->adj[0], s->adj[1], s->adj[2],
                fd_vec(s, res, pitch, {rho, s->adj[0], s->adj[1], s->adj[2]}));
            for (int c = 0; c < 3; ++c)
                djb::k_mesh_affine<<<cb, 256, 0, s->stream>>>(s->adj[c], res, pitch, 1.0f, 0.0f, o + (c + 1) * cells);
            if (cudaGetLastError() != cudaSuccess) rc = fail(DJB_ERR_CUDA, "mesh field kernels failed");
        }
    }
    if (rc == DJB_OK && mem == DJB_MEM_HOST) rc = copy_out(s, out, o, size_t(4 * cells), DJB_MEM_HOST);
    stage_free(s, sp);
    stage_free(s, so);
    if (rc != DJB_OK) return rc;
    return check_err(s);
}

int djb_solver_attach_nn(djb_solver* s, djb_nn* net, double delta_scale, double force_scale, double out_scale) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (!net) {
        s->nn = nullptr;
        return DJB_OK;
    }
    int32_t layers = 0, cin = 0, hidden = 0, cout = 0, dev = -1;
    TRY(djb_nn_info(net, &layers, &cin, &hidden, &cout, &dev));
    if (cin != 4 || cout != 3)
        return fail(DJB_ERR_INVALID, "the force correction needs a network with 4 inputs and 3 outputs (got %d, %d)",
                    cin, cout);
    if (dev != s->cfg.device) return fail(DJB_ERR_INVALID, "network and solver are on different devices");
    // the pipeline reads the unshifted density and potential of its first shift from the
    // dense meshes of the finite-difference path
    const bool zero_first = s->shifts.size() >= 3 && s->shifts[0] == 0.0 && s->shifts[1] == 0.0 &&
                            s->shifts[2] == 0.0;
    if (!s->phi[0] || s->cfg.grad_order == 0 || s->cfg.n_resample > 1 || !zero_first)
        return fail(DJB_ERR_INVALID,
                    "the force correction needs a finite-difference gradient (2/4/6), no resampling, a PMSolver "
                    "(not lean) with res divisible by 4, and antialias 0 or 1");
    if (!(std::isfinite(delta_scale) && std::isfinite(force_scale) && std::isfinite(out_scale)))
        return fail(DJB_ERR_INVALID, "scales must be finite");
    const int64_t cells = int64_t(s->res) * s->res * s->res;
    if (!s->nnf) TRY(dmalloc(s, (void**)&s->nnf, sizeof(float) * size_t(4 * cells)));
    if (!s->nnd) TRY(dmalloc(s, (void**)&s->nnd, sizeof(float) * size_t(3 * cells)));
    if (!s->nnacc) TRY(dmalloc(s, (void**)&s->nnacc, sizeof(float) * size_t(3 * s->np)));
    s->nn = net;
    s->nn_in = float(delta_scale);
    s->nn_fin = float(force_scale);
    s->nn_out = float(out_scale);
    s->nn_steps = 0;
    s->nn_valid = false;
    return DJB_OK;
}

int djb_solver_nn_schedule(djb_solver* s, int32_t every, int32_t start) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    if (every < 1 || start < 0) return fail(DJB_ERR_INVALID, "every must be at least 1 and start at least 0");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->nn_every = every;
    s->nn_start = start;
    s->nn_steps = 0;
    s->nn_valid = false;
    return DJB_OK;
}

int djb_mesh_interp3(djb_solver* s, const float* psi, const float* mesh3, float* out, int32_t mem) {
    djb::clear_error();
    if (!s || !psi || !mesh3 || !out) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    const size_t count = size_t(3 * s->np);
    const size_t mcount = size_t(3) * s->res * s->res * s->res;
    Stage sp, sm, so;
    int rc = stage_in(s, sp, psi, count, mem, true, 0);
    if (rc == DJB_OK) rc = stage_in(s, sm, mesh3, mcount, mem, true, 1);
    if (rc == DJB_OK && mem == DJB_MEM_HOST) rc = stage_in(s, so, nullptr, count, mem, false, 2);
    float* o = (mem == DJB_MEM_HOST) ? so.p : out;
    if (rc == DJB_OK) {
#define DJB_INTERP(W_)                                                                                         \
    if (s->W == W_)                                                                                            \
        djb::k_interp3<W_><<<blocks(s->np), kThreads, 0, s->stream>>>(sp.p, s->q1, s->n, s->np, s->Lf, s->res, \
                                                                      sm.p, 1.0f, o, s->err);
        DJB_INTERP(2)
        DJB_INTERP(3)
        DJB_INTERP(4)
#undef DJB_INTERP
        if (cudaGetLastError() != cudaSuccess) rc = fail(DJB_ERR_CUDA, "interpolation kernel launch failed");
    }
    if (rc == DJB_OK && mem == DJB_MEM_HOST) rc = copy_out(s, out, o, count, DJB_MEM_HOST);
    stage_free(s, sp);
    stage_free(s, sm);
    stage_free(s, so);
    if (rc != DJB_OK) return rc;
    return check_err(s);
}

int djb_mesh_deposit3(djb_solver* s, const float* psi, const float* vec, float* mesh3, int32_t mem) {
    djb::clear_error();
    if (!s || !psi || !vec || !mesh3) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    const size_t count = size_t(3 * s->np);
    const size_t mcount = size_t(3) * s->res * s->res * s->res;
    Stage sp, sv, so;
    int rc = stage_in(s, sp, psi, count, mem, true, 0);
    if (rc == DJB_OK) rc = stage_in(s, sv, vec, count, mem, true, 1);
    if (rc == DJB_OK && mem == DJB_MEM_HOST) rc = stage_in(s, so, nullptr, mcount, mem, false, 2);
    float* o = (mem == DJB_MEM_HOST) ? so.p : mesh3;
    if (rc == DJB_OK && mem == DJB_MEM_DEVICE) {
        cudaError_t e = cudaMemsetAsync(o, 0, mcount * sizeof(float), s->stream);
        if (e != cudaSuccess) rc = fail(DJB_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    }
    if (rc == DJB_OK) {
#define DJB_DEPOSIT(W_)                                                                                         \
    if (s->W == W_)                                                                                             \
        djb::k_deposit3<W_><<<blocks(s->np), kThreads, 0, s->stream>>>(sp.p, s->q1, s->n, s->np, s->Lf, s->res, \
                                                                       sv.p, o, s->err);
        DJB_DEPOSIT(2)
        DJB_DEPOSIT(3)
        DJB_DEPOSIT(4)
#undef DJB_DEPOSIT
        if (cudaGetLastError() != cudaSuccess) rc = fail(DJB_ERR_CUDA, "deposit kernel launch failed");
    }
    if (rc == DJB_OK && mem == DJB_MEM_HOST) rc = copy_out(s, mesh3, o, mcount, DJB_MEM_HOST);
    stage_free(s, sp);
    stage_free(s, sv);
    stage_free(s, so);
    if (rc != DJB_OK) return rc;
    return check_err(s);
}

int djb_pm_acceleration(djb_solver* s, const float* psi, float* acc, int32_t mem) {
    djb::clear_error();
    if (!s || !psi || !acc) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    // The displacements are staged in a stream-ordered buffer so that the resident
    // particle state of run_nbody survives a force call (pm.jl:507-521 uses S.X).
    float* saved = s->psi;
    float* stage = nullptr;
    const size_t count = size_t(3 * s->np);
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&stage), count * sizeof(float), s->stream);
    if (e != cudaSuccess) return fail(DJB_ERR_ALLOC, "staging allocation failed: %s", cudaGetErrorString(e));
    int rc = copy_in(s, stage, psi, count, mem);
    if (rc == DJB_OK) {
        s->psi = stage;
        rc = force(s, false, 0, 0, 0, 0);
        s->psi = saved;
    }
    if (rc == DJB_OK) rc = copy_out(s, acc, s->acc, count, mem);
    cudaFreeAsync(stage, s->stream);
    if (rc != DJB_OK) return rc;
    return check_err(s);
}

int djb_set_state(djb_solver* s, const float* psi, const float* mom, double mom_scale, int32_t mem) {
    djb::clear_error();
    if (!s || !psi || !mom) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    s->nn_steps = 0;      // a new state: the next step evaluates the network
    s->nn_valid = false;
    const size_t count = size_t(3 * s->np);
    TRY(copy_in(s, s->psi, psi, count, mem));
    if (mom_scale == 1.0) {
        TRY(copy_in(s, s->mom, mom, count, mem));
    } else {
        TRY(copy_in(s, s->acc, mom, count, mem));
        djb::k_set_mom<<<grid_for(count), kThreads, 0, s->stream>>>(s->mom, s->acc, mom_scale, int64_t(count));
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->have_state = true;
    return DJB_OK;
}

int djb_get_state(djb_solver* s, float* psi, float* mom, int32_t mem) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    if (!s->have_state) return fail(DJB_ERR_STATE, "no particle state set");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    const size_t count = size_t(3 * s->np);
    if (psi) TRY(copy_out(s, psi, s->psi, count, mem));
    if (mom) TRY(copy_out(s, mom, s->mom, count, mem));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return check_err(s);
}

int djb_step(djb_solver* s, double dd1, double alpha, double beta, double dd2) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    if (!s->have_state) return fail(DJB_ERR_STATE, "no particle state set");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    if (s->cfg.n_resample > 1) {
        // Resampling reads the drifted positions per shift; drift first, then the
        // unfused force and kick-drift.
        djb::k_drift<<<grid_for(3 * s->np), kThreads, 0, s->stream>>>(s->psi, s->mom, float(dd1), 3 * s->np);
        TRY(force(s, false, 0, 0, 0, 0));
        djb::k_kick_drift<<<grid_for(3 * s->np), kThreads, 0, s->stream>>>(
            s->psi, s->mom, s->acc, float(alpha), float(beta), float(dd2), 3 * s->np);
        CUDA_TRY(cudaGetLastError());
        return DJB_OK;
    }
    return force(s, true, dd1, alpha, beta, dd2);
}

int djb_run(djb_solver* s, int32_t n_steps, const double* dd1, const double* alpha, const double* beta,
            const double* dd2) {
    djb::clear_error();
    if (!s || !dd1 || !alpha || !beta || !dd2) return fail(DJB_ERR_INVALID, "null argument");
    for (int k = 0; k < n_steps; ++k) TRY(djb_step(s, dd1[k], alpha[k], beta[k], dd2[k]));
    return djb_synchronize(s);
}

int djb_get_output(djb_solver* s, float* x_out, float* p_out, int32_t wrap, double p_div, double p_mul,
                   int32_t mem) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    if (!s->have_state) return fail(DJB_ERR_STATE, "no particle state set");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    const size_t count = size_t(3 * s->np);
    float* xo = nullptr;
    float* po = nullptr;
    float* stage = nullptr;
    if (mem == DJB_MEM_HOST) {
        TRY(scratch(s, 3, 2 * count, &stage));  // kept between calls, like the adjoint's work areas
        xo = x_out ? stage : nullptr;
        po = p_out ? stage + count : nullptr;
    } else {
        xo = x_out;
        po = p_out;
    }
    djb::k_output<<<grid_for(count), kThreads, 0, s->stream>>>(s->psi, s->mom, s->q1, s->n, s->np, s->Lf, wrap,
                                                               p_div, p_mul, xo, po);
    int rc = DJB_OK;
    if (cudaGetLastError() != cudaSuccess) rc = fail(DJB_ERR_CUDA, "output kernel launch failed");
    if (rc == DJB_OK && mem == DJB_MEM_HOST) {
        if (x_out) rc = copy_out(s, x_out, xo, count, DJB_MEM_HOST);
        if (rc == DJB_OK && p_out) rc = copy_out(s, p_out, po, count, DJB_MEM_HOST);
    }
    if (rc != DJB_OK) return rc;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return check_err(s);
}

int djb_state_write_snapshot(djb_solver* s, const char* path, double D, double L, double p_div, double p_mul) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    if (!s->have_state) return fail(DJB_ERR_STATE, "no particle state set");
    if (!path || !*path) return fail(DJB_ERR_INVALID, "snapshot path is empty");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    const size_t count = size_t(3 * s->np);
    float* stage = nullptr;
    TRY(scratch(s, 3, 2 * count, &stage));
    djb::k_output<<<grid_for(count), kThreads, 0, s->stream>>>(s->psi, s->mom, s->q1, s->n, s->np, s->Lf, 0, p_div,
                                                               p_mul, stage, stage + count);
    if (cudaGetLastError() != cudaSuccess) return fail(DJB_ERR_CUDA, "output kernel launch failed");

    // two pinned pieces: the copy of piece k+1 runs while piece k goes to the file
    constexpr size_t kPiece = size_t(16) << 20;
    float* host[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int rc = DJB_OK;
    for (int i = 0; i < 2 && rc == DJB_OK; ++i) {
        if (cudaHostAlloc(reinterpret_cast<void**>(&host[i]), kPiece * sizeof(float), cudaHostAllocDefault) !=
                cudaSuccess ||
            cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(DJB_ERR_ALLOC, "pinned snapshot buffers could not be allocated");
        }
    }
    if (rc == DJB_OK) {
        const uint64_t nn = uint64_t(s->n);
        const std::vector<uint64_t> dims = {3, nn, nn, nn};
        rc = djb::h5_write_arrays(
            path, {{"Psi", dims, 4}, {"Pi", dims, 4}}, {{"D", D}, {"L", L}}, [&](size_t a, FILE* fp) -> int {
                const float* src = stage + a * count;
                const size_t pieces = (count + kPiece - 1) / kPiece;
                auto issue = [&](size_t k) -> int {
                    const size_t off = k * kPiece;
                    const size_t len = std::min(kPiece, count - off);
                    if (cudaMemcpyAsync(host[k & 1], src + off, len * sizeof(float), cudaMemcpyDeviceToHost,
                                        s->stream) != cudaSuccess ||
                        cudaEventRecord(ev[k & 1], s->stream) != cudaSuccess) {
                        cudaGetLastError();
                        return fail(DJB_ERR_CUDA, "snapshot copy failed");
                    }
                    return DJB_OK;
                };
                int r = issue(0);
                for (size_t k = 0; k < pieces && r == DJB_OK; ++k) {
                    if (k + 1 < pieces) r = issue(k + 1);
                    if (r != DJB_OK) break;
                    if (cudaEventSynchronize(ev[k & 1]) != cudaSuccess) {
                        cudaGetLastError();
                        r = fail(DJB_ERR_CUDA, "snapshot copy failed");
                        break;
                    }
                    r = djb::h5_write_floats(fp, host[k & 1], std::min(kPiece, count - k * kPiece));
                }
                return r;
            });
    }
    cudaError_t e = cudaStreamSynchronize(s->stream);   // no copy into the pinned pieces is left in flight
    for (int i = 0; i < 2; ++i) {
        if (host[i]) cudaFreeHost(host[i]);
        if (ev[i]) cudaEventDestroy(ev[i]);
    }
    if (rc != DJB_OK) return rc;
    if (e != cudaSuccess) return fail(DJB_ERR_CUDA, "%s", cudaGetErrorString(e));
    return check_err(s);
}

int djb_solver_profile(djb_solver* s, int32_t enable) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->prof.reset();
    s->prof.on = enable != 0;
    return DJB_OK;
}

int djb_solver_profile_read(djb_solver* s, double* ms, int64_t* launches, int64_t* calls, int32_t nphase) {
    djb::clear_error();
    if (!s || !ms || !launches || !calls) return fail(DJB_ERR_INVALID, "null argument");
    if (nphase < PH_COUNT) return fail(DJB_ERR_INVALID, "need room for %d phases", int(PH_COUNT));
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    for (int i = 0; i < nphase; ++i) {
        ms[i] = 0.0;
        launches[i] = i < PH_COUNT ? s->prof.launches[i] : 0;
        calls[i] = i < PH_COUNT ? s->prof.calls[i] : 0;
    }
    for (const auto& r : s->prof.recs) {
        float t = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&t, r.a, r.b));
        ms[r.phase] += double(t);
    }
    s->prof.reset();
    return DJB_OK;
}

int djb_synchronize(djb_solver* s) {
    djb::clear_error();
    if (!s) return fail(DJB_ERR_INVALID, "null solver");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    CUDA_TRY(cudaGetLastError());
    return check_err(s);
}

}  // extern "C"

// Exposed to power.cu: the solver's CIC deposit of its state for P(k).
namespace djb {
cufftHandle solver_r2c(const djb_solver* s) { return s->r2c; }
cufftHandle solver_c2r(const djb_solver* s) { return s->c2r; }
// psibar += Σ_n ∂W_CIC(X − n)/∂X · mesh(n) for the resident state (shift 0); device arrays.
int solver_cic_gather_grad(djb_solver* s, const float* mesh, int pitch, float* psibar) {
    djb::k_gather_grad<2><<<blocks(s->np), 256, 0, s->stream>>>(s->psi, s->q1, s->n, s->np, s->Lf, s->res, pitch,
                                                                 0.0f, 0.0f, 0.0f, mesh, nullptr, nullptr, nullptr,
                                                                 1.0f, psibar, s->err);
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}
int solver_check_err(djb_solver* s) { return check_err(s); }
double solver_boxsize(const djb_solver* s) { return s->L; }
int solver_deposit_cic(djb_solver* s, float** mesh_out, int* res, int* pitch, cudaStream_t* st) {
    if (!s->have_state) return fail(DJB_ERR_STATE, "no particle state set");
    CUDA_TRY(cudaSetDevice(s->cfg.device));
    CUDA_TRY(cudaMemsetAsync(s->mesh[0], 0, size_t(s->mesh_floats) * sizeof(float), s->stream));
    GroupShifts g{};
    s->cur_perm = nullptr;  // the P(k) deposit uses Lagrangian tiles
    launch_scatter_t<2, 1>(s, nullptr, 0.0f, g, s->mesh[0], nullptr, s->pitch, false);
    CUDA_TRY(cudaGetLastError());
    *mesh_out = s->mesh[0];
    *res = s->res;
    *pitch = s->pitch;
    *st = s->stream;
    return DJB_OK;
}
int64_t solver_np(const djb_solver* s) { return s->np; }
int solver_res(const djb_solver* s) { return s->res; }
}  // namespace djb
