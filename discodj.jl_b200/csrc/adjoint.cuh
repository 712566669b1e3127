// Adjoint (vector-Jacobian product) kernels of the PM force and of the P(k) loss.
//
// The reference has no adjoint; these are the transposes of the forward operators
// (mass assignment pm.jl:57-74, Kφ pm.jl:389-391, FD gradient pm.jl:330-342,
// interpolation pm.jl:344-364). Per shift, with G_c = −D_c φ and φ = K ∗ ρ:
//   Ψ̄_a += Σ_c ā_c Σ_n ∂_a W(X − n) G_c(n)          k_gather_grad (three fields)
//   Ḡ_c  = Σ_p ā_c W(X_p − n)                         k_scatter_weighted
//   φ̄    = Σ_c D_c Ḡ_c   (the FD stencil is antisymmetric: (−D)ᵀ = D)   k_fd_div3
//   ρ̄    = K ∗ φ̄        (Kφ is real and even: the Poisson operator is symmetric)
//   Ψ̄_a += Σ_n ∂_a W(X − n) ρ̄(n)                     k_gather_grad (one field)
// The weight derivatives differentiate pm.jl:49-51; the CIC adjoint gather has the
// shape of `_cic_gather_kernel!` (src/field/sheet_deposit.jl:75-94). Meshes are
// [iz][iy][ix] with row pitch `pitch`; these are one-thread-per-particle (or per cell)
// kernels with global float atomics where they accumulate.
#pragma once

#include <cstdint>

#include "pm_kernels.cuh"

namespace djb {

// d/dd of wk<W>(|d|) for the signed distance d = g − node.
template <int W>
__device__ __forceinline__ float dwk(float d) {
    const float a = fabsf(d);
    const float s = d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f);
    if (W == 2) return a > 1.0f ? 0.0f : -s;
    if (W == 3) {
        if (a > 1.5f) return 0.0f;
        if (a > 0.5f) return -(1.5f - a) * s;
        return -2.0f * d;
    }
    if (a > 2.0f) return 0.0f;
    if (a > 1.0f) return -0.5f * (2.0f - a) * (2.0f - a) * s;
    return -2.0f * d + 1.5f * d * a;
}

// Weights, weight derivatives with respect to the position (grid units per length:
// res/L) and wrapped node indices along one axis.
template <int W>
__device__ __forceinline__ void axis_wdw(float g, int res, float dgdx, float* w, float* dw, int* idx) {
    const int b = wbase<W>(g);
#pragma unroll
    for (int o = 0; o < W; ++o) {
        const int node = b + WLo<W>::v + o;
        const float d = g - float(node);
        w[o] = wk<W>(fabsf(d));
        dw[o] = dwk<W>(d) * dgdx;
        idx[o] = wrapi(node, res);
    }
}

// Position X = q + Ψ (+ shift) of particle p and its per-axis stencil.
template <int W>
__device__ __forceinline__ void particle_stencil(const float* __restrict__ psi, const float* __restrict__ q1, int n,
                                                 int64_t np, int64_t p, float L, int res, const float sh[3],
                                                 int* err, float (&w)[3][W], float (&dw)[3][W], int (&idx)[3][W]) {
    LatticeDiv ld;
    ld.init(n);
    int ijk[3];
    ld.ijk(p, ijk[0], ijk[1], ijk[2]);
    const float resf = float(res);
    const float dgdx = resf / L;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float X = psi[p + a * np] + q1[ijk[a]];
        const float g = grid_coord(X + sh[a], L, resf, err);
        axis_wdw<W>(g, res, dgdx, w[a], dw[a], idx[a]);
    }
}

// Thread t takes particle perm[t] (or t): brick order keeps the mesh traffic local.
// f1 == null: Ψ̄_a += scale · Σ_n ∂_a W · f0(n).
// else:       Ψ̄_a += scale · Σ_c ā_c Σ_n ∂_a W · f_c(n).
template <int W>
__global__ void __launch_bounds__(256) k_gather_grad(const float* __restrict__ psi, const float* __restrict__ q1,
                                                     int n, int64_t np, float L, int res, int pitch, float sx,
                                                     float sy, float sz, const float* __restrict__ f0,
                                                     const float* __restrict__ f1, const float* __restrict__ f2,
                                                     const float* __restrict__ abar, float scale,
                                                     float* __restrict__ psibar, int* err,
                                                     const int* __restrict__ perm = nullptr) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int64_t p = perm ? int64_t(perm[t]) : t;
    const float sh[3] = {sx, sy, sz};
    float w[3][W], dw[3][W];
    int idx[3][W];
    particle_stencil<W>(psi, q1, n, np, p, L, res, sh, err, w, dw, idx);
    const bool vec = f1 != nullptr;
    const float a0 = vec ? abar[p] : 0.0f, a1 = vec ? abar[p + np] : 0.0f, a2 = vec ? abar[p + 2 * np] : 0.0f;
    float v[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
        for (int b = 0; b < W; ++b) {
            const int64_t row = (int64_t(idx[2][c]) * res + idx[1][b]) * pitch;
#pragma unroll
            for (int a = 0; a < W; ++a) {
                const int64_t node = row + idx[0][a];
                const float f = vec ? (a0 * f0[node] + a1 * f1[node] + a2 * f2[node]) : f0[node];
                v[0] += dw[0][a] * w[1][b] * w[2][c] * f;
                v[1] += w[0][a] * dw[1][b] * w[2][c] * f;
                v[2] += w[0][a] * w[1][b] * dw[2][c] * f;
            }
        }
#pragma unroll
    for (int a = 0; a < 3; ++a) psibar[p + a * np] += scale * v[a];
}

// m_c(n) += scale · ā_c · W(X − n) for the three components.
template <int W>
__global__ void __launch_bounds__(256) k_scatter_weighted(const float* __restrict__ psi,
                                                          const float* __restrict__ q1, int n, int64_t np, float L,
                                                          int res, int pitch, float sx, float sy, float sz,
                                                          const float* __restrict__ abar, float scale,
                                                          float* __restrict__ m0, float* __restrict__ m1,
                                                          float* __restrict__ m2, int* err,
                                                          const int* __restrict__ perm = nullptr) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const int64_t p = perm ? int64_t(perm[t]) : t;
    const float sh[3] = {sx, sy, sz};
    float w[3][W], dw[3][W];
    int idx[3][W];
    particle_stencil<W>(psi, q1, n, np, p, L, res, sh, err, w, dw, idx);
    const float a0 = scale * abar[p], a1 = scale * abar[p + np], a2 = scale * abar[p + 2 * np];
#pragma unroll
    for (int c = 0; c < W; ++c)
#pragma unroll
        for (int b = 0; b < W; ++b) {
            const int64_t row = (int64_t(idx[2][c]) * res + idx[1][b]) * pitch;
#pragma unroll
            for (int a = 0; a < W; ++a) {
                const float wt = w[0][a] * w[1][b] * w[2][c];
                atomicAdd(m0 + row + idx[0][a], a0 * wt);
                atomicAdd(m1 + row + idx[0][a], a1 * wt);
                atomicAdd(m2 + row + idx[0][a], a2 * wt);
            }
        }
}

// g_c = −D_c φ, (D_c f)(n) = Σ_t c_t (f(n + t e_c) − f(n − t e_c)) (pm.jl:330-342).
__global__ void __launch_bounds__(256) k_fd_grad3(const float* __restrict__ phi, int res, int pitch, float c1,
                                                  float c2, float c3, float* __restrict__ g0,
                                                  float* __restrict__ g1, float* __restrict__ g2) {
    const int64_t total = int64_t(res) * res * res;
    const float cc[3] = {c1, c2, c3};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int x = int(t % res), y = int((t / res) % res), z = int(t / (int64_t(res) * res));
        float d[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int s = k + 1;
            if (cc[k] == 0.0f) continue;
            const float fxp = phi[(int64_t(z) * res + y) * pitch + wrapi(x + s, res)];
            const float fxm = phi[(int64_t(z) * res + y) * pitch + wrapi(x - s, res)];
            const float fyp = phi[(int64_t(z) * res + wrapi(y + s, res)) * pitch + x];
            const float fym = phi[(int64_t(z) * res + wrapi(y - s, res)) * pitch + x];
            const float fzp = phi[(int64_t(wrapi(z + s, res)) * res + y) * pitch + x];
            const float fzm = phi[(int64_t(wrapi(z - s, res)) * res + y) * pitch + x];
            d[0] += cc[k] * (fxp - fxm);
            d[1] += cc[k] * (fyp - fym);
            d[2] += cc[k] * (fzp - fzm);
        }
        const int64_t o = (int64_t(z) * res + y) * pitch + x;
        g0[o] = -d[0];
        g1[o] = -d[1];
        g2[o] = -d[2];
    }
}

// out = Σ_c D_c g_c.
__global__ void __launch_bounds__(256) k_fd_div3(const float* __restrict__ g0, const float* __restrict__ g1,
                                                 const float* __restrict__ g2, int res, int pitch, float c1,
                                                 float c2, float c3, float* __restrict__ out) {
    const int64_t total = int64_t(res) * res * res;
    const float cc[3] = {c1, c2, c3};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int x = int(t % res), y = int((t / res) % res), z = int(t / (int64_t(res) * res));
        float d = 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int s = k + 1;
            if (cc[k] == 0.0f) continue;
            d += cc[k] * (g0[(int64_t(z) * res + y) * pitch + wrapi(x + s, res)] -
                          g0[(int64_t(z) * res + y) * pitch + wrapi(x - s, res)]);
            d += cc[k] * (g1[(int64_t(z) * res + wrapi(y + s, res)) * pitch + x] -
                          g1[(int64_t(z) * res + wrapi(y - s, res)) * pitch + x]);
            d += cc[k] * (g2[(int64_t(wrapi(z + s, res)) * res + y) * pitch + x] -
                          g2[(int64_t(wrapi(z - s, res)) * res + y) * pitch + x]);
        }
        out[(int64_t(z) * res + y) * pitch + x] = d;
    }
}

// Step adjoint helpers over 3·np components.
// psi1 = psi0 + dd1·mom0 (the drifted positions at which the step's force is taken).
__global__ void k_drifted(const float* __restrict__ psi0, const float* __restrict__ mom0, float dd1,
                          float* __restrict__ psi1, int64_t m) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m; t += int64_t(gridDim.x) * blockDim.x)
        psi1[t] = psi0[t] + dd1 * mom0[t];
}
// M̄ += dd2·Ψ̄; ā = β·M̄.
__global__ void k_step_vjp_pre(const float* __restrict__ psibar, float* __restrict__ mombar, float dd2, float beta,
                               float* __restrict__ abar, int64_t m) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m; t += int64_t(gridDim.x) * blockDim.x) {
        const float mb = mombar[t] + dd2 * psibar[t];
        mombar[t] = mb;
        abar[t] = beta * mb;
    }
}
// M̄ = α·M̄ + dd1·Ψ̄.
__global__ void k_step_vjp_post(const float* __restrict__ psibar, float* __restrict__ mombar, float alpha,
                                float dd1, int64_t m) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m; t += int64_t(gridDim.x) * blockDim.x)
        mombar[t] = alpha * mombar[t] + dd1 * psibar[t];
}

// out = scale·in − offset on the res³ cells of a pitched mesh, written densely.
__global__ void k_mesh_affine(const float* __restrict__ in, int res, int pitch, float scale, float offset,
                              float* __restrict__ out) {
    const int64_t total = int64_t(res) * res * res;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t row = t / res;
        const int x = int(t - row * res);
        out[t] = scale * in[row * pitch + x] - offset;
    }
}

}  // namespace djb
