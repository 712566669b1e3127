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

#include "brick.cuh"
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

// Both stencil kernels sweep a column of kFdTX × kFdTY cells along z over kFdZ planes,
// 256 threads with two rows each. The planes come into shared memory by asynchronous
// copies (16 bytes where the row pitch and the mesh width allow it, else 4 bytes),
// four planes ahead of the plane being computed, so the loads of later planes overlap
// the arithmetic of this one; the z stencil reads a ring of staged planes.
constexpr int kFdTX = 32, kFdTY = 16, kFdZ = 64, kFdR = 3;
constexpr int kFdThreads = 256;
constexpr int kFdRing = 8;   // planes z − 3 .. z + 3 and the one in flight

// Periodic index of any integer (tiles and windows reach past 2·res on small meshes);
// indices inside the mesh, the common case, take one unsigned comparison.
__device__ __forceinline__ int fd_wrap(int v, int res) {
    if (unsigned(v) < unsigned(res)) return v;
    v %= res;
    return v < 0 ? v + res : v;
}

// Copies rows ys .. ys + rows − 1, columns xs .. xs + NCOL − 1 of plane z (periodic) into
// t[rows][NCOL]. vec: xs, res and pitch are multiples of 4 and f is 16-byte aligned.
template <int NCOL>
__device__ __forceinline__ void fd_issue(float* t, const float* __restrict__ f, int xs, int ys, int rows, int z,
                                         int res, int pitch, bool vec) {
    const int64_t pz = int64_t(fd_wrap(z, res)) * res;
    if (vec) {
        constexpr int N4 = NCOL / 4;
        for (int i = threadIdx.x; i < rows * N4; i += kFdThreads) {
            const int r = i / N4, c = i - r * N4;
            const float* src = f + (pz + fd_wrap(ys + r, res)) * pitch + fd_wrap(xs + 4 * c, res);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(t + r * NCOL + 4 * c)), "l"(src)
                         : "memory");
        }
    } else {
        for (int i = threadIdx.x; i < rows * NCOL; i += kFdThreads) {
            const int r = i / NCOL, c = i - r * NCOL;
            const float* src = f + (pz + fd_wrap(ys + r, res)) * pitch + fd_wrap(xs + c, res);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(t + r * NCOL + c)), "l"(src)
                         : "memory");
        }
    }
}
__device__ __forceinline__ void fd_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most one copy group of this thread is still in flight.
__device__ __forceinline__ void fd_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ int fd_slot(int z, int z0) { return (z - z0 + kFdR) & (kFdRing - 1); }

// g_c = −D_c φ, (D_c f)(n) = Σ_t c_t (f(n + t e_c) − f(n − t e_c)) (pm.jl:330-342).
// Staged planes: rows y0 − 3 .. y0 + 18, columns x0 − 4 .. x0 + 35.
__global__ void __launch_bounds__(kFdThreads) k_fd_grad3(const float* __restrict__ phi, int res, int pitch, float c1,
                                                          float c2, float c3, float* __restrict__ g0,
                                                          float* __restrict__ g1, float* __restrict__ g2, int vec) {
    constexpr int NC = kFdTX + 8, NR = kFdTY + 2 * kFdR;
    __shared__ __align__(16) float ring[kFdRing][NR * NC];
    const float cc[kFdR] = {c1, c2, c3};
    const int tx = threadIdx.x % kFdTX, ty = threadIdx.x / kFdTX;
    const int x0 = blockIdx.x * kFdTX, y0 = blockIdx.y * kFdTY, z0 = blockIdx.z * kFdZ;
    const int z1 = min(z0 + kFdZ, res);
    const int x = x0 + tx;
    for (int z = z0 - kFdR; z <= z0 + kFdR; ++z) {   // one copy group per plane
        fd_issue<NC>(ring[fd_slot(z, z0)], phi, x0 - 4, y0 - kFdR, NR, z, res, pitch, vec != 0);
        fd_commit();
    }
    for (int z = z0; z < z1; ++z) {
        if (z + 1 < z1) fd_issue<NC>(ring[fd_slot(z + kFdR + 1, z0)], phi, x0 - 4, y0 - kFdR, NR, z + kFdR + 1, res,
                                     pitch, vec != 0);
        fd_commit();
        fd_wait1();   // planes up to z + 3 have landed
        __syncthreads();
        const float* pc = ring[fd_slot(z, z0)];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int yy = ty + 8 * h, y = y0 + yy;
            if (x < res && y < res) {
                const int off = (yy + kFdR) * NC + tx + 4;
                const float* c0 = pc + off;
                float d0 = 0.0f, d1 = 0.0f, d2 = 0.0f;
#pragma unroll
                for (int k = 0; k < kFdR; ++k) {
                    const int t = k + 1;
                    d0 += cc[k] * (c0[t] - c0[-t]);
                    d1 += cc[k] * (c0[t * NC] - c0[-t * NC]);
                    d2 += cc[k] * (ring[fd_slot(z + t, z0)][off] - ring[fd_slot(z - t, z0)][off]);
                }
                const int64_t o = (int64_t(z) * res + y) * pitch + x;
                g0[o] = -d0;
                g1[o] = -d1;
                g2[o] = -d2;
            }
        }
        __syncthreads();   // the slot of plane z − 3 is refilled next
    }
}

// out = Σ_c D_c g_c. Staged: g0 rows y0 .. y0 + 15 with columns x0 − 4 .. x0 + 35 and g1
// rows y0 − 3 .. y0 + 18 with columns x0 .. x0 + 31 (plane z and z + 1), g2 rows
// y0 .. y0 + 15, columns x0 .. x0 + 31 in the ring of planes.
__global__ void __launch_bounds__(kFdThreads) k_fd_div3(const float* __restrict__ g0, const float* __restrict__ g1,
                                                         const float* __restrict__ g2, int res, int pitch, float c1,
                                                         float c2, float c3, float* __restrict__ out, int vec) {
    constexpr int NX = kFdTX + 8, NY = kFdTY + 2 * kFdR;
    __shared__ __align__(16) float ring[kFdRing][kFdTY * kFdTX];
    __shared__ __align__(16) float tx_tile[2][kFdTY * NX];
    __shared__ __align__(16) float ty_tile[2][NY * kFdTX];
    const float cc[kFdR] = {c1, c2, c3};
    const int tx = threadIdx.x % kFdTX, ty = threadIdx.x / kFdTX;
    const int x0 = blockIdx.x * kFdTX, y0 = blockIdx.y * kFdTY, z0 = blockIdx.z * kFdZ;
    const int z1 = min(z0 + kFdZ, res);
    const int x = x0 + tx;
    const bool v4 = vec != 0;
    for (int z = z0 - kFdR; z <= z0 + kFdR; ++z) {
        fd_issue<kFdTX>(ring[fd_slot(z, z0)], g2, x0, y0, kFdTY, z, res, pitch, v4);
        if (z == z0) {
            fd_issue<NX>(tx_tile[0], g0, x0 - 4, y0, kFdTY, z0, res, pitch, v4);
            fd_issue<kFdTX>(ty_tile[0], g1, x0, y0 - kFdR, NY, z0, res, pitch, v4);
        }
        fd_commit();
    }
    for (int z = z0; z < z1; ++z) {
        const int b = (z - z0) & 1;
        if (z + 1 < z1) {
            fd_issue<kFdTX>(ring[fd_slot(z + kFdR + 1, z0)], g2, x0, y0, kFdTY, z + kFdR + 1, res, pitch, v4);
            fd_issue<NX>(tx_tile[b ^ 1], g0, x0 - 4, y0, kFdTY, z + 1, res, pitch, v4);
            fd_issue<kFdTX>(ty_tile[b ^ 1], g1, x0, y0 - kFdR, NY, z + 1, res, pitch, v4);
        }
        fd_commit();
        fd_wait1();   // g2 up to plane z + 3, g0 and g1 of plane z have landed
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int yy = ty + 8 * h, y = y0 + yy;
            if (x < res && y < res) {
                const float* a0 = tx_tile[b] + yy * NX + tx + 4;
                const float* a1 = ty_tile[b] + (yy + kFdR) * kFdTX + tx;
                const int zc = yy * kFdTX + tx;
                float d = 0.0f;
#pragma unroll
                for (int k = 0; k < kFdR; ++k) {
                    const int t = k + 1;
                    d += cc[k] * (a0[t] - a0[-t]);
                    d += cc[k] * (a1[t * kFdTX] - a1[-t * kFdTX]);
                    d += cc[k] * (ring[fd_slot(z + t, z0)][zc] - ring[fd_slot(z - t, z0)][zc]);
                }
                out[(int64_t(z) * res + y) * pitch + x] = d;
            }
        }
        __syncthreads();
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

// ── brick-owned forms (particles sorted by brick, see brick.cuh) ─────────────────
// One CTA owns one brick and its particles; its W-node stencils fall inside the
// brick's deposit box (BrickList::ssx, sSs, sos), which lives in shared memory.

// Position of particle p and, per axis, the weights, their derivatives (grid units per
// length dgdx) and the stencil's first node relative to the box (clamped into the box
// with error bit 2 when the binning and this evaluation disagree).
// p: the particle (its lattice site); io: where its Ψ lives in `psi` (p, or its slot in
// brick order when the arrays were gathered into that order).
// DW = false: the weights only (dw is left unset).
template <int W, bool DW = true>
__device__ __forceinline__ void brick_stencil(const float* __restrict__ psi, const float* __restrict__ q1,
                                              const LatticeDiv& ld, int64_t np, int64_t p, int64_t io, float L,
                                              float resf, int res, const float sh[3], const TileBox& box, int* err,
                                              float (&w)[3][W], float (&dw)[3][W], int (&d)[3]) {
    int ijk[3];
    ld.ijk(p, ijk[0], ijk[1], ijk[2]);
    const float dgdx = resf / L;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float X = psi[io + a * np] + q1[ijk[a]];
        const float g = grid_coord(X + sh[a], L, resf, err);
        const int bb = wbase<W>(g);
#pragma unroll
        for (int o = 0; o < W; ++o) {
            const float dd = g - float(bb + WLo<W>::v + o);
            w[a][o] = wk<W>(fabsf(dd));
            if constexpr (DW) dw[a][o] = dwk<W>(dd) * dgdx;
        }
        d[a] = box_rel(bb + WLo<W>::v, box.o[a], res);
        if (d[a] < 0 || d[a] > box.S[a] - W) {
            if (err) atomicOr(err, 2);
            d[a] = d[a] < 0 ? 0 : box.S[a] - W;
        }
    }
}

// m_c(n) += scale · ā_c(p) · W(X_p − n) for c = 0, 1, 2: one component per pass over the
// brick's particles into a shared-memory box, then added to the mesh with vector
// reductions. Bricks of at most kFixedMax particles accumulate in 32-bit fixed point
// (integer shared atomics, signed values in two's complement): the node sums are
// bounded by cnt · max|scale · ā| (a particle's weights sum to 1), kept below 2^30, so
// the unit is at most 4096 · max|scale · ā| · 2^−30. Denser bricks use float shared
// atomics.
constexpr unsigned kFixedMax = 4096;

// `tma` != 0: m0..m2 are dense [res]^3 meshes described by tm0..tm2 (boxes of the deposit
// box's shape); boxes that do not wrap are then converted to float in place and added to
// the mesh with one bulk tensor reduction each.
template <int W>
__global__ void __launch_bounds__(kTileThreads, DJB_BRICK_SCATTER_BLOCKS) k_scatter_weighted_brick(
    const float* __restrict__ psi, const float* __restrict__ q1, int n, int64_t np, float L, int res, int pitch,
    float sx, float sy, float sz, const float* __restrict__ abar, float scale, float* __restrict__ m0,
    float* __restrict__ m1, float* __restrict__ m2, int* err, BrickList bl, int sorted_io,
    const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
    const __grid_constant__ CUtensorMap tm2, int tma) {
    extern __shared__ __align__(128) float wbox[];
    unsigned* qbox = reinterpret_cast<unsigned*>(wbox);
    __shared__ float s_max[kTileThreads / 32];
    const int b = brick_of_block(bl, blockIdx.x);
    unsigned start, cnt;
    brick_range(bl, b, start, cnt);
    if (cnt == 0) return;
    const int tid = threadIdx.x;
    const TileBox box = aligned_box(bl, b, bl.sos, bl.sSs, bl.ssx);
    const bool vec = ((pitch | res) & 3) == 0;
    const bool bulk = tma && box_inside(box, res) && (smem_u32(wbox) & 127u) == 0u;
    const float resf = float(res);
    const int cells = box.plane * box.S[2];   // a multiple of 4
    const float sh[3] = {sx, sy, sz};
    const bool fixed = cnt <= kFixedMax;
    LatticeDiv ld;
    ld.init(n);
#pragma unroll 1
    for (int comp = 0; comp < 3; ++comp) {
        float up = 1.0f, down = 1.0f;
        for (int t = 4 * tid; t < cells; t += 4 * kTileThreads)
            *reinterpret_cast<uint4*>(qbox + t) = make_uint4(0u, 0u, 0u, 0u);
        if (fixed) {   // the largest |scale · ā_c| of the brick sets the unit
            float m = 0.0f;
            for (unsigned slot = tid; slot < cnt; slot += kTileThreads)
                m = fmaxf(m, fabsf(scale * abar[(sorted_io ? int64_t(start + slot) : int64_t(bl.perm[start + slot])) +
                                                comp * np]));
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if ((tid & 31) == 0) s_max[tid >> 5] = m;
        }
        __syncthreads();
        if (fixed) {
            float amax = 0.0f;
            for (int i = 0; i < kTileThreads / 32; ++i) amax = fmaxf(amax, s_max[i]);
            if (!(amax > 0.0f) || !isfinite(amax)) {   // nothing to deposit (or not finite: skip)
                __syncthreads();
                continue;
            }
            int ex;
            frexpf(amax * float(cnt), &ex);            // amax · cnt < 2^ex
            const int e = min(30 - ex, 120);
            up = ldexpf(1.0f, e);
            down = ldexpf(1.0f, -e);
        }
        for (unsigned r0 = 0; r0 < cnt; r0 += kTileThreads) {
            // lanes 8 slots apart: particles of one cell land in different warps
            const unsigned slot = r0 + unsigned((tid & 31) * (kTileThreads / 32) + (tid >> 5));
            if (slot >= cnt) continue;
            const int64_t p = bl.perm[start + slot];
            const int64_t io = sorted_io ? int64_t(start + slot) : p;
            const float av = scale * abar[io + comp * np] * up;
            float w[3][W], dw[3][W];
            int d[3];
            brick_stencil<W, false>(psi, q1, ld, np, p, io, L, resf, res, sh, box, comp == 0 ? err : nullptr, w, dw,
                                    d);
#pragma unroll
            for (int c = 0; c < W; ++c)
#pragma unroll
                for (int bb = 0; bb < W; ++bb) {
                    const int o = ((d[2] + c) * box.S[1] + d[1] + bb) * box.P + d[0];
                    const float wyz = av * w[1][bb] * w[2][c];
#pragma unroll
                    for (int a = 0; a < W; ++a) {
                        if (fixed) atomicAdd(qbox + o + a, unsigned(__float2int_rn(w[0][a] * wyz)));
                        else atomicAdd(wbox + o + a, w[0][a] * wyz);
                    }
                }
        }
        __syncthreads();
        if (bulk) {
            // signed fixed point -> float in place (float sums stay), then one bulk reduction
            if (fixed)
                for (int t = 4 * tid; t < cells; t += 4 * kTileThreads) {
                    const uint4 u = *reinterpret_cast<const uint4*>(qbox + t);
                    *reinterpret_cast<float4*>(wbox + t) =
                        make_float4(float(int(u.x)) * down, float(int(u.y)) * down, float(int(u.z)) * down,
                                    float(int(u.w)) * down);
                }
            fence_proxy_async_smem();   // the conversions are read by the bulk copy below
            __syncthreads();
            if (tid == 0) {
                tma_reduce_add_3d(comp == 0 ? &tm0 : (comp == 1 ? &tm1 : &tm2), box.o[0], box.o[1], box.o[2], wbox);
                bulk_commit_and_wait_read();   // the box is zeroed for the next component after this
            }
            __syncthreads();
            continue;
        }
        float* mesh = comp == 0 ? m0 : (comp == 1 ? m1 : m2);
        for_box_wrapped(box, res, pitch, vec, [&](int so, int64_t go) {
            if (vec) {
                const uint4 u = *reinterpret_cast<const uint4*>(qbox + so);
                if ((u.x | u.y | u.z | u.w) == 0u) return;
                if (fixed)
                    red_add_v4(mesh + go, float(int(u.x)) * down, float(int(u.y)) * down, float(int(u.z)) * down,
                               float(int(u.w)) * down);
                else
                    red_add_v4(mesh + go, __uint_as_float(u.x), __uint_as_float(u.y), __uint_as_float(u.z),
                               __uint_as_float(u.w));
            } else {
                const unsigned u = qbox[so];
                if (u != 0u) atomicAdd(mesh + go, fixed ? float(int(u)) * down : __uint_as_float(u));
            }
        });
        __syncthreads();
    }
}

// f1 == null: Ψ̄_a += scale · Σ_n ∂_a W · f0(n); else Ψ̄_a += scale · Σ_c ā_c Σ_n ∂_a W · f_c(n).
// One field at a time is staged over the brick's deposit box (16-byte copies); every
// particle of the brick adds its share to Ψ̄ per field (a particle belongs to one
// brick, so no other CTA writes it). sorted_io: psi, abar and psibar are in brick order
// (slot start + i), read and written coalesced.
// `tma` != 0: f0 (.. f2) are dense [res]^3 meshes described by tm0 (.. tm2), boxes of the
// deposit box's shape; boxes that do not wrap are then staged with one bulk tensor copy.
template <int W>
__global__ void __launch_bounds__(kTileThreads, DJB_BRICK_SCATTER_BLOCKS) k_gather_grad_brick(
    const float* __restrict__ psi, const float* __restrict__ q1, int n, int64_t np, float L, int res, int pitch,
    float sx, float sy, float sz, const float* __restrict__ f0, const float* __restrict__ f1,
    const float* __restrict__ f2, const float* __restrict__ abar, float scale, float* __restrict__ psibar, int* err,
    BrickList bl, int sorted_io, const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
    const __grid_constant__ CUtensorMap tm2, int tma) {
    extern __shared__ __align__(128) float fbox[];
    __shared__ __align__(8) uint64_t s_bar;
    const int b = brick_of_block(bl, blockIdx.x);
    unsigned start, cnt;
    brick_range(bl, b, start, cnt);
    if (cnt == 0) return;
    const int tid = threadIdx.x;
    const bool vec = ((pitch | res) & 3) == 0;
    const float resf = float(res);
    const float sh[3] = {sx, sy, sz};
    const int nf = f1 ? 3 : 1;
    LatticeDiv ld;
    ld.init(n);
    const TileBox box = aligned_box(bl, b, bl.sos, bl.sSs, bl.ssx);
    const bool bulk = tma && box_inside(box, res) && (smem_u32(fbox) & 127u) == 0u;
    const unsigned box_bytes = unsigned(box.plane) * unsigned(box.S[2]) * 4u;
    if (bulk && tid == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    unsigned parity = 0;
#pragma unroll 1
    for (int f = 0; f < nf; ++f) {
        if (bulk) {
            if (tid == 0) {
                fence_proxy_async_smem();   // the previous field's reads precede the refill
                mbar_arrive_expect_tx(&s_bar, box_bytes);
                tma_load_3d(fbox, f == 0 ? &tm0 : (f == 1 ? &tm1 : &tm2), box.o[0], box.o[1], box.o[2], &s_bar);
            }
            const bool ok = mbar_wait(&s_bar, parity);
            parity ^= 1u;
            if (__syncthreads_or(!ok)) {   // the copy never completed: report, do not spin
                if (tid == 0) atomicOr(err, 8);
                return;
            }
        } else {
            stage_box_wrapped(fbox, f == 0 ? f0 : (f == 1 ? f1 : f2), box, res, pitch, vec);
            __syncthreads();
        }
        for (unsigned slot = tid; slot < cnt; slot += kTileThreads) {
            const int64_t p = bl.perm[start + slot];
            const int64_t io = sorted_io ? int64_t(start + slot) : p;
            float w[3][W], dw[3][W];
            int d[3];
            brick_stencil<W>(psi, q1, ld, np, p, io, L, resf, res, sh, box, f == 0 ? err : nullptr, w, dw, d);
            const float af = scale * (f1 ? abar[io + f * np] : 1.0f);
            // separable sums: rows along x (∂_x W and W), then y, then z
            float v[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int c = 0; c < W; ++c) {
                float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
                for (int bb = 0; bb < W; ++bb) {
                    const float* row = fbox + ((d[2] + c) * box.S[1] + d[1] + bb) * box.P + d[0];
                    float r0 = 0.0f, r1 = 0.0f;
#pragma unroll
                    for (int a = 0; a < W; ++a) {
                        const float fv = row[a];
                        r0 += dw[0][a] * fv;
                        r1 += w[0][a] * fv;
                    }
                    s0 += w[1][bb] * r0;
                    s1 += dw[1][bb] * r1;
                    s2 += w[1][bb] * r1;
                }
                v[0] += w[2][c] * s0;
                v[1] += w[2][c] * s1;
                v[2] += dw[2][c] * s2;
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) psibar[io + a * np] += af * v[a];
        }
        __syncthreads();
    }
}

// dst[c·np + t] = src[c·np + perm[t]]: three components into brick order.
__global__ void k_gather_sorted3(const float* __restrict__ src, const int* __restrict__ perm, int64_t np,
                                 float* __restrict__ dst) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < np; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t p = perm[t];
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c * np + t] = src[c * np + p];
    }
}

// dst[c·np + perm[t]] += src[c·np + t]: back from brick order (perm is a permutation).
__global__ void k_scatter_add_sorted3(const float* __restrict__ src, const int* __restrict__ perm, int64_t np,
                                      float* __restrict__ dst) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < np; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t p = perm[t];
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c * np + p] += src[c * np + t];
    }
}

}  // namespace djb
