// Shared-memory tiled mass assignment and force interpolation.
//
// A CTA owns a tile of 256 particles: either 256 consecutive entries of the brick
// sort (`perm`, sort.cuh) or, without a sort, a Lagrangian tile of kTX x kTY x kTZ
// particles (consecutive i, j, k of the particle lattice). Its particles' W-node stencils cover an Eulerian
// box that the CTA sizes from a min/max reduction of their base nodes (relative to
// the tile's first particle, periodic differences unwrapped). The box is processed
// in z-chunks that fit the shared-memory budget:
//   mass assignment  : 32-bit fixed-point accumulation with native shared-memory
//                      integer atomics (scale 2^23 / 2^24 / 2^25 for CIC / TSC / PCS:
//                      a tile of 256 particles on one node, each at the kernel's
//                      largest node weight 1, 0.75^3, (2/3)^3, stays below 2^32), then
//                      one coalesced flush of the chunk's non-zero cells to the float
//                      mesh with global reductions. Within a tile the sum is
//                      order-independent;
//   interpolation    : the chunk of the potential (with the finite-difference halo R
//                      on every side) is staged with asynchronous global->shared
//                      copies, then every particle applies its FD-convolved separable
//                      weights to the staged values.
// Box cells are enumerated without per-element division (reciprocal multiply) and
// with the periodic wrap precomputed per row and per column in shared tables.
// A tile whose box rows or columns exceed those tables, or whose single z-plane
// exceeds the budget, falls back to per-particle global access for that shift.
#pragma once

#include "pm_kernels.cuh"

namespace djb {

constexpr int kTX = 8, kTY = 8, kTZ = 4;
constexpr int kTileThreads = kTX * kTY * kTZ;  // 256
constexpr int kTileWarps = kTileThreads / 32;
constexpr int kMaxRows = 2048;  // box rows (y, z) per chunk
constexpr int kMaxCols = 512;   // box extent along x

// Periodic index for box coordinates: valid on [-2 res, 3 res). A box origin lies at
// >= -res/2 - 4 and a box spans < 1.5 res + 6 nodes, which stays inside for res >= 8.
__device__ __forceinline__ int wrap2(int i, int res) { return wrapi(wrapi(i, res), res); }

__device__ __forceinline__ int unwrap_rel(int d, int res) {
    if (d >= res / 2) d -= res;
    else if (d < -res / 2) d += res;
    return d;
}

// t / d for 0 <= t < 2^20 and 2 <= d < 2^11 by a multiply-high with m = ceil(2^32 / d)
// (exact when t * d < 2^32).
struct FastDiv {
    unsigned m;
    int d;
    __device__ __forceinline__ void init(int dd) {
        d = dd;
        m = 0xffffffffu / unsigned(dd) + 1u;
    }
    __device__ __forceinline__ int div(int t) const { return int(__umulhi(unsigned(t), m)); }
};

struct TileBox {
    int o[3];   // global node of box coordinate 0 (may lie outside [0,res): wrapped on access)
    int S[3];   // box extent per axis
    int P;      // row pitch in shared memory (odd, >= S[0])
    int plane;  // P * S[1]
};

// CTA-wide box of the nodes [b + lo, b + lo + ext) over active particles; `d` returns
// each thread's base relative to the box origin.
__device__ __forceinline__ void tile_box(const int b[3], bool active, int lo, int ext, int res,
                                         TileBox& box, int d[3]) {
    __shared__ int s_ref[3];
    __shared__ int s_mn[kTileWarps][3];
    __shared__ int s_mx[kTileWarps][3];
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_ref[0] = b[0];
        s_ref[1] = b[1];
        s_ref[2] = b[2];
    }
    __syncthreads();
    int rel[3], mn[3], mx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        rel[a] = active ? unwrap_rel(b[a] - s_ref[a], res) : 0;  // thread 0 is active with rel 0
        mn[a] = __reduce_min_sync(0xffffffffu, rel[a]);
        mx[a] = __reduce_max_sync(0xffffffffu, rel[a]);
    }
    if ((tid & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            s_mn[tid >> 5][a] = mn[a];
            s_mx[tid >> 5][a] = mx[a];
        }
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int lo_a = s_mn[0][a], hi_a = s_mx[0][a];
#pragma unroll
        for (int w = 1; w < kTileWarps; ++w) {
            lo_a = min(lo_a, s_mn[w][a]);
            hi_a = max(hi_a, s_mx[w][a]);
        }
        box.o[a] = s_ref[a] + lo_a + lo;
        box.S[a] = hi_a - lo_a + ext;
        d[a] = rel[a] - lo_a;
    }
    box.P = box.S[0] | 1;
    box.plane = box.P * box.S[1];
    __syncthreads();  // s_ref / s_mn reused by the next call
}

// Wrapped column table (once per box) and row table (per chunk): s_col[x] = global x,
// s_row[r] = global z * res + global y for the chunk rows r = z * S1 + y.
__device__ __forceinline__ void box_columns(const TileBox& box, int res, int* s_col) {
    for (int x = threadIdx.x; x < box.S[0]; x += kTileThreads) s_col[x] = wrap2(box.o[0] + x, res);
}

__device__ __forceinline__ void chunk_rows(const TileBox& box, int res, int z0, int nz, int* s_row) {
    FastDiv fs;
    fs.init(box.S[1] > 1 ? box.S[1] : 2);
    const int rows = box.S[1] * nz;
    for (int r = threadIdx.x; r < rows; r += kTileThreads) {
        const int z = (box.S[1] > 1) ? fs.div(r) : r;
        const int y = r - z * box.S[1];
        s_row[r] = wrap2(box.o[2] + z0 + z, res) * res + wrap2(box.o[1] + y, res);
    }
}

// ── mass assignment ───────────────────────────────────────────────────────────
template <int W>
struct FixScale {
    static constexpr float up = (W == 2) ? 8388608.0f : (W == 3) ? 16777216.0f : 33554432.0f;  // 2^23..2^25
    static constexpr float down = 1.0f / up;
};

// Largest 3-D weight a particle gives one node: 1 (CIC, d = 0), 0.75^3 (TSC), (2/3)^3 (PCS).
template <int W>
struct MaxW3 {
    static constexpr float v = (W == 2) ? 1.0f : (W == 3) ? 0.421875f : 0.2962963f;
};

// A tile deposits at most kTileThreads particles, so no node sum of the tiled kernel can
// pass 2^32 at FixScale (each rounded weight is below its value + 1).
static_assert(double(kTileThreads) * (MaxW3<2>::v * FixScale<2>::up + 1.0) < 4294967296.0, "CIC tile sum");
static_assert(double(kTileThreads) * (MaxW3<3>::v * FixScale<3>::up + 1.0) < 4294967296.0, "TSC tile sum");
static_assert(double(kTileThreads) * (MaxW3<4>::v * FixScale<4>::up + 1.0) < 4294967296.0, "PCS tile sum");

#ifndef DJB_SCATTER_MIN_BLOCKS
#define DJB_SCATTER_MIN_BLOCKS 2
#endif

// The particle a thread of the tile handles: the tile's sorted slot, or its lattice cell.
struct TileParticle {
    int i, j, k;
    int64_t p;
    bool active;
};

__device__ __forceinline__ TileParticle tile_particle(const int* __restrict__ perm, int n, int64_t np) {
    TileParticle t;
    const int tid = threadIdx.x;
    if (perm) {
        const int64_t slot = int64_t(blockIdx.x) * kTileThreads + tid;
        t.active = slot < np;  // slot 0 of every tile exists, so thread 0 is active
        t.p = t.active ? int64_t(perm[slot]) : 0;
        LatticeDiv ld;
        ld.init(n);
        ld.ijk(t.p, t.i, t.j, t.k);
    } else {
        t.i = blockIdx.x * kTX + (tid % kTX);
        t.j = blockIdx.y * kTY + ((tid / kTX) % kTY);
        t.k = blockIdx.z * kTZ + (tid / (kTX * kTY));
        t.active = (t.i < n) && (t.j < n) && (t.k < n);
        t.p = t.active ? int64_t(t.i) + int64_t(n) * (t.j + int64_t(n) * t.k) : 0;
    }
    return t;
}

template <int W, int NS>
__global__ void __launch_bounds__(kTileThreads, DJB_SCATTER_MIN_BLOCKS) k_scatter_tiled(
    float* __restrict__ psi, const float* __restrict__ mom, float dd1, const float* __restrict__ q1, int n,
    int64_t np, float L, int res, int pitch, GroupShifts sh, float* __restrict__ mesh0,
    float* __restrict__ mesh1, int* err, int budget, const int* __restrict__ perm) {
    extern __shared__ unsigned int sacc[];
    __shared__ int s_row[kMaxRows];
    __shared__ int s_col[kMaxCols];
    const int tid = threadIdx.x;
    const TileParticle tp = tile_particle(perm, n, np);
    const int i = tp.i, j = tp.j, k = tp.k;
    const bool active = tp.active;
    const int64_t p = tp.p;
    float X[3] = {0.0f, 0.0f, 0.0f};
    if (active) {
        float ps[3] = {psi[p], psi[p + np], psi[p + 2 * np]};
        if (mom) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                ps[c] = ps[c] + dd1 * mom[p + c * np];
                psi[p + c * np] = ps[c];
            }
        }
        X[0] = ps[0] + q1[i];
        X[1] = ps[1] + q1[j];
        X[2] = ps[2] + q1[k];
    }
    const float resf = float(res);
#pragma unroll 1
    for (int g = 0; g < NS; ++g) {
        float* mesh = (g == 0) ? mesh0 : mesh1;
        const Shift3 sg = (g == 0) ? sh.s[0] : sh.s[NS > 1 ? 1 : 0];  // no runtime index into params
        float w[3][W];
        int bb[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float s = (a == 0) ? sg.x : (a == 1) ? sg.y : sg.z;
            const float gc = active ? grid_coord(X[a] + s, L, resf, err) : 0.0f;
            bb[a] = wbase<W>(gc);
#pragma unroll
            for (int o = 0; o < W; ++o) w[a][o] = wk<W>(fabsf(gc - float(bb[a] + WLo<W>::v + o)));
        }
        TileBox box;
        int d[3];
        tile_box(bb, active, WLo<W>::v, W, res, box, d);
        if (box.plane > budget || box.S[0] > kMaxCols || box.S[1] > kMaxRows) {
            // extreme spread: per-particle global atomics
            if (active) {
                int ix[W], iy[W], iz[W];
#pragma unroll
                for (int o = 0; o < W; ++o) {
                    ix[o] = wrapi(bb[0] + WLo<W>::v + o, res);
                    iy[o] = wrapi(bb[1] + WLo<W>::v + o, res);
                    iz[o] = wrapi(bb[2] + WLo<W>::v + o, res);
                }
#pragma unroll
                for (int c = 0; c < W; ++c)
#pragma unroll
                    for (int b = 0; b < W; ++b) {
                        float* row = mesh + (int64_t(iz[c]) * res + iy[b]) * pitch;
#pragma unroll
                        for (int a = 0; a < W; ++a) atomicAdd(row + ix[a], w[0][a] * w[1][b] * w[2][c]);
                    }
            }
            continue;
        }
        box_columns(box, res, s_col);
        FastDiv fp;
        fp.init(box.P);
        const int zc = min(budget / box.plane, kMaxRows / box.S[1]);
        for (int z0 = 0; z0 < box.S[2]; z0 += zc) {
            const int nz = min(zc, box.S[2] - z0);
            const int cells = box.plane * nz;
            for (int t = tid; t < cells; t += kTileThreads) sacc[t] = 0u;
            chunk_rows(box, res, z0, nz, s_row);
            __syncthreads();
            if (active) {
#pragma unroll
                for (int c = 0; c < W; ++c) {
                    const int zl = d[2] + c - z0;
                    if (zl < 0 || zl >= nz) continue;
#pragma unroll
                    for (int b = 0; b < W; ++b) {
                        unsigned int* row = sacc + (zl * box.S[1] + d[1] + b) * box.P + d[0];
                        const float wyz = w[1][b];
#pragma unroll
                        for (int a = 0; a < W; ++a) {
                            const float v = w[0][a] * wyz * w[2][c];
                            atomicAdd(row + a, __float2uint_rn(v * FixScale<W>::up));
                        }
                    }
                }
            }
            __syncthreads();
            // flush the chunk's non-zero cells (consecutive threads -> consecutive x)
            for (int t = tid; t < cells; t += kTileThreads) {
                const unsigned int v = sacc[t];
                if (v == 0u) continue;
                const int r = fp.div(t);
                const int x = t - r * box.P;
                atomicAdd(mesh + int64_t(s_row[r]) * pitch + s_col[x], __uint2float_rn(v) * FixScale<W>::down);
            }
            __syncthreads();
        }
    }
}

// ── force interpolation (finite-difference gradient of order 2R) ─────────────
// Out-of-line per-particle interpolation from global memory (extreme-spread tiles).
template <int W, int R>
__device__ __noinline__ void gather_fd_global(const float* __restrict__ phi, int res, int pitch, float gx,
                                              float gy, float gz, float c1, float c2, float c3, float* s) {
    gather_fd<W, R>(phi, res, pitch, gx, gy, gz, c1, c2, c3, s[0], s[1], s[2]);
}

#ifndef DJB_GATHER_MIN_BLOCKS
#define DJB_GATHER_MIN_BLOCKS 2
#endif

template <int W, int R, int NS>
__global__ void __launch_bounds__(kTileThreads, DJB_GATHER_MIN_BLOCKS) k_gather_tiled(GatherArgs A, int budget) {
    extern __shared__ float sbox[];
    __shared__ int s_row[kMaxRows];
    __shared__ int s_col[kMaxCols];
    constexpr int E = W + 2 * R;
    const int tid = threadIdx.x;
    const int n = A.n;
    const int64_t np = A.np;
    const int res = A.res;
    const TileParticle tp = tile_particle(A.perm, n, np);
    const int i = tp.i, j = tp.j, k = tp.k;
    const bool active = tp.active;
    const int64_t p = tp.p;
    float ps[3] = {0.0f, 0.0f, 0.0f};
    float acc[3] = {0.0f, 0.0f, 0.0f};
    if (active) {
        ps[0] = A.psi[p];
        ps[1] = A.psi[p + np];
        ps[2] = A.psi[p + 2 * np];
        if (!A.first) {
            acc[0] = A.acc[p];
            acc[1] = A.acc[p + np];
            acc[2] = A.acc[p + 2 * np];
        }
    }
    const float X[3] = {ps[0] + (active ? A.q1[i] : 0.0f), ps[1] + (active ? A.q1[j] : 0.0f),
                        ps[2] + (active ? A.q1[k] : 0.0f)};
    const float resf = float(res);
    const float cc[4] = {0.0f, A.c1, A.c2, A.c3};
#pragma unroll 1
    for (int g = 0; g < NS; ++g) {
        const float* phi = (g == 0) ? A.mesh[0] : A.mesh[NS > 1 ? 1 : 0];
        const Shift3 sg = (g == 0) ? A.sh.s[0] : A.sh.s[NS > 1 ? 1 : 0];
        float w[3][W], u[3][E];
        float gcs[3];
        int bb[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float s = (a == 0) ? sg.x : (a == 1) ? sg.y : sg.z;
            const float gc = active ? grid_coord(X[a] + s, A.L, resf, A.err) : 0.0f;
            gcs[a] = gc;
            bb[a] = wbase<W>(gc);
#pragma unroll
            for (int o = 0; o < W; ++o) w[a][o] = wk<W>(fabsf(gc - float(bb[a] + WLo<W>::v + o)));
            // weights convolved with the antisymmetric stencil: coefficient of φ(node + t)
            // in F(node) is -c_t (t > 0) and +c_|t| (t < 0)
#pragma unroll
            for (int e = 0; e < E; ++e) {
                float sacc = 0.0f;
#pragma unroll
                for (int o = 0; o < W; ++o) {
                    const int t = e - R - o;
                    if (t > 0 && t <= R) sacc -= w[a][o] * cc[t > 0 ? t : 0];
                    if (t < 0 && -t <= R) sacc += w[a][o] * cc[t < 0 ? -t : 0];
                }
                u[a][e] = sacc;
            }
        }
        TileBox box;
        int d[3];
        tile_box(bb, active, WLo<W>::v - R, E, res, box, d);
        float sX = 0.0f, sY = 0.0f, sZ = 0.0f;
        if (box.plane > budget || box.S[0] > kMaxCols || box.S[1] > kMaxRows) {
            if (active) {
                float sv[3];
                gather_fd_global<W, R>(phi, res, A.pitch, gcs[0], gcs[1], gcs[2], A.c1, A.c2, A.c3, sv);
                sX = sv[0];
                sY = sv[1];
                sZ = sv[2];
            }
        } else {
            box_columns(box, res, s_col);
            FastDiv fp;
            fp.init(box.P);
            const int zc = min(budget / box.plane, kMaxRows / box.S[1]);
            for (int z0 = 0; z0 < box.S[2]; z0 += zc) {
                const int nz = min(zc, box.S[2] - z0);
                const int cells = box.plane * nz;
                chunk_rows(box, res, z0, nz, s_row);
                __syncthreads();
                // stage the chunk with asynchronous global->shared copies (all in flight at once)
                for (int t = tid; t < cells; t += kTileThreads) {
                    const int r = fp.div(t);
                    const int x = t - r * box.P;
                    if (x >= box.S[0]) continue;
                    const float* src = phi + int64_t(s_row[r]) * A.pitch + s_col[x];
                    const unsigned sa = unsigned(__cvta_generic_to_shared(sbox + t));
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(src));
                }
                asm volatile("cp.async.wait_all;\n" ::);
                __syncthreads();
                if (active) {
#pragma unroll
                    for (int e = 0; e < E; ++e) {
                        const int zl = d[2] + e - z0;
                        if (zl < 0 || zl >= nz) continue;
                        const float* pl = sbox + zl * box.plane + d[0];
                        if (e >= R && e < R + W) {
                            const int c = e - R;
#pragma unroll
                            for (int b = 0; b < W; ++b) {
                                const float* row = pl + (d[1] + R + b) * box.P;
                                float rx = 0.0f, rc = 0.0f;
#pragma unroll
                                for (int x = 0; x < E; ++x) {
                                    const float v = row[x];
                                    rx += u[0][x] * v;
                                    if (x >= R && x < R + W) rc += w[0][x - R] * v;
                                }
                                sX += (w[1][b] * w[2][c]) * rx;
                                sY += (u[1][b + R] * w[2][c]) * rc;
                                sZ += (u[2][e] * w[1][b]) * rc;
                            }
#pragma unroll
                            for (int h = 0; h < 2 * R; ++h) {
                                const int ey = (h < R) ? h : h + W;
                                const float* row = pl + (d[1] + ey) * box.P + R;
                                float rc = 0.0f;
#pragma unroll
                                for (int a = 0; a < W; ++a) rc += w[0][a] * row[a];
                                sY += (u[1][ey] * w[2][c]) * rc;
                            }
                        } else {
#pragma unroll
                            for (int b = 0; b < W; ++b) {
                                const float* row = pl + (d[1] + R + b) * box.P + R;
                                float rc = 0.0f;
#pragma unroll
                                for (int a = 0; a < W; ++a) rc += w[0][a] * row[a];
                                sZ += (u[2][e] * w[1][b]) * rc;
                            }
                        }
                    }
                }
                __syncthreads();
            }
        }
        acc[0] += sX;
        acc[1] += sY;
        acc[2] += sZ;
    }
    if (!active) return;
    if (A.last && A.divide) {
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

}  // namespace djb
