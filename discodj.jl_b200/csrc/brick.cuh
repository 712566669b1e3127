// Brick-owned mass assignment and force interpolation.
//
// The particles are binned by the B^3-cell brick holding their (drifted) cell
// floor(g) (sort.cuh, linear brick order). One CTA owns one brick and every particle
// binned into it. The brick's Eulerian box is known in advance. The host bounds the
// base node of a particle relative to its cell over the configuration's shifts, to
// [lo, hi] (0 and 0 or 1 for shift 0; for a shift s the floor or round-to-nearest of
// [c + s, c + 1 + s) widened by 0.01 cells of round-off, and by one more node below
// for the ties of round-to-nearest). Then per axis:
//   mass assignment  : nodes [B*b + lo + lo_W, B*b + B - 1 + hi + lo_W + W), i.e.
//                      B + hi - lo + W - 1 nodes (BrickList::sos, sSs);
//   interpolation    : the same box widened by the finite-difference halo R (so, sS).
// A particle outside its box (the binning and the kernel disagree) sets error bit 2
// and is clamped into the box.
// An empty brick costs one read of its count; a dense brick loops over its particles
// in rounds of 256 while its box stays in shared memory. The staged volume per step
// is (number of non-empty bricks) x (box volume), independent of how far particles
// have moved from their Lagrangian positions.
#pragma once

#include "tiled.cuh"
#include "sort.cuh"
#include "tma.cuh"

namespace djb {

// Interpolation: the resident CTAs per SM its registers are sized for (3 x 256 threads at
// <= 85 registers; the 28 x 26 x 26-node PCS box of 76 KB lets 3 CTAs share an SM's
// shared memory).
#ifndef DJB_BRICK_GATHER_BLOCKS
#define DJB_BRICK_GATHER_BLOCKS 3
#endif

struct BrickList {
    const unsigned* offset;  // block-local exclusive scan of the key counts
    const unsigned* bsum;    // scan of the block totals
    const int* perm;         // particles in key order
    int nb;                  // bricks per axis
    int brick;               // cells per brick side
    int nsub;                // sort keys per brick (2^3-cell sub-blocks)
    int64_t nkeys;           // keys in total
    unsigned np;             // particles
    int sx;                  // interpolation box: width along x (aligned_box),
    int sS;                  //   extent along y and z,
    int so;                  //   first node relative to the brick's first cell
    int ssx;                 // mass-assignment box: width along x,
    int sSs;                 //   extent along y and z,
    int sos;                 //   first node relative to the brick's first cell
};

__device__ __forceinline__ unsigned key_start(const BrickList& bl, int64_t key) {
    return key >= bl.nkeys ? bl.np : bl.offset[key] + bl.bsum[key / kScanBlock];
}

// Brick processed by CTA `blk`. DJB_BRICK_MORTON = 1 and a power-of-two number of bricks
// per axis: Morton (Z-order) order, so that CTAs running at the same time own bricks
// that are neighbours along all three axes and share their boxes' overlap in L2;
// otherwise linear order (x fastest).
#ifndef DJB_BRICK_MORTON
#define DJB_BRICK_MORTON 1
#endif
__device__ __forceinline__ int compact3(unsigned v) {  // every third bit of v, from bit 0
    v &= 0x09249249u;
    v = (v ^ (v >> 2)) & 0x030c30c3u;
    v = (v ^ (v >> 4)) & 0x0300f00fu;
    v = (v ^ (v >> 8)) & 0xff0000ffu;
    v = (v ^ (v >> 16)) & 0x000003ffu;
    return int(v);
}
__device__ __forceinline__ int brick_of_block(const BrickList& bl, unsigned blk) {
#if DJB_BRICK_MORTON
    if ((bl.nb & (bl.nb - 1)) == 0 && bl.nb <= 1024) {
        const int bx = compact3(blk), by = compact3(blk >> 1), bz = compact3(blk >> 2);
        return (bz * bl.nb + by) * bl.nb + bx;
    }
#endif
    return int(blk);
}

// Sorted range [start, start + cnt) of the particles of brick b.
__device__ __forceinline__ void brick_range(const BrickList& bl, int b, unsigned& start, unsigned& cnt) {
    start = key_start(bl, int64_t(b) * bl.nsub);
    cnt = key_start(bl, int64_t(b + 1) * bl.nsub) - start;
}

// Box of brick b: origin B*b + first per axis, S nodes per axis.
__device__ __forceinline__ TileBox brick_box(const BrickList& bl, int b, int first, int S) {
    TileBox box;
    const int bx = b % bl.nb, by = (b / bl.nb) % bl.nb, bz = b / (bl.nb * bl.nb);
    box.o[0] = bx * bl.brick + first;
    box.o[1] = by * bl.brick + first;
    box.o[2] = bz * bl.brick + first;
    box.S[0] = box.S[1] = box.S[2] = S;
    box.P = S | 1;
    box.plane = box.P * S;
    return box;
}

// Offset of a node from the box origin, periodic differences taken in [-4, res - 4):
// valid offsets lie in [0, sx - 1] and res > sx + 4 (the host sizes the bricks so).
// node - origin lies in [-res - 4, 2 res - 4) (nodes in [-5, res + 2], origins in
// [-5, res)), so one correction either way suffices.
__device__ __forceinline__ int box_rel(int node, int origin, int res) {
    int v = node - origin;
    if (v < -4) v += res;
    if (v >= res - 4) v -= res;
    return v;
}

// Box of brick b with the x origin rounded down to a multiple of 4 nodes (so that
// every row starts on a 16-byte boundary of a dense mesh) and `sx` nodes along x (a
// multiple of 4 covering the S nodes after the rounding); y and z as brick_box.
// Shared memory holds the box densely, [z][y][x] with rows of sx elements.
__device__ __forceinline__ TileBox aligned_box(const BrickList& bl, int b, int first, int S, int sx) {
    TileBox box = brick_box(bl, b, first, S);
    box.o[0] &= ~3;
    box.S[0] = sx;
    box.P = sx;
    box.plane = sx * S;
    return box;
}

// Elements reserved per box in shared memory: a multiple of 32 (128 bytes, the alignment
// of a bulk tensor copy's shared-memory operand).
__host__ __device__ __forceinline__ int box_stride(int cells) { return (cells + 31) & ~31; }

__device__ __forceinline__ bool box_inside(const TileBox& box, int res) {
    return box.o[0] >= 0 && box.o[0] + box.S[0] <= res && box.o[1] >= 0 && box.o[1] + box.S[1] <= res &&
           box.o[2] >= 0 && box.o[2] + box.S[2] <= res;
}

// Walks the box in copies of `per` elements (4 when `vec`: pitch and res multiples of 4,
// so a 16-byte group never straddles the periodic wrap; else 1) and calls
// f(shared offset, global offset) with the wrapped global element offset.
template <class F>
__device__ __forceinline__ void for_box_wrapped(const TileBox& box, int res, int pitch, bool vec, F f) {
    const int S1 = box.S[1];
    FastDiv fy;
    fy.init(S1);
    const int per = vec ? 4 : 1;
    const int cpr = box.S[0] / per;  // copies per row
    FastDiv fc;
    fc.init(cpr);
    const int total = cpr * S1 * box.S[2];
    for (int t = threadIdx.x; t < total; t += kTileThreads) {
        const int r = fc.div(t);
        const int c = t - r * cpr;
        const int z = fy.div(r);
        const int y = r - z * S1;
        const int gx = wrap2(box.o[0] + per * c, res);
        const int gy = wrap2(box.o[1] + y, res);
        const int gz = wrap2(box.o[2] + z, res);
        f(r * box.S[0] + per * c, (int64_t(gz) * res + gy) * pitch + gx);
    }
}

// ── mass assignment ───────────────────────────────────────────────────────────
// Box: the deposit box (BrickList::ssx, sSs, sos); kScatterBoxes shifts of the group
// are filled per pass over the brick's particles, one box each. One box per pass (45 KB
// for PCS) and registers sized for 5 resident CTAs per SM (48 registers, no spills)
// measured faster than both shifts per pass at 2 CTAs per SM, and than 4 CTAs per SM. `tma` != 0: the meshes are dense [res]^3
// (pitch == res) described by tm0/tm1 with boxes of the deposit box's shape; boxes that
// do not wrap are then added to the mesh with one bulk tensor reduction each.
#ifndef DJB_SCATTER_BOXES
#define DJB_SCATTER_BOXES 1
#endif
#ifndef DJB_BRICK_SCATTER_BLOCKS
#define DJB_BRICK_SCATTER_BLOCKS 5
#endif
constexpr int kScatterBoxes = DJB_SCATTER_BOXES;

// Fixed-point unit of a brick of `cnt` particles. A node sum is at most
// cnt * (MaxW3 * up + 1) (each rounded weight is below its value + 1), which must stay
// below 2^32. Sparse bricks keep FixScale<W>::up; denser ones take the largest power of
// two that keeps the bound. The rounding error of a fixed-point sum is at most half a unit
// per particle whatever the sum's size, while a float sum of many equal weights (a
// collapsed clump) drifts by a fraction of its own ulp per addition; so fixed point stays
// the more accurate form down to units of 2^8 (bricks of ~5.6e7 particles), below which
// the brick accumulates in float with shared float atomics (returns 0).
template <int W>
__device__ __forceinline__ float brick_fixed_unit(unsigned cnt) {
    const float room = 4294967296.0f / float(cnt) - 1.0f;  // MaxW3 * up must stay below this
    if (room >= MaxW3<W>::v * FixScale<W>::up) return FixScale<W>::up;
    int e;
    frexpf(room / MaxW3<W>::v, &e);  // room / MaxW3 in [2^(e-1), 2^e)
    return (e - 1 >= 8) ? ldexpf(1.0f, e - 1) : 0.0f;
}

template <int W, int NS>
__global__ void __launch_bounds__(kTileThreads, DJB_BRICK_SCATTER_BLOCKS) k_scatter_brick(
    const float* __restrict__ psi, const float* __restrict__ q1, int n, int64_t np, float L, int res, int pitch,
    GroupShifts sh, float* __restrict__ mesh0, float* __restrict__ mesh1, int* err, BrickList bl,
    const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1, int tma) {
    constexpr int NB = kScatterBoxes < NS ? kScatterBoxes : NS;  // boxes per particle pass
    extern __shared__ __align__(128) unsigned int sacc[];
    const int b = brick_of_block(bl, blockIdx.x);
    unsigned start, cnt;
    brick_range(bl, b, start, cnt);
    if (cnt == 0) return;
    const int tid = threadIdx.x;
    const TileBox box = aligned_box(bl, b, bl.sos, bl.sSs, bl.ssx);
    const bool bulk = tma && box_inside(box, res) && (smem_u32(sacc) & 127u) == 0u;
    const bool vec = ((pitch | res) & 3) == 0;
    const float resf = float(res);
    const int cells = box.plane * box.S[2];  // a multiple of 4
    const int stride = box_stride(cells);    // boxes start on 128-byte boundaries (bulk tensor copies)
    // 32-bit fixed point with a unit that keeps every node sum of this brick below 2^32;
    // bricks too dense for that accumulate float sums (sacc then holds floats)
    const float up = brick_fixed_unit<W>(cnt);
    const bool fixed = up > 0.0f;
    const float down = fixed ? 1.0f / up : 1.0f;
    LatticeDiv ld;
    ld.init(n);
#pragma unroll 1
    for (int g0 = 0; g0 < NS; g0 += NB) {
        for (int t = 4 * tid; t < NB * stride; t += 4 * kTileThreads)
            *reinterpret_cast<uint4*>(sacc + t) = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        for (unsigned r0 = 0; r0 < cnt; r0 += kTileThreads) {
            // lanes 8 slots apart: particles of one cell land in different warps, which
            // keeps same-address shared atomics out of a single instruction
            const unsigned slot = r0 + unsigned((tid & 31) * (kTileThreads / 32) + (tid >> 5));
            if (slot >= cnt) continue;
            const int64_t p = bl.perm[start + slot];
            int i, j, k;
            ld.ijk(p, i, j, k);
            const float X[3] = {psi[p] + q1[i], psi[p + np] + q1[j], psi[p + 2 * np] + q1[k]};
#pragma unroll 1
            for (int gb = 0; gb < NB; ++gb) {
                const int g = g0 + gb;
                const Shift3 sg = (g == 0) ? sh.s[0] : sh.s[NS > 1 ? 1 : 0];
                unsigned int* acc = sacc + gb * stride;
                float w[3][W];
                int d[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float s = (a == 0) ? sg.x : (a == 1) ? sg.y : sg.z;
                    const float gc = grid_coord(X[a] + s, L, resf, err);
                    const int bb = wbase<W>(gc);
#pragma unroll
                    for (int o = 0; o < W; ++o) w[a][o] = wk<W>(fabsf(gc - float(bb + WLo<W>::v + o)));
                    d[a] = box_rel(bb + WLo<W>::v, box.o[a], res);
                    if (d[a] < 0 || d[a] > box.S[a] - W) {  // not binned consistently: report, stay in bounds
                        atomicOr(err, 2);
                        d[a] = d[a] < 0 ? 0 : box.S[a] - W;
                    }
                }
                if (fixed) {
#pragma unroll
                    for (int c = 0; c < W; ++c)
#pragma unroll
                        for (int bb = 0; bb < W; ++bb) {
                            unsigned int* row = acc + ((d[2] + c) * box.S[1] + d[1] + bb) * box.P + d[0];
                            const float wyz = w[1][bb] * up;
#pragma unroll
                            for (int a = 0; a < W; ++a) atomicAdd(row + a, __float2uint_rn(w[0][a] * wyz * w[2][c]));
                        }
                } else {
#pragma unroll
                    for (int c = 0; c < W; ++c)
#pragma unroll
                        for (int bb = 0; bb < W; ++bb) {
                            float* row =
                                reinterpret_cast<float*>(acc) + ((d[2] + c) * box.S[1] + d[1] + bb) * box.P + d[0];
                            const float wyz = w[1][bb];
#pragma unroll
                            for (int a = 0; a < W; ++a) atomicAdd(row + a, w[0][a] * wyz * w[2][c]);
                        }
                }
            }
        }
        __syncthreads();
        if (bulk) {
            // fixed point -> float in place, then one bulk reduction per box
            if (fixed)
                for (int t = 4 * tid; t < NB * stride; t += 4 * kTileThreads) {
                    const uint4 v = *reinterpret_cast<const uint4*>(sacc + t);
                    *reinterpret_cast<float4*>(sacc + t) =
                        make_float4(__uint2float_rn(v.x) * down, __uint2float_rn(v.y) * down,
                                    __uint2float_rn(v.z) * down, __uint2float_rn(v.w) * down);
                }
            fence_proxy_async_smem();  // the conversions are read by the bulk copies below
            __syncthreads();
            if (tid == 0) {
                for (int gb = 0; gb < NB; ++gb)
                    tma_reduce_add_3d((g0 + gb == 0) ? &tm0 : &tm1, box.o[0], box.o[1], box.o[2], sacc + gb * stride);
                bulk_commit_and_wait_read();  // shared memory stays allocated until read
            }
            __syncthreads();
        } else {
#pragma unroll 1
            for (int gb = 0; gb < NB; ++gb) {
                float* mesh = (g0 + gb == 0) ? mesh0 : mesh1;
                const unsigned int* acc = sacc + gb * stride;
                for_box_wrapped(box, res, pitch, vec, [&](int so, int64_t go) {
                    // float sums (dense bricks) are read as their bit patterns: +0.0f is 0u
                    const auto val = [&](unsigned v) { return fixed ? __uint2float_rn(v) * down : __uint_as_float(v); };
                    if (vec) {
                        const uint4 v = *reinterpret_cast<const uint4*>(acc + so);
                        if ((v.x | v.y | v.z | v.w) == 0u) return;
                        red_add_v4(mesh + go, val(v.x), val(v.y), val(v.z), val(v.w));
                    } else {
                        const unsigned v = acc[so];
                        if (v != 0u) atomicAdd(mesh + go, val(v));
                    }
                });
            }
            __syncthreads();
        }
    }
}

// Stages the potential over `box` with asynchronous copies that take the periodic wrap.
__device__ __forceinline__ void stage_box_wrapped(float* sbox, const float* __restrict__ phi, const TileBox& box,
                                                  int res, int pitch, bool vec) {
    for_box_wrapped(box, res, pitch, vec, [&](int so, int64_t go) {
        const unsigned sa = smem_u32(sbox + so);
        if (vec)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(phi + go));
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(phi + go));
    });
    asm volatile("cp.async.wait_all;\n" ::);
}

// Force interpolation of one brick's particles: FD gradient of the staged potential,
// interpolation with the mass-assignment weights, mean over the interlacing shifts, then
// the kick and drift. The shifts are the outer loop: the brick's box is staged once per
// shift for all of its particles, and the sums over the shifts go through the
// acceleration array (the last shift applies the mean, the correction and the
// kick-drift). With `A.part` (6 blocks of np floats) they go through it instead, in
// sorted order, together with a copy of Ψ made in the call's first shift: a thread
// visits the same sorted positions in every shift of a force call (the same `perm`,
// the same slots), so it reads back only what it wrote, and its accesses are coalesced
// where the particle-order ones are scattered. `tma` != 0: the potentials are dense [res]^3 meshes (pitch == res)
// described by tm0/tm1 (box sx x S x S); boxes that do not wrap are then fetched with one
// bulk tensor copy.
template <int W, int R, int NS>
__global__ void __launch_bounds__(kTileThreads, DJB_BRICK_GATHER_BLOCKS) k_gather_brick(
    GatherArgs A, BrickList bl, const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
    int tma) {
    extern __shared__ __align__(128) float sbox[];
    __shared__ __align__(8) uint64_t s_bar;
    constexpr int E = W + 2 * R;
    const int b = brick_of_block(bl, blockIdx.x);
    unsigned start, cnt;
    brick_range(bl, b, start, cnt);
    if (cnt == 0) return;
    const int tid = threadIdx.x;
    const int n = A.n;
    const int64_t np = A.np;
    const int res = A.res;
    const TileBox box = aligned_box(bl, b, bl.so, bl.sS, bl.sx);
    const bool bulk = tma && box_inside(box, res) && (smem_u32(sbox) & 127u) == 0u;
    const bool vec = ((A.pitch | res) & 3) == 0;
    const unsigned box_bytes = unsigned(box.plane) * unsigned(box.S[2]) * 4u;
    if (bulk && tid == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    unsigned parity = 0;
    const float resf = float(res);
    const float cc[4] = {0.0f, A.c1, A.c2, A.c3};
    LatticeDiv ld;
    ld.init(n);
#pragma unroll 1
    for (int g = 0; g < NS; ++g) {
        const Shift3 sgs = (g == 0) ? A.sh.s[0] : A.sh.s[NS > 1 ? 1 : 0];
        if (bulk) {
            if (tid == 0) {
                fence_proxy_async_smem();  // the previous shift's reads precede the refill
                mbar_arrive_expect_tx(&s_bar, box_bytes);
                tma_load_3d(sbox, (g == 0) ? &tm0 : &tm1, box.o[0], box.o[1], box.o[2], &s_bar);
            }
            const bool ok = mbar_wait(&s_bar, parity);
            parity ^= 1u;
            if (__syncthreads_or(!ok)) {  // the copy never completed: report, do not spin
                if (tid == 0) atomicOr(A.err, 8);
                return;
            }
        } else {
            stage_box_wrapped(sbox, (g == 0) ? A.mesh[0] : A.mesh[NS > 1 ? 1 : 0], box, res, A.pitch, vec);
            __syncthreads();
        }
        const bool first_sum = A.first && g == 0;   // no partial sum to continue
        const bool finish = A.last && g == NS - 1;  // mean, correction, kick-drift
#pragma unroll 1
        for (unsigned slot = tid; slot < cnt; slot += kTileThreads) {
            const int64_t at = int64_t(start) + slot;  // sorted position: this thread's in every shift
            const int64_t p = bl.perm[at];
            int i, j, k;
            ld.ijk(p, i, j, k);
            // after the call's first shift, Ψ comes from the sorted copy (coalesced)
            const bool from_part = A.part && !first_sum;
            const float ps[3] = {from_part ? A.part[at + 3 * np] : A.psi[p],
                                 from_part ? A.part[at + 4 * np] : A.psi[p + np],
                                 from_part ? A.part[at + 5 * np] : A.psi[p + 2 * np]};
            const float X[3] = {ps[0] + A.q1[i], ps[1] + A.q1[j], ps[2] + A.q1[k]};
            float w[3][W], u[3][E];
            int d[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float s = (a == 0) ? sgs.x : (a == 1) ? sgs.y : sgs.z;
                const float gc = grid_coord(X[a] + s, A.L, resf, A.err);
                const int bb = wbase<W>(gc);
#pragma unroll
                for (int o = 0; o < W; ++o) w[a][o] = wk<W>(fabsf(gc - float(bb + WLo<W>::v + o)));
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
                d[a] = box_rel(bb + WLo<W>::v - R, box.o[a], res);
                if (d[a] < 0 || d[a] > box.S[a] - E) {  // not binned consistently: report, stay in bounds
                    atomicOr(A.err, 2);
                    d[a] = d[a] < 0 ? 0 : box.S[a] - E;
                }
            }
            float sX = 0.0f, sY = 0.0f, sZ = 0.0f;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const float* pl = sbox + (d[2] + e) * box.plane + d[0];
                if (e >= R && e < R + W) {
                    const int c = e - R;
#pragma unroll
                    for (int bb = 0; bb < W; ++bb) {
                        const float* row = pl + (d[1] + R + bb) * box.P;
                        float rx = 0.0f, rc = 0.0f;
#pragma unroll
                        for (int x = 0; x < E; ++x) {
                            const float v = row[x];
                            rx += u[0][x] * v;
                            if (x >= R && x < R + W) rc += w[0][x - R] * v;
                        }
                        sX += (w[1][bb] * w[2][c]) * rx;
                        sY += (u[1][bb + R] * w[2][c]) * rc;
                        sZ += (u[2][e] * w[1][bb]) * rc;
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
                    for (int bb = 0; bb < W; ++bb) {
                        const float* row = pl + (d[1] + R + bb) * box.P + R;
                        float rc = 0.0f;
#pragma unroll
                        for (int a = 0; a < W; ++a) rc += w[0][a] * row[a];
                        sZ += (u[2][e] * w[1][bb]) * rc;
                    }
                }
            }
            float a3[3] = {sX, sY, sZ};
            if (!first_sum) {
                if (A.part) {
                    a3[0] += A.part[at];
                    a3[1] += A.part[at + np];
                    a3[2] += A.part[at + 2 * np];
                } else {
                    a3[0] += A.acc[p];
                    a3[1] += A.acc[p + np];
                    a3[2] += A.acc[p + 2 * np];
                }
            }
            if (finish) {
                if (A.divide) {
                    a3[0] = a3[0] / A.nshift_f;
                    a3[1] = a3[1] / A.nshift_f;
                    a3[2] = a3[2] / A.nshift_f;
                }
                if (A.extra) {
                    a3[0] += A.extra[p];
                    a3[1] += A.extra[p + np];
                    a3[2] += A.extra[p + 2 * np];
                }
            }
            if (finish && A.step) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float m = A.alpha * A.mom[p + c * np] + A.beta * a3[c];
                    A.mom[p + c * np] = m;
                    A.psi[p + c * np] = ps[c] + A.dd2 * m;
                }
            } else if (finish || !A.part) {
                A.acc[p] = a3[0];
                A.acc[p + np] = a3[1];
                A.acc[p + 2 * np] = a3[2];
            } else {  // partial sums (and, after the first shift, Ψ) in sorted order
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    A.part[at + c * np] = a3[c];
                    if (first_sum) A.part[at + (3 + c) * np] = ps[c];
                }
            }
        }
        __syncthreads();  // the box is read before the next shift's copy
    }
}

// Interpolation of three node fields (the force correction on the mesh) to the brick's
// particles with the mass-assignment weights at their unshifted positions: out_c(p) =
// scale * sum_n W(X_p - n) f_c(n). One CTA per brick; the brick's deposit boxes of the
// three fields (rows of sx nodes) are staged together, one bulk tensor copy each where
// the box does not wrap (`tma` != 0: f is three dense [res]^3 meshes described by
// tm0..tm2), so each particle's 3 W^3 loads come from shared memory.
template <int W>
__global__ void __launch_bounds__(kTileThreads, 2) k_interp3_brick(
    const float* __restrict__ psi, const float* __restrict__ q1, int n, int64_t np, float L, int res,
    const float* __restrict__ f, float scale, float* __restrict__ out, int* err, BrickList bl, int sx,
    const __grid_constant__ CUtensorMap tm0, const __grid_constant__ CUtensorMap tm1,
    const __grid_constant__ CUtensorMap tm2, int tma) {
    extern __shared__ __align__(128) float fbox[];
    __shared__ __align__(8) uint64_t s_bar;
    const int b = brick_of_block(bl, blockIdx.x);
    unsigned start, cnt;
    brick_range(bl, b, start, cnt);
    if (cnt == 0) return;
    const int tid = threadIdx.x;
    const int64_t cells = int64_t(res) * res * res;
    const TileBox box = aligned_box(bl, b, bl.sos, bl.sSs, sx);
    const int bcells = box.plane * box.S[2];
    const int stride = box_stride(bcells);   // boxes on 128-byte boundaries
    const bool bulk = tma && box_inside(box, res) && (smem_u32(fbox) & 127u) == 0u;
    if (bulk) {
        if (tid == 0) mbar_init(&s_bar, 1);
        __syncthreads();
        if (tid == 0) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&s_bar, 3u * unsigned(bcells) * 4u);
            tma_load_3d(fbox, &tm0, box.o[0], box.o[1], box.o[2], &s_bar);
            tma_load_3d(fbox + stride, &tm1, box.o[0], box.o[1], box.o[2], &s_bar);
            tma_load_3d(fbox + 2 * stride, &tm2, box.o[0], box.o[1], box.o[2], &s_bar);
        }
        const bool ok = mbar_wait(&s_bar, 0);
        if (__syncthreads_or(!ok)) {   // the copies never completed: report, do not spin
            if (tid == 0) atomicOr(err, 8);
            return;
        }
    } else {
        const bool vec = (res & 3) == 0;
        for (int c = 0; c < 3; ++c) stage_box_wrapped(fbox + c * stride, f + c * cells, box, res, res, vec);
        __syncthreads();
    }
    const float resf = float(res);
    LatticeDiv ld;
    ld.init(n);
#pragma unroll 1
    for (unsigned slot = tid; slot < cnt; slot += kTileThreads) {
        const int64_t p = bl.perm[start + slot];
        int ijk[3];
        ld.ijk(p, ijk[0], ijk[1], ijk[2]);
        float w[3][W];
        int d[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float gc = grid_coord(psi[p + a * np] + q1[ijk[a]], L, resf, err);
            const int bb = wbase<W>(gc);
#pragma unroll
            for (int o = 0; o < W; ++o) w[a][o] = wk<W>(fabsf(gc - float(bb + WLo<W>::v + o)));
            d[a] = box_rel(bb + WLo<W>::v, box.o[a], res);
            if (d[a] < 0 || d[a] > box.S[a] - W) {   // not binned consistently: report, stay in bounds
                atomicOr(err, 2);
                d[a] = d[a] < 0 ? 0 : box.S[a] - W;
            }
        }
        float v[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int z = 0; z < W; ++z) {
            float sy[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int y = 0; y < W; ++y) {
                const float* row = fbox + ((d[2] + z) * box.S[1] + d[1] + y) * box.P + d[0];
                float sxv[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int x = 0; x < W; ++x) {
                    sxv[0] += w[0][x] * row[x];
                    sxv[1] += w[0][x] * row[stride + x];
                    sxv[2] += w[0][x] * row[2 * stride + x];
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) sy[c] += w[1][y] * sxv[c];
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] += w[2][z] * sy[c];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) out[p + c * np] = scale * v[c];
    }
}

}  // namespace djb
