// Force-correction network: a 3-D CNN on the PM mesh (no counterpart in the reference).
//
// Layers: L convolutions with 3³ kernels and periodic boundaries (the box is periodic),
// cin → hidden → … → hidden → cout channels, ReLU after every layer but the last.
// Inputs and outputs cross the C ABI as float32 meshes in the solver's layout,
// [channel][z][y][x]; inside, activations are bf16 channels-last, [voxel][channel].
//
// Every convolution whose padded channel counts are at most 32 runs on the tensor cores
// (tcgen05.mma, `conv_tc.cuh`), forward and backward:
//   forward        k_conv3_tc: input planes staged in shared memory once, the taps
//                  read as shifted operand views, accumulators in tensor memory, bias
//                  + ReLU fused into the epilogue (the first layer from x-pair rows);
//   data gradient  k_conv3_tc with the weights flipped and transposed, ReLU′ of the
//                  layer below fused into the epilogue;
//   weight grad.   k_conv3_wgrad (inputs narrower than 32 channels zero-widened first).
// Wider layers, and every layer after djb_nn_set_conv(h, 1), make the implicit GEMM
// explicit per chunk of z planes:
//   col[v][tap·C + c] = X[v + offset(tap)][c]        k_im2col (bf16, periodic wrap)
//   Y = col · W  (M = voxels, K = 27·C, N = channels out; bf16 operands, float32
//                 accumulation on the tensor cores through cuBLAS)
//   X' = relu(Y + b) → bf16                           k_bias_act
// and their backward: dW = colᵀ·dY and dcol = dY·Wᵀ (cuBLAS), dX[v] = Σ_tap
// dcol[v − offset(tap)][tap] (k_col2im, a gather: no atomics). db = Σ_v dY (a block
// reduction). Loss: mean squared error over all outputs. Optimizer: Adam on float32
// master weights, then the bf16 copies the kernels read.
// Channel counts are padded to multiples of 8 (16-byte rows for the tensor cores);
// the padding channels hold zeros and their weights stay zero.
#include <cublas_v2.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <new>
#include <random>
#include <vector>

#include "common.h"
#include "conv_tc.cuh"
#include "djb200.h"

using djb::fail;

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(DJB_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));      \
    } while (0)

#define CUBLAS_TRY(expr)                                                                        \
    do {                                                                                        \
        cublasStatus_t st_ = (expr);                                                            \
        if (st_ != CUBLAS_STATUS_SUCCESS) return fail(DJB_ERR_CUDA, "%s failed (cuBLAS %d)", #expr, int(st_)); \
    } while (0)

namespace {

constexpr int kMaxLayers = 8;
constexpr int kNT = 256;

__host__ __device__ inline int pad8(int c) { return (c + 7) & ~7; }

// voxel index of (x, y, z) + (dx, dy, dz) on the periodic res³ mesh, v = (z·res + y)·res + x
__device__ __forceinline__ int64_t nbr(int x, int y, int z, int dx, int dy, int dz, int res) {
    x += dx;
    y += dy;
    z += dz;
    x = x < 0 ? x + res : (x >= res ? x - res : x);
    y = y < 0 ? y + res : (y >= res ? y - res : y);
    z = z < 0 ? z + res : (z >= res ? z - res : z);
    return (int64_t(z) * res + y) * res + x;
}

// float32 [c][z][y][x] (c < cin) → bf16 [v][cp] (zeros beyond cin, cp a multiple of 8),
// one voxel per thread. `pair` (cin <= 4, may be null): also the x-pair rows
// [v][8] = (4 channels of v, 4 channels of its +x neighbour, periodic), the first
// layer's tensor-core input.
__global__ void k_pack(const float* __restrict__ in, int cin, int cp, int res, int64_t nvox,
                       __nv_bfloat16* __restrict__ out, __nv_bfloat16* __restrict__ pair) {
    for (int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < nvox; v += int64_t(gridDim.x) * blockDim.x) {
        const int x = int(v % res);
        const int64_t vn = v - x + (x + 1 == res ? 0 : x + 1);
        float f[8], g[4];
#pragma unroll
        for (int c = 0; c < 8; ++c) f[c] = c < cin ? in[int64_t(c) * nvox + v] : 0.0f;
        uint4* o = reinterpret_cast<uint4*>(out + v * cp);
        o[0] = make_uint4(djb::conv::pack_bf16(f[0], f[1]), djb::conv::pack_bf16(f[2], f[3]),
                          djb::conv::pack_bf16(f[4], f[5]), djb::conv::pack_bf16(f[6], f[7]));
        for (int c8 = 1; c8 < cp / 8; ++c8) {
            float h[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) h[j] = c8 * 8 + j < cin ? in[int64_t(c8 * 8 + j) * nvox + v] : 0.0f;
            o[c8] = make_uint4(djb::conv::pack_bf16(h[0], h[1]), djb::conv::pack_bf16(h[2], h[3]),
                               djb::conv::pack_bf16(h[4], h[5]), djb::conv::pack_bf16(h[6], h[7]));
        }
        if (pair) {
#pragma unroll
            for (int c = 0; c < 4; ++c) g[c] = c < cin ? in[int64_t(c) * nvox + vn] : 0.0f;
            reinterpret_cast<uint4*>(pair)[v] =
                make_uint4(djb::conv::pack_bf16(f[0], f[1]), djb::conv::pack_bf16(f[2], f[3]),
                           djb::conv::pack_bf16(g[0], g[1]), djb::conv::pack_bf16(g[2], g[3]));
        }
    }
}

// col[v][tap·C + c] for the m voxels starting at v0 (C a multiple of 8: 16-byte copies).
__global__ void k_im2col(const __nv_bfloat16* __restrict__ X, int res, int C, int64_t v0, int64_t m,
                         __nv_bfloat16* __restrict__ col) {
    const int groups = C / 8;
    const int64_t total = m * 27 * groups;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int g = int(t % groups);
        const int64_t r = t / groups;
        const int tap = int(r % 27);
        const int64_t vl = r / 27;
        const int64_t v = v0 + vl;
        const int x = int(v % res), y = int((v / res) % res), z = int(v / (int64_t(res) * res));
        const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
        const int64_t src = nbr(x, y, z, dx, dy, dz, res);
        reinterpret_cast<uint4*>(col + (vl * 27 + tap) * C)[g] = reinterpret_cast<const uint4*>(X + src * C)[g];
    }
}

// out[v][c] = act(Y[v][c] + b[c]) for c < n, zero for n <= c < np (bf16); `relu` or identity.
__global__ void k_bias_act(const float* __restrict__ Y, int n, const float* __restrict__ b, int np, int relu,
                           int64_t m, __nv_bfloat16* __restrict__ out) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m * np; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = t / np;
        const int c = int(t - v * np);
        float y = 0.0f;
        if (c < n) {
            y = Y[v * n + c] + b[c];
            if (relu) y = fmaxf(y, 0.0f);
        }
        out[t] = __float2bfloat16_rn(y);
    }
}

// last layer: out = Y + b (float32 [v][n]) for voxels [v0, v0 + m) → channel-major mesh
__global__ void k_bias_out(const float* __restrict__ Y, int n, const float* __restrict__ b, int64_t nvox, int64_t v0,
                           int64_t m, float* __restrict__ out) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m * n; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = t / n;
        const int c = int(t - v * n);
        out[int64_t(c) * nvox + v0 + v] = Y[t] + b[c];
    }
}

// dY[v][c] = 2 (out − target) / count and Σ (out − target)² into *sum (double).
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ target, int n, int64_t nvox,
                      double inv_count, float* __restrict__ dY, double* __restrict__ sum) {
    __shared__ double part[kNT];
    double acc = 0.0;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nvox * n; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = t / n;
        const int c = int(t - v * n);
        const float d = out[int64_t(c) * nvox + v] - target[int64_t(c) * nvox + v];
        acc += double(d) * d;
        dY[t] = float(2.0 * inv_count) * d;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(sum, part[0]);
}

// dY[v][c] = dout[c][v]: a given gradient of the output mesh, in the layout k_mse writes.
__global__ void k_out_grad(const float* __restrict__ dout, int n, int64_t nvox, float* __restrict__ dY) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nvox * n; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = t / n;
        const int c = int(t - v * n);
        dY[t] = dout[int64_t(c) * nvox + v];
    }
}

// float32 [v][n] → bf16 [v][np] (zeros beyond n), optionally masked by A > 0 (ReLU backward).
__global__ void k_grad_bf16(const float* __restrict__ dA, int n, int np, const __nv_bfloat16* __restrict__ A,
                            int64_t m, __nv_bfloat16* __restrict__ dY) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < m * np; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = t / np;
        const int c = int(t - v * np);
        float g = 0.0f;
        if (c < n) {
            g = dA[v * n + c];
            if (A && !(__bfloat162float(A[t]) > 0.0f)) g = 0.0f;
        }
        dY[t] = __float2bfloat16_rn(g);
    }
}

// db[c] += Σ_v dY[v][c] (bf16 [v][np], c < n, np a multiple of 8): thread t of a block
// sums the 8-channel chunk t % (np/8) of every (blockDim / (np/8))-th voxel of a
// grid-stride run; the block's partial sums meet in shared memory and leave with one
// atomic per channel.
__global__ void k_bias_grad(const __nv_bfloat16* __restrict__ dY, int n, int np, int64_t m, float* __restrict__ db) {
    __shared__ float part[kNT][8];
    const int chunks = np / 8;
    const int vpb = kNT / chunks;                       // voxels per block and pass
    const int c8 = threadIdx.x % chunks, r = threadIdx.x / chunks;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (r < vpb) {
        for (int64_t v = int64_t(blockIdx.x) * vpb + r; v < m; v += int64_t(gridDim.x) * vpb) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(dY + v * np) + c8);
            const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[j]);
                acc[2 * j] += __bfloat162float(h.x);
                acc[2 * j + 1] += __bfloat162float(h.y);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) part[threadIdx.x][j] = acc[j];
    __syncthreads();
    if (int(threadIdx.x) < n) {
        const int c = threadIdx.x, ch = c / 8, j = c % 8;
        float s = 0.0f;
        for (int q = 0; q < vpb; ++q) s += part[q * chunks + ch][j];
        atomicAdd(db + c, s);
    }
}

// dX[v][c] = Σ_tap dcol[v − offset(tap)][tap][c] over all voxels (float32, C channels)
__global__ void k_col2im(const float* __restrict__ dcol, int res, int C, int64_t nvox, float* __restrict__ dX) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nvox * C; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = t / C;
        const int c = int(t - v * C);
        const int x = int(v % res), y = int((v / res) % res), z = int(v / (int64_t(res) * res));
        float acc = 0.0f;
#pragma unroll
        for (int tap = 0; tap < 27; ++tap) {
            const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
            const int64_t src = nbr(x, y, z, -dx, -dy, -dz, res);
            acc += dcol[(src * 27 + tap) * C + c];
        }
        dX[t] = acc;
    }
}

// Adam (float32 master weights) and the bf16 copy of the weights.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, int64_t count, float lr, float b1, float b2, float eps, float c1,
                       float c2, const uint8_t* __restrict__ frozen, __nv_bfloat16* __restrict__ pb) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < count; t += int64_t(gridDim.x) * blockDim.x) {
        if (frozen && frozen[t]) continue;
        const float gi = g[t];
        const float a = b1 * m1[t] + (1.0f - b1) * gi;
        const float b = b2 * m2[t] + (1.0f - b2) * gi * gi;
        m1[t] = a;
        m2[t] = b;
        const float mh = a / c1, vh = b / c2;
        p[t] -= lr * mh / (sqrtf(vh) + eps);
        if (pb) pb[t] = __float2bfloat16_rn(p[t]);
    }
}

__global__ void k_to_bf16(const float* __restrict__ a, int64_t count, __nv_bfloat16* __restrict__ b) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < count; t += int64_t(gridDim.x) * blockDim.x)
        b[t] = __float2bfloat16_rn(a[t]);
}

int grid_of(int64_t count) { return int(std::min<int64_t>((count + kNT - 1) / kNT, 148LL * 32)); }

}  // namespace

struct djb_nn {
    int layers = 0;
    int cin[kMaxLayers] = {}, cout[kMaxLayers] = {};   // real channel counts per layer
    int cinp[kMaxLayers] = {}, coutp[kMaxLayers] = {};  // padded to 8
    int64_t woff[kMaxLayers] = {}, boff[kMaxLayers] = {};
    int64_t nparam = 0;
    int device = 0;
    cudaStream_t stream = nullptr, own = nullptr;
    cublasHandle_t blas = nullptr;
    // parameters: float32 master, bf16 copy, Adam moments, gradients, frozen mask (padding)
    float* p = nullptr;
    __nv_bfloat16* pb = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    float* g = nullptr;
    uint8_t* frozen = nullptr;
    int64_t step = 0;
    // work areas for a mesh of `res`³ voxels processed in chunks of `chunk` voxels
    int res = 0;
    int64_t chunk = 0;
    __nv_bfloat16* act[kMaxLayers + 1] = {};  // [v][cinp] per layer input (act[L] unused)
    __nv_bfloat16* act0p = nullptr;            // [v][8] x-pair rows of the input (use_pair)
    __nv_bfloat16* actw = nullptr;             // [v][32] a narrow layer input widened (training)
    __nv_bfloat16* col = nullptr;              // [chunk][27·Cmax]
    float* Y = nullptr;                        // [chunk][Nmax] (also dA)
    float* dcol = nullptr;                     // [nvox][27·Cmax] (training only)
    float* dA = nullptr;                       // [nvox][Cmax]
    __nv_bfloat16* dY = nullptr;               // [nvox][Cmax]
    __nv_bfloat16* dY2 = nullptr;              // [nvox][Cmax] (the next layer's, ping-pong)
    float* outm = nullptr;                     // [cout][nvox] float32
    double* lsum = nullptr;
    int* derr = nullptr;                       // set by a tensor-core convolution whose wait ran out
    int conv_mode = 0;                         // 0: tensor-core convolutions where possible; 1: im2col
    bool tma = true;                           // interior planes by bulk tensor copy
    bool tma_used = false;                     // a plane map was accepted by the driver
    bool work_train = false;                   // work areas sized for training
    bool work_im2col = false;                  // work areas hold the im2col buffers
    std::vector<void*> work;
};

namespace {

int dalloc(djb_nn* h, void** p, size_t bytes, bool work) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DJB_ERR_ALLOC, "cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    if (work) h->work.push_back(*p);
    return DJB_OK;
}

#define TRYN(expr)                  \
    do {                            \
        int rc_ = (expr);           \
        if (rc_ != DJB_OK) return rc_; \
    } while (0)

void free_work(djb_nn* h) {
    for (void* q : h->work) cudaFree(q);
    h->work.clear();
    for (auto& a : h->act) a = nullptr;
    h->act0p = nullptr;
    h->actw = nullptr;
    h->col = nullptr;
    h->Y = nullptr;
    h->work_train = false;
    h->work_im2col = false;
    h->dcol = nullptr;
    h->dA = nullptr;
    h->dY = nullptr;
    h->dY2 = nullptr;
    h->outm = nullptr;
    h->res = 0;
}

int cmax(const djb_nn* h) {
    int c = 8;
    for (int l = 0; l < h->layers; ++l) c = std::max({c, h->cinp[l], h->coutp[l]});
    return c;
}

// Layer l runs on the tensor-core implicit GEMM (padded channel counts up to 32).
bool use_tc(const djb_nn* h, int l) { return h->conv_mode == 0 && h->cinp[l] <= 32 && h->coutp[l] <= 32; }

bool any_im2col(const djb_nn* h) {
    for (int l = 0; l < h->layers; ++l)
        if (!use_tc(h, l)) return true;
    return false;
}

// Tensor map of a bf16 [res]^3 × (8·cc) channels-last activation as the 5-D tensor
// [z][chunk][y][x][8] with boxes of bx × by positions of one plane, all chunks (a
// staged plane with its halo: 10 × 18; a dY tile: 8 × 16). false when the driver does
// not accept it (the kernels then copy with cp.async).
bool act_map(CUtensorMap* m, const __nv_bfloat16* X, int res, int cc, int bx, int by) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess && fn)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        cudaGetLastError();
    }
    if (!encode) return false;
    using namespace djb::conv;
    const cuuint64_t r = cuuint64_t(res), row = cuuint64_t(cc) * 16;
    const cuuint64_t dims[5] = {8, r, r, cuuint64_t(cc), r};
    const cuuint64_t strides[4] = {row, r * row, 16, r * r * row};
    const cuuint32_t box[5] = {8, cuuint32_t(bx), cuuint32_t(by), cuuint32_t(cc), 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(X), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of a bf16 [res]^3 × cout output as [z][y][x][cout] with boxes of one output
// tile (8 × 16 voxels of one plane, all channels), for the bulk tensor stores.
bool out_map(CUtensorMap* m, __nv_bfloat16* Y, int res, int cout) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess && fn)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        cudaGetLastError();
    }
    if (!encode || !Y) return false;
    using namespace djb::conv;
    const cuuint64_t r = cuuint64_t(res), row = cuuint64_t(cout) * 2;
    const cuuint64_t dims[4] = {cuuint64_t(cout), r, r, r};
    const cuuint64_t strides[3] = {row, r * row, r * r * row};
    const cuuint32_t box[4] = {cuuint32_t(cout), cuuint32_t(kTX), cuuint32_t(kTY), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, Y, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int CC, int N, int MODE, bool PAIR = false>
int launch_tc_inst(djb_nn* h, const djb::conv::Args& a0, cudaStream_t st) {
    using namespace djb::conv;
    constexpr int KC = PAIR ? 1 : (CC + 1) / 2 * 2;
    constexpr int bytes = smem_bytes<KC, N, PAIR>();
    auto kern = k_conv3_tc<CC, N, MODE, PAIR>;
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    int occ = 0, sms = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, bytes));
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    if (occ < 1) return fail(DJB_ERR_CUDA, "tensor-core convolution does not fit on an SM (%d bytes)", bytes);
    Args a = a0;
    a.ntx = (a.res + kTX - 1) / kTX;
    a.nty = (a.res + kTY - 1) / kTY;
    // z segments of at most kMaxSegment tiles (one tensor-memory accumulator each); the
    // two planes beyond a segment's ends feed only its first and last tile
    const int64_t slots = int64_t(occ) * sms;
    a.zlen = std::min(a.res, kMaxSegment);
    a.nzs = (a.res + a.zlen - 1) / a.zlen;
    CUtensorMap map{}, omap{};
    a.use_tma = h->tma && a.res >= kBY && act_map(&map, a.X, a.res, CC, kBX, kBY) ? 1 : 0;
    h->tma_used = h->tma_used || a.use_tma;
    a.use_ostore = (MODE != kLast && h->tma && a.cout == N && a.res >= kTY && out_map(&omap, a.Y, a.res, a.cout)) ? 1 : 0;
    const int64_t items = int64_t(a.ntx) * a.nty * a.nzs;
    const int grid = int(std::min<int64_t>(items, slots));
    kern<<<grid, kThreads, bytes, st>>>(a, map, omap);
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

template <int N, int MODE>
int launch_tc_cc(djb_nn* h, int cc, const djb::conv::Args& a, cudaStream_t st) {
    switch (cc) {
        case 1: return launch_tc_inst<1, N, MODE>(h, a, st);
        case 2: return launch_tc_inst<2, N, MODE>(h, a, st);
        case 3: return launch_tc_inst<3, N, MODE>(h, a, st);
        case 4: return launch_tc_inst<4, N, MODE>(h, a, st);
        default: return fail(DJB_ERR_INVALID, "tensor-core convolution: %d input channels", cc * 8);
    }
}

template <int MODE>
int launch_tc(djb_nn* h, const djb::conv::Args& a) {
    const int cc = a.cin / 8;
    return a.cout <= 16 ? launch_tc_cc<16, MODE>(h, cc, a, h->stream) : launch_tc_cc<32, MODE>(h, cc, a, h->stream);
}

// The first layer reads the x-pair rows (at most 4 input channels, not the last layer).
bool use_pair(const djb_nn* h) { return use_tc(h, 0) && h->cin[0] <= 4 && h->cinp[0] == 8 && h->layers > 1; }

// Layer l on the tensor cores: act[l] → act[l + 1] (hidden) or outm (last).
int conv_tc(djb_nn* h, int l) {
    using namespace djb::conv;
    const bool last = (l == h->layers - 1);
    Args a{};
    a.X = h->act[l];
    a.W = h->pb + h->woff[l];
    a.bias = h->p + h->boff[l];
    a.Y = last ? nullptr : h->act[l + 1];
    a.Yf = last ? h->outm : nullptr;
    a.res = h->res;
    a.cin = h->cinp[l];
    a.cout = h->coutp[l];
    a.nout = h->cout[l];
    a.err = h->derr;
    if (l == 0 && use_pair(h)) {
        a.X = h->act0p;
        return h->coutp[0] <= 16 ? launch_tc_inst<1, 16, kHidden, true>(h, a, h->stream)
                                 : launch_tc_inst<1, 32, kHidden, true>(h, a, h->stream);
    }
    return last ? launch_tc<kLast>(h, a) : launch_tc<kHidden>(h, a);
}

// Data gradient of layer l > 0 on the tensor cores: dY (bf16 [v][coutp]) → the next
// dY down, (act[l] > 0) · Σ_tap Σ_o dY[v − offset(tap)][o] W[tap][c][o] (bf16 [v][cinp]).
int conv_tc_back(djb_nn* h, int l, const __nv_bfloat16* dy, __nv_bfloat16* dy_next) {
    using namespace djb::conv;
    Args a{};
    a.X = dy;
    a.W = h->pb + h->woff[l];
    a.M = h->act[l];
    a.Y = dy_next;
    a.res = h->res;
    a.cin = h->coutp[l];
    a.cout = h->cinp[l];
    a.nout = h->cinp[l];
    a.flip = 1;
    a.err = h->derr;
    return launch_tc<kBackData>(h, a);
}

template <int CCO, int N>
int launch_wg_inst(djb_nn* h, const djb::conv::WArgs& a0) {
    using namespace djb::conv;
    constexpr int bytes = wg_smem_bytes<N>();
    auto kern = k_conv3_wgrad<CCO, N>;
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    WArgs a = a0;
    a.ntx = (a.res + kTX - 1) / kTX;
    a.nty = (a.res + kTY - 1) / kTY;
    a.zlen = a.res;
    while (a.zlen > 4 && int64_t(a.ntx) * a.nty * ((a.res + a.zlen - 1) / a.zlen) < 4 * int64_t(sms))
        a.zlen = (a.zlen + 1) / 2;
    a.nzs = (a.res + a.zlen - 1) / a.zlen;
    CUtensorMap xmap{}, ymap{};
    a.use_tma = h->tma && a.res >= kBY && act_map(&xmap, a.X, a.res, 4, kBX, kBY) &&
                        act_map(&ymap, a.dY, a.res, CCO, kTX, kTY)
                    ? 1
                    : 0;
    h->tma_used = h->tma_used || a.use_tma;
    const int64_t items = int64_t(a.ntx) * a.nty * a.nzs;
    const int grid = int(std::min<int64_t>(items, sms));
    kern<<<grid, kThreads, bytes, h->stream>>>(a, xmap, ymap);
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

// Layer l's weight gradient on the tensor cores, accumulated into the zeroed gradient
// buffer. The kernel reads 32 input channels: narrower inputs are first widened with
// zeros into h->actw, and only the layer's own rows of dW are written.
bool use_tc_wgrad(const djb_nn* h, int l) { return use_tc(h, l); }

// [v][c] (c < cp, a multiple of 8) → [v][32], zeros beyond cp.
__global__ void k_widen32(const __nv_bfloat16* __restrict__ in, int cp, int64_t nvox, __nv_bfloat16* __restrict__ out) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < nvox * 4; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t v = t / 4;
        const int c8 = int(t - v * 4);
        reinterpret_cast<uint4*>(out)[t] =
            c8 * 8 < cp ? reinterpret_cast<const uint4*>(in + v * cp)[c8] : make_uint4(0u, 0u, 0u, 0u);
    }
}

int conv_tc_wgrad(djb_nn* h, int l, const __nv_bfloat16* dy) {
    djb::conv::WArgs a{};
    a.X = h->act[l];
    const int64_t nvox = int64_t(h->res) * h->res * h->res;
    if (h->cinp[l] < 32) {
        k_widen32<<<grid_of(nvox * 4), kNT, 0, h->stream>>>(h->act[l], h->cinp[l], nvox, h->actw);
        a.X = h->actw;
    }
    a.cin_w = h->cinp[l];
    a.dY = dy;
    a.dW = h->g + h->woff[l];
    a.res = h->res;
    a.cout = h->coutp[l];
    a.err = h->derr;
    const int cco = h->coutp[l] / 8;
    if (h->coutp[l] <= 16) {
        switch (cco) {
            case 1: return launch_wg_inst<1, 16>(h, a);
            case 2: return launch_wg_inst<2, 16>(h, a);
        }
    } else {
        switch (cco) {
            case 3: return launch_wg_inst<3, 32>(h, a);
            case 4: return launch_wg_inst<4, 32>(h, a);
        }
    }
    return fail(DJB_ERR_INVALID, "tensor-core weight gradient: %d output channels", h->coutp[l]);
}

// Reads the device error word of the tensor-core convolutions (after a stream sync).
int check_derr(djb_nn* h) {
    int e = 0;
    CUDA_TRY(cudaMemcpyAsync(&e, h->derr, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (e) {
        cudaMemsetAsync(h->derr, 0, sizeof(int), h->stream);
        return fail(DJB_ERR_CUDA, "tensor-core convolution: a wait for the tensor cores ran out");
    }
    return DJB_OK;
}

// Work areas for res³ voxels; training needs the whole mesh at once (chunk = nvox).
// The im2col buffers exist only for layers that do not fit the tensor-core kernels (or
// every layer after djb_nn_set_conv(h, 1)): col, Y, and dcol when training.
int ensure_work(djb_nn* h, int res, bool train) {
    const int64_t nvox = int64_t(res) * res * res;
    const bool im2col = any_im2col(h);
    if (h->res == res && (h->work_train || !train) && (h->work_im2col || !im2col) && (h->act0p || !use_pair(h)))
        return DJB_OK;
    free_work(h);
    const int C = cmax(h);
    // chunks of whole z planes holding at most 4 Mi voxels (col: 27·C bf16 per voxel,
    // 7 GB for C = 32)
    int64_t planes = std::max<int64_t>(1, (int64_t(1) << 22) / (int64_t(res) * res));
    planes = std::min<int64_t>(planes, res);
    h->chunk = train ? nvox : planes * res * res;
    for (int l = 0; l < h->layers; ++l)
        TRYN(dalloc(h, (void**)&h->act[l], size_t(nvox) * h->cinp[l] * sizeof(__nv_bfloat16), true));
    if (use_pair(h)) TRYN(dalloc(h, (void**)&h->act0p, size_t(nvox) * 8 * sizeof(__nv_bfloat16), true));
    if (im2col) TRYN(dalloc(h, (void**)&h->col, size_t(h->chunk) * 27 * C * sizeof(__nv_bfloat16), true));
    if (im2col) TRYN(dalloc(h, (void**)&h->Y, size_t(h->chunk) * C * sizeof(float), true));
    TRYN(dalloc(h, (void**)&h->outm, size_t(nvox) * h->cout[h->layers - 1] * sizeof(float), true));
    TRYN(dalloc(h, (void**)&h->lsum, sizeof(double), true));
    if (train) {
        if (im2col) TRYN(dalloc(h, (void**)&h->dcol, size_t(nvox) * 27 * C * sizeof(float), true));
        TRYN(dalloc(h, (void**)&h->dA, size_t(nvox) * C * sizeof(float), true));
        TRYN(dalloc(h, (void**)&h->dY, size_t(nvox) * C * sizeof(__nv_bfloat16), true));
        TRYN(dalloc(h, (void**)&h->dY2, size_t(nvox) * C * sizeof(__nv_bfloat16), true));
        TRYN(dalloc(h, (void**)&h->actw, size_t(nvox) * 32 * sizeof(__nv_bfloat16), true));
    }
    h->work_train = train;
    h->work_im2col = im2col;
    h->res = res;
    return DJB_OK;
}

// Forward over all voxels: input (float32 mesh, device) → h->outm (float32 mesh).
int forward(djb_nn* h, const float* in) {
    const int res = h->res;
    const int64_t nvox = int64_t(res) * res * res;
    const float one = 1.0f, zero = 0.0f;
    k_pack<<<grid_of(nvox), kNT, 0, h->stream>>>(in, h->cin[0], h->cinp[0], res, nvox, h->act[0],
                                                 use_pair(h) ? h->act0p : nullptr);
    for (int l = 0; l < h->layers; ++l) {
            if (use_tc(h, l)) {
            TRYN(conv_tc(h, l));
            continue;
        }
        const int C = h->cinp[l], K = 27 * C;
        const bool last = (l == h->layers - 1);
        const int N = last ? h->cout[l] : h->coutp[l];
        for (int64_t v0 = 0; v0 < nvox; v0 += h->chunk) {
            const int64_t m = std::min(h->chunk, nvox - v0);
            k_im2col<<<grid_of(m * 27 * (C / 8)), kNT, 0, h->stream>>>(h->act[l], res, C, v0, m, h->col);
            // Yᶜ (N×m) = Wᶜ (N×K) · colᶜ (K×m); W row-major [K][coutp]
            CUBLAS_TRY(cublasGemmEx(h->blas, CUBLAS_OP_N, CUBLAS_OP_N, N, int(m), K, &one, h->pb + h->woff[l],
                                    CUDA_R_16BF, h->coutp[l], h->col, CUDA_R_16BF, K, &zero, h->Y, CUDA_R_32F, N,
                                    CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT));
            if (last)
                k_bias_out<<<grid_of(m * N), kNT, 0, h->stream>>>(h->Y, N, h->p + h->boff[l], nvox, v0, m, h->outm);
            else
                k_bias_act<<<grid_of(m * h->cinp[l + 1]), kNT, 0, h->stream>>>(
                    h->Y, N, h->p + h->boff[l], h->cinp[l + 1], 1, m, h->act[l + 1] + v0 * h->cinp[l + 1]);
        }
    }
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

// Backward from the MSE loss against `target` (float32 mesh, device), or from a given
// gradient `dout` of the output mesh (target null), into h->g; *loss (MSE only).
int backward(djb_nn* h, const float* target, double* loss, const float* dout = nullptr) {
    const int res = h->res;
    const int64_t nvox = int64_t(res) * res * res;
    const float one = 1.0f, zero = 0.0f;
    const int L = h->layers;
    const int nout = h->cout[L - 1];
    CUDA_TRY(cudaMemsetAsync(h->g, 0, size_t(h->nparam) * sizeof(float), h->stream));
    CUDA_TRY(cudaMemsetAsync(h->lsum, 0, sizeof(double), h->stream));
    if (target)
        k_mse<<<grid_of(nvox * nout), kNT, 0, h->stream>>>(h->outm, target, nout, nvox, 1.0 / double(nvox * nout),
                                                          h->dA, h->lsum);
    else
        k_out_grad<<<grid_of(nvox * nout), kNT, 0, h->stream>>>(dout, nout, nvox, h->dA);
    // dY of the last layer (bf16, [v][coutp], no activation)
    __nv_bfloat16* dy = h->dY;
    __nv_bfloat16* dy_next = h->dY2;
    k_grad_bf16<<<grid_of(nvox * h->coutp[L - 1]), kNT, 0, h->stream>>>(h->dA, nout, h->coutp[L - 1], nullptr, nvox,
                                                                       dy);
    for (int l = L - 1; l >= 0; --l) {
        const int C = h->cinp[l], K = 27 * C;
        const int N = h->coutp[l];
        const int n = (l == L - 1) ? nout : h->cout[l];
        k_bias_grad<<<int(std::min<int64_t>((nvox + 255) / 256, 148 * 4)), kNT, 0, h->stream>>>(dy, n, N, nvox,
                                                                                              h->g + h->boff[l]);
        if (use_tc_wgrad(h, l)) {
            TRYN(conv_tc_wgrad(h, l, dy));
        } else {
            k_im2col<<<grid_of(nvox * 27 * (C / 8)), kNT, 0, h->stream>>>(h->act[l], res, C, 0, nvox, h->col);
            // dWᶜ (N×K) = dYᶜ (N×M) · colᶜᵀ (M×K)
            CUBLAS_TRY(cublasGemmEx(h->blas, CUBLAS_OP_N, CUBLAS_OP_T, N, K, int(nvox), &one, dy, CUDA_R_16BF, N,
                                    h->col, CUDA_R_16BF, K, &zero, h->g + h->woff[l], CUDA_R_32F, N,
                                    CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT));
        }
        if (l == 0) break;
        // dY of layer l − 1: the data gradient of this layer, masked by ReLU'(act[l])
        if (use_tc(h, l)) {
            TRYN(conv_tc_back(h, l, dy, dy_next));
        } else {
            // dcolᶜ (K×M) = Wᶜᵀ (K×N) · dYᶜ (N×M)
            CUBLAS_TRY(cublasGemmEx(h->blas, CUBLAS_OP_T, CUBLAS_OP_N, K, int(nvox), N, &one, h->pb + h->woff[l],
                                    CUDA_R_16BF, N, dy, CUDA_R_16BF, N, &zero, h->dcol, CUDA_R_32F, K,
                                    CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT));
            k_col2im<<<grid_of(nvox * C), kNT, 0, h->stream>>>(h->dcol, res, C, nvox, h->dA);
            k_grad_bf16<<<grid_of(nvox * C), kNT, 0, h->stream>>>(h->dA, C, C, h->act[l], nvox, dy_next);
        }
        std::swap(dy, dy_next);
    }
    if (loss && target) {
        double s = 0.0;
        CUDA_TRY(cudaMemcpyAsync(&s, h->lsum, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        *loss = s / double(nvox * nout);
    }
    CUDA_TRY(cudaGetLastError());
    return DJB_OK;
}

// Stages a float32 mesh of `count` floats to the device (host memory) or uses it in place.
int stage(djb_nn* h, const float* src, size_t count, int mem, float** out, bool* owned) {
    *owned = false;
    if (mem == DJB_MEM_DEVICE) {
        *out = const_cast<float*>(src);
        return DJB_OK;
    }
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(out), count * sizeof(float), h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DJB_ERR_ALLOC, "staging allocation failed: %s", cudaGetErrorString(e));
    }
    *owned = true;
    CUDA_TRY(cudaMemcpyAsync(*out, src, count * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    return DJB_OK;
}

}  // namespace

extern "C" {

int djb_nn_create(int32_t layers, int32_t cin, int32_t hidden, int32_t cout, uint64_t seed, int32_t device,
                  djb_nn** out) {
    djb::clear_error();
    if (!out) return fail(DJB_ERR_INVALID, "null argument");
    if (layers < 2 || layers > kMaxLayers || cin < 1 || hidden < 1 || cout < 1 || hidden > 256 || cin > 256 ||
        cout > 256)
        return fail(DJB_ERR_INVALID, "layers must be in 2..%d and channel counts in 1..256", kMaxLayers);
    CUDA_TRY(cudaSetDevice(device));
    djb_nn* h = new (std::nothrow) djb_nn();
    if (!h) return fail(DJB_ERR_ALLOC, "host allocation failed");
    *out = h;
    h->layers = layers;
    h->device = device;
    int64_t off = 0;
    for (int l = 0; l < layers; ++l) {
        h->cin[l] = (l == 0) ? cin : hidden;
        h->cout[l] = (l == layers - 1) ? cout : hidden;
        h->cinp[l] = pad8(h->cin[l]);
        h->coutp[l] = pad8(h->cout[l]);
        h->woff[l] = off;
        off += int64_t(27) * h->cinp[l] * h->coutp[l];
        h->boff[l] = off;
        off += h->coutp[l];
    }
    h->nparam = off;
    // Kaiming-uniform weights (bound sqrt(6 / fan_in)), zero biases; padding frozen at 0
    std::vector<float> p(size_t(off), 0.0f);
    std::vector<uint8_t> fr(size_t(off), 1);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < layers; ++l) {
        const double bound = std::sqrt(6.0 / (27.0 * h->cin[l]));
        std::uniform_real_distribution<double> U(-bound, bound);
        for (int tap = 0; tap < 27; ++tap)
            for (int c = 0; c < h->cin[l]; ++c)
                for (int o = 0; o < h->cout[l]; ++o) {
                    const int64_t i = h->woff[l] + (int64_t(tap) * h->cinp[l] + c) * h->coutp[l] + o;
                    p[size_t(i)] = float(U(rng));
                    fr[size_t(i)] = 0;
                }
        for (int o = 0; o < h->cout[l]; ++o) fr[size_t(h->boff[l] + o)] = 0;
    }
    CUDA_TRY(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
    h->stream = h->own;
    CUBLAS_TRY(cublasCreate(&h->blas));
    CUBLAS_TRY(cublasSetStream(h->blas, h->stream));
    CUBLAS_TRY(cublasSetMathMode(h->blas, CUBLAS_DEFAULT_MATH));
    TRYN(dalloc(h, (void**)&h->p, size_t(off) * sizeof(float), false));
    TRYN(dalloc(h, (void**)&h->pb, size_t(off) * sizeof(__nv_bfloat16), false));
    TRYN(dalloc(h, (void**)&h->m1, size_t(off) * sizeof(float), false));
    TRYN(dalloc(h, (void**)&h->m2, size_t(off) * sizeof(float), false));
    TRYN(dalloc(h, (void**)&h->g, size_t(off) * sizeof(float), false));
    TRYN(dalloc(h, (void**)&h->frozen, size_t(off), false));
    TRYN(dalloc(h, (void**)&h->derr, sizeof(int), false));
    CUDA_TRY(cudaMemset(h->derr, 0, sizeof(int)));
    CUDA_TRY(cudaMemcpy(h->p, p.data(), size_t(off) * sizeof(float), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(h->frozen, fr.data(), size_t(off), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(h->m1, 0, size_t(off) * sizeof(float)));
    CUDA_TRY(cudaMemset(h->m2, 0, size_t(off) * sizeof(float)));
    k_to_bf16<<<grid_of(off), kNT>>>(h->p, off, h->pb);
    CUDA_TRY(cudaDeviceSynchronize());
    return DJB_OK;
}

int djb_nn_destroy(djb_nn* h) {
    if (!h) return DJB_OK;
    cudaSetDevice(h->device);
    free_work(h);
    for (void* q : {(void*)h->p, (void*)h->pb, (void*)h->m1, (void*)h->m2, (void*)h->g, (void*)h->frozen,
                    (void*)h->derr})
        if (q) cudaFree(q);
    if (h->blas) cublasDestroy(h->blas);
    if (h->own) cudaStreamDestroy(h->own);
    delete h;
    return DJB_OK;
}

int djb_nn_param_count(const djb_nn* h, int64_t* count) {
    djb::clear_error();
    if (!h || !count) return fail(DJB_ERR_INVALID, "null argument");
    *count = h->nparam;
    return DJB_OK;
}

int djb_nn_get_params(djb_nn* h, float* params) {
    djb::clear_error();
    if (!h || !params) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMemcpyAsync(params, h->p, size_t(h->nparam) * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DJB_OK;
}

int djb_nn_load(djb_nn* h, const float* params) {
    djb::clear_error();
    if (!h || !params) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMemcpyAsync(h->p, params, size_t(h->nparam) * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemsetAsync(h->m1, 0, size_t(h->nparam) * sizeof(float), h->stream));
    CUDA_TRY(cudaMemsetAsync(h->m2, 0, size_t(h->nparam) * sizeof(float), h->stream));
    k_to_bf16<<<grid_of(h->nparam), kNT, 0, h->stream>>>(h->p, h->nparam, h->pb);
    h->step = 0;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DJB_OK;
}

int djb_nn_set_stream(djb_nn* h, void* stream) {
    djb::clear_error();
    if (!h) return fail(DJB_ERR_INVALID, "null argument");
    h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own;
    CUBLAS_TRY(cublasSetStream(h->blas, h->stream));
    return DJB_OK;
}

int djb_nn_set_conv(djb_nn* h, int32_t mode) {
    djb::clear_error();
    if (!h) return fail(DJB_ERR_INVALID, "null argument");
    if (mode != 0 && mode != 1) return fail(DJB_ERR_INVALID, "conv mode must be 0 (tensor-core) or 1 (im2col)");
    h->conv_mode = mode;
    return DJB_OK;
}

int djb_nn_get_conv(const djb_nn* h, int32_t* mode, int32_t* tma_used) {
    djb::clear_error();
    if (!h || !mode || !tma_used) return fail(DJB_ERR_INVALID, "null argument");
    *mode = h->conv_mode;
    *tma_used = h->tma_used ? 1 : 0;
    return DJB_OK;
}

int djb_nn_apply(djb_nn* h, const float* in, int32_t res, float* out, int32_t mem) {
    djb::clear_error();
    if (!h || !in || !out) return fail(DJB_ERR_INVALID, "null argument");
    if (res < 3) return fail(DJB_ERR_INVALID, "res must be >= 3");
    CUDA_TRY(cudaSetDevice(h->device));
    TRYN(ensure_work(h, res, false));
    const int64_t nvox = int64_t(res) * res * res;
    float* din = nullptr;
    bool own_in = false;
    TRYN(stage(h, in, size_t(nvox) * h->cin[0], mem, &din, &own_in));
    int rc = forward(h, din);
    const size_t nout = size_t(nvox) * h->cout[h->layers - 1];
    if (rc == DJB_OK && cudaMemcpyAsync(out, h->outm, nout * sizeof(float),
                                        mem == DJB_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                        h->stream) != cudaSuccess)
        rc = fail(DJB_ERR_CUDA, "output copy failed");
    if (own_in) cudaFreeAsync(din, h->stream);
    if (rc != DJB_OK) return rc;
    return check_derr(h);
}

// Gradients of the mean squared error of net(in) against target, into the network's
// gradient buffer (read with djb_nn_grads, replaced with djb_nn_set_grads).
int djb_nn_backward(djb_nn* h, const float* in, const float* target, int32_t res, double* loss, int32_t mem) {
    djb::clear_error();
    if (!h || !in || !target) return fail(DJB_ERR_INVALID, "null argument");
    if (res < 3) return fail(DJB_ERR_INVALID, "res must be >= 3");
    CUDA_TRY(cudaSetDevice(h->device));
    TRYN(ensure_work(h, res, true));
    const int64_t nvox = int64_t(res) * res * res;
    float *din = nullptr, *dt = nullptr;
    bool own_in = false, own_t = false;
    TRYN(stage(h, in, size_t(nvox) * h->cin[0], mem, &din, &own_in));
    int rc = stage(h, target, size_t(nvox) * h->cout[h->layers - 1], mem, &dt, &own_t);
    if (rc == DJB_OK) rc = forward(h, din);
    if (rc == DJB_OK) rc = backward(h, dt, loss);
    if (own_in) cudaFreeAsync(din, h->stream);
    if (own_t) cudaFreeAsync(dt, h->stream);
    if (rc != DJB_OK) return rc;
    return check_derr(h);
}

// Gradients of Σ dout · net(in) (dout: the loss gradient with respect to the output mesh)
// into the network's gradient buffer.
int djb_nn_backward_output_grad(djb_nn* h, const float* in, const float* dout, int32_t res, int32_t mem) {
    djb::clear_error();
    if (!h || !in || !dout) return fail(DJB_ERR_INVALID, "null argument");
    if (res < 3) return fail(DJB_ERR_INVALID, "res must be >= 3");
    CUDA_TRY(cudaSetDevice(h->device));
    TRYN(ensure_work(h, res, true));
    const int64_t nvox = int64_t(res) * res * res;
    float *din = nullptr, *dd = nullptr;
    bool own_in = false, own_d = false;
    TRYN(stage(h, in, size_t(nvox) * h->cin[0], mem, &din, &own_in));
    int rc = stage(h, dout, size_t(nvox) * h->cout[h->layers - 1], mem, &dd, &own_d);
    if (rc == DJB_OK) rc = forward(h, din);
    if (rc == DJB_OK) rc = backward(h, nullptr, nullptr, dd);
    if (own_in) cudaFreeAsync(din, h->stream);
    if (own_d) cudaFreeAsync(dd, h->stream);
    if (rc != DJB_OK) return rc;
    return check_derr(h);
}

int djb_nn_info(const djb_nn* h, int32_t* layers, int32_t* cin, int32_t* hidden, int32_t* cout, int32_t* device) {
    djb::clear_error();
    if (!h) return fail(DJB_ERR_INVALID, "null network");
    if (layers) *layers = h->layers;
    if (cin) *cin = h->cin[0];
    if (hidden) *hidden = h->layers > 1 ? h->cout[0] : 0;
    if (cout) *cout = h->cout[h->layers - 1];
    if (device) *device = h->device;
    return DJB_OK;
}

int djb_nn_grads(djb_nn* h, float* grads, int32_t mem) {
    djb::clear_error();
    if (!h || !grads) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMemcpyAsync(grads, h->g, size_t(h->nparam) * sizeof(float),
                             mem == DJB_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DJB_OK;
}

int djb_nn_set_grads(djb_nn* h, const float* grads, int32_t mem) {
    djb::clear_error();
    if (!h || !grads) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaMemcpyAsync(h->g, grads, size_t(h->nparam) * sizeof(float),
                             mem == DJB_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DJB_OK;
}

// One Adam step (beta 0.9/0.999, eps 1e-8) with the gradients in the gradient buffer.
int djb_nn_adam_step(djb_nn* h, double lr) {
    djb::clear_error();
    if (!h) return fail(DJB_ERR_INVALID, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    ++h->step;
    const float c1 = float(1.0 - std::pow(0.9, double(h->step)));
    const float c2 = float(1.0 - std::pow(0.999, double(h->step)));
    k_adam<<<grid_of(h->nparam), kNT, 0, h->stream>>>(h->p, h->g, h->m1, h->m2, h->nparam, float(lr), 0.9f, 0.999f,
                                                       1e-8f, c1, c2, h->frozen, h->pb);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return DJB_OK;
}

int djb_nn_train_step(djb_nn* h, const float* in, const float* target, int32_t res, double lr, double* loss,
                      int32_t mem) {
    TRYN(djb_nn_backward(h, in, target, res, loss, mem));
    return djb_nn_adam_step(h, lr);
}

}  // extern "C"
