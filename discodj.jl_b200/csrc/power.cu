// Isotropic power spectrum with float64 shell sums
// (native/DiscoDJNative/src/analysis/power_spectrum.jl:25-79).
//
// The field is transformed in float32 by cuFFT (R2C, x axis halved). Each mode's
// |δ(k)|²·V/res⁶, its weight (0.5 on the two self-conjugate planes of the halved
// axis, power_spectrum.jl:59-60) and |k| are formed in float64 and summed per
// shell: per-block shared-memory partials, then float64 atomics.
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "common.h"

using djb::fail;

struct djb_solver;
namespace djb {
int solver_deposit_cic(djb_solver* s, float** mesh_out, int* res, int* pitch, cudaStream_t* st);
int solver_res(const djb_solver* s);
int64_t solver_np(const djb_solver* s);
cufftHandle solver_r2c(const djb_solver* s);
cufftHandle solver_c2r(const djb_solver* s);
double solver_boxsize(const djb_solver* s);
int solver_cic_gather_grad(djb_solver* s, const float* mesh, int pitch, float* psibar);
int solver_check_err(djb_solver* s);
}  // namespace djb

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBins = 1024;

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

// Shell sums: sums[4*b + 0] = Σ w·P, [1] = Σ w, [2] = Σ |k|, counts[b] = modes.
__global__ void __launch_bounds__(kThreads) k_shells(const float2* __restrict__ f, int res, double dk,
                                                      double norm, const double* __restrict__ edges,
                                                      int bins, double* __restrict__ sums,
                                                      unsigned long long* __restrict__ counts) {
    extern __shared__ double sm[];
    double* s_wp = sm;
    double* s_w = sm + bins;
    double* s_k = sm + 2 * bins;
    unsigned long long* s_n = reinterpret_cast<unsigned long long*>(sm + 3 * bins);
    for (int b = threadIdx.x; b < bins; b += blockDim.x) {
        s_wp[b] = 0.0;
        s_w[b] = 0.0;
        s_k[b] = 0.0;
        s_n[b] = 0ull;
    }
    __syncthreads();
    const int nh = res / 2 + 1;
    const int64_t total = int64_t(res) * res * nh;
    const double kmin = edges[0], kmax = edges[bins];
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int kx = int(t % nh);
        const int iy = int((t / nh) % res);
        const int iz = int(t / (int64_t(nh) * res));
        // full axes: index <= res/2 positive (power_spectrum.jl:40)
        const double ky = double(iy <= res / 2 ? iy : iy - res) * dk;
        const double kz = double(iz <= res / 2 ? iz : iz - res) * dk;
        const double kh = double(kx) * dk;
        // same association as the reference's kx²+ky²+kz² with its halved axis last
        const double k = sqrt((kz * kz + ky * ky) + kh * kh);
        if (!(k >= kmin && k < kmax)) continue;
        int lo = 0, hi = bins;  // edges[lo] <= k < edges[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (edges[mid] <= k) lo = mid;
            else hi = mid;
        }
        const float2 v = f[t];
        const double p = (double(v.x) * v.x + double(v.y) * v.y) * norm;
        const double w = (kx == 0 || kx == nh - 1) ? 0.5 : 1.0;
        atomicAdd(&s_wp[lo], w * p);
        atomicAdd(&s_w[lo], w);
        atomicAdd(&s_k[lo], k);
        atomicAdd(&s_n[lo], 1ull);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < bins; b += blockDim.x) {
        if (s_n[b] == 0ull) continue;
        atomicAdd(&sums[4 * b + 0], s_wp[b]);
        atomicAdd(&sums[4 * b + 1], s_w[b]);
        atomicAdd(&sums[4 * b + 2], s_k[b]);
        atomicAdd(&counts[b], s_n[b]);
    }
}

// spec[k] *= coef[bin(k)] (0 outside every bin): the bins of k_shells.
__global__ void __launch_bounds__(kThreads) k_shell_scale(float2* __restrict__ f, int res, double dk,
                                                          const double* __restrict__ edges, int bins,
                                                          const double* __restrict__ coef) {
    const int nh = res / 2 + 1;
    const int64_t total = int64_t(res) * res * nh;
    const double kmin = edges[0], kmax = edges[bins];
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int kx = int(t % nh);
        const int iy = int((t / nh) % res);
        const int iz = int(t / (int64_t(nh) * res));
        const double ky = double(iy <= res / 2 ? iy : iy - res) * dk;
        const double kz = double(iz <= res / 2 ? iz : iz - res) * dk;
        const double kh = double(kx) * dk;
        const double k = sqrt((kz * kz + ky * ky) + kh * kh);
        double c = 0.0;
        if (k >= kmin && k < kmax) {
            int lo = 0, hi = bins;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (edges[mid] <= k) lo = mid;
                else hi = mid;
            }
            c = coef[lo];
        }
        const float cf = float(c);
        float2 v = f[t];
        v.x *= cf;
        v.y *= cf;
        f[t] = v;
    }
}

// Julia LinRange element j of n (power_spectrum.jl:50-52).
double linrange(double a, double b, int j, int n) {
    if (j == 0) return a;
    if (j == n - 1) return b;
    const double t = double(j) / double(n - 1);
    return (1.0 - t) * a + t * b;
}

std::vector<double> bin_edges(int res, double boxsize, int bins, bool logarithmic) {
    const double dk = 2 * M_PI / boxsize;
    const double kny = M_PI * res / boxsize;
    const double kmin = dk, kmax = kny * std::sqrt(3.0);
    std::vector<double> e(bins + 1);
    for (int j = 0; j <= bins; ++j)
        e[j] = logarithmic ? std::pow(10.0, linrange(std::log10(kmin), std::log10(kmax), j, bins + 1))
                           : linrange(kmin, kmax, j, bins + 1);
    return e;
}

// Bins the spectrum `spec` (already transformed) and writes k, P, N on the host.
int shells(const float2* spec, int res, double boxsize, double scale2, int bins, bool logarithmic,
           double* k_out, double* pk_out, int64_t* n_out, cudaStream_t st, double* wsum_out = nullptr) {
    std::vector<double> e = bin_edges(res, boxsize, bins, logarithmic);
    double* d_edges = nullptr;
    double* d_sums = nullptr;
    unsigned long long* d_counts = nullptr;
    int rc = DJB_OK;
    auto cleanup = [&]() {
        if (d_edges) cudaFreeAsync(d_edges, st);
        if (d_sums) cudaFreeAsync(d_sums, st);
        if (d_counts) cudaFreeAsync(d_counts, st);
    };
    if (cudaMallocAsync((void**)&d_edges, sizeof(double) * (bins + 1), st) != cudaSuccess ||
        cudaMallocAsync((void**)&d_sums, sizeof(double) * 4 * bins, st) != cudaSuccess ||
        cudaMallocAsync((void**)&d_counts, sizeof(unsigned long long) * bins, st) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        return fail(DJB_ERR_ALLOC, "power spectrum work area allocation failed");
    }
    std::vector<double> sums(4 * size_t(bins));
    std::vector<unsigned long long> counts(bins);
    do {
        if (cudaMemcpyAsync(d_edges, e.data(), sizeof(double) * (bins + 1), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemsetAsync(d_sums, 0, sizeof(double) * 4 * bins, st) != cudaSuccess ||
            cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * bins, st) != cudaSuccess) {
            rc = fail(DJB_ERR_CUDA, "power spectrum set-up copy failed");
            break;
        }
        const double V = boxsize * boxsize * boxsize;
        const double r3 = double(res) * res * res;
        const double norm = V / (r3 * r3) * scale2;
        const int64_t total = int64_t(res) * res * (res / 2 + 1);
        int grid = int(std::min<int64_t>((total + kThreads - 1) / kThreads, 148 * 8));
        const size_t smem = size_t(bins) * 4 * sizeof(double);
        k_shells<<<grid, kThreads, smem, st>>>(spec, res, 2 * M_PI / boxsize, norm, d_edges, bins, d_sums, d_counts);
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) {
            rc = fail(DJB_ERR_CUDA, "shell kernel launch failed: %s", cudaGetErrorString(le));
            break;
        }
        if (cudaMemcpyAsync(sums.data(), d_sums, sizeof(double) * 4 * bins, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(counts.data(), d_counts, sizeof(unsigned long long) * bins, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = fail(DJB_ERR_CUDA, "power spectrum read-back failed");
            break;
        }
    } while (false);
    cleanup();
    if (rc != DJB_OK) return rc;
    for (int b = 0; b < bins; ++b) {
        const unsigned long long n = counts[b];
        if (wsum_out) wsum_out[b] = sums[4 * b + 1];
        if (n == 0) {
            k_out[b] = std::sqrt(e[b] * e[b + 1]);
            pk_out[b] = 0.0;
            n_out[b] = 0;
        } else {
            k_out[b] = sums[4 * b + 2] / double(n);
            pk_out[b] = sums[4 * b + 0] / sums[4 * b + 1];
            n_out[b] = int64_t(n);
        }
    }
    return DJB_OK;
}

// ── non-allocating shell sums ─────────────────────────────────────────────────
// Work area of djb_power_spectrum_shells_noalloc: bin edges, the four per-bin sums
// and the per-bin mode counts, for at most kNoAllocBins bins. It lives in a
// file-scope device array that every GPU loading the library holds until exit;
// every call shares it, and it keeps the previous call's contents.
constexpr int kNoAllocBins = 512;
constexpr size_t kEdgesBytes = ((kNoAllocBins + 1) * sizeof(double) + 255) / 256 * 256;
constexpr size_t kSumsBytes = 4 * kNoAllocBins * sizeof(double);
constexpr size_t kCountsBytes = kNoAllocBins * sizeof(unsigned long long);
constexpr size_t kNoAllocBytes = kEdgesBytes + kSumsBytes + kCountsBytes;  // 24,832 bytes
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device. In host code the symbol's name is
// only a host-side stand-in, so the address comes from cudaGetSymbolAddress, taken
// once per device with that device current.
void* g_noalloc_addr[kMaxDevices] = {};
std::mutex g_noalloc_mu;

int noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return fail(DJB_ERR_INVALID, "device ordinal %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(DJB_ERR_CUDA, "cudaGetSymbolAddress of the shell-sum scratch failed: %s",
                        cudaGetErrorString(e));
        g_noalloc_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[device]);
    return DJB_OK;
}

// Density-contrast Fourier modes δ̂(m)/res³ / W_CIC(m) of a CIC mesh's half spectrum
// (in place, rows of nh = res/2 + 1 complex, [kz][ky][kx]); m = (mx, my, mz) in
// (−res/2, res/2], modes with mx < 0 read the conjugate of −m. `f` = res³/n³ scales the
// mesh to 1 + δ; the m = 0 mode is δ's mean, 0. W_CIC = Π_d sinc²(π m_d / res).
__global__ void k_density_modes(const float2* __restrict__ spec, int res, const int* __restrict__ modes, int nm,
                                double f, double2* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nm) return;
    int mx = modes[3 * i], my = modes[3 * i + 1], mz = modes[3 * i + 2];
    if (mx == 0 && my == 0 && mz == 0) {
        out[i] = make_double2(0.0, 0.0);
        return;
    }
    const bool conj = mx < 0;
    if (conj) {
        mx = -mx;
        my = -my;
        mz = -mz;
    }
    const int nh = res / 2 + 1;
    const int ky = (my % res + res) % res, kz = (mz % res + res) % res;
    const float2 v = spec[(int64_t(kz) * res + ky) * nh + mx];
    double w = 1.0;
    const int md[3] = {mx, my, mz};
    for (int d = 0; d < 3; ++d) {
        if (md[d] == 0) continue;
        const double x = M_PI * double(md[d]) / double(res);
        const double sc = sin(x) / x;
        w *= sc * sc;
    }
    const double r3 = double(res) * res * res;
    const double sc = f / (r3 * w);
    out[i] = make_double2(double(v.x) * sc, (conj ? -double(v.y) : double(v.y)) * sc);
}

int res_limit(const djb_solver* s) { return djb::solver_res(s) / 2; }

// Makes a device current for the guard's lifetime and gives the calling thread its
// previous current device back on every return path.
struct DeviceGuard {
    int prev = -1;
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" {

int djb_power_spectrum_shells_noalloc(const void* spectrum, int32_t res, double boxsize, int32_t bins,
                                      int32_t logarithmic, double scale2, double* k, double* pk,
                                      int64_t* nmodes, void* stream, int32_t device) {
    djb::clear_error();
    if (!spectrum || !k || !pk || !nmodes) return fail(DJB_ERR_INVALID, "null argument");
    if (res < 2 || (res & 1)) return fail(DJB_ERR_INVALID, "field must be cubic with an even side");
    if (bins < 1 || bins > kNoAllocBins)
        return fail(DJB_ERR_INVALID,
                    "bins = %d exceeds the %d bins of the non-allocating shell sums (use djb_power_spectrum)",
                    bins, kNoAllocBins);
    if (!(boxsize > 0)) return fail(DJB_ERR_INVALID, "boxsize must be positive");
    DeviceGuard guard;  // the caller's current device is restored on return
    CUDA_TRY(cudaGetDevice(&guard.prev));
    CUDA_TRY(cudaSetDevice(device));
    unsigned char* base = nullptr;
    int rc = noalloc_scratch(device, &base);
    if (rc != DJB_OK) return rc;
    double* d_edges = reinterpret_cast<double*>(base);
    double* d_sums = reinterpret_cast<double*>(base + kEdgesBytes);
    unsigned long long* d_counts = reinterpret_cast<unsigned long long*>(base + kEdgesBytes + kSumsBytes);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // host-side work lives on the stack: nothing is allocated
    double e[kNoAllocBins + 1];
    double sums[4 * kNoAllocBins];
    unsigned long long counts[kNoAllocBins];
    {
        const double dk = 2 * M_PI / boxsize;
        const double kny = M_PI * res / boxsize;
        const double kmin = dk, kmax = kny * std::sqrt(3.0);
        for (int j = 0; j <= bins; ++j)
            e[j] = logarithmic ? std::pow(10.0, linrange(std::log10(kmin), std::log10(kmax), j, bins + 1))
                               : linrange(kmin, kmax, j, bins + 1);
    }
    CUDA_TRY(cudaMemcpyAsync(d_edges, e, sizeof(double) * (bins + 1), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(d_sums, 0, kSumsBytes, st));     // the previous call's sums remain otherwise
    CUDA_TRY(cudaMemsetAsync(d_counts, 0, kCountsBytes, st));
    const double V = boxsize * boxsize * boxsize;
    const double r3 = double(res) * res * res;
    const double norm = V / (r3 * r3) * scale2;
    const int64_t total = int64_t(res) * res * (res / 2 + 1);
    const int grid = int(std::min<int64_t>((total + kThreads - 1) / kThreads, 148 * 8));
    k_shells<<<grid, kThreads, size_t(bins) * 4 * sizeof(double), st>>>(
        static_cast<const float2*>(spectrum), res, 2 * M_PI / boxsize, norm, d_edges, bins, d_sums, d_counts);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(sums, d_sums, sizeof(double) * 4 * bins, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(counts, d_counts, sizeof(unsigned long long) * bins, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (int b = 0; b < bins; ++b) {
        if (counts[b] == 0) {
            k[b] = std::sqrt(e[b] * e[b + 1]);
            pk[b] = 0.0;
            nmodes[b] = 0;
        } else {
            k[b] = sums[4 * b + 2] / double(counts[b]);
            pk[b] = sums[4 * b + 0] / sums[4 * b + 1];
            nmodes[b] = int64_t(counts[b]);
        }
    }
    return DJB_OK;
}

int djb_power_spectrum(const float* field, int32_t res, double boxsize, int32_t bins, int32_t logarithmic,
                       double* k, double* pk, int64_t* nmodes, int32_t mem, int32_t device) {
    djb::clear_error();
    if (!field || !k || !pk || !nmodes) return fail(DJB_ERR_INVALID, "null argument");
    if (res < 2 || (res & 1)) return fail(DJB_ERR_INVALID, "field must be cubic with an even side");
    if (bins < 1 || bins > kMaxBins) return fail(DJB_ERR_INVALID, "bins must be in 1..%d", kMaxBins);
    if (!(boxsize > 0)) return fail(DJB_ERR_INVALID, "boxsize must be positive");
    CUDA_TRY(cudaSetDevice(device));
    cudaStream_t st;
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const int pitch = res + 2;
    float* mesh = nullptr;
    cufftHandle plan = 0;
    bool have_plan = false;
    int rc = DJB_OK;
    do {
        if (cudaMallocAsync((void**)&mesh, sizeof(float) * size_t(res) * res * pitch, st) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(DJB_ERR_ALLOC, "power spectrum mesh allocation failed");
            break;
        }
        // column-major (res,res,res) [ix,iy,iz] rows of res floats into rows of res+2
        if (cudaMemcpy2DAsync(mesh, sizeof(float) * pitch, field, sizeof(float) * res, sizeof(float) * res,
                              size_t(res) * res,
                              mem == DJB_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                              st) != cudaSuccess) {
            rc = fail(DJB_ERR_CUDA, "field copy failed");
            break;
        }
        long long dims[3] = {res, res, res};
        long long rembed[3] = {res, res, pitch};
        long long cembed[3] = {res, res, res / 2 + 1};
        size_t work = 0;
        if (cufftCreate(&plan) != CUFFT_SUCCESS) {
            rc = fail(DJB_ERR_CUFFT, "cufftCreate failed");
            break;
        }
        have_plan = true;
        if (cufftMakePlanMany64(plan, 3, dims, rembed, 1, rembed[0] * rembed[1] * rembed[2], cembed, 1,
                                cembed[0] * cembed[1] * cembed[2], CUFFT_R2C, 1, &work) != CUFFT_SUCCESS ||
            cufftSetStream(plan, st) != CUFFT_SUCCESS ||
            cufftExecR2C(plan, mesh, reinterpret_cast<cufftComplex*>(mesh)) != CUFFT_SUCCESS) {
            rc = fail(DJB_ERR_CUFFT, "power spectrum transform failed");
            break;
        }
        rc = shells(reinterpret_cast<const float2*>(mesh), res, boxsize, 1.0, bins, logarithmic != 0, k, pk,
                    nmodes, st);
    } while (false);
    if (have_plan) cufftDestroy(plan);
    if (mesh) cudaFreeAsync(mesh, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return rc;
}

int djb_state_power_spectrum(djb_solver* s, int32_t bins, int32_t logarithmic, double* k, double* pk,
                             int64_t* nmodes) {
    djb::clear_error();
    if (!s || !k || !pk || !nmodes) return fail(DJB_ERR_INVALID, "null argument");
    if (bins < 1 || bins > kMaxBins) return fail(DJB_ERR_INVALID, "bins must be in 1..%d", kMaxBins);
    float* mesh = nullptr;
    int res = 0, pitch = 0;
    cudaStream_t st = nullptr;
    int rc = djb::solver_deposit_cic(s, &mesh, &res, &pitch, &st);
    if (rc != DJB_OK) return rc;
    CUFFT_TRY(cufftExecR2C(djb::solver_r2c(s), mesh, reinterpret_cast<cufftComplex*>(mesh)));
    // δ = mesh·res³/n³ − 1: for k ≠ 0 the spectrum scales by (res³/n³)²
    const double f = double(res) * res * res / double(djb::solver_np(s));
    return shells(reinterpret_cast<const float2*>(mesh), res, djb::solver_boxsize(s), f * f, bins,
                  logarithmic != 0, k, pk, nmodes, st);
}

int djb_state_density_modes(djb_solver* s, int32_t nmodes, const int32_t* modes, double* out) {
    djb::clear_error();
    if (!s || (nmodes > 0 && (!modes || !out))) return fail(DJB_ERR_INVALID, "null argument");
    if (nmodes < 0) return fail(DJB_ERR_INVALID, "nmodes must be >= 0");
    float* mesh = nullptr;
    int res = 0, pitch = 0;
    cudaStream_t st = nullptr;
    for (int32_t i = 0; i < 3 * nmodes; ++i)
        if (modes[i] <= -res_limit(s) || modes[i] > res_limit(s))
            return fail(DJB_ERR_INVALID, "mode component %d outside (-res/2, res/2]", int(modes[i]));
    int rc = djb::solver_deposit_cic(s, &mesh, &res, &pitch, &st);
    if (rc != DJB_OK) return rc;
    if (nmodes == 0) return djb::solver_check_err(s);
    CUFFT_TRY(cufftExecR2C(djb::solver_r2c(s), mesh, reinterpret_cast<cufftComplex*>(mesh)));
    int* d_modes = nullptr;
    double2* d_out = nullptr;
    auto cleanup = [&]() {
        if (d_modes) cudaFreeAsync(d_modes, st);
        if (d_out) cudaFreeAsync(d_out, st);
    };
    if (cudaMallocAsync(reinterpret_cast<void**>(&d_modes), sizeof(int) * 3 * size_t(nmodes), st) != cudaSuccess ||
        cudaMallocAsync(reinterpret_cast<void**>(&d_out), sizeof(double2) * size_t(nmodes), st) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        return fail(DJB_ERR_ALLOC, "mode buffers allocation failed");
    }
    const double f = double(res) * res * res / double(djb::solver_np(s));
    cudaError_t e = cudaMemcpyAsync(d_modes, modes, sizeof(int) * 3 * size_t(nmodes), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_density_modes<<<(nmodes + 127) / 128, 128, 0, st>>>(reinterpret_cast<const float2*>(mesh), res, d_modes,
                                                              nmodes, f, d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out, sizeof(double2) * size_t(nmodes), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cleanup();
    if (e != cudaSuccess) return fail(DJB_ERR_CUDA, "density modes failed: %s", cudaGetErrorString(e));
    return djb::solver_check_err(s);
}

// Ψ̄ of Σ_b P̄_b·P_b for the solver's particle state, P as djb_state_power_spectrum.
// P_b = (V/res⁶)·Σ_half w|δ̂|²/Σ_half w with δ = mesh·res³/n³ − 1, so
// ∂/∂mesh(n) = Σ_b P̄_b·(V/res⁶)/(Σ_half w)_b·(res³/n³)²·Σ_{k∈b, full} f_k e^{ik·n}
// with f the R2C of the CIC mesh: the spectrum is scaled per bin and brought back by the
// unnormalised C2R, and the CIC weight derivatives gather it to the particles.
int djb_state_power_spectrum_vjp(djb_solver* s, int32_t bins, int32_t logarithmic, const double* pk_bar,
                                 float* psi_bar, int32_t mem) {
    djb::clear_error();
    if (!s || !pk_bar || !psi_bar) return fail(DJB_ERR_INVALID, "null argument");
    if (bins < 1 || bins > kMaxBins) return fail(DJB_ERR_INVALID, "bins must be in 1..%d", kMaxBins);
    float* mesh = nullptr;
    int res = 0, pitch = 0;
    cudaStream_t st = nullptr;
    int rc = djb::solver_deposit_cic(s, &mesh, &res, &pitch, &st);
    if (rc != DJB_OK) return rc;
    CUFFT_TRY(cufftExecR2C(djb::solver_r2c(s), mesh, reinterpret_cast<cufftComplex*>(mesh)));
    const double boxsize = djb::solver_boxsize(s);
    const double f = double(res) * res * res / double(djb::solver_np(s));
    std::vector<double> kk(bins), pk(bins), wsum(bins), coef(bins);
    std::vector<int64_t> nm(bins);
    rc = shells(reinterpret_cast<const float2*>(mesh), res, boxsize, f * f, bins, logarithmic != 0, kk.data(),
                pk.data(), nm.data(), st, wsum.data());
    if (rc != DJB_OK) return rc;
    const double V = boxsize * boxsize * boxsize;
    const double r3 = double(res) * res * res;
    for (int b = 0; b < bins; ++b) coef[b] = (wsum[b] > 0.0) ? pk_bar[b] * (V / (r3 * r3)) / wsum[b] * f * f : 0.0;
    const size_t count = size_t(3 * djb::solver_np(s));
    std::vector<double> e = bin_edges(res, boxsize, bins, logarithmic != 0);
    double* d_edges = nullptr;
    double* d_coef = nullptr;
    float* d_bar = nullptr;
    auto cleanup = [&]() {
        if (d_edges) cudaFreeAsync(d_edges, st);
        if (d_coef) cudaFreeAsync(d_coef, st);
        if (d_bar && mem == DJB_MEM_HOST) cudaFreeAsync(d_bar, st);
    };
    if (cudaMallocAsync((void**)&d_edges, sizeof(double) * (bins + 1), st) != cudaSuccess ||
        cudaMallocAsync((void**)&d_coef, sizeof(double) * bins, st) != cudaSuccess ||
        (mem == DJB_MEM_HOST && cudaMallocAsync((void**)&d_bar, sizeof(float) * count, st) != cudaSuccess)) {
        cudaGetLastError();
        cleanup();
        return fail(DJB_ERR_ALLOC, "P(k) VJP work area allocation failed");
    }
    if (mem != DJB_MEM_HOST) d_bar = psi_bar;
    do {
        if (cudaMemcpyAsync(d_edges, e.data(), sizeof(double) * (bins + 1), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(d_coef, coef.data(), sizeof(double) * bins, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemsetAsync(d_bar, 0, sizeof(float) * count, st) != cudaSuccess) {
            rc = fail(DJB_ERR_CUDA, "P(k) VJP set-up copy failed");
            break;
        }
        const int64_t total = int64_t(res) * res * (res / 2 + 1);
        const int grid = int(std::min<int64_t>((total + kThreads - 1) / kThreads, 148 * 16));
        k_shell_scale<<<grid, kThreads, 0, st>>>(reinterpret_cast<float2*>(mesh), res, 2 * M_PI / boxsize, d_edges,
                                                 bins, d_coef);
        if (cufftExecC2R(djb::solver_c2r(s), reinterpret_cast<cufftComplex*>(mesh), mesh) != CUFFT_SUCCESS) {
            rc = fail(DJB_ERR_CUFFT, "C2R of the P(k) cotangent failed");
            break;
        }
        rc = djb::solver_cic_gather_grad(s, mesh, pitch, d_bar);
        if (rc != DJB_OK) break;
        if (mem == DJB_MEM_HOST &&
            cudaMemcpyAsync(psi_bar, d_bar, sizeof(float) * count, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
            rc = fail(DJB_ERR_CUDA, "P(k) VJP read-back failed");
            break;
        }
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = fail(DJB_ERR_CUDA, "P(k) VJP failed");
    } while (false);
    cleanup();
    if (rc != DJB_OK) return rc;
    return djb::solver_check_err(s);
}

}  // extern "C"
