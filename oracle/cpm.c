/*
 * cpm.c — CPU restatement of the PM particle kernels (OpenMP, float32 and float64).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the larger parity cases and the CPU
 * baseline timed by bench.py. Follows native/DiscoDJNative/src/nbody/pm.jl:
 *   cpm_scatter_*   `_pm_scatter!` (pm.jl:57-74): atomic W-order assignment
 *   cpm_fdgrad_*    `_k_fdgrad!`   (pm.jl:330-342): F_c = -D_c phi, orders 2/4/6
 *   cpm_gather3_*   `_k_gather3!`  (pm.jl:344-364): acc += sum w F (3 components)
 *   cpm_gather1_*   `_pm_gather!`  (pm.jl:76-95)
 * Layouts are the reference's column-major ones: meshes (res,res,res) with x
 * fastest, idx = ix + res*(iy + res*iz); particle positions as three component
 * blocks of np values.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static inline int wrapi(int i, int res) {
    i = (i >= res) ? i - res : i;
    return (i < 0) ? i + res : i;
}

#define DEFINE_CPM(T, SUF, FLOOR, RINT, FMOD, FABS)                                               \
    static inline T jmod_##SUF(T x, T y) {                                                        \
        T r = FMOD(x, y);                                                                         \
        if (r < 0) r += y;                                                                        \
        return r;                                                                                 \
    }                                                                                             \
    static inline T wk_##SUF(int W, T d) {                                                        \
        if (W == 2) return d > 1 ? (T)0 : (T)1 - d;                                               \
        if (W == 3) {                                                                             \
            if (d > (T)1.5) return 0;                                                             \
            if (d > (T)0.5) return (T)0.5 * (((T)1.5 - d) * ((T)1.5 - d));                        \
            return (T)0.75 - d * d;                                                               \
        }                                                                                         \
        if (d > 2) return 0;                                                                      \
        if (d > 1) return ((T)2 - d) * ((T)2 - d) * ((T)2 - d) / (T)6;                            \
        return ((T)4 - (T)6 * (d * d) + (T)3 * (d * d * d)) / (T)6;                               \
    }                                                                                             \
    static inline void weights_##SUF(int W, T g, int res, T* w, int* idx) {                       \
        const int b = (W % 2 == 0) ? (int)FLOOR(g) : (int)RINT(g);                                \
        const int lo = (W == 2) ? 0 : -1;                                                         \
        for (int o = 0; o < W; ++o) {                                                             \
            const int node = b + lo + o;                                                          \
            w[o] = wk_##SUF(W, FABS(g - (T)node));                                                \
            idx[o] = wrapi(node, res);                                                            \
        }                                                                                         \
    }                                                                                             \
    void cpm_scatter_##SUF(const T* X, int64_t np, int res, T L, int W, T* mesh) {                \
        const T resf = (T)res;                                                                    \
        _Pragma("omp parallel for schedule(static)")                                              \
        for (int64_t p = 0; p < np; ++p) {                                                        \
            T wx[4], wy[4], wz[4];                                                                \
            int ix[4], iy[4], iz[4];                                                              \
            weights_##SUF(W, jmod_##SUF(X[p], L) / L * resf, res, wx, ix);                        \
            weights_##SUF(W, jmod_##SUF(X[p + np], L) / L * resf, res, wy, iy);                   \
            weights_##SUF(W, jmod_##SUF(X[p + 2 * np], L) / L * resf, res, wz, iz);               \
            for (int c = 0; c < W; ++c)                                                           \
                for (int b = 0; b < W; ++b) {                                                     \
                    T* row = mesh + ((int64_t)iz[c] * res + iy[b]) * res;                         \
                    for (int a = 0; a < W; ++a) {                                                 \
                        const T v = wx[a] * wy[b] * wz[c];                                        \
                        _Pragma("omp atomic") row[ix[a]] += v;                                    \
                    }                                                                             \
                }                                                                                 \
        }                                                                                         \
    }                                                                                             \
    void cpm_fdgrad_##SUF(const T* phi, int res, T c1, T c2, T c3, T* F) {                        \
        const int64_t N = (int64_t)res * res * res;                                               \
        _Pragma("omp parallel for schedule(static)")                                              \
        for (int64_t t = 0; t < (int64_t)res * res; ++t) {                                        \
            const int iy = (int)(t % res), iz = (int)(t / res);                                   \
            const T* row = phi + t * res;                                                         \
            for (int ix = 0; ix < res; ++ix) {                                                    \
                const int64_t o = t * res + ix;                                                   \
                F[o] = -(c1 * (row[wrapi(ix + 1, res)] - row[wrapi(ix - 1, res)]) +               \
                         c2 * (row[wrapi(ix + 2, res)] - row[wrapi(ix - 2, res)]) +               \
                         c3 * (row[wrapi(ix + 3, res)] - row[wrapi(ix - 3, res)]));               \
                const T* py = phi + (int64_t)iz * res * res + ix;                                 \
                F[N + o] = -(c1 * (py[(int64_t)wrapi(iy + 1, res) * res] - py[(int64_t)wrapi(iy - 1, res) * res]) + \
                             c2 * (py[(int64_t)wrapi(iy + 2, res) * res] - py[(int64_t)wrapi(iy - 2, res) * res]) + \
                             c3 * (py[(int64_t)wrapi(iy + 3, res) * res] - py[(int64_t)wrapi(iy - 3, res) * res])); \
                const T* pz = phi + (int64_t)iy * res + ix;                                       \
                const int64_t pl = (int64_t)res * res;                                            \
                F[2 * N + o] = -(c1 * (pz[wrapi(iz + 1, res) * pl] - pz[wrapi(iz - 1, res) * pl]) + \
                                 c2 * (pz[wrapi(iz + 2, res) * pl] - pz[wrapi(iz - 2, res) * pl]) + \
                                 c3 * (pz[wrapi(iz + 3, res) * pl] - pz[wrapi(iz - 3, res) * pl])); \
            }                                                                                     \
        }                                                                                         \
    }                                                                                             \
    void cpm_gather3_##SUF(const T* F, const T* X, int64_t np, int res, T L, int W, T* acc) {     \
        const T resf = (T)res;                                                                    \
        const int64_t N = (int64_t)res * res * res;                                               \
        _Pragma("omp parallel for schedule(static)")                                              \
        for (int64_t p = 0; p < np; ++p) {                                                        \
            T wx[4], wy[4], wz[4];                                                                \
            int ix[4], iy[4], iz[4];                                                              \
            weights_##SUF(W, jmod_##SUF(X[p], L) / L * resf, res, wx, ix);                        \
            weights_##SUF(W, jmod_##SUF(X[p + np], L) / L * resf, res, wy, iy);                   \
            weights_##SUF(W, jmod_##SUF(X[p + 2 * np], L) / L * resf, res, wz, iz);               \
            T s1 = 0, s2 = 0, s3 = 0;                                                             \
            for (int c = 0; c < W; ++c)                                                           \
                for (int b = 0; b < W; ++b) {                                                     \
                    const int64_t r = ((int64_t)iz[c] * res + iy[b]) * res;                       \
                    for (int a = 0; a < W; ++a) {                                                 \
                        const T w = wx[a] * wy[b] * wz[c];                                        \
                        s1 += F[r + ix[a]] * w;                                                   \
                        s2 += F[N + r + ix[a]] * w;                                               \
                        s3 += F[2 * N + r + ix[a]] * w;                                           \
                    }                                                                             \
                }                                                                                 \
            acc[p] += s1;                                                                         \
            acc[p + np] += s2;                                                                    \
            acc[p + 2 * np] += s3;                                                                \
        }                                                                                         \
    }                                                                                             \
    void cpm_gather1_##SUF(const T* mesh, const T* X, int64_t np, int res, T L, int W, T* out) {  \
        const T resf = (T)res;                                                                    \
        _Pragma("omp parallel for schedule(static)")                                              \
        for (int64_t p = 0; p < np; ++p) {                                                        \
            T wx[4], wy[4], wz[4];                                                                \
            int ix[4], iy[4], iz[4];                                                              \
            weights_##SUF(W, jmod_##SUF(X[p], L) / L * resf, res, wx, ix);                        \
            weights_##SUF(W, jmod_##SUF(X[p + np], L) / L * resf, res, wy, iy);                   \
            weights_##SUF(W, jmod_##SUF(X[p + 2 * np], L) / L * resf, res, wz, iz);               \
            T s = 0;                                                                              \
            for (int c = 0; c < W; ++c)                                                           \
                for (int b = 0; b < W; ++b) {                                                     \
                    const int64_t r = ((int64_t)iz[c] * res + iy[b]) * res;                       \
                    for (int a = 0; a < W; ++a) s += mesh[r + ix[a]] * (wx[a] * wy[b] * wz[c]);  \
                }                                                                                 \
            out[p] = s;                                                                           \
        }                                                                                         \
    }

DEFINE_CPM(float, f32, floorf, rintf, fmodf, fabsf)
DEFINE_CPM(double, f64, floor, rint, fmod, fabs)

int cpm_threads(void) {
    int n = 1;
#pragma omp parallel
    {
#pragma omp single
        n = 0 +
#ifdef _OPENMP
            omp_get_num_threads();
#else
            1;
#endif
    }
    return n;
}
