/*
 * djb200.h — C ABI of libdjb200.so, a B200 (sm_100a) particle-mesh step for
 * DiscoDJNative's `run_nbody` (yipihey/DiscoDJ.jl).
 *
 * Every function returns an int status (DJB_OK = 0). On failure the message is
 * available from djb_last_error() (per calling thread). Invalid options raise
 * DJB_ERR_INVALID with the same wording the reference uses in its Julia
 * `error(...)` calls.
 *
 * Array conventions (the reference's, native/DiscoDJNative/src/nbody/pm.jl:15-17):
 *   particle fields are Julia (n,n,n,3) Float32 arrays in column-major order,
 *   i.e. three component blocks of n^3 floats, x index fastest. A pointer is host
 *   memory when `mem` = DJB_MEM_HOST and device memory (a CuArray's pointer on
 *   the solver's device) when `mem` = DJB_MEM_DEVICE.
 *   A field mesh for djb_power_spectrum is (res,res,res) Float32 column-major
 *   [ix,iy,iz] (x fastest).
 *
 * Threading: one solver per stream; calls on one solver are not re-entrant.
 * Calls are synchronous with respect to the host unless stated otherwise.
 * Entry points make the device they work on (the solver's, the network's, or the
 * `device` argument) current on the calling thread and leave it current, except
 * djb_power_spectrum_shells_noalloc, which restores the caller's device.
 */
#ifndef DJB200_H
#define DJB200_H

#include <stdint.h>

#if defined(__GNUC__)
#define DJB_API __attribute__((visibility("default")))
#else
#define DJB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DJB_OK 0
#define DJB_ERR_INVALID 1   /* invalid option or argument */
#define DJB_ERR_CUDA 2      /* CUDA runtime error */
#define DJB_ERR_CUFFT 3     /* cuFFT error */
#define DJB_ERR_ALLOC 4     /* device or host allocation failed */
#define DJB_ERR_STATE 5     /* call made in the wrong state (e.g. no particle state set) */
#define DJB_ERR_DEVICE 6    /* a device-side check failed (error word set by a kernel) */
#define DJB_ERR_IO 7        /* a file could not be written */

#define DJB_MEM_HOST 0
#define DJB_MEM_DEVICE 1

/* steppers (run_nbody.jl:48-101) */
#define DJB_STEPPER_BULLFROG 0
#define DJB_STEPPER_FASTPM 1
#define DJB_STEPPER_SYMPLECTIC 2

/* time variables (run_nbody.jl:27-40); DJB_TIME_ARRAY = explicit vector of a */
#define DJB_TIME_A 0
#define DJB_TIME_LOG_A 1
#define DJB_TIME_D 2
#define DJB_TIME_SUPERCONFT 3
#define DJB_TIME_ARRAY 4

/* sheet resampling methods (pm.jl:45) */
#define DJB_RESAMPLE_FOURIER 0
#define DJB_RESAMPLE_LINEAR 1

/* Options of the PM force. Mirrors `PMConfig` (pm.jl:35-46) field by field;
 * `lean` selects the `PMSolverLean` restrictions (pm.jl:569-571). */
typedef struct djb_pm_config {
    int32_t res_pm;      /* mesh cells per side (even, >= 8) */
    int32_t n_part;      /* particles per side (n_part^3 particles) */
    double boxsize;      /* box side L */
    int32_t worder;      /* 2 CIC, 3 TSC, 4 PCS */
    int32_t deconvolve;  /* 0/1: divide by the assignment window twice */
    int32_t antialias;   /* -1, 0, 1, 2, 3 interlacing shift sets */
    int32_t grad_order;  /* 0 (ik), 2, 4, 6 finite-difference gradient */
    int32_t lap_order;   /* 0 (-1/k^2), 2, 4, 6 finite-difference inverse Laplacian */
    int32_t n_resample;  /* sheet resampling factor per axis (1 = off) */
    int32_t resampling;  /* DJB_RESAMPLE_FOURIER or DJB_RESAMPLE_LINEAR */
    int32_t lean;        /* 0/1: apply the PMSolverLean option restrictions */
    int32_t device;      /* CUDA device ordinal */
} djb_pm_config;

typedef struct djb_cosmology djb_cosmology;
typedef struct djb_solver djb_solver;

/* ── library ─────────────────────────────────────────────────────────────── */
DJB_API const char* djb_version(void);
/* Message of the last failed call on this thread ("" if none). */
DJB_API const char* djb_last_error(void);

/* ── cosmology and time tables (host, float64) ───────────────────────────── */
/* Replaces `Cosmology(; Omega_c, Omega_b, h, sigma8, n_s, Omega_k, w0, wa)` +
 * `compute_timetables(c; n_pts, a_ini)`
 * (native/DiscoDJNative/src/cosmology/Cosmology.jl:22-45,86-115).
 * params = {Omega_c, Omega_b, h, sigma8, n_s, Omega_k, w0, wa}. */
DJB_API int djb_cosmology_create(const double params[8], int32_t n_pts, double a_ini,
                         djb_cosmology** out);
/* Replaces `Cosmology(name::String)` (Cosmology.jl:158-165). */
DJB_API int djb_cosmology_create_named(const char* name, djb_cosmology** out);
DJB_API int djb_cosmology_destroy(djb_cosmology* c);
/* Number of table points (2500 by default). */
DJB_API int djb_cosmology_table_size(const djb_cosmology* c, int32_t* n);
/* Copies one table: 0 a, 1 Dplus (D1), 2 dDplus/da, 3 D2plus, 4 dD2plus/da,
 * 5 superconformal time, 6 f1, 7 f2, 8 D3a, 9 D3b, 10 D3c
 * (timetables.jl:23-24; Cosmology.jl:32-44). */
DJB_API int djb_cosmology_table(const djb_cosmology* c, int32_t which, double* out, int32_t n);
/* The eight parameters {Omega_c, Omega_b, h, sigma8, n_s, Omega_k, w0, wa}
 * (Cosmology.jl:22-30). */
DJB_API int djb_cosmology_params(const djb_cosmology* c, double out[8]);
/* Unnormalised D1(a=1) (`_D1_unnormed_at_1`). */
DJB_API int djb_cosmology_d1_unnormed(const djb_cosmology* c, double* out);
/* Evaluates one timetable lookup at x: 0 Dplus(a) (`_Dplus`, timetables.jl:44),
 * 1 dDplus/da (`growth_Dplusda` :30), 2 D2plus(a) (`_D2plus` :45),
 * 3 dD2plus/da (:32), 4 superconft(a) (:34), 5 a_of_superconft(s) (:36),
 * 6 a_of_Dplus(D) (:38), 7 Fplus(a) (:40), 8 hubble_E(a) (Cosmology.jl:55),
 * 9 Omega_m (Cosmology.jl:47; x ignored). */
DJB_API int djb_cosmology_eval(const djb_cosmology* c, int32_t what, double x, double* out);
/* Replaces `stepper_coefficients(cosmo, stepper, a_ini, a_end, n_steps; time_var)`
 * (native/DiscoDJNative/src/nbody/run_nbody.jl:48-101). Outputs have n_steps
 * entries, all_a has n_steps+1. `time_var_array` (n_steps+1 scale factors) is
 * read only when time_var == DJB_TIME_ARRAY. */
DJB_API int djb_stepper_coefficients(const djb_cosmology* c, int32_t stepper, int32_t time_var,
                             const double* time_var_array, double a_ini, double a_end,
                             int32_t n_steps, double* alpha, double* beta, double* ddrift1,
                             double* ddrift2, double* all_a);

/* ── PM solver ───────────────────────────────────────────────────────────── */
/* Replaces `PMSolver(cfg, like)` / `PMSolverLean(cfg, like)` (pm.jl:385-414,569-585):
 * validates the options (pm.jl:136,146,214,245,423,570-571), allocates the
 * device meshes, FFT plans and particle state on cfg->device. */
DJB_API int djb_solver_create(const djb_pm_config* cfg, djb_solver** out);
DJB_API int djb_solver_destroy(djb_solver* s);
/* Runs subsequent work of this solver on `stream` (a cudaStream_t; NULL = the
 * solver's own stream). */
DJB_API int djb_solver_set_stream(djb_solver* s, void* stream);
/* Device bytes held by the solver (meshes, particle state, cuFFT work areas). */
DJB_API int djb_solver_device_bytes(const djb_solver* s, int64_t* bytes);

/* Replaces `pm_acceleration!(S, psi)` (pm.jl:507-521, lean :623-641): writes
 * acc = -grad(phi) at X = q + psi, (n,n,n,3) Float32, for displacements psi. */
DJB_API int djb_pm_acceleration(djb_solver* s, const float* psi, float* acc, int32_t mem);

/* Particle state (Psi, Mom) resident in HBM (run_nbody.jl:143-144).
 * Mom is set to float(double(mom_in[i]) * mom_scale): mom_scale = Fplus(a_ini) for
 * the symplectic stepper (`_pi_to_v`, run_nbody.jl:104), 1 otherwise. */
DJB_API int djb_set_state(djb_solver* s, const float* psi, const float* mom, double mom_scale,
                  int32_t mem);
DJB_API int djb_get_state(djb_solver* s, float* psi, float* mom, int32_t mem);
/* One drift-kick-drift step (run_nbody.jl:156-158):
 *   Psi += dd1*Mom;  Mom = alpha*Mom + beta*acc(Psi);  Psi += dd2*Mom.
 * The first drift is fused into the mass assignment and the kick and second drift
 * into the force interpolation. Asynchronous on the solver's stream. */
DJB_API int djb_step(djb_solver* s, double ddrift1, double alpha, double beta, double ddrift2);
/* n_steps consecutive steps with per-step coefficients (the loop of run_nbody.jl:155-163). */
DJB_API int djb_run(djb_solver* s, int32_t n_steps, const double* ddrift1, const double* alpha,
            const double* beta, const double* ddrift2);
/* Output of run_nbody.jl:148-171: x_out = Psi (wrap = 0), mod(q + Psi + L, L)
 * (wrap = 1, the wrapped positions) or q + Psi (wrap = 2, `addq`), and
 * p_out = float((double(Mom) / p_div) * p_mul) (`canon`, run_nbody.jl:149).
 * Either pointer may be NULL. */
DJB_API int djb_get_output(djb_solver* s, float* x_out, float* p_out, int32_t wrap, double p_div,
                   double p_mul, int32_t mem);
/* Snapshot file of the study driver's snapshot writer
 * (studies/eft_shell_crossing/scripts/run_jobs.jl:41-48, called at
 * studies/eft_shell_crossing/src/runners.jl:154-156): HDF5 with the datasets "Psi" and "Pi"
 * ((n,n,n,3) Float32 column-major; HDF5 dimensions (3,n,n,n)) and the float64 root
 * attributes "D" and "L". The oldest HDF5 file format (superblock 0), readable by every
 * HDF5 library. psi and pi are host arrays. DJB_ERR_IO when the file cannot be written
 * (a partial file is removed). */
DJB_API int djb_write_snapshot_h5(const char* path, const float* psi, const float* pi, int32_t n, double D,
                                  double L);
/* The same file from the resident state, Psi = the displacement and
 * Pi = float((double(Mom) / p_div) * p_mul) as in djb_get_output (the reference passes
 * Pi = P / Fplus(a), p_div = Fplus(a), p_mul = 1); the arrays stream from HBM through
 * pinned host buffers in 64 MiB pieces, so no host copy of the state is made. */
DJB_API int djb_state_write_snapshot(djb_solver* s, const char* path, double D, double L, double p_div,
                                     double p_mul);
/* Per-phase timing with CUDA events on the solver's stream (enable = 1) and launch
 * counts of this library's kernels. Phases: 0 mesh clear, 1 mass assignment,
 * 2 sheet resampling, 3 R2C, 4 k-space multiply, 5 C2R, 6 force interpolation
 * (fused kick-drift), 7 particle brick sort, 8 network force correction (network inputs,
 * network, interpolation of its output). Enabling or disabling resets the sums. */
DJB_API int djb_solver_profile(djb_solver* s, int32_t enable);
/* Reads and resets the sums: ms[phase] device milliseconds (0 when timing is off),
 * launches[phase] kernel launches of this library, calls[phase] phase executions.
 * nphase >= 9. */
DJB_API int djb_solver_profile_read(djb_solver* s, double* ms, int64_t* launches, int64_t* calls,
                                    int32_t nphase);
/* Waits for the solver's queued work and reports a device-side error word, if any. */
DJB_API int djb_synchronize(djb_solver* s);

/* ── power spectrum (shell sums in float64) ──────────────────────────────── */
/* Replaces `evaluate_power_spectrum(field, boxsize; bins, logarithmic)`
 * (native/DiscoDJNative/src/analysis/power_spectrum.jl:25-79). `field` is a
 * (res,res,res) Float32 column-major mesh. k, pk: `bins` doubles; nmodes: `bins`
 * int64. Allocates its own device work area per call. */
DJB_API int djb_power_spectrum(const float* field, int32_t res, double boxsize, int32_t bins,
                       int32_t logarithmic, double* k, double* pk, int64_t* nmodes,
                       int32_t mem, int32_t device);
/* P(k) of the solver's current particle state: CIC deposit of q + Psi on the
 * solver's mesh, delta = mesh*res^3/n^3 - 1, then the shell sums above (the
 * snapshot measurement of studies/eft_shell_crossing/src/measure.jl:430-447). */
DJB_API int djb_state_power_spectrum(djb_solver* s, int32_t bins, int32_t logarithmic, double* k,
                             double* pk, int64_t* nmodes);

/* CIC density-contrast Fourier modes of the solver's particle state, the snapshot
 * measurement `density_modes` of studies/eft_shell_crossing/src/measure.jl:80-91: CIC
 * deposit of X = q + Psi on the solver's mesh, delta = mesh*res^3/n^3 - 1, R2C, and per
 * mode m = modes[3i..3i+2] (integers in (-res/2, res/2], x, y, z) the coefficient
 * delta(m)/res^3 divided by the CIC window prod_d sinc^2(pi m_d/res), with
 * delta(m) = sum_x delta(x) exp(-2 pi i m.x/res). out: host double[2*nmodes] (re, im).
 * The particle state stays on the device. */
DJB_API int djb_state_density_modes(djb_solver* s, int32_t nmodes, const int32_t* modes, double* out);

/* ── initial conditions (2LPT, 3LPT) ─────────────────────────────────────────
 * Replaces the GPU path of `nbody_ics_lpt` at n_order = 2 (src/ics/grf.jl:118-144,
 * src/lpt/nlpt_core.jl:44-311, src/nbody/run_nbody.jl:180-208): white noise w (device, n^3
 * float32, x fastest) -> phi(k) = rfft(w) * (-sqrt(P(|k|) (n/L)^3) / k^2) with P linearly
 * interpolated in the host table (k_tab, p_tab, npk points, clamped at its ends) ->
 * psi_1 = -D phi and the second-order shape from the 3/2-padded source
 * mu2 = sum_{a<b} (psi_aa psi_bb - psi_ab^2) -> Psi = D psi_1 + D^2 psi_2 and
 * Pi = dPsi/dD = psi_1 + 2 D psi_2 at growth factor D, written to psi and pi (device,
 * (n,n,n,3) float32). n a multiple of 4. Runs on `stream` (a cudaStream_t, NULL = legacy
 * default) and waits for it; allocates its work areas (about 6 (3n/2)^3 + 6 n^3 floats)
 * for the call. */
DJB_API int djb_lpt2_ics(const float* white, int32_t n, double boxsize, const double* k_tab, const double* p_tab,
                         int32_t npk, double D, float* psi, float* pi, int32_t device, void* stream);
/* The same chain at n_order = 2 or 3 (`compute_core`, src/lpt/nlpt_core.jl:311, EdS
 * growth): for 3, psi_3 from the longitudinal source -5/9 mu2(psi_1, psi_2) -
 * 1/3 mu3(psi_1, psi_1, psi_1) and the transverse source 1/3 C(psi_1, psi_2) of
 * nlpt_core.jl:223-280 (products of the 3/2-padded derivative fields in real space),
 * Psi = sum_m D^m psi_m, Pi = sum_m m D^(m-1) psi_m. `work`: a device area of at least
 * djb_lpt_ics_work_bytes bytes (about 14 (3n/2)^3 + 6 n^3 floats for n_order = 3, 5 and 6
 * for 2), or NULL to have the call allocate and free one. */
DJB_API int djb_lpt_ics(const float* white, int32_t n, double boxsize, const double* k_tab, const double* p_tab,
                        int32_t npk, int32_t n_order, double D, float* psi, float* pi, void* work,
                        int64_t work_bytes, int32_t device, void* stream);
DJB_API int djb_lpt_ics_work_bytes(int32_t n, int32_t n_order, int32_t npk, int64_t* bytes);

/* ── adjoints (vector-Jacobian products) ────────────────────────────────────
 * No counterpart in the reference, which has no adjoint; these are the transposes
 * of the forward operators above, checked against finite differences of float64
 * restatements. They cover finite-difference gradients (grad_order 2/4/6) without
 * sheet resampling (DJB_ERR_INVALID otherwise). Arrays are (n,n,n,3) Float32 in
 * the memory `mem` names; the calls wait for the GPU before returning. The solver
 * keeps its adjoint work areas between calls (three meshes and up to nine particle
 * arrays of 3*n^3 floats) until djb_solver_destroy.
 *
 * psi_bar = (d acc / d psi)^T acc_bar, acc = djb_pm_acceleration(psi): the
 * transposes of the interpolation (weight derivatives, pm.jl:344-364), of the FD
 * gradient (pm.jl:330-342; antisymmetric stencil), of Kphi (pm.jl:389-391; real and
 * even) and of the mass assignment (pm.jl:57-74), averaged over the shifts like the
 * force (pm.jl:513-519). */
DJB_API int djb_pm_acceleration_vjp(djb_solver* s, const float* psi, const float* acc_bar, float* psi_bar,
                                    int32_t mem);
/* Adjoint of one djb_step from the state (psi0, mom0) it started from: on entry
 * psi_bar, mom_bar hold the cotangents of the state after the step, on return
 * those of (psi0, mom0). The step is Psi1 = Psi0 + dd1*Mom0, Mom1 = alpha*Mom0 +
 * beta*acc(Psi1), Psi2 = Psi1 + dd2*Mom1 (run_nbody.jl:156-158). */
DJB_API int djb_step_vjp(djb_solver* s, double ddrift1, double alpha, double beta, double ddrift2,
                         const float* psi0, const float* mom0, float* psi_bar, float* mom_bar, int32_t mem);
/* psi_bar = d(sum_b pk_bar[b] * P_b)/d psi for P(k) of the solver's particle state as
 * djb_state_power_spectrum computes it (same bins); pk_bar: host double[bins]. */
DJB_API int djb_state_power_spectrum_vjp(djb_solver* s, int32_t bins, int32_t logarithmic, const double* pk_bar,
                                         float* psi_bar, int32_t mem);

/* The PM fields on the solver's mesh for displacements psi: out = [delta, F_x, F_y,
 * F_z], four float32 res^3 meshes [z][y][x] (delta = mesh*res^3/n^3 - 1 of the W-order
 * deposit without shift; F_c = -D_c phi, the FD gradient of the potential the force
 * interpolates, pm.jl:330-342). No counterpart in the reference: the inputs of the
 * force-correction network. FD gradients (2/4/6) without resampling. */
DJB_API int djb_mesh_fields(djb_solver* s, const float* psi, float* out, int32_t mem);

/* ── force-correction network ──────────────────────────────────────────────────
 * No counterpart in the reference. A 3-D CNN on the PM mesh: `layers` convolutions
 * with 3^3 kernels and periodic boundaries, cin -> hidden -> ... -> cout channels, ReLU
 * between layers (for the force correction: in = delta and the three force
 * components, out = the three components of a force correction). bf16 operands with
 * float32 accumulation on the tensor cores, float32 master
 * weights and Adam. Meshes cross the ABI as float32 [channel][z][y][x] of res^3
 * voxels in the memory `mem` names. Parameters: per layer the weights
 * [27 taps (dz, dy, dx) x cin_pad x cout_pad] then cout_pad biases, channel counts
 * padded to multiples of 8 (padding entries are zero and stay zero). */
typedef struct djb_nn djb_nn;
DJB_API int djb_nn_create(int32_t layers, int32_t cin, int32_t hidden, int32_t cout, uint64_t seed,
                          int32_t device, djb_nn** out);
DJB_API int djb_nn_destroy(djb_nn* h);
DJB_API int djb_nn_param_count(const djb_nn* h, int64_t* count);
/* Host float32 arrays of djb_nn_param_count entries; load also resets the optimizer. */
DJB_API int djb_nn_get_params(djb_nn* h, float* params);
DJB_API int djb_nn_load(djb_nn* h, const float* params);
DJB_API int djb_nn_set_stream(djb_nn* h, void* stream);
/* Convolution path: 0 (default) = implicit GEMMs on the tcgen05 tensor cores, forward
 * and backward, for the layers whose padded channel counts are at most 32 (wider ones
 * use im2col + cuBLAS GEMMs); 1 = im2col + cuBLAS for every layer. */
DJB_API int djb_nn_set_conv(djb_nn* h, int32_t mode);
/* The convolution path in use; *tma_used = 1 once a tensor-core convolution has staged
 * planes by bulk tensor copies (the driver accepted the plane tensor map). */
DJB_API int djb_nn_get_conv(const djb_nn* h, int32_t* mode, int32_t* tma_used);
/* out = net(in); large meshes are processed in chunks of z planes. */
DJB_API int djb_nn_apply(djb_nn* h, const float* in, int32_t res, float* out, int32_t mem);
/* Gradients of the mean squared error of net(in) against target into the network's
 * gradient buffer; *loss (may be null) receives the loss. For data-parallel training
 * the buffer is read (djb_nn_grads), summed across replicas and written back
 * (djb_nn_set_grads) before djb_nn_adam_step. */
DJB_API int djb_nn_backward(djb_nn* h, const float* in, const float* target, int32_t res, double* loss,
                            int32_t mem);
DJB_API int djb_nn_grads(djb_nn* h, float* grads, int32_t mem);
DJB_API int djb_nn_set_grads(djb_nn* h, const float* grads, int32_t mem);
/* One Adam step (beta 0.9/0.999, eps 1e-8, learning rate lr) with the buffered gradients. */
DJB_API int djb_nn_adam_step(djb_nn* h, double lr);
/* djb_nn_backward then djb_nn_adam_step; *loss is the loss before the step. */
DJB_API int djb_nn_train_step(djb_nn* h, const float* in, const float* target, int32_t res, double lr,
                              double* loss, int32_t mem);
/* Gradients of sum(dout * net(in)) into the gradient buffer, for a loss defined outside the
 * network: dout (float32 [channel][z][y][x], cout meshes) is the loss gradient with respect
 * to the network's output (e.g. the transpose of an interpolation to particles,
 * djb_mesh_deposit3). */
DJB_API int djb_nn_backward_output_grad(djb_nn* h, const float* in, const float* dout, int32_t res, int32_t mem);
/* Layer count, input, hidden (0 for one layer) and output channels, and device. */
DJB_API int djb_nn_info(const djb_nn* h, int32_t* layers, int32_t* cin, int32_t* hidden, int32_t* cout,
                        int32_t* device);

/* ── NN-corrected PM force ──────────────────────────────────────────────────────
 * No counterpart in the reference. Attaches a network (4 inputs, 3 outputs) to the solver:
 * every force evaluation (djb_pm_acceleration, djb_step, djb_run) then adds
 *   out_scale * interp(net([delta_scale * delta, force_scale * F]))(X_p)
 * to the PM acceleration of pm.jl:507-521, where delta and F are the unshifted density
 * contrast and finite-difference force on the mesh (as djb_mesh_fields computes them) and
 * interp is the solver's W-order interpolation at X = q + Psi (djb_mesh_interp3), at
 * the positions the force sees (after the step's first drift). Needs a finite-difference gradient
 * (2/4/6), no resampling, a non-lean solver with res divisible by 4 and antialias 0 or 1;
 * net = NULL detaches. The solver keeps 4 + 3 meshes and 3*n^3 floats for it. The
 * network runs on the solver's stream (its stream is set to the solver's at every force). */
DJB_API int djb_solver_attach_nn(djb_solver* s, djb_nn* net, double delta_scale, double force_scale,
                                 double out_scale);
/* Network schedule: steps of djb_step/djb_run are counted from djb_set_state,
 * djb_solver_attach_nn or this call (0-based); the attached network corrects the force
 * from step `start` on (earlier steps are uncorrected) and runs on every `every`-th of
 * those steps (the first always), each particle keeping the correction it was last given
 * in between; djb_pm_acceleration always runs it. Default: every = 1, start = 0. */
DJB_API int djb_solver_nn_schedule(djb_solver* s, int32_t every, int32_t start);
/* out (n,n,n,3) = the solver's W-order interpolation (pm.jl:344-364, no shift) of the three
 * res^3 meshes mesh3 ([channel][z][y][x]) at X = q + psi. */
DJB_API int djb_mesh_interp3(djb_solver* s, const float* psi, const float* mesh3, float* out, int32_t mem);
/* The transpose of djb_mesh_interp3: mesh3[c](node) = sum_p W(X_p - node) vec_c(p). */
DJB_API int djb_mesh_deposit3(djb_solver* s, const float* psi, const float* vec, float* mesh3, int32_t mem);

/* ── self-test ───────────────────────────────────────────────────────────────
 * No counterpart in the reference. Runs the bounded mbarrier wait that the library's
 * bulk-copy kernels use on a barrier of its own: with arrive = 1 the barrier completes
 * and *err_word = 0; with arrive = 0 nothing arrives, the wait gives up after
 * limit_cycles SM cycles (at most 2^31, the kernels' own limit) and *err_word has bit 8
 * set, the kernels' "a wait ran out" flag. No copy is in flight; the device stays usable. */
DJB_API int djb_selftest_bounded_wait(int32_t device, int32_t arrive, int64_t limit_cycles, int32_t* err_word);

/* ── non-allocating shell sums ──────────────────────────────────────────────
 * No counterpart in the reference. For callers that cannot allocate device
 * memory at the point of the call: applications whose device memory is owned by
 * a pool or an external framework that forbids allocations outside it, and step
 * loops that must not synchronise the device through an allocator (cudaMalloc
 * and cudaFree can wait for the whole device). The caller passes the half spectrum of a (res,res,res)
 * field (device memory, complex64 [kz][ky][kx], kx in [0, res/2], as an in-place
 * R2C of the x-fastest field produces it) and host outputs k, pk (double) and
 * nmodes (int64) of `bins` entries; scale2 multiplies |delta(k)|^2 (1 for a field
 * given directly). The per-bin work area is a file-scope device array for at
 * most 512 bins (about 24 KB, held by every GPU that loads the library until
 * exit); more bins are rejected with DJB_ERR_INVALID. The call allocates no
 * device memory and calls no allocating library routine. The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and caches
 * it. All calls share
 * the one array, which keeps the last call's contents (each call clears the sums
 * it uses): calls that overlap on the GPU, on different streams or threads, race.
 * Runs on `stream` (a cudaStream_t, NULL = legacy default) of `device`. Every call
 * copies the sums into host stack arrays and synchronises `stream` before it
 * returns, so no call can be recorded into a CUDA graph. The calling thread's current device is the same after the call as
 * before it. Same results as djb_power_spectrum for the same field. */
DJB_API int djb_power_spectrum_shells_noalloc(const void* spectrum, int32_t res, double boxsize,
                                              int32_t bins, int32_t logarithmic, double scale2,
                                              double* k, double* pk, int64_t* nmodes, void* stream,
                                              int32_t device);

#ifdef __cplusplus
}
#endif

#endif /* DJB200_H */
