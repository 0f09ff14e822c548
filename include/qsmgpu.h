/*
 * qsmgpu.h — C ABI of the B200 (sm_100a) implementation of QSM.rs's FFT-driven
 * reconstruction path: TV-ADMM, TKD/TSVD, Tikhonov, Laplacian unwrapping and
 * SMV/SHARP/V-SHARP background removal, plus the pipeline dispatchers.
 *
 * Every entry point mirrors one function of the reference crate (astewartau/QSM.rs);
 * the citation beside each declaration is the Rust function it replaces.  Conventions:
 *   - volumes are flat arrays of nx*ny*nz values in Fortran order, index
 *     i + j*nx + k*nx*ny (src/fft.rs:236-241); masks are uint8 (0 = outside);
 *   - inputs are borrowed, outputs are caller-allocated buffers of the same length
 *     (the Rust wrapper allocates the Vec and passes its pointer);
 *   - plain entry points take HOST pointers and are synchronous; the *_device
 *     variants take pointers to device memory on the context's GPU and return once
 *     the result is written (the context's stream is synchronised);
 *   - every function returns a qsm_status; qsm_last_error(ctx) describes the last
 *     failure on that context.  A context is not thread-safe.
 */
#ifndef QSMGPU_H
#define QSMGPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define QSM_API __attribute__((visibility("default")))
#else
#define QSM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status -- */
typedef enum {
  QSM_OK = 0,
  QSM_ERR_INVALID_ARGUMENT = 1, /* null pointer, non-finite or out-of-range parameter */
  QSM_ERR_DIMENSION_MISMATCH = 2, /* PipelineError::DimensionMismatch (src/pipeline/config.rs:343-368) */
  QSM_ERR_UNSUPPORTED_SIZE = 3, /* an axis length above 4096, or above 2048 with a prime factor > 13 */
  QSM_ERR_ALLOC = 4,
  QSM_ERR_CUDA = 5,
  QSM_ERR_INVALID_CONFIG = 6, /* PipelineError::InvalidConfig */
  QSM_ERR_NO_DEVICE = 7,
  QSM_ERR_IO = 8 /* file access, malformed or unsupported NIfTI data */
} qsm_status;

/* Arithmetic used by a context.  QSM_PRECISION_F64 runs every FFT, stencil and
 * reduction in double (the reference's arithmetic).  QSM_PRECISION_MIXED runs FFTs
 * and stencils in float with FP64 reductions (convergence tests, norms) and FP64
 * k-space multipliers; inputs and outputs stay double. */
typedef enum { QSM_PRECISION_F64 = 0, QSM_PRECISION_MIXED = 1 } qsm_precision;

typedef struct qsm_ctx qsm_ctx;

/* Progress callback (current, max) — the reference's `impl FnMut(usize, usize)`. */
typedef void (*qsm_progress_fn)(void* user, size_t current, size_t max);

/* Grid — src/grid.rs:9-13 (dims, voxel_size in mm). */
typedef struct {
  size_t nx, ny, nz;
  double vsx, vsy, vsz;
} qsm_grid;

/* ----------------------------------------------------------------- context -- */
/* Create a context on CUDA device `device` with the given precision. */
QSM_API qsm_status qsm_ctx_create(int device, int precision, qsm_ctx** out);
QSM_API qsm_status qsm_ctx_destroy(qsm_ctx* ctx);
QSM_API qsm_status qsm_ctx_set_precision(qsm_ctx* ctx, int precision);
QSM_API int qsm_ctx_get_precision(const qsm_ctx* ctx);
/* Free cached device workspaces (they are otherwise reused between calls). */
QSM_API qsm_status qsm_ctx_release_workspace(qsm_ctx* ctx);
QSM_API const char* qsm_last_error(const qsm_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), so callers can order their own work
 * and timing events with the library's launches. */
QSM_API void* qsm_ctx_stream(const qsm_ctx* ctx);
/* Number of kernels this context has launched (cumulative). */
QSM_API uint64_t qsm_ctx_kernel_launches(const qsm_ctx* ctx);
QSM_API const char* qsm_version(void);
/* Per-kernel timing: while on, every launch on this context is bracketed by CUDA
 * events on its stream (iterative solvers then run without graph capture).  Totals
 * accumulate per kernel name until qsm_ctx_profile_reset. */
QSM_API qsm_status qsm_ctx_set_profiling(qsm_ctx* ctx, int on);
QSM_API qsm_status qsm_ctx_profile_reset(qsm_ctx* ctx);
QSM_API size_t qsm_ctx_profile_count(qsm_ctx* ctx);
QSM_API qsm_status qsm_ctx_profile_entry(qsm_ctx* ctx, size_t i, char* name, size_t name_cap, uint64_t* launches,
                                         double* total_ms);
/* Which FFT pass kernels a context launches.  QSM_PLANS_COMPILED (the default) takes
 * the compile-time pass kernel wherever an axis length has one (loop bounds, radices and
 * shared-memory addressing folded into constants) and the runtime Stockham engine
 * elsewhere.  QSM_PLANS_RUNTIME takes the runtime engine for every pass: the same plan
 * and radices, so results agree to rounding.  No reference counterpart (rustfft has one
 * transform per length); tests use it to pin each compile-time pass against the runtime
 * engine. */
typedef enum { QSM_PLANS_COMPILED = 0, QSM_PLANS_RUNTIME = 1 } qsm_plan_mode;
QSM_API qsm_status qsm_ctx_set_plan_mode(qsm_ctx* ctx, int mode);
QSM_API int qsm_ctx_get_plan_mode(const qsm_ctx* ctx);
/* Arithmetic of the Krylov solvers inside iLSQR (its LSQR and LSMR steps) in a mixed
 * context; no reference counterpart.  QSM_PRECISION_F64 (the default) runs their vectors
 * and operator transforms in double: the reference stops LSQR after 50 iterations short
 * of its tolerance, so its result is the truncated Krylov iterate, and float rounding in
 * the operator moves that iterate by ~1e-3 (amplified about a thousandfold).
 * QSM_PRECISION_MIXED runs them in float with FP64 norms and recurrences (faster, about
 * 2e-3 relative L2 from the reference).  An FP64 context always runs double. */
QSM_API qsm_status qsm_ctx_set_krylov_precision(qsm_ctx* ctx, int precision);
QSM_API int qsm_ctx_get_krylov_precision(const qsm_ctx* ctx);
/* Input check (no reference counterpart; off by default, as the reference lets NaN and
 * infinities propagate into the result).  When on, every solver first scans its input
 * volume and returns QSM_ERR_INVALID_ARGUMENT, naming the count, if a voxel is NaN or
 * infinite. */
QSM_API qsm_status qsm_ctx_set_input_check(qsm_ctx* ctx, int on);
/* Autotuner of the compile-time Y/Z pass launch shapes (no reference counterpart; on by
 * default).  The first TV-ADMM-family solve of a grid on a context times each candidate
 * shape of its Y and fused Z passes once, on the solve's own buffers before they hold
 * data, and keeps the fastest per (pass, grid, precision) for the context's lifetime.
 * Candidates differ in grid form (resident blocks walking the tiles, or one block per
 * tile) and in how a narrow remainder of columns is tiled; all compute the same values,
 * so results do not depend on the choice.  Off: the resident-block shape always.
 * qsm_ctx_autotune_entry reports entry i (0 <= i < qsm_ctx_autotune_count): its key,
 * the chosen candidate, and up to `cap` (candidate, microseconds per launch) pairs;
 * *count receives the number of candidates timed. */
QSM_API qsm_status qsm_ctx_set_autotune(qsm_ctx* ctx, int on);
/* Test hook: launch every tunable pass in candidate shape `shape` (0..63: bit 0 edge
 * tiles where the grid has a narrow column remainder, bit 1 one block per tile, bits 2-5
 * resident blocks per SM of the persistent grid, 0 = as many as fit), or -1 to return to
 * the autotuner's choice. */
QSM_API qsm_status qsm_ctx_force_launch_shape(qsm_ctx* ctx, int shape);
QSM_API size_t qsm_ctx_autotune_count(const qsm_ctx* ctx);
QSM_API qsm_status qsm_ctx_autotune_entry(const qsm_ctx* ctx, size_t i, char* key, size_t key_cap, int* choice,
                                          int* candidates, float* us, size_t cap, size_t* count);
/* Fault injection for callers' error-path tests: after `after` more successful device
 * allocations, the context's next allocation fails with QSM_ERR_ALLOC (the failure is
 * simulated on the host; nothing reaches the GPU), then allocations succeed again.  A
 * negative value cancels.  The context stays usable after the failed call. */
QSM_API qsm_status qsm_ctx_inject_alloc_failure(qsm_ctx* ctx, long long after);
/* 1 when every axis length of `grid` has a transform plan: lengths up to 4096 whose prime
 * factors are at most 13, and any length up to 2048 (a Bluestein transform). */
QSM_API int qsm_grid_supported(const qsm_grid* grid);

/* ---------------------------------------------------------------- params --- */
/* TvParams — src/inversion/tv.rs:23-43 (defaults 2e-4, 2e-2, 1e-3, 250). */
typedef struct { double lambda, rho, tol; size_t max_iter; } qsm_tv_params;
/* TkdParams — src/inversion/tkd.rs:23-32 (default threshold 0.15). */
typedef struct { double threshold; } qsm_tkd_params;
/* Regularization + TikhonovParams — src/inversion/tikhonov.rs:26-49. */
typedef enum { QSM_REG_IDENTITY = 0, QSM_REG_GRADIENT = 1, QSM_REG_LAPLACIAN = 2 } qsm_regularization;
typedef struct { double lambda; int reg; } qsm_tikhonov_params;
/* SharpParams — src/bgremove/sharp.rs:22-37 (0.05, 6.0). */
typedef struct { double threshold, radius; } qsm_sharp_params;
/* VsharpParams — src/bgremove/vsharp.rs:22-40 (0.05, 12.0, 1.0). */
typedef struct { double threshold, max_radius, min_radius; } qsm_vsharp_params;
/* TgvParams — src/inversion/tgv.rs:39-76 (alpha1 5e-4, alpha0 1.5e-3, 1000 iterations,
 * 3 erosions, step 3, 3 T, TE 20 ms, tol 1e-5); single precision like the reference. */
typedef struct {
  float alpha1, alpha0;
  size_t iterations, erosions;
  float step_size, fieldstrength, te, tol;
} qsm_tgv_params;
/* ResharpParams — src/bgremove/resharp.rs:22-45 (radius 6 mm, tik_reg 1e-4, tol 1e-6, 30). */
typedef struct { double radius, tik_reg, tol; size_t max_iter; } qsm_resharp_params;
/* IsmvParams — src/bgremove/ismv.rs:19-35 (tol 1e-6, max_iter 50, radius 5 mm). */
typedef struct { double tol; size_t max_iter; double radius; } qsm_ismv_params;
/* RtsParams — src/inversion/rts.rs:22-51 (delta 0.15, mu 1e5, rho 10, tol 1e-2, 20, 4). */
typedef struct { double delta, mu, rho, tol; size_t max_iter, lsmr_iter; } qsm_rts_params;
/* NltvParams — src/inversion/nltv.rs:24-48 (lambda 1e-3, mu 1, tol 1e-3, max_iter 250 per
 * pass, newton_iter 10 passes). */
typedef struct { double lambda, mu, tol; size_t max_iter, newton_iter; } qsm_nltv_params;
/* IlsqrParams — src/inversion/ilsqr.rs:20-34 (tol 0.01, max_iter 50: the LSMR step's
 * tolerance and iteration cap). */
typedef struct { double tol; size_t max_iter; } qsm_ilsqr_params;

QSM_API void qsm_tv_params_default(qsm_tv_params* p);
QSM_API void qsm_tkd_params_default(qsm_tkd_params* p);
QSM_API void qsm_tikhonov_params_default(qsm_tikhonov_params* p);
QSM_API void qsm_sharp_params_default(qsm_sharp_params* p);
QSM_API void qsm_vsharp_params_default(qsm_vsharp_params* p);
QSM_API void qsm_ilsqr_params_default(qsm_ilsqr_params* p);
QSM_API void qsm_rts_params_default(qsm_rts_params* p);
QSM_API void qsm_nltv_params_default(qsm_nltv_params* p);
QSM_API void qsm_ismv_params_default(qsm_ismv_params* p);
QSM_API void qsm_resharp_params_default(qsm_resharp_params* p);
QSM_API void qsm_tgv_params_default(qsm_tgv_params* p);

/* -------------------------------------------------------- dipole inversion -- */
/* inversion::tv_admm — src/inversion/tv.rs:63-97 (+ admm.rs:76-178). */
QSM_API qsm_status qsm_tv_admm(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                       const double bdir[3], const qsm_tv_params* params, qsm_progress_fn progress, void* user,
                       double* out_chi);
QSM_API qsm_status qsm_tv_admm_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask,
                              const qsm_grid* grid, const double bdir[3], const qsm_tv_params* params,
                              qsm_progress_fn progress, void* user, double* d_out_chi);
/* Iterations actually run by the last tv_admm call on this context (early exit). */
QSM_API size_t qsm_tv_last_iterations(const qsm_ctx* ctx);

/* One volume of a batch: its own grid, field direction, input, mask and output (host
 * pointers for the plain batch call, device pointers for the *_device one). */
typedef struct {
  const double* local_field;
  const uint8_t* mask;
  double* out_chi;
  qsm_grid grid;
  double bdir[3];
} qsm_volume;

/* inversion::tv_admm over a batch of volumes of any sizes and field directions, one
 * call (no counterpart in the reference, which solves one volume per call; each volume's
 * result equals a qsm_tv_admm call with the same parameters).  One CUDA graph advances
 * every volume by two iterations, the volumes running as parallel branches.  progress
 * is (volumes finished, n); out_iterations (may be NULL) receives each volume's
 * iteration count. */
QSM_API qsm_status qsm_tv_admm_batch(qsm_ctx* ctx, const qsm_volume* volumes, size_t n, const qsm_tv_params* params,
                                     qsm_progress_fn progress, void* user, size_t* out_iterations);
QSM_API qsm_status qsm_tv_admm_batch_device(qsm_ctx* ctx, const qsm_volume* volumes, size_t n,
                                            const qsm_tv_params* params, qsm_progress_fn progress, void* user,
                                            size_t* out_iterations);
/* Placement of a batch over n_parts GPUs (no counterpart in the reference, which solves
 * one volume per call on one host).  Volumes are independent, so a batch shards with no
 * exchange: each GPU (one process or context per GPU) solves the volumes placed on it as
 * one batched call, and the results are gathered on the host at the end.  Placement is
 * longest-processing-time-first on cost N*log2(N)*iterations (N = voxels; iterations may
 * be NULL for equal counts): volumes in decreasing cost (ties in batch order), each on
 * the part with the least total cost so far (ties to the lowest index).  out_part[b]
 * receives volume b's part; out_load (may be NULL) the n_parts total costs.  Host only:
 * needs no GPU and no context. */
QSM_API qsm_status qsm_batch_partition(const qsm_grid* grids, const size_t* iterations, size_t n, size_t n_parts,
                                       uint32_t* out_part, double* out_load);
/* inversion::tkd over a batch of volumes (no counterpart in the reference). */
QSM_API qsm_status qsm_tkd_batch_device(qsm_ctx* ctx, const qsm_volume* volumes, size_t n,
                                        const qsm_tkd_params* params);

/* Differentiable unrolled TV-ADMM (no counterpart in the reference): `iterations` fixed
 * iterations of inversion::tv_admm (tol = 0, so the forward result equals qsm_tv_admm_device
 * with max_iter = iterations) and, when d_grad_chi (dL/dchi, nx*ny*nz values) is not NULL,
 * the vector-Jacobian product: dL/d(local_field) into d_out_grad_field and dL/dlambda into
 * *out_grad_lambda (rho is held fixed).  The adjoint sweep recomputes the forward states
 * from checkpoints taken every `checkpoint_every` iterations.  The shrink derivative
 * is 1 where |v| > lambda/rho, else 0.  Device pointers; every axis >= 1, fewer than
 * 2^32 voxels. */
QSM_API qsm_status qsm_tv_admm_unrolled_vjp_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask,
                                                   const qsm_grid* grid, const double bdir[3], double lambda,
                                                   double rho, size_t iterations, size_t checkpoint_every,
                                                   const double* d_grad_chi, double* d_out_chi,
                                                   double* d_out_grad_field, double* out_grad_lambda);

/* inversion::rts — src/inversion/rts.rs:72-211 (the pipeline's default inversion).
 * Progress (iter, max_iter) per ADMM iteration and (iters, iters) on convergence. */
QSM_API qsm_status qsm_rts(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                           const double bdir[3], const qsm_rts_params* params, qsm_progress_fn progress, void* user,
                           double* out_chi);
QSM_API qsm_status qsm_rts_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask,
                                  const qsm_grid* grid, const double bdir[3], const qsm_rts_params* params,
                                  qsm_progress_fn progress, void* user, double* d_out_chi);

/* inversion::nltv — src/inversion/nltv.rs:62-131.  Progress (k, max_iter * newton_iter)
 * before every inner ADMM step, k running over all passes; no (k, k) call. */
QSM_API qsm_status qsm_nltv(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                            const double bdir[3], const qsm_nltv_params* params, qsm_progress_fn progress, void* user,
                            double* out_chi);
QSM_API qsm_status qsm_nltv_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask,
                                   const qsm_grid* grid, const double bdir[3], const qsm_nltv_params* params,
                                   qsm_progress_fn progress, void* user, double* d_out_chi);

/* inversion::tkd — src/inversion/tkd.rs:48-99. */
QSM_API qsm_status qsm_tkd(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                   const double bdir[3], const qsm_tkd_params* params, double* out_chi);
QSM_API qsm_status qsm_tkd_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask, const qsm_grid* grid,
                          const double bdir[3], const qsm_tkd_params* params, double* d_out_chi);
/* TKD in f64 that allocates no device memory (no counterpart in the reference).
 * For callers that cannot call cudaMalloc: another allocator holds the GPU, a
 * real-time loop must avoid cudaMalloc's implicit synchronisation, or a fixed memory
 * budget applies.  Same result as qsm_tkd_device in f64, without a context: pointers
 * are device pointers on the current device, work runs on `stream` (a cudaStream_t,
 * NULL = default stream) and the call returns after the stream has finished.  Scratch
 * is a 48 MiB array in the library's own device memory (held by every GPU that loads
 * the library); volumes whose scratch exceeds it (above about 160^3) return
 * QSM_ERR_UNSUPPORTED_SIZE.  Calls share that array, so calls that overlap on the GPU
 * race and must be serialised by the caller.  Every call resolves the array's address
 * on the current device.  The call uploads small tables and synchronises its stream,
 * so it must never be called while that stream is capturing a CUDA graph (refused with
 * QSM_ERR_INVALID_ARGUMENT). */
QSM_API qsm_status qsm_tkd_device_noalloc(const double* d_local_field, const uint8_t* d_mask, const qsm_grid* grid,
                                          const double bdir[3], const qsm_tkd_params* params, double* d_out_chi,
                                          void* stream);
/* inversion::tsvd — src/inversion/tkd.rs:105-153. */
QSM_API qsm_status qsm_tsvd(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                    const double bdir[3], const qsm_tkd_params* params, double* out_chi);
QSM_API qsm_status qsm_tsvd_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask,
                           const qsm_grid* grid, const double bdir[3], const qsm_tkd_params* params,
                           double* d_out_chi);
/* inversion::ilsqr — src/inversion/ilsqr.rs:1307-1351, returning (chi, xsa, xfs, xlsqr).
 * out_xsa, out_xfs and out_xlsqr may be NULL when the caller does not need them.  Progress
 * is (1,4) .. (4,4) as in the reference.  Every axis length must be >= 2 (the reference's
 * one-sided Laplacian stencils read outside a length-1 axis). */
QSM_API qsm_status qsm_ilsqr(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                             const double bdir[3], const qsm_ilsqr_params* params, qsm_progress_fn progress,
                             void* user, double* out_chi, double* out_xsa, double* out_xfs, double* out_xlsqr);
QSM_API qsm_status qsm_ilsqr_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask,
                                    const qsm_grid* grid, const double bdir[3], const qsm_ilsqr_params* params,
                                    qsm_progress_fn progress, void* user, double* d_out_chi, double* d_out_xsa,
                                    double* d_out_xfs, double* d_out_xlsqr);
/* The operator of iLSQR's LSQR step — the apply_a closure of lsqr_step,
 * src/inversion/ilsqr.rs:988-1010: y = D * FFT(w * Re(IFFT(D * x))), D the dipole kernel
 * of (grid, bdir).  x and y are full complex spectra of nx*ny*nz values (interleaved re,
 * im; Fortran order; 16-byte aligned device memory), w is real (nx*ny*nz values).  Runs
 * the five passes of the solver's own loop, in float in a mixed context (whatever its
 * Krylov precision) and in double otherwise. */
QSM_API qsm_status qsm_ilsqr_lsqr_operator_device(qsm_ctx* ctx, const qsm_grid* grid, const double bdir[3],
                                                  const double* d_weights, const double* d_x, double* d_y);
/* inversion::tgv_qsm — src/inversion/tgv.rs:1045-1299: susceptibility (ppm) from WRAPPED
 * phase, parameters before the field direction as in the reference.  Progress is
 * (iter, iterations) for every iteration started, then (final_iter, iterations).  The
 * iterations always run in float (the reference's arithmetic), whatever the context's
 * precision.  A mask that is empty after the erosions returns QSM_ERR_INVALID_ARGUMENT
 * (the reference panics on it). */
QSM_API qsm_status qsm_tgv_qsm(qsm_ctx* ctx, const double* phase, const uint8_t* mask, const qsm_grid* grid,
                               const qsm_tgv_params* params, const double b0_dir[3], qsm_progress_fn progress,
                               void* user, double* out_chi);
QSM_API qsm_status qsm_tgv_qsm_device(qsm_ctx* ctx, const double* d_phase, const uint8_t* d_mask,
                                      const qsm_grid* grid, const qsm_tgv_params* params, const double b0_dir[3],
                                      qsm_progress_fn progress, void* user, double* d_out_chi);
/* inversion::tgv::compute_oblique_stencil — src/inversion/tgv.rs:272-479 (host only):
 * out_stencil[(di*3 + dj)*3 + dk] for offsets di, dj, dk in {-1, 0, 1} shifted by one. */
QSM_API qsm_status qsm_tgv_oblique_stencil(const double res[3], const double b0_dir[3], float out_stencil[27]);
/* inversion::tikhonov — src/inversion/tikhonov.rs:62-138. */
QSM_API qsm_status qsm_tikhonov(qsm_ctx* ctx, const double* local_field, const uint8_t* mask, const qsm_grid* grid,
                        const double bdir[3], const qsm_tikhonov_params* params, double* out_chi);
QSM_API qsm_status qsm_tikhonov_device(qsm_ctx* ctx, const double* d_local_field, const uint8_t* d_mask,
                               const qsm_grid* grid, const double bdir[3], const qsm_tikhonov_params* params,
                               double* d_out_chi);

/* Forward dipole model out = Re IFFT(D * FFT(chi)) (src/fft.rs:214-233,
 * apply_dipole_inplace), used to synthesise local fields. */
QSM_API qsm_status qsm_dipole_forward(qsm_ctx* ctx, const double* chi, const qsm_grid* grid, const double bdir[3],
                              double* out_field);
QSM_API qsm_status qsm_dipole_forward_device(qsm_ctx* ctx, const double* d_chi, const qsm_grid* grid,
                                             const double bdir[3], double* d_out_field);

/* ---------------------------------------------------------------- unwrap ---- */
/* unwrap::laplacian_unwrap — src/unwrap/laplacian.rs:135-161. */
QSM_API qsm_status qsm_laplacian_unwrap(qsm_ctx* ctx, const double* phase, const uint8_t* mask, const qsm_grid* grid,
                                double* out_unwrapped);
QSM_API qsm_status qsm_laplacian_unwrap_device(qsm_ctx* ctx, const double* d_phase, const uint8_t* d_mask,
                                       const qsm_grid* grid, double* d_out_unwrapped);

/* ----------------------------------------------------- background removal -- */
/* bgremove::smv — src/bgremove/smv.rs:31-59. */
QSM_API qsm_status qsm_smv(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid, double radius,
                   double* out_local, uint8_t* out_mask);
/* bgremove::ismv — src/bgremove/ismv.rs:48-166: (local field, eroded mask).  Progress
 * (iter, max_iter) per iteration and (iter, iter) when the change falls below tol. */
QSM_API qsm_status qsm_ismv(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                            const qsm_ismv_params* params, qsm_progress_fn progress, void* user, double* out_local,
                            uint8_t* out_mask);
QSM_API qsm_status qsm_ismv_device(qsm_ctx* ctx, const double* d_field, const uint8_t* d_mask, const qsm_grid* grid,
                                   const qsm_ismv_params* params, qsm_progress_fn progress, void* user,
                                   double* d_out_local, uint8_t* d_out_mask);
/* bgremove::sharp — src/bgremove/sharp.rs:51-131. */
QSM_API qsm_status qsm_sharp(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                     const qsm_sharp_params* params, double* out_local, uint8_t* out_mask);
/* bgremove::vsharp — src/bgremove/vsharp.rs:55-63. */
QSM_API qsm_status qsm_vsharp(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                      const qsm_vsharp_params* params, qsm_progress_fn progress, void* user, double* out_local,
                      uint8_t* out_mask);
/* bgremove::vsharp_with_radii — src/bgremove/vsharp.rs:88-199 (radii in mm, any order). */
QSM_API qsm_status qsm_vsharp_with_radii(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                                 const double* radii, size_t n_radii, double threshold, qsm_progress_fn progress,
                                 void* user, double* out_local, uint8_t* out_mask);
QSM_API qsm_status qsm_vsharp_with_radii_device(qsm_ctx* ctx, const double* d_field, const uint8_t* d_mask,
                                        const qsm_grid* grid, const double* radii, size_t n_radii,
                                        double threshold, qsm_progress_fn progress, void* user,
                                        double* d_out_local, uint8_t* d_out_mask);

/* bgremove::resharp — src/bgremove/resharp.rs:58-125: Tikhonov-regularised SHARP solved
 * by conjugate gradients on (H^T H + tik_reg I) x = H^T H field. */
QSM_API qsm_status qsm_resharp(qsm_ctx* ctx, const double* field, const uint8_t* mask, const qsm_grid* grid,
                               const qsm_resharp_params* params, qsm_progress_fn progress, void* user,
                               double* out_local, uint8_t* out_mask);
QSM_API qsm_status qsm_resharp_device(qsm_ctx* ctx, const double* d_field, const uint8_t* d_mask,
                                      const qsm_grid* grid, const qsm_resharp_params* params,
                                      qsm_progress_fn progress, void* user, double* d_out_local,
                                      uint8_t* d_out_mask);

/* ------------------------------------------------------------------ solvers -- */
/* solvers::cg_solve_with_progress — src/solvers/cg.rs:34-101 — for one fixed operator
 * (closures cannot cross the C ABI):
 *   A x = Re IFFT(K * FFT(w * Re IFFT(K * FFT(x)))) + lambda * x,
 * the normal operator of H x = w * IFFT(K * FFT(x)).  d_kernel_spectrum holds K as
 * nx*ny*nz real values in natural FFT order (the reference's fft_real_kernel output);
 * K must be even (K(k) = K(-k)), as every real symmetric image-space kernel's is; the
 * GPU applies (K(k) + K(-k))/2.  d_weight (w) may be NULL for w = 1, d_x0 NULL for a
 * zero start.  Same stopping rules as the reference: |p.Ap| < 1e-20 or
 * ||r|| < tol ||b||; progress(iter, max_iter) for every iteration begun. */
QSM_API qsm_status qsm_cg_kspace_normal_device(qsm_ctx* ctx, const qsm_grid* grid, const double* d_kernel_spectrum,
                                               const double* d_weight, double lambda, const double* d_b,
                                               const double* d_x0, double tol, size_t max_iter,
                                               qsm_progress_fn progress, void* user, double* d_x);

/* ----------------------------------------------------------------- pipeline -- */
/* InversionAlgorithm — src/pipeline/config.rs:47-58, same variant order.  Variants
 * this library does not compute return QSM_ERR_INVALID_CONFIG; Tgv and Qsmart return
 * it as the reference does (src/pipeline/inversion.rs:106-110). */
typedef enum {
  QSM_INV_TKD = 0,
  QSM_INV_TSVD = 1,
  QSM_INV_TIKHONOV = 2,
  QSM_INV_TV = 3,
  QSM_INV_RTS = 4,
  QSM_INV_NLTV = 5,
  QSM_INV_MEDI = 6,
  QSM_INV_ILSQR = 7,
  QSM_INV_TGV = 8,
  QSM_INV_QSMART = 9
} qsm_inversion_algorithm;

/* ScanMetadata — src/pipeline/config.rs:302-324 (echo times not needed on this path). */
typedef struct {
  size_t nx, ny, nz;
  double vsx, vsy, vsz;
  double field_strength;
  double b0_direction[3];
} qsm_scan_metadata;

/* InversionConfig subset — src/pipeline/config.rs:234-264. */
typedef struct {
  int algorithm;
  qsm_tkd_params tkd;
  qsm_tkd_params tsvd;
  qsm_tikhonov_params tikhonov;
  qsm_tv_params tv;
  qsm_ilsqr_params ilsqr;
  qsm_rts_params rts;
  qsm_nltv_params nltv;
} qsm_inversion_config;

/* BgRemovalAlgorithm — src/pipeline/config.rs:33-42, same variant order.  Variants
 * this library does not compute return QSM_ERR_INVALID_CONFIG. */
typedef enum {
  QSM_BG_VSHARP = 0,
  QSM_BG_PDF = 1,
  QSM_BG_LBV = 2,
  QSM_BG_ISMV = 3,
  QSM_BG_SHARP = 4,
  QSM_BG_RESHARP = 5,
  QSM_BG_HARPERELLA = 6,
  QSM_BG_IHARPERELLA = 7
} qsm_bg_algorithm;

/* BgRemovalConfig subset — src/pipeline/config.rs:204-230 (default V-SHARP). */
typedef struct {
  int algorithm;
  qsm_vsharp_params vsharp;
  qsm_sharp_params sharp;
  qsm_resharp_params resharp;
  qsm_ismv_params ismv;
} qsm_bg_removal_config;

QSM_API void qsm_inversion_config_default(qsm_inversion_config* c);
QSM_API void qsm_bg_removal_config_default(qsm_bg_removal_config* c);

/* pipeline::run_dipole_inversion — src/pipeline/inversion.rs:28-114.  `len` is the
 * length of local_field (checked against nx*ny*nz -> QSM_ERR_DIMENSION_MISMATCH). */
QSM_API qsm_status qsm_run_dipole_inversion(qsm_ctx* ctx, const double* local_field_ppm, size_t len, const uint8_t* mask,
                                    const qsm_scan_metadata* metadata, const qsm_inversion_config* config,
                                    qsm_progress_fn progress, void* user, double* out_chi);
/* pipeline::run_bg_removal — src/pipeline/bg_removal.rs:20-92. */
QSM_API qsm_status qsm_run_bg_removal(qsm_ctx* ctx, const double* field_ppm, size_t len, const uint8_t* mask,
                              const qsm_scan_metadata* metadata, const qsm_bg_removal_config* config,
                              qsm_progress_fn progress, void* user, double* out_local_field,
                              uint8_t* out_eroded_mask);

/* ------------------------------------------------------ order statistics -- */
/* prctile (src/inversion/ilsqr.rs:937-946) of the values d_vals[i] with d_mask[i] != 0
 * (all n values when d_mask is NULL), for each of the np percents in p; results in
 * out[0..np) on the host.  The reference sorts the selected values; this computes the
 * same order statistics by radix selection.  Returns 0 for an empty selection, as the
 * reference's prctile does. */
QSM_API qsm_status qsm_prctile_device(qsm_ctx* ctx, const double* d_vals, const uint8_t* d_mask, size_t n,
                                      const double* p, size_t np, double* out);

/* ------------------------------------------------- multi-echo field mapping -- */
/* B0WeightType — src/utils/multi_echo.rs:78-91, same variant order. */
typedef enum {
  QSM_B0W_PHASE_SNR = 0,
  QSM_B0W_PHASE_VAR = 1,
  QSM_B0W_AVERAGE = 2,
  QSM_B0W_TES = 3,
  QSM_B0W_MAG = 4
} qsm_b0_weight_type;

/* LinearFitParams — src/utils/multi_echo.rs:33-48 (estimate_offset true, percentile 90). */
typedef struct {
  int estimate_offset;
  double reliability_threshold_percentile;
} qsm_linear_fit_params;
QSM_API void qsm_linear_fit_params_default(qsm_linear_fit_params* p);

/* utils::multi_echo::calculate_b0_weighted — src/utils/multi_echo.rs:450-506.  phases and
 * mags hold n_echoes volumes of n values each, echo-major (echo e at e*n); tes holds the
 * n_echoes echo times in seconds (host memory, at most 64).  Output: B0 in Hz. */
QSM_API qsm_status qsm_calculate_b0_weighted(qsm_ctx* ctx, const double* phases, const double* mags,
                                             const double* tes, size_t n_echoes, const uint8_t* mask, size_t n,
                                             int weight_type, double* out_b0_hz);
QSM_API qsm_status qsm_calculate_b0_weighted_device(qsm_ctx* ctx, const double* d_phases, const double* d_mags,
                                                    const double* tes, size_t n_echoes, const uint8_t* d_mask,
                                                    size_t n, int weight_type, double* d_out_b0_hz);
/* utils::multi_echo::multi_echo_linear_fit — src/utils/multi_echo.rs:631-768 (layout as
 * above): LinearFitResult's field (rad/s), phase_offset, fit_residual and
 * reliability_mask. */
QSM_API qsm_status qsm_multi_echo_linear_fit(qsm_ctx* ctx, const double* phases, const double* mags,
                                             const double* tes, size_t n_echoes, const uint8_t* mask, size_t n,
                                             const qsm_linear_fit_params* params, double* out_field,
                                             double* out_phase_offset, double* out_fit_residual,
                                             uint8_t* out_reliability);
QSM_API qsm_status qsm_multi_echo_linear_fit_device(qsm_ctx* ctx, const double* d_phases, const double* d_mags,
                                                    const double* tes, size_t n_echoes, const uint8_t* d_mask,
                                                    size_t n, const qsm_linear_fit_params* params,
                                                    double* d_out_field, double* d_out_phase_offset,
                                                    double* d_out_fit_residual, uint8_t* d_out_reliability);

/* --------------------------------------------------------------- NIfTI I/O -- */
/* io.rs:62-460.  Single-file NIfTI-1 (.nii, and .nii.gz detected by its gzip magic),
 * either byte order.  The host functions need no context or GPU; they report errors
 * through `err` (err_cap bytes, may be NULL). */
typedef enum {
  QSM_NIFTI_UINT8 = 2,
  QSM_NIFTI_INT16 = 4,
  QSM_NIFTI_INT32 = 8,
  QSM_NIFTI_FLOAT32 = 16,
  QSM_NIFTI_FLOAT64 = 64,
  QSM_NIFTI_INT8 = 256,
  QSM_NIFTI_UINT16 = 512,
  QSM_NIFTI_UINT32 = 768,
  QSM_NIFTI_INT64 = 1024,
  QSM_NIFTI_UINT64 = 1280
} qsm_nifti_datatype;

/* NiftiData's metadata (io.rs:13-27) and what decoding needs. */
typedef struct {
  size_t nx, ny, nz, nt;  /* dim[1..4]; nt = 1 for 3D */
  double voxel_size[3];   /* pixdim[1..3] */
  double affine[16];      /* row-major: sform rows when sform_code > 0, else diag(pixdim) (io.rs:226-253) */
  double scl_slope;       /* 1 when the file stores 0 (io.rs:96) */
  double scl_inter;
  double raw_slope;       /* scl_slope as stored: voxels are raw * slope + inter unless it is 0 */
  int datatype;           /* qsm_nifti_datatype of the stored voxels */
  int ndim;               /* dim[0] */
  int big_endian;
  int gzip;
  size_t vox_offset;      /* byte offset of the voxels in the uncompressed image */
} qsm_nifti_header;

QSM_API qsm_status qsm_nifti_parse_header(const uint8_t* bytes, size_t len, qsm_nifti_header* out, char* err,
                                          size_t err_cap);
/* io::load_nifti (all_volumes = 0: nx*ny*nz values, the first volume of 4D data) and
 * io::load_nifti_4d (all_volumes = 1: nx*ny*nz*nt values); x fastest.  out_len must be
 * that count (QSM_ERR_DIMENSION_MISMATCH otherwise).  hdr may be NULL. */
QSM_API qsm_status qsm_nifti_load(const uint8_t* bytes, size_t len, int all_volumes, double* out, size_t out_len,
                                  qsm_nifti_header* hdr, char* err, size_t err_cap);
/* io::save_nifti / io::save_nifti_gz (gzip = 1): float32 voxels after a 352-byte
 * header.  out == NULL: *out_len = the size (uncompressed), or an upper bound (gzip). */
QSM_API qsm_status qsm_nifti_save(const double* data, size_t nx, size_t ny, size_t nz, const double voxel_size[3],
                                  const double affine[16], int gzip, uint8_t* out, size_t out_cap, size_t* out_len,
                                  char* err, size_t err_cap);
/* io::read_nifti_dims (io.rs:366-421). */
QSM_API qsm_status qsm_nifti_read_dims(const char* path, size_t dims[3], char* err, size_t err_cap);
QSM_API qsm_status qsm_nifti_read_file_header(const char* path, qsm_nifti_header* out, char* err, size_t err_cap);
/* io::read_nifti_file (io.rs:424-431), with the all_volumes choice of qsm_nifti_load. */
QSM_API qsm_status qsm_nifti_read_file(const char* path, int all_volumes, double* out, size_t out_len,
                                       qsm_nifti_header* hdr, char* err, size_t err_cap);
/* io::save_nifti_to_file (io.rs:434-452): gzip when the path ends in .nii.gz. */
QSM_API qsm_status qsm_nifti_save_file(const char* path, const double* data, size_t nx, size_t ny, size_t nz,
                                       const double voxel_size[3], const double affine[16], char* err,
                                       size_t err_cap);
/* qsm_nifti_load into device memory (no counterpart in the reference): the stored voxels
 * cross to the GPU in their own type through pinned staging buffers and are decoded
 * and scaled there. */
QSM_API qsm_status qsm_nifti_load_device(qsm_ctx* ctx, const uint8_t* bytes, size_t len, int all_volumes,
                                         double* d_out, size_t out_len, qsm_nifti_header* hdr);
/* qsm_nifti_save from device memory (no counterpart in the reference): float32
 * conversion on the GPU, 4 bytes per voxel back to the host through pinned staging. */
QSM_API qsm_status qsm_nifti_save_device(qsm_ctx* ctx, const double* d_data, size_t nx, size_t ny, size_t nz,
                                         const double voxel_size[3], const double affine[16], int gzip, uint8_t* out,
                                         size_t out_cap, size_t* out_len);

/* QsmReference — src/pipeline/config.rs:69-72. */
typedef enum { QSM_REFERENCE_MEAN = 0, QSM_REFERENCE_NONE = 1 } qsm_reference;

/* pipeline::referencing::apply_reference — src/pipeline/referencing.rs:12-43 (host
 * pointers, n values): Mean subtracts the mean over mask > 0; both zero outside it. */
QSM_API qsm_status qsm_apply_reference(qsm_ctx* ctx, const double* chi, const uint8_t* mask, size_t n, int method,
                                       double* out);

/* pipeline::run_tgv — src/pipeline/inversion.rs:124-157 for a single echo: wrapped phase ->
 * tgv_qsm -> apply_reference.  `phases` holds n_echoes pointers to `len` values each;
 * more than one echo needs field mapping, which this library does not provide, and
 * returns QSM_ERR_INVALID_CONFIG.  len != nx*ny*nz -> QSM_ERR_DIMENSION_MISMATCH. */
QSM_API qsm_status qsm_run_tgv(qsm_ctx* ctx, const double* const* phases, size_t n_echoes, size_t len,
                               const uint8_t* mask, const qsm_scan_metadata* metadata, const qsm_tgv_params* params,
                               int reference, qsm_progress_fn progress, void* user, double* out_chi);

/* ---------------------------------------------------------- FFT primitives -- */
/* Forward 3D transform of a real volume, returned as the full complex spectrum
 * (interleaved re, im; nx*ny*nz complex values) — src/fft.rs:412-430 fft3d on real
 * data.  Exposed for parity testing of the transform engine. */
QSM_API qsm_status qsm_fft3d_real(qsm_ctx* ctx, const double* in, const qsm_grid* grid, double* out_complex);

#ifdef __cplusplus
}
#endif

#endif /* QSMGPU_H */
