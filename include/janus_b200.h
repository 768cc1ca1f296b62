/*
 * janus_b200 — C ABI of the B200-native Lippmann–Schwinger hot path.
 *
 * Plain C types only: device pointers are `void*` / typed pointers into GPU
 * memory the caller owns, streams are `cudaStream_t` passed as `void*`
 * (NULL = legacy default stream), shapes are `int64_t` arrays.  Every entry
 * point returns an `int` status: JB_OK (0) on success, a negative JB_E*
 * code on failure, with a message in jb_last_error() (per calling thread).
 * No exception crosses this boundary.  Host wrappers map JB_EINVAL to
 * ValueError and every other code to RuntimeError, like the reference's
 * checkarray/green validation (janus/utils/checkarray.pyx:3-53,
 * janus/green.pyx:102-109, 146-161).
 *
 * Conventions (those of the reference): fields are row-major
 * `T[n0][n1][(n2)][s]` with the Mandel component fastest, s = 3 (2D) or 6
 * (3D), Mandel order (xx, yy, xy) / (xx, yy, zz, √2 yz, √2 zx, √2 xy).
 * Spectra are `T[n0][(n1)][n_last/2+1][2]` (real/imaginary interleaved along
 * the last axis, the reference's FFT output layout).  A "batch" L of fields
 * is L such arrays back to back.  T is double (JB_F64) or float (JB_F32).
 *
 * Each entry point below names the reference interface it replaces.
 */
#ifndef JANUS_B200_H
#define JANUS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define JB_OK 0
#define JB_EINVAL (-1)   /* invalid argument (shape, size, range) */
#define JB_ECUDA (-2)    /* CUDA runtime error */
#define JB_ENOMEM (-3)   /* device allocation failed */
#define JB_ESTATE (-4)   /* call not valid in the handle's state */
#define JB_EFAULT (-5)   /* a kernel gave up a bounded wait for an asynchronous copy
                            (device fault word set): this call's results are invalid */

/* Per-load-case outcome of a solve (status[] of the run calls below).  No
 * counterpart in the reference, whose tutorial loop only records the
 * residuals (sphinx/tutorials/square_basic/square_basic.py:88-92).  A load
 * case stops taking part in the stopping test as soon as it is
 * non-finite or diverging; the call returns once every load case has
 * converged or stopped, or at the iteration limit. */
#define JB_SOLVE_CONVERGED 0   /* residual <= tol */
#define JB_SOLVE_MAX_ITER 1    /* iteration limit reached above tol */
#define JB_SOLVE_NON_FINITE 2  /* a residual was NaN or infinite */
#define JB_SOLVE_DIVERGING 3   /* a residual grew 1e4-fold over the smallest one seen */

#define JB_F64 0
#define JB_F32 1

#define JB_TRUNCATED 0
#define JB_FILTERED 1
/* FiniteDifferences2D/3D, janus.green.willot2015 (janus/green.pyx:976-1036):
 * Gamma0 at k_i = sin(phi_i) prod_{j != i} cos(phi_j), phi_i = pi b_i / n_i */
#define JB_WILLOT 2

typedef struct jb_fft_s jb_fft;
typedef struct jb_green_s jb_green;
typedef struct jb_local_s jb_local;
typedef struct jb_solver_s jb_solver;

/* Library version (major*10000 + minor*100 + patch). */
int jb_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char *jb_last_error(void);
/* Largest supported length of one grid axis for a precision. */
int jb_max_axis_length(int dtype);
/* Device-side fault word of the current device, read and cleared: bit 0 set
 * means a kernel gave up a bounded wait on its own asynchronous copies and
 * skipped its tile (no reference counterpart; the reference has no device
 * code).  Synchronises with the device. */
int jb_device_status(unsigned *fault);
/* Polls of the first bounded wait of every asynchronous copy in the pass
 * kernels (a negative value restores the default, 2^24).  For tests of the
 * failure path only: 0 makes every first wait give up at once, while its
 * copy is still in flight; the kernel then sets the fault word, waits at the
 * full limit for its own copy and returns, and the solvers report JB_EFAULT
 * at their next synchronisation.  No reference counterpart. */
int jb_set_wait_limit(int polls);

/* ---- real FFT objects ------------------------------------------------- */

/* Replaces janus.fft.serial.create_real (janus/fft/serial/_serial_fft.pyx:
 * 20-53) and the _RealFFT2D/_RealFFT3D constructors (55-74, 179-200).
 * `flags` is accepted for interface parity (FFTW planner flags, 10-18). */
int jb_fft_create(int dim, const int64_t *shape, int dtype, unsigned flags,
                  jb_fft **out);
int jb_fft_destroy(jb_fft *fft);
/* _RealFFT2D/3D.r2c (152-163, 296-309): unnormalised forward transform.
 * r: real T[n0][n1][(n2)] with element strides r_strides (dim entries,
 * in elements, may be NULL for C-contiguous); c: T[oshape] contiguous. */
int jb_fft_r2c(jb_fft *fft, const void *r, const int64_t *r_strides, void *c,
               void *stream);
/* _RealFFT2D/3D.c2r (165-177, 311-325): inverse transform scaled by 1/N.
 * c is not modified. */
int jb_fft_c2r(jb_fft *fft, const void *c, void *r, const int64_t *r_strides,
               void *stream);

/* ---- continuous Green operator (host, per wave-vector) ---------------- */

/* _GreenOperatorForStrains2D/3D.c_set_frequency + c_to_memoryview
 * (janus/material/elastic/linear/isotropic.pyx:158-206, 227-353): the
 * s x s Mandel matrix of Gamma0(k) for shear modulus g, Poisson ratio nu,
 * row-major into out. Same operations as the reference. */
int jb_green_continuous_matrix(int dim, double g, double nu, const double *k,
                               double *out);
/* _GreenOperatorForStrains2D/3D.c_apply (isotropic.pyx:186-193, 294-313):
 * y = Gamma0(k) x for one s-vector, host, reference operation order. */
int jb_green_continuous_apply(int dim, double g, double nu, const double *k,
                              const double *x, double *y);
/* FourthRankIsotropicTensor2D/3D.c_apply (janus/operators.pyx:317-324,
 * 354-365): y = (sph J + dev K) x for one s-vector, host, reference
 * operation order; x == y allowed. */
int jb_isotropic_apply(int dim, double sph, double dev, const double *x,
                       double *y);

/* ---- discrete Green operators ----------------------------------------- */

/* Replaces janus.green.truncated / filtered / willot2015 (janus/green.pyx:
 * 22-36, 1030-1036) and the TruncatedGreenOperator2D/3D,
 * FilteredGreenOperator2D/3D, FiniteDifferences2D/3D constructors (100-141,
 * 261-307, 428-430, 501-503, 593-605, 708-728, 976-1027). */
int jb_green_create(int dim, const int64_t *shape, double h, double g,
                    double nu, int variant, int dtype, jb_green **out);
int jb_green_destroy(jb_green *green);
/* DiscreteGreenOperator2D/3D.c_apply and the fused truncated loops
 * (green.pyx:185-216, 356-390, 456-495, 534-580): y = Gamma0[x] for a batch
 * of `batch` contiguous fields; x == y is allowed. */
int jb_green_apply(jb_green *green, const void *x, void *y, int64_t batch,
                   void *stream);
/* No counterpart in the reference.  y = Gamma0[x] (FP64, one field, x == y
 * allowed) for callers that cannot allocate device memory at all: code under
 * an allocator that owns the whole GPU, a host application that forbids
 * cudaMalloc/cudaFree outside its set-up phase, or a plug-in that is handed
 * only its input and output buffers.  It takes no handle and allocates
 * nothing: twiddles, Green tables and the spectral scratch live in one
 * 32 MiB file-scope device array that every GPU loading this library holds
 * until exit.  Limit: the half spectrum n0*(n1)*(n_last/2+1)*s*16 bytes must
 * fit in 31 MiB (FP64 2D up to about 1024 x 1024, 3D up to about 80^3) and
 * no axis may exceed 4096; larger grids get JB_EINVAL with the size in the
 * message.  x and y must be memory of the current device and `stream` one
 * of its streams (else JB_EINVAL).  The first call on a device (with that
 * device current) looks up the array's address and caches it (the cache
 * does not survive cudaDeviceReset), so make it before any stream capture.
 * Each call fills the twiddles and tables with a kernel on `stream` (no host
 * copies).  Calls share the array: calls that overlap on the GPU race. */
int jb_green_apply_noalloc(int dim, const int64_t *shape, double h, double g,
                           double nu, int variant, const double *x, double *y,
                           void *stream);
/* Column-pass tile schedule of this operator (no reference counterpart; the
 * reference plans with FFTW).  v[6] = {plain width, plain input tiles, plain
 * compile-time tiles allowed, Green width, Green input tiles, Green
 * compile-time tiles allowed}; widths in complex columns (the Green one a
 * multiple of s), input tiles 2 or 3, 0 = built-in rule; a Green
 * compile-time value of 2 transforms the Green tiles in place (24 columns at
 * n = 128, 12 at n = 256, no partner tile), 3 takes the register-tile Green
 * pass (n0 = 32 ... 1024, a power of two: the axis-0 transforms and the
 * contraction in registers between shared-memory exchanges; the built-in
 * rule except 3D n0 = 256 and 3D FP32 n0 = 128 on the fly).  A width whose tiles do not fit the
 * shared-memory budget is narrowed.  An optional 7th value selects the Green
 * contraction: 0 built-in rule (the table for the filtered operator, on the
 * fly for the truncated and finite-difference ones), 1 the table of
 * per-coefficient symmetric Mandel matrices, 2 on the fly.  Set by the
 * autotuner (janus_b200.autotune) from timed candidates; count is 6 or 7. */
int jb_green_set_tuning(jb_green *green, const int *v, int count);
int jb_green_get_tuning(jb_green *green, int *v, int count);
/* set_frequency + to_memoryview at index b (green.pyx:146-171, 312-342 and
 * the subclasses' c_set_frequency / c_to_memoryview): host, FP64, with the
 * reference's range checks (0 <= b_i < n_i). */
int jb_green_matrix(jb_green *green, const int32_t *b, double *out);
/* apply_by_freq (green.pyx:173-180, 344-351): eta = Gamma(b) tau, host. */
int jb_green_apply_by_freq(jb_green *green, const int32_t *b,
                           const double *tau, double *eta);
/* Device form of apply_by_freq over `count` indices: b int32[count][dim],
 * tau/eta complex T[count][s][2] (may alias). Uses the same spectral
 * contraction as jb_green_apply. */
int jb_green_apply_by_freq_device(jb_green *green, int64_t count,
                                  const int32_t *b, const void *tau,
                                  void *eta, void *stream);

/* ---- local operators (C - C0):eps ------------------------------------- */

/* Replaces BlockDiagonalOperator2D/3D built from FourthRankIsotropicTensor
 * local operators (janus/operators.pyx:617-716, 257-408): phase-map form.
 * sph/dev: host arrays of nphase coefficients; phase: device array of
 * n0*n1*(n2) indices, uint8 (index_bytes 1) or int32 (4), copied.
 * index_bytes 0: one (sph, dev) pair per voxel (a stiffness field such as
 * mu(x)); nphase must equal the voxel count and phase must be NULL. */
int jb_local_create(int dim, const int64_t *shape, int nphase,
                    const double *sph, const double *dev, const void *phase,
                    int index_bytes, int dtype, jb_local **out);
/* BlockDiagonalOperator2D/3D over general linear local operators
 * (LinearOperator, FourthRankCubicTensor2D: janus/operators.pyx:195-254,
 * 411-450): one row-major s x s matrix (C - C0 of the phase) per table entry,
 * mats host double[nphase][s][s]; phase / index_bytes as jb_local_create.
 * Applied as y_i = sum_j m_ij x_j in j order without FMA contraction (the
 * reference's c_apply order). */
int jb_local_create_matrix(int dim, const int64_t *shape, int nphase,
                           const double *mats, const void *phase,
                           int index_bytes, int dtype, jb_local **out);
int jb_local_destroy(jb_local *local);
/* BlockDiagonalOperator2D/3D.c_apply (657-664, 708-716), bitwise the
 * reference arithmetic; x == y allowed. */
int jb_local_apply(jb_local *local, const void *x, void *y, int64_t batch,
                   void *stream);
/* Per-voxel strain / adjoint-strain contraction for the gradient of mean
 * stresses with respect to a stiffness field (no reference counterpart: the
 * reference has no derivatives).  eps, zeta: [nload][nvox][s] fields of
 * `dtype` on the device; out: double[nvox][2] on the device, receiving
 *   out[v][0] = scale * sum_j tr(zeta_j) tr(eps_j) / dim        (d/d sph)
 *   out[v][1] = scale * sum_j (zeta_j . eps_j - tr(zeta_j) tr(eps_j) / dim)
 *                                                             (d/d dev)
 * i.e. zeta : J : eps and zeta : K : eps with J, K the isotropic projectors
 * of sph J + dev K (operators.pyx:257-303), in Mandel form. */
int jb_local_gradient(int dim, int dtype, int64_t nvox, int nload,
                      const void *eps, const void *zeta, double scale,
                      double *out, void *stream);
/* BlockDiagonalLinearOperator2D/3D.c_apply / c_apply_transpose (739-774,
 * 823-861): y[v] = a[v] x[v] (or a[v]^T x[v]); a: T[nvox][osz][isz]. */
int jb_block_linear_apply(int dtype, int64_t nvox, int osz, int isz,
                          const void *a, const void *x, void *y,
                          int transpose, void *stream);

/* ---- basic fixed-point scheme ----------------------------------------- */

/* The loop of sphinx/tutorials/square_basic/square_basic.py:83-97 over
 * `nload` load cases at once: eps_{k+1} = E - Gamma0[(C - C0):eps_k],
 * res_k = ||eps_{k+1} - eps_k|| / (sqrt(N) ||E||). */
int jb_solver_create(jb_green *green, jb_local *local, int nload,
                     jb_solver **out);
int jb_solver_destroy(jb_solver *solver);
/* eps: device T[nload][grid][s]; E: host double[nload][s]. If init != 0,
 * eps is set to E first.  Runs until every load case has res <= tol (or has
 * stopped, non-finite or diverging) or max_iter iterations.  residuals: host
 * double[max_iter][nload] (may be NULL); iters_out: iterations done;
 * mean_tau: host double[nload][s], the grid mean of (C - C0):eps at the
 * final eps (may be NULL); status: host int[nload], JB_SOLVE_* (may be
 * NULL).  The device fault word is read at every iteration (JB_EFAULT).
 * The call returns after the work on `stream` has completed. */
int jb_solver_run(jb_solver *solver, const double *E, void *eps, int init,
                  int max_iter, double tol, double *residuals, int *iters_out,
                  double *mean_tau, int *status, void *stream);
/* Set the macroscopic strains E (host double[nload][s]) used by
 * jb_solver_step. */
int jb_solver_set_load(jb_solver *solver, const double *E);
/* One iteration on `stream`, asynchronous: eps is updated in place and the
 * normalised residual of each load case is written to res_dev (device
 * double[nload], may be NULL). */
int jb_solver_step(jb_solver *solver, void *eps, double *res_dev,
                   void *stream);
/* ---- restarted GMRES(m) ------------------------------------------------- */

/* Replaces the reference's Krylov usage, scipy's gmres over a LinearOperator
 * whose matvec is x + Gamma0[(C - C0):x]
 * (examples/square_inclusion_scipy.py:52-59, 88), for `nload` load cases at
 * once (one Krylov space each), FP64 only, basis of restart + 1 fields kept
 * on the device.  The handles are borrowed and must outlive the solver. */
typedef struct jb_gmres_s jb_gmres;
int jb_gmres_create(jb_green *green, jb_local *local, int nload, int restart,
                    jb_gmres **out);
int jb_gmres_destroy(jb_gmres *solver);
/* Solves (I + Gamma0 (C - C0)) eps = E from eps (set to E first if init).
 * Stops when every load case has ||E - eps - Gamma0[(C - C0):eps]|| /
 * (sqrt(N) ||E||) <= tol (the basic scheme's residual measure), checked on
 * the true residual at each restart, or after max_iter Arnoldi steps.
 * residuals: host double[max_iter][nload], the Givens estimate of each step
 * (may be NULL); iters_out: Arnoldi steps done; final_residuals: host
 * double[nload], the true residual at exit (may be NULL); mean_tau and
 * status as for jb_solver_run (a load case whose residual estimate is not
 * finite stops).  Returns after the work on `stream` has completed. */
int jb_gmres_run(jb_gmres *solver, const double *E, void *eps, int init,
                 int max_iter, double tol, double *residuals, int *iters_out,
                 double *final_residuals, double *mean_tau, int *status,
                 void *stream);

/* ---- mixed-precision basic scheme (defect correction) ------------------- */

/* No counterpart in the reference (its solver loop is FP64 only).  Solves the
 * same equation as jb_solver_run with FP32 bulk iterations and FP64 defect
 * correction: each outer step computes, in FP64, the basic scheme's residual
 * r = E - eps - Gamma0[(C - C0):eps] and its norm (the stopping test, same
 * normalisation as jb_solver_run), then runs `inner - 1` FP32 iterations of
 * d <- r - Gamma0[(C - C0):d] from d = r, and adds d to the FP64 eps.
 * g64/l64 and g32/l32 are the same operators built with JB_F64 and JB_F32;
 * g32/l32 may also be JB_F64 operators (the FP64 ones themselves), which
 * runs the same algorithm with FP64 corrections (a control that separates
 * the inner solver's gain from precision's).  The handles are borrowed and
 * must outlive the solver. */
typedef struct jb_mixed_s jb_mixed;
int jb_mixed_create(jb_green *g64, jb_local *l64, jb_green *g32, jb_local *l32,
                    int nload, jb_mixed **out);
int jb_mixed_destroy(jb_mixed *solver);
/* Inner solver of the correction equation A d = r, A d = d + Gamma0[(C -
 * C0):d] (the basic scheme's operator, FP32): JB_INNER_BASIC runs `inner - 1`
 * basic iterations (the default); JB_INNER_BICGSTAB runs up to `inner`
 * BiCGSTAB iterations (two applications of A each) from d = 0, batched over
 * the load cases with device-side scalars: after the first correction,
 * jb_mixed_run sizes each one by the residual reduction per iteration seen
 * over the previous one, extrapolated to half the tolerance (jb_batch_run
 * always runs `inner`).  The outer FP64 residual and stopping test are the
 * same for both; fp32_iters_out counts applications of A. */
#define JB_INNER_BASIC 0
#define JB_INNER_BICGSTAB 1
#define JB_INNER_BICGSTAB_FIXED 2 /* always `inner` iterations per correction */
int jb_mixed_set_method(jb_mixed *solver, int method);
/* eps: device double[nload][grid][s]; E host double[nload][s]; residuals:
 * host double[max_outer][nload] (FP64 residual at each outer step, may be
 * NULL); outer_out / fp32_iters_out: counts done; status: host int[nload],
 * JB_SOLVE_* of the FP64 residual (may be NULL).  Returns after the work on
 * `stream` has completed. */
int jb_mixed_run(jb_mixed *solver, const double *E, void *eps, int init,
                 int max_outer, int inner, double tol, double *residuals,
                 int *outer_out, int *fp32_iters_out, double *mean_tau,
                 int *status, void *stream);

/* Batched mixed-precision solves (no reference counterpart): `count`
 * problems, each a jb_mixed solver of its own grid (sizes may differ) and
 * load cases.  jb_batch_run evaluates every problem's first FP64 residual,
 * then runs the outer steps (the FP32 correction sweeps and the next FP64
 * residual of every problem still iterating) in one CUDA graph launch (see
 * jb_batch_set_persistent; per-step form: one launch per outer step, the
 * problems on `branches` parallel streams inside the graph, largest first
 * onto the least loaded, captured again only when a problem leaves the
 * iteration, converged or at max_outer).  Arrays are
 * concatenated in problem order: E host double[L_p][s_p]; eps device
 * pointers (FP64 fields [L_p][grid_p][s_p]); residuals host
 * double[max_outer][L_p] per problem (may be NULL); outer_out /
 * fp32_iters_out int[count]; mean_tau host double[L_p][s_p] (may be NULL);
 * graph_launches_out: graph launches made; status host int[L_p] per
 * problem, JB_SOLVE_* (may be NULL; a problem leaves the iteration when all
 * its load cases have converged or stopped).  The handles are borrowed. */
typedef struct jb_batch_s jb_batch;
int jb_batch_create(int count, jb_mixed *const *problems, int branches,
                    jb_batch **out);
int jb_batch_destroy(jb_batch *batch);
/* on != 0 (the default): jb_batch_run makes ONE graph launch for the whole
 * run: a while node whose body runs a decision kernel (each problem's
 * residuals recorded and its load cases' outcomes updated on the device,
 * problems retired as on the host) and, per problem, an if node holding its
 * correction and FP64 residual; no host readback until the end.  on == 0:
 * one graph launch per outer step with the decision on the host.  Results
 * are bitwise the same.  Where conditional graph nodes are unavailable the
 * run falls back to the per-step form. */
int jb_batch_set_persistent(jb_batch *batch, int on);
int jb_batch_run(jb_batch *batch, const double *E, void *const *eps, int init,
                 int max_outer, int inner, double tol, double *residuals,
                 int *outer_out, int *fp32_iters_out, double *mean_tau,
                 int *graph_launches_out, int *status, void *stream);

/* Benchmark support: record CUDA events around every pass of the next
 * `max_steps` calls of jb_solver_step (on their stream). */
int jb_solver_timing_begin(jb_solver *solver, int max_steps);
/* Wait for the recorded steps; pass_ms[i] = total device time of pass i
 * (ms, summed over the steps; room for 8 passes), npass and nsteps out. */
int jb_solver_timing_end(jb_solver *solver, double *pass_ms, int *npass,
                         int *nsteps);
/* Name of pass i of one solver step ("" if out of range). */
const char *jb_solver_pass_name(jb_solver *solver, int i);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* JANUS_B200_H */
