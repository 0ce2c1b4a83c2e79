/* esc.h -- C ABI of the B200 Cahn-Hilliard stepper for embedded core-shell particles.
 *
 * This library replaces the body of the time loop of the reference Julia model
 * (saswataiith/embedded-spinodal-core-shell-julia, core_shell.jl:84-103,
 * `run_simulation`): per step it records the history row
 * [s*dt, mean c, energy, min c, max c, dissipation] of the current field and
 * then applies the stabilised semi-implicit Fourier update
 * (core_shell.jl:72-76).  All work runs in hand-written sm_100a CUDA kernels on
 * one GPU; there is no CPU fallback.
 *
 * Conventions
 *   - Fields are n x n real arrays in the memory order of a Julia Matrix{Float64}
 *     (column-major, dimension 1 = x contiguous); a C-ordered NumPy array a[y][x]
 *     has the same bytes.
 *   - history is (steps+1) x 6 Float64, column-major like Julia's
 *     zeros(steps+1, 6): row s (0-based) at history[s + col*(steps+1)].
 *   - All pointers are host memory unless a function name says `_device`.
 *   - Supported grid sizes (esc_supported_size): any n with 2 <= n <= 4096 whose prime
 *     factors are all <= 127, and any n <= 512, odd n included (the reference's make_grid
 *     and FFTW take any n, core_shell.jl:17-25).  Tuned kernel sets serve
 *     n = 8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024, 1536, 2048,
 *     3072, 4096; every other size runs on runtime-size kernels with the same results.
 *     esc_adjoint, esc_batch_adjoint and esc_run_noalloc need a tuned size.
 *   - Functions return esc_status and never exit, abort or trap.  The message of
 *     the last failure is available from esc_last_error / esc_batch_last_error.
 *   - One context per host thread at a time; calls on a context are not re-entrant.
 *     Contexts on different threads run concurrently; their creations
 *     (esc_create, esc_batch_create) are serialised inside the library.
 */
#ifndef ESC_H
#define ESC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Model constants: field-for-field the Julia `Parameters` struct, core_shell.jl:4-15
 * (defaults A=2, B=4, chi=0.5, P=5, ca=0.5, cb=0, cc=1, kappa=2, mobility=1, Q=0.5). */
typedef struct {
  double A, B, chi, P, ca, cb, cc, kappa, mobility, Q;
} esc_params;

typedef enum {
  ESC_OK = 0,
  ESC_EINVAL = 1,      /* bad argument or unsupported grid size */
  ESC_ECUDA = 2,       /* CUDA runtime error (message in esc_last_error) */
  ESC_ENONFINITE = 3,  /* composition became non-finite (core_shell.jl:93); *bad_step holds s */
  ESC_ETIMEOUT = 4,    /* a bounded device-side wait gave up */
  ESC_ENOMEM = 5,      /* device allocation failed */
  ESC_EMASS = 6        /* coupled model: the mean composition moved by more than comperr in one step
                          (original/2023-3d/evolve.cu:145-155) */
} esc_status;

typedef enum {
  ESC_FP64 = 0,  /* plain drop-in: every field, transform and reduction in FP64 */
  ESC_MIXED = 1  /* FP64 state c, its transforms and all history reductions;
                    FP32 for f'(c), mu, grad mu and flux transforms */
} esc_precision;

typedef struct esc_ctx esc_ctx;
typedef struct esc_batch esc_batch;

/* Fills `p` with the defaults of core_shell.jl:4-15. */
void esc_default_params(esc_params *p);

/* 1 if n is a supported grid size, else 0. */
int esc_supported_size(int n);

/* Library version string. */
const char *esc_version(void);

/* Creates a single-particle context: grid n x n with spacing dx, fixed particle
 * field phi (n*n), model constants p.  Replaces make_grid + geometry
 * (core_shell.jl:86-87, :17-25, :39-43). */
esc_status esc_create(esc_ctx **out, int n, double dx, const double *phi, const esc_params *p,
                      esc_precision prec);

/* Runs `steps` steps from c (n*n, in/out) like run_simulation(c0, phi; dt, steps)
 * (core_shell.jl:84-103): fills history ((steps+1) x 6, column-major; may be NULL)
 * and overwrites c with the final field.  On a non-finite field returns
 * ESC_ENONFINITE with *bad_step = s (the step whose row was being recorded, as in
 * core_shell.jl:93); rows before s are valid and c is left unchanged.  Otherwise
 * *bad_step = -1.  bad_step may be NULL. */
esc_status esc_run(esc_ctx *ctx, double *c, int steps, double dt, double *history, int64_t *bad_step);

/* Same as esc_run with c (n*n) and history ((steps+1)*6, may be NULL) in device
 * memory.  The work is queued on the context's stream (esc_set_stream) and the
 * call returns when it has finished. */
esc_status esc_run_device(esc_ctx *ctx, double *c, int steps, double dt, double *history, int64_t *bad_step);

/* Queues the work of esc_run_device on the context's stream and returns without
 * waiting: an event the caller records on that stream afterwards completes with
 * the run, so the run can be timed on the device alone.  esc_wait must follow
 * before c or the history is read and before any other call on the context (a
 * second run before it returns ESC_EINVAL).  Argument errors are reported here;
 * the outcome of the run (ESC_ENONFINITE and the step, ESC_ETIMEOUT) by esc_wait.
 * No counterpart in the reference. */
esc_status esc_run_device_async(esc_ctx *ctx, double *c, int steps, double dt, double *history);

/* Waits for the run queued by esc_run_device_async and reports it as esc_run_device
 * would (*bad_step = -1 or the step of a non-finite field). */
esc_status esc_wait(esc_ctx *ctx, int64_t *bad_step);

/* Uses `stream` (a cudaStream_t) for all later work of the context; NULL restores
 * the context's own stream. */
esc_status esc_set_stream(esc_ctx *ctx, void *stream);

/* 1 when runs of ctx go through the cluster-resident kernel: a single FP64 grid of n = 128
 * or 256 whose whole time loop runs in one launch of one thread-block cluster of 16 CTAs
 * with the state in distributed shared memory.  Chosen at creation when the device can place
 * the cluster and 16 timed steps ran faster than the four-launch path (ESC_CLUSTER=1 forces
 * it, 0 forbids it); else 0. */
int esc_uses_cluster(const esc_ctx *ctx);

/* Message of the last failure on ctx (ctx may be NULL: last failure of this thread). */
const char *esc_last_error(const esc_ctx *ctx);

void esc_destroy(esc_ctx *ctx);

/* Gradient of L = 1/2 sum_x (c_T - c_target)^2 + lambda_F * F[c_T] (F the energy
 * of core_shell.jl:78-82, c_T after `steps` steps from c0) with respect to c0
 * (dL_dc0, n*n) and to theta = (P, chi, kappa, M0) (dL_dparams, 4 values), by a
 * hand-written FP64 adjoint of the stabilised update with checkpoint-and-
 * recompute every ckpt_every steps (<= 0: ceil(sqrt(steps))).  The forward and
 * recomputed passes run in the context's precision.  Any output may be NULL.
 * No counterpart in the reference (which has no gradients); it serves parameter
 * calibration. */
esc_status esc_adjoint(esc_ctx *ctx, const double *c0, int steps, double dt, const double *c_target,
                       double lambda_F, int ckpt_every, double *dL_dc0, double *dL_dparams, double *L);

/* Batched ensemble: `count` independent particles with their own grid size n[i],
 * spacing dx[i], particle phi[i] (n[i]^2) and constants p[i], advanced together
 * (same dt, same step count).  Grid sizes may differ. */
esc_status esc_batch_create(esc_batch **out, int count, const int *n, const double *dx,
                            const double *const *phi, const esc_params *p, esc_precision prec);

/* Runs all instances for `steps` steps.  c[i] (n[i]^2, in/out) and history[i]
 * ((steps+1) x 6 each, entries may be NULL) are host arrays; bad_steps (count
 * entries, may be NULL) receives -1 or the step at which instance i became
 * non-finite.  Returns ESC_ENONFINITE if any instance did; such an instance's c
 * is left unchanged and its history rows before that step are valid, while the
 * others still run to the end and their outputs are valid. */
esc_status esc_batch_run(esc_batch *b, double *const *c, int steps, double dt, double *const *history,
                         int64_t *bad_steps);

/* Device-memory variant of esc_batch_run (same outputs, the same non-finite
 * handling): c[i] are device pointers; history, if not NULL, is ONE device array
 * of count*(steps+1)*6 doubles, instance i at offset i*(steps+1)*6. */
esc_status esc_batch_run_device(esc_batch *b, double *const *c, int steps, double dt, double *history,
                                int64_t *bad_steps);

/* esc_batch_run_device split in two, as esc_run_device_async / esc_wait: the first
 * queues the whole run (the fork into the size groups' streams, their graph
 * launches, and the join back into the batch's stream) and returns at once; the
 * second waits and reports the outcome (bad_steps, count entries, may be NULL). */
esc_status esc_batch_run_device_async(esc_batch *b, double *const *c, int steps, double dt, double *history);
esc_status esc_batch_wait(esc_batch *b, int64_t *bad_steps);

esc_status esc_batch_set_stream(esc_batch *b, void *stream);

/* Gradients for a whole batch of one grid size (all n[i] equal; otherwise
 * ESC_EINVAL): for every particle i the loss, dL/dc0 and dL/d(P, chi, kappa, M0)
 * of esc_adjoint, computed together (every adjoint kernel runs over all
 * particles at once).  c0[i], c_target[i] and dL_dc0[i] (n*n each, entries of
 * dL_dc0 may be NULL) are host arrays; dL_dparams receives count*4 values
 * (particle-major), L count values; either may be NULL.  No counterpart in the
 * reference; it serves the batched parameter fit. */
esc_status esc_batch_adjoint(esc_batch *b, const double *const *c0, int steps, double dt,
                             const double *const *c_target, double lambda_F, int ckpt_every, double *const *dL_dc0,
                             double *dL_dparams, double *L);

/* Measurement aid: runs `steps` further steps on the batch's current device state
 * (left by the last run) launching each phase kernel separately between CUDA
 * events, and reports the mean duration in milliseconds of the four phase
 * kernels (row A, column A, row B, column B) of every size group:
 * ms[4*g + phase].  *n_groups receives the number of groups; call first with
 * the arrays NULL to size them.  The history buffer row 0 is overwritten. */
esc_status esc_batch_profile_phases(esc_batch *b, int steps, int *n_groups, int *group_n, int *group_count,
                                    double *ms);
/* Writes a JSON description of the kernel families the autotuner chose for each
 * size group (with the per-family timings it measured) into buf; returns the
 * length needed including the terminating zero.  The tuner runs once per
 * (n, precision, instance count) at creation on a synthetic state; ESC_TUNE=0
 * disables it and ESC_TUNE_CACHE=<file> persists its decisions. */
int esc_batch_describe(const esc_batch *b, char *buf, int buflen);
const char *esc_batch_last_error(const esc_batch *b);

/* Particle shapes for esc_particle_device.  Coordinates x = (i - n/2) dx along
 * the contiguous index i and y = (j - n/2) dx; S(r, R) = (1 - tanh((r - R)/w))/2.
 * params holds four values (unused ones ignored):
 *   DISC           S(r, p0)                                   (core_shell.jl:29-30)
 *   BAND           (tanh((y - p0)/w) - tanh((y - p1)/w))/2     (band p0 < y < p1)
 *   ELLIPSE        S(sqrt((x p1/p0)^2 + y^2), p1)             (semi-axes p0 along x, p1 along y)
 *   ANNULUS        S(r, p1) - S(r, p0)                        (radii p0 < p1)
 *   SQUIRCLE       S((x^4 + y^4)^(1/4), p0)
 *   ELLIPTIC_SHELL ellipse (p0, p1) minus a disc of radius p2
 *   ELLIPTIC_HOLE  disc of radius p0 minus an ellipse (p1 along x, p2 along y)
 * The last six restate, in physical coordinates, the shape set of the
 * historical 2-D program of the reference (original/2022-2d/init_conf.cu:77-147). */
typedef enum {
  ESC_SHAPE_DISC = 0,
  ESC_SHAPE_BAND = 1,
  ESC_SHAPE_ELLIPSE = 2,
  ESC_SHAPE_ANNULUS = 3,
  ESC_SHAPE_SQUIRCLE = 4,
  ESC_SHAPE_ELLIPTIC_SHELL = 5,
  ESC_SHAPE_ELLIPTIC_HOLE = 6
} esc_shape;

/* Fills the DEVICE array phi (n*n) with a particle shape of interface width w.
 * Runs on `stream` (NULL = default) and returns when done.  Replaces the host
 * generation of core_shell.jl:29-30 for large grids. */
esc_status esc_particle_device(int shape, int n, double dx, const double *params, double width, double *phi,
                               void *stream);

/* Fills the DEVICE array c (n*n) with mean + amplitude (2u - 1), u uniform from
 * SplitMix64(seed, element index).  With a DEVICE particle field phi (n*n), the
 * noise is applied only where phi >= 0.5 and its mean there is removed, c = mean
 * elsewhere (core_shell.jl:31-35, with our counter-based generator instead of
 * MersenneTwister); with phi NULL the whole field is noisy. */
esc_status esc_noise_device(int n, const double *phi, double mean, double amplitude, uint64_t seed, double *c,
                            void *stream);

/* Fills out[0..count) with the first `count` values of Julia's
 * rand(MersenneTwister(seed), count): the stream the reference's initial_fields
 * draws its noise from (core_shell.jl:32, rand(MersenneTwister(seed), n, n) in
 * the memory order of the n x n matrix).  The seed is hashed with SHA2-256 into
 * the key of dSFMT-19937, as Julia 1.12's Random library does, and the values lie
 * in [0, 1).  Host code only (no GPU); replaces nothing on the time loop, it
 * reproduces the reference's inputs. */
esc_status esc_julia_rand(uint64_t seed, double *out, int64_t count);

/* Allocation-free single-particle run.  No counterpart in the reference: it
 * exists for callers that may not call cudaMalloc themselves or through this
 * library (device memory owned by another allocator or a fixed budget, or a
 * loop that cannot take the device-wide synchronisation of cudaMalloc/cudaFree).
 * Inputs and outputs are caller-owned DEVICE buffers: phi (n*n), c (n*n, in/out),
 * history ((steps+1) x 6 column-major, may be NULL).  FP64 only, same results as
 * esc_run_device.  Every intermediate lives in one fixed __device__ array of the
 * library (about 2.1 MiB per GPU, held until exit), so n is limited to 256:
 * larger n returns ESC_EINVAL.  All calls share that array: calls that overlap on
 * the GPU race and must be serialised by the caller.  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress).  No call can run inside a
 * stream capture (each call copies a host descriptor and waits for its stream);
 * a call on a capturing stream returns ESC_EINVAL.  The first call of a grid size
 * on a device fills that size's process-wide twiddle tables; creating a context of
 * the same size rewrites them with identical values, which is harmless to kernels
 * reading them at that moment.  Work is queued on `stream` (a cudaStream_t, NULL =
 * default stream) and the call returns when it has finished.  Failures are
 * described by esc_last_error(NULL). */
esc_status esc_run_noalloc(int n, double dx, const double *phi, const esc_params *p, double *c, int steps,
                           double dt, double *history, int64_t *bad_step, void *stream);
void esc_batch_destroy(esc_batch *b);

/* ---- Coupled c-phi model (3-D) ------------------------------------------------------------
 * Conserved composition c (Cahn-Hilliard, variable mobility M = mobility h(phi)) coupled to
 * an order parameter phi that relaxes by Allen-Cahn dynamics: the step of the reference's
 * 2023 3-D program (original/2023-3d/evolve.cu:86-186, kernels original/2023-3d/EvoKernels.h).
 * Per step: df/dc and df/dphi of f(c, phi) = (1-h)(A(c-ca)^2 + A0) + h B (c-cb1)^2 (c-cb2)^2
 * + P (1 - chi c) g; mu^ = FFT(df/dc) + 2 kappa_c k^2 c^; div = sum_a D_a(M D_a mu) with the
 * fourth-order central difference D_a; c^ <- (dt div^ + lhs c^)/lhs, lhs = 1 + 2 Q kappa_c k^4 dt;
 * phi^ <- (phi^ - relax dt FFT(df/dphi)) / (1 + 2 relax kappa_phi k^2 dt).  FP64 throughout.
 * The z-gradient of mu uses dz (the reference passes dy there, evolve.cu:124).
 * Fields are nx*ny*nz real arrays in the reference's order a[k + nz*(j + ny*i)] (z
 * contiguous).  Each of nx, ny, nz must be one of 8, 12, 16, 24, 32, 48, 64, 96, 128, 192,
 * 256, 384, 512 (esc_cphi_supported_size). */
typedef struct {
  double A, B, chi, P, ca, cb1, cb2, A0, kappa_c, kappa_phi, mobility, relax, Q;
} esc_cphi_params;
typedef struct esc_cphi esc_cphi;

/* stop reasons reported by esc_cphi_run */
#define ESC_CPHI_COMPLETED 0    /* all steps ran */
#define ESC_CPHI_CONVERGED 1    /* max|c - c_prev| <= tolerance after a step (evolve.cu:168-181) */
#define ESC_CPHI_OUT_OF_BOUNDS 2 /* some c < -0.4 or c > 1.4 after a step (EvoKernels.h:489-508) */
#define ESC_CPHI_MASS_ERROR 3   /* mean composition drift > comperr (returns ESC_EMASS) */
#define ESC_CPHI_NONFINITE 4    /* non-finite c or phi (returns ESC_ENONFINITE) */

/* Fills p with the constants of original/2023-3d/InputParams:13-22
 * (A=2, B=1, chi=0.5, P=6, ca=0.5, cb1=0, cb2=1, A0=0.08, kappa_c=2, kappa_phi=10,
 * mobility=1, relax=0.001, Q=0.5). */
void esc_cphi_default_params(esc_cphi_params *p);

/* 1 if n is a supported size of one axis of the coupled model, else 0. */
int esc_cphi_supported_size(int n);

/* Creates a coupled-model context for an nx x ny x nz grid with spacings dx, dy, dz.
 * Replaces the set-up of original/2023-3d/main.cu:80-110 (k-vectors, plans). */
esc_status esc_cphi_create(esc_cphi **out, int nx, int ny, int nz, double dx, double dy, double dz,
                           const esc_cphi_params *p);

/* Runs up to `steps` steps from (c, phi) (host arrays, in/out), the loop of
 * original/2023-3d/evolve.cu:74-186.  history ((steps+1) x 6 column-major, may be NULL)
 * gets row s = [s*dt, mean c, mean phi, min c, max c, max|c_s - c_(s-1)|] for the fields
 * after s steps (row 0: the input, last column 0); rows after the last step run stay 0.
 * The run ends early when max|c - c_prev| <= tolerance (tolerance 0: never, unless c stops
 * changing), when c leaves [-0.4, 1.4] (both return ESC_OK with the fields after that
 * step), when the mean composition of c^'s k = 0 mode moves from the input mean by more
 * than comperr (1e-8 in the reference; returns ESC_EMASS with the fields before the
 * failing step), or on a non-finite value (ESC_ENONFINITE, fields of that step).
 * *steps_done gets the number of steps whose fields are returned, *stop_reason one of
 * ESC_CPHI_*. */
esc_status esc_cphi_run(esc_cphi *ctx, double *c, double *phi, int steps, double dt, double tolerance,
                        double comperr, double *history, int64_t *steps_done, int *stop_reason);

/* esc_cphi_run with DEVICE arrays c, phi and history (history may be NULL). */
esc_status esc_cphi_run_device(esc_cphi *ctx, double *c, double *phi, int steps, double dt, double tolerance,
                               double comperr, double *history, int64_t *steps_done, int *stop_reason);

/* Queues later runs on `stream` (a cudaStream_t; NULL = the context's own stream). */
esc_status esc_cphi_set_stream(esc_cphi *ctx, void *stream);

/* Measurement aid: steps on from the fields the last run left, `steps` times, timing
 * each of the twelve stages of a step with CUDA events on the context's stream (the two
 * x passes are two kernels each, timed together); ms[k] (12 values) gets the mean time
 * of stage k in launch order: z forward of the
 * local terms, y forward (2 fields), x pass with mu^ and the phi update, y inverse,
 * z inverse of mu with the z stencil, y stencil, x stencil, z forward of div,
 * y forward, x pass with the c update, y inverse (2 fields), z inverse to c and phi. */
esc_status esc_cphi_profile(esc_cphi *ctx, int steps, double *ms);

/* Message of the context's last failure (esc_last_error(NULL) for a failed creation). */
const char *esc_cphi_last_error(const esc_cphi *ctx);

void esc_cphi_destroy(esc_cphi *ctx);

#ifdef __cplusplus
}
#endif

#endif /* ESC_H */
