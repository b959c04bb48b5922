/* sns_b200.h — C ABI of the B200 pseudo-spectral Taylor-Green solver (libsns_b200.so).
 *
 * Plain pointers and sizes only.  Every entry point returns SNS_OK (0) or an SNS_ERR_*
 * code; no C++ exception crosses this boundary; sns_last_error() gives the message.
 * A handle owns all its device memory and one CUDA stream on the device that was current
 * when it was created.  Calls are synchronous on that stream (they return after the GPU
 * work finished).  One handle per host thread: there is no internal locking.
 *
 * Layouts on the host side are the reference's (ovankerm/Spectral_solver):
 *   physical field: N^3 doubles, x fastest, id = ix + N*(iy + N*iz)
 *                   (FftwFft3D::for_each_physical, src/fftw_fft.hpp:30-40);
 *   spectral field: 2*N^3 doubles, interleaved complex, same index order, mode
 *                   m = i <= N/2 ? i : i - N on each axis (fftw_fft.hpp:45-71).
 * On the device the spectra live on the half spectrum mx in [0, N/2].
 *
 * Solver handles (sns_create): N = 8, 12, 16, 24, 32, 48, 64, 96, 128, 256, 512 on the
 * domain [0, 2*pi)^3, so the wavenumber equals the integer mode.  Any other grid or box
 * goes through the generic-shape handle (sns_fft3d_*, below).
 */
#ifndef SNS_B200_H
#define SNS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SNS_OK = 0,
  SNS_ERR_INVALID = 1,        /* bad argument (null pointer, non-positive Re, ...) */
  SNS_ERR_UNSUPPORTED = 2,    /* grid size without an FFT plan, or mode not built */
  SNS_ERR_CUDA = 3,           /* CUDA runtime error (message has the CUDA string) */
  SNS_ERR_NOMEM = 4,          /* device allocation failed or exceeds the HBM budget */
  SNS_ERR_NO_DEVICE = 5,      /* no CUDA device visible */
  SNS_ERR_INJECTED = 6        /* failure forced by sns_debug_fail_after (tests only) */
};

/* Storage precision of a solver: FP64 plain form (the drop-in), or the FP32 precision form
 * (fields in FP32; twiddles and phases generated in FP64 and rounded; energy, enstrophy,
 * dissipation and the Nyquist-plane sums accumulated in FP64).  Host buffers are doubles
 * for both. */
enum { SNS_PRECISION_FP64 = 0, SNS_PRECISION_FP32 = 1 };
/* Viscous treatment: the reference's explicit term -nu*k^2*u_hat inside the RHS (the drop-in),
 * or an integrating factor: the RHS is the projected nonlinear term alone and each RK3
 * stage multiplies u_hat and g by exp(-nu*k^2*(c_{s+1} - c_s)*dt), stage times
 * c = (0, 1/3, 3/4, 1), exponent evaluated in FP64.  In that mode sns_rhs returns the
 * projected nonlinear term (the RHS of the transformed equation at the current time). */
enum { SNS_VISCOUS_EXPLICIT = 0, SNS_VISCOUS_INTEGRATING_FACTOR = 1 };

typedef struct sns_handle sns_handle;

/* Diagnostics row, the reference's Diagnostics (src/ava_taylor_green.hpp:8-19) minus the
 * run-loop columns (dt, cfl, main_dt, main_cfl), which the driver fills. */
typedef struct sns_diag {
  double t;
  double kinetic_energy;
  double dissipation;
  double enstrophy;
  double max_spectral_divergence;
  double max_velocity;
} sns_diag;

/* Library version string. */
const char* sns_version(void);

/* Bytes of device memory a solver handle of size n and the given precision needs
 * (state + work + tables); 0 for an unknown precision. */
size_t sns_bytes_required(int n, int precision);

/* Create a solver: Taylor-Green initial field (u = sin x cos y cos z, v = -cos x sin y cos z,
 * w = 0 at cell centres), plus, if pert_amp > 0, the seeded solenoidal k^(-5/3)
 * perturbation with 1 <= |m| <= pert_kmax scaled to rms |u'| = pert_amp; then the Leray
 * projection and sphere truncation.  nu = 1/Re.
 * Replaces TaylorGreenSolver::TaylorGreenSolver(int n, double reynolds)
 * (src/ava_taylor_green.hpp:40, impl :703-716); errors as its std::runtime_error. */
int sns_create(int n, double nu, int precision, int viscous_mode, uint64_t seed, double pert_amp, int pert_kmax,
               sns_handle** out);
int sns_destroy(sns_handle* h);

/* Message of the last failed call on h (or, when h is NULL, of the last failed call made
 * without a handle: sns_create, sns_forward_r2c_noalloc). */
const char* sns_last_error(const sns_handle* h);

/* FFT-backend contract (FftwFft3D::forward / backward, src/fftw_fft.cpp:53-85):
 * forward: N^3 real -> 2*N^3 doubles, unnormalised, sign -1;
 * backward: 2*N^3 doubles -> N^3 real = Re(IDFT(c)) / N^3 for any input, Hermitian or not. */
int sns_forward_r2c(sns_handle* h, const double* host_physical, double* host_spectral);
int sns_backward_c2r(sns_handle* h, const double* host_spectral, double* host_physical);

/* State exchange in the reference's full complex layout (3 arrays of 2*N^3 doubles).
 * set_state keeps mx in [0, N/2]; the rest of a reference state is its conjugate mirror. */
int sns_set_state(sns_handle* h, const double* const uhat_full[3]);
int sns_get_state(sns_handle* h, double* const uhat_full[3]);

/* Projected right-hand side of the reference's compute_rhs (ava_taylor_green_impl.hpp:847-977)
 * for the given state (full layout in and out).  The handle's own state is not changed. */
int sns_rhs(sns_handle* h, const double* const uhat_full[3], double* const rhs_full[3]);

/* Masked nonlinear term alone, -i k_j FFT(u_i u_j) dealiased and truncated, without the
 * viscous term or the projection (SpectralNavierStokes::nonlinear_rhs,
 * src/spectral_solver.cpp:160-240).  The handle's own state is not changed. */
int sns_nonlinear(sns_handle* h, const double* const uhat_full[3], double* const out_full[3]);

/* nsteps Williamson RK3 steps of size dt (TaylorGreenSolver::step_rk3, :979-1045). */
int sns_step(sns_handle* h, double dt, int nsteps);

/* Adaptive CFL stepping on the device (the reference's rule of run_taylor_green,
 * ava_taylor_green_impl.hpp:1363-1378, dt = min(dt_max, cfl * (2 pi / N) / vmax) clipped to
 * the horizon, evaluated before every step from the current state's vmax).  sns_set_clock
 * starts the handle's clock at t with horizon t_end (INFINITY: none); each sns_step_cfl step
 * computes vmax, the step size and the new time on the device (nothing waits for the host,
 * so batches and servers replay it from graphs) and stops the clock at the horizon, after
 * which a step leaves the state as it is.  sns_get_clock writes {t, last step size, steps
 * taken, stopped (0/1)}.  The steps equal, bit for bit, those of the host loop that calls
 * sns_max_velocity and sns_step with the same rule. */
int sns_set_clock(sns_handle* h, double t, double t_end, double cfl, double dt_max);
int sns_step_cfl(sns_handle* h, int nsteps);
int sns_get_clock(sns_handle* h, double* out, int count);

/* Diagnostics of the current state (TaylorGreenSolver::diagnostics, :1122-1179) and the
 * maximum velocity magnitude (TaylorGreenSolver::max_velocity, :1105-1120). */
int sns_diagnostics(sns_handle* h, double t, sns_diag* out);
int sns_max_velocity(sns_handle* h, double* out);

/* Final physical velocity: 3 arrays of N^3 doubles (the reference's layout). */
int sns_dump_velocity(sns_handle* h, double* const phys[3]);

/* Change the viscosity nu used by later RHS / step calls (SpectralNavierStokes passes its
 * own viscosity to the backend's handle). */
int sns_set_viscosity(sns_handle* h, double nu);

/* Nonlinear term: the reference's conservative form -i k_j FFT(u_i u_j) (default), or the
 * rotational form FFT(u x omega), omega_hat = i k x u_hat, with the same phase-shift
 * dealiasing, sphere mask and projection.  The two differ by a gradient (removed by the
 * projection) and by their aliasing residue, so the rotational form is not a parity mode.
 * It needs 3 more device fields (allocated by the first switch to it). */
enum { SNS_FORM_CONSERVATIVE = 0, SNS_FORM_ROTATIONAL = 1 };
int sns_set_nonlinear_form(sns_handle* h, int form);

/* Sphere pruning of the RK update (on by default; grids with the fused forward-z + sweep
 * pass, N = 128, 256, 512).  The column-block tiles (my, mx block) of the z pencils that hold
 * only modes outside the sphere |k| <= N/2 are zero in the state and zeroed by every stage,
 * so the fused pass skips them: no load, no transform, no sweep (about a fifth of its tiles).
 * The results are bitwise those of the full computation; enabled = 0 runs every tile. */
int sns_set_sphere_pruning(sns_handle* h, int enabled);

/* Compensated state of the FP32 precision form (on by default there; no counterpart in the
 * reference, whose FP32 build rounds u to FP32 after every stage).  Each complex value of u
 * is kept as its FP32 value plus a 16-bit word holding the remainder of each part as an
 * int8 multiple of 1/255 of its FP32 ulp, and the k-space sweep forms the RK update
 * u += b*dt*g and the projection of u in FP64 from the two.  Without it the FP32 rounding of
 * u drops the low bits of each stage's small increment, which over thousands of steps
 * dominates the form's error against FP64.  Costs 3 words (6 bytes) per mode of device
 * memory and 12 bytes per mode of traffic in the sweep.  get_state returns the compensated
 * value and set_state fills both parts, so a state round-trips exactly.  Enabling it after
 * it was off restarts the remainder at zero.  The FP64 form accepts 0 only
 * (SNS_ERR_UNSUPPORTED for 1). */
int sns_set_compensation(sns_handle* h, int enabled);

/* Persistent grids chosen at creation: out[0] TMA y/z passes, out[1] two-stage x pass
 * (0 = generic), out[2] fused forward-z + sweep (0 = two kernels), out[3] SM count. */
int sns_launch_config(const sns_handle* h, int* out, int count);

/* Grid size and device bytes held by the handle. */
int sns_grid_size(const sns_handle* h);
size_t sns_device_bytes(const sns_handle* h);

/* Time `nsteps` steps on the device with CUDA events (no host copies); writes the elapsed
 * milliseconds.  Used by the benchmark; the state advances as with sns_step. */
int sns_time_steps(sns_handle* h, double dt, int nsteps, double* elapsed_ms);

/* Per-pass device time: runs nsteps steps (the state advances) with CUDA events between
 * the passes of every stage on the handle's stream and writes the mean milliseconds per
 * stage of each pass into pass_ms[SNS_NUM_PASSES], in the order
 * inverse z (+phase), inverse y, fused x (products), Nyquist sums, forward y, forward z,
 * k-space sweep.  Benchmark/profiling aid; not for timed runs. */
#define SNS_NUM_PASSES 7
int sns_profile_passes(sns_handle* h, double dt, int nsteps, double* pass_ms);

/* ---------------------------------------------------------------------------------------
 * Batched ensembles (no counterpart in the reference, which runs one solve per process).
 * Many independent solves of uneven N, Re and precision live on one device; every solve
 * keeps its own handle (fields resident in HBM) and its own fixed time step.  One RK3 step
 * of the whole batch is one CUDA graph launch: the graph forks into one branch per solve
 * (the solve's passes in order on its own stream), so the solves' kernels overlap on the
 * device.  Results are bitwise those of the same solve stepped alone (fixed-order
 * reductions, no shared state between solves). */
typedef struct sns_batch sns_batch;

typedef struct sns_solve_spec {
  int n;             /* grid size (a supported N) */
  double nu;         /* viscosity 1/Re */
  int precision;     /* SNS_PRECISION_* */
  int viscous_mode;  /* SNS_VISCOUS_* */
  uint64_t seed;     /* perturbation seed */
  double pert_amp;   /* perturbation rms amplitude (0: pure Taylor-Green) */
  int pert_kmax;     /* perturbation shell 1 <= |m| <= pert_kmax */
  double dt;         /* > 0: fixed time step; <= 0: the CFL step, recomputed on the device before
                        every step from the current vmax (sns_step_cfl; no horizon) */
  double cfl;        /* CFL number for dt <= 0 (dt = min(dt_max, cfl * (2 pi / N) / vmax)) */
  double dt_max;     /* cap of the CFL step */
} sns_solve_spec;

/* Create `count` solves and capture the batch step graph.  With autotune_trials > 0 the
 * launch shape of each distinct (N, precision) is chosen by sns_autotune on a scratch handle
 * (cached in autotune_cache when non-NULL) and used by every solve of that key.  out_dt
 * (may be NULL) receives each solve's fixed step, or the first step of a CFL solve (its
 * later steps follow its vmax; sns_get_clock on sns_batch_handle(b, i) reads them). */
int sns_batch_create(const sns_solve_spec* specs, int count, int autotune_trials, const char* autotune_cache,
                     sns_batch** out, double* out_dt);
int sns_batch_destroy(sns_batch* b);
/* nsteps graph launches (every solve advances nsteps steps), then a synchronisation. */
int sns_batch_step(sns_batch* b, int nsteps);
/* Same, timed with CUDA events around the launches; writes the elapsed milliseconds. */
int sns_batch_time_steps(sns_batch* b, int nsteps, double* elapsed_ms);
/* The handle of solve i (owned by the batch: get_state, diagnostics, ... work on it). */
sns_handle* sns_batch_handle(sns_batch* b, int i);
int sns_batch_size(const sns_batch* b);
/* Message of the last failed batch call. */
const char* sns_batch_last_error(const sns_batch* b);

/* Launch-shape autotuner (no counterpart in the reference).  Times the pass variants a
 * handle can run -- the x pass as the two-stage 16 x M plan or the generic Stockham plan
 * (N = 256, 512), the forward z pass fused with the k-space sweep or as two kernels
 * (N >= 128), and the persistent grid of the TMA y/z passes (1 .. max CTAs per SM) -- over
 * `trial_steps` steps each (the state advances; results do not depend on the choice) and
 * keeps the fastest.  With a non-NULL cache_path the choice is read from / appended to that
 * file, one line per (device, N, precision) key, so later handles skip the trials.
 * out_config (may be NULL) receives {tma_grid, x2_grid, p5_grid}. */
int sns_autotune(sns_handle* h, int trial_steps, const char* cache_path, int* out_config);

/* ---------------------------------------------------------------------------------------
 * Serving with continuous batching (no counterpart in the reference).  Requests queue on
 * the host; each sns_server_step (one tick, which never waits for GPU work) admits queued
 * requests in arrival order while their device bytes fit the HBM budget, queues the next
 * batch of steps of every resident solve that has fewer than two batches in flight, on the
 * solve's own stream (so their work overlaps on the device) -- the largest resident solve by
 * one step, smaller ones by N_max^3/N^3 steps (at most 64) -- and retires the solves whose
 * last step has completed (final diagnostics returned).  A retired solve's device memory
 * is kept in an idle pool and the next request of the same N re-initialises it in place, so
 * a steady stream admits and retires without cudaMalloc / cudaFree; the budget counts
 * resident and idle memory, and idle handles of another N are freed only to make room.
 * Every step of a solve is the reference's adaptive CFL step, computed on the device from
 * the solve's current vmax and clipped to its horizon (sns_step_cfl); each result is bitwise
 * that of the same request solved alone. */
typedef struct sns_server sns_server;

typedef struct sns_request {
  int n;             /* grid size */
  double nu;         /* viscosity 1/Re */
  double t_end;      /* horizon */
  uint64_t seed;     /* perturbation seed */
  double pert_amp;   /* perturbation rms amplitude */
  int pert_kmax;     /* perturbation shell */
  double cfl;        /* CFL number of every step */
  double dt_max;     /* cap of the step */
} sns_request;

typedef struct sns_result {
  int64_t id;        /* id returned by sns_server_submit */
  int n;
  int steps;         /* RK3 steps taken (the last one clipped to t_end) */
  double dt;         /* the mean step, t_end / steps */
  sns_diag final;    /* diagnostics at t_end */
} sns_result;

int sns_server_create(size_t hbm_budget_bytes, int precision, sns_server** out);
int sns_server_destroy(sns_server* s);
int sns_server_submit(sns_server* s, const sns_request* r, int64_t* out_id);
/* One serving step; finished solves are written to done[0 .. *ndone) (at most max_done,
 * the rest are returned by later calls).  resident / queued (may be NULL) receive the
 * counts after the step; bytes_in_use (may be NULL) the admitted device bytes. */
int sns_server_step(sns_server* s, sns_result* done, int max_done, int* ndone, int* resident, int* queued,
                    size_t* bytes_in_use);
const char* sns_server_last_error(const sns_server* s);
/* Pool figures: idle_bytes (may be NULL) the device bytes of retired handles kept for reuse;
 * handles_created (may be NULL) how many handles the server has allocated so far (a request
 * that found an idle handle of its N allocated nothing). */
int sns_server_stats(const sns_server* s, size_t* idle_bytes, long long* handles_created);

/* Forward transform that allocates no device memory (no counterpart in the reference).
 * For callers that cannot let a library call cudaMalloc: applications that reserve the
 * GPU's memory up front and serve it from their own pool, runs close to the HBM limit,
 * and loops that cannot take the device-wide synchronisation an allocation may cause.
 * Same result as sns_forward_r2c, but on device buffers the caller owns:
 *   dev_physical: N^3 doubles (x fastest), dev_spectral: 2*N^3 doubles (16-byte aligned),
 * both on the current device; stream is a cudaStream_t (NULL = the default stream) and the
 * call returns after the work on it finished.  N <= SNS_NOALLOC_MAX_N (sizes 8 12 16 24 32
 * 48 64); larger grids return SNS_ERR_UNSUPPORTED.  The intermediate spectrum lives in one
 * fixed __device__ array (about 2.5 MiB) that every GPU loading the library holds until
 * exit and that all calls on a device share: calls whose GPU work overlaps race on it.
 * The first call on a device sets that array up (with the device current).  Every call
 * returns after its work on `stream` finished (it synchronises that stream), so a stream
 * that is being captured is refused with SNS_ERR_INVALID.  Errors: sns_last_error(NULL). */
#define SNS_NOALLOC_MAX_N 64
int sns_forward_r2c_noalloc(int n, const double* dev_physical, double* dev_spectral, void* stream);

/* 1 when the fused passes have a plan for an n^3 grid (sns_create accepts n), else 0. */
int sns_grid_supported(int n);

/* ---------------------------------------------------------------------------------------
 * Generic-shape transforms: the FFT-backend contract of FftwFft3D for any grid
 * (src/fftw_fft.hpp:13-81, src/fftw_fft.cpp:8-85), nx, ny, nz > 1 and box lengths > 0.  The
 * sns_create handle serves the benchmark domain (cubic, L = 2 pi, N from a fixed list) on the
 * half spectrum; this handle serves any shape in the reference's own full complex storage.
 * It holds one complex and one real field (24 bytes per grid point) plus the per-axis
 * twiddles; the solver calls below add their working set (18 complex and 8 real fields) on
 * first use.  Axis lengths factor into radices up to 16, run as register butterflies, and
 * any larger prime, run as a direct DFT of that length (slow for large primes); one CTA's
 * shared memory bounds an axis to 6400 points.  Errors: sns_fft3d_last_error
 * (sns_last_error(NULL) for sns_fft3d_create).  Calls are synchronous on the handle's own
 * stream. */
typedef struct sns_fft3d sns_fft3d;
int sns_fft3d_create(int nx, int ny, int nz, double lx, double ly, double lz, sns_fft3d** out);
int sns_fft3d_destroy(sns_fft3d* h);
const char* sns_fft3d_last_error(const sns_fft3d* h);
size_t sns_fft3d_device_bytes(const sns_fft3d* h);
/* forward: nx*ny*nz real (x fastest) -> 2*nx*ny*nz doubles, unnormalised, sign -1;
 * backward: 2*nx*ny*nz doubles -> Re(IDFT) / (nx ny nz) (FftwFft3D::forward / backward). */
int sns_fft3d_forward(sns_fft3d* h, const double* host_physical, double* host_spectral);
int sns_fft3d_backward(sns_fft3d* h, const double* host_spectral, double* host_physical);
/* SpectralNavierStokes numerics on this grid, k = 2 pi m / L, in the reference's full layout
 * (src/spectral_solver.cpp of ovankerm/Spectral_solver):
 *   rhs: full = 0 -> nonlinear_rhs (:160-240), -i k_j FFT(u_i u_j) with the phase-shift pair
 *        when dealias = 1 or the plain product when 0, truncated to the ellipsoid mask;
 *        full = 1 -> rhs (:242-260), minus nu k^2 u_hat, projected, zero mean, truncated;
 *   step: nsteps Williamson RK3 steps (step_rk3, :262-309) on uhat in place;
 *   diagnostics: E and max |u| of the physical field, enstrophy 0.5 <|omega|^2>,
 *        dissipation 2 nu enstrophy, max |k . u_hat| (:311-386);
 *   product: product_dealiased(a_hat, b_hat) (:122-158), one field each;
 *   vorticity_slice: |omega| on the physical plane iz, nx*ny doubles (x fastest), the data
 *        behind write_vorticity_ppm (:421-486). */
int sns_fft3d_rhs(sns_fft3d* h, double nu, int dealias, int full, const double* const uhat[3], double* const out[3]);
int sns_fft3d_step(sns_fft3d* h, double nu, int dealias, double dt, int nsteps, double* const uhat[3]);
int sns_fft3d_diagnostics(sns_fft3d* h, double nu, const double* const uhat[3], double t, sns_diag* out);
int sns_fft3d_product(sns_fft3d* h, const double* a_hat, const double* b_hat, double* out);
int sns_fft3d_vorticity_slice(sns_fft3d* h, const double* const uhat[3], int iz, double* host_mag);

/* Test hook: the k-th following call into the handle fails with SNS_ERR_INJECTED
 * (k <= 0 disables).  Exercises the error paths without touching the GPU. */
int sns_debug_fail_after(sns_handle* h, int k);

/* Test hook: write `code` into the handle's device error word, where a pass kernel records a
 * bounded wait that ran out (1 = a TMA tile did not land).  The next call that synchronises
 * the handle reports it as SNS_ERR_CUDA and clears the word; the call after that runs
 * normally.  Exercises the host side of the device error path without a device fault. */
int sns_debug_set_error_word(sns_handle* h, int code);

/* Test hook: one thread arms a shared-memory barrier for bytes no copy will deliver and
 * polls it `polls` times (1 .. 2^22) as the pass kernels poll their tiles; *status receives
 * 1 when the wait ran out (the pass kernels' timeout code), 0 if it landed.  Runs on the
 * current device and synchronises it.  Errors: sns_last_error(NULL). */
int sns_debug_bounded_wait(unsigned polls, int* status);

/* Debug-build hook: the index checks of libsns_b200_check.so (the same sources compiled with
 * -DSNS_BOUNDS_CHECK; every shared-memory, tensor-memory and global index of the TMA-fed
 * y/z passes, the two-stage x pass and the fused forward-z + sweep is checked against its
 * buffer, recorded when outside it and replaced by 0).  *count receives the number of
 * indices found outside their buffers so far in this process (-1 in the normal build, which
 * has no checks), *line (may be NULL) the source line and *index (may be NULL) the value of
 * the first. */
int sns_debug_bounds(long long* count, int* line, long long* index);

/* Measurement hook: `count` (a positive multiple of 128) 16-point complex DFTs (sign -1,
 * unnormalised; FP32 re/im interleaved, 32 floats per sequence, device buffers 16-byte
 * aligned) from dev_in to dev_out on `stream`, either on the register butterflies the pass
 * kernels use (use_tensor_cores = 0) or as tcgen05.mma kind::tf32 tiles of 128 sequences
 * with the 3xTF32 split (1).  *elapsed_ms (may be NULL) receives the kernel's CUDA-event
 * time.  Synchronises the stream.  Errors: sns_last_error(NULL). */
int sns_dft16_batch(const float* dev_in, float* dev_out, long long count, int use_tensor_cores, void* stream,
                    double* elapsed_ms);

#ifdef __cplusplus
}
#endif

#endif /* SNS_B200_H */
