/*
 * hit3d_gpu.h -- C-ABI of the B200 pseudospectral step for HIT3DP.
 *
 * The reference has no plugin API: its hot path is a set of argument-less
 * Fortran subroutines acting on module globals (call sites main.f90:124-167).
 * Each entry point below replaces one of those calls or module set-ups, takes
 * plain pointers and fixed-width integers (the reference compiles with -i8 -r8,
 * Makefile:11-12,53-56, so a binding must use c_int32_t/c_int64_t/c_double
 * explicitly, never default INTEGER/REAL), and returns 0 on success or a
 * negative code; hit3d_gpu_last_error() then describes the failure (the
 * reference's equivalent is call my_exit(-1), my_exit.f90:23-62).
 *
 * Layouts at the boundary are the reference's:
 *   fields(nx+2, ny, nz, nfields) real*8, column-major.  Fourier space is
 *   (kx re/im interleaved, kz, ky) (x_fftw.f90:321-327); physical space is
 *   (x, y, z) with two padding entries per x row.
 * Inside the library the state lives in HBM in a transposed, row-padded layout;
 * it is converted only on upload/download.
 *
 * One context = one simulation on one GPU, driven from one host thread, on one
 * CUDA stream.  Contexts are independent; calls on one context are not
 * thread-safe.
 */
#ifndef HIT3D_GPU_H
#define HIT3D_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hit3d_ctx hit3d_ctx;

#define HIT3D_MAX_SCALARS 8
/* les_model of the learned closure; outside the reference's model numbers 0-10 */
#define HIT3D_LES_LEARNED 20

/* Run parameters; the values the reference reads from <run_name>.in
 * (m_parameters.f90:172-512) and derives at start-up. */
typedef struct hit3d_params {
    int32_t nx;          /* cubic grid size N = nx = ny = nz_all (m_parameters.f90:202)  */
    int32_t dealias;     /* 0: 2/3 rule, 1: phase shift + truncation (m_parameters.f90:330) */
    int32_t flow_type;   /* 0: decaying, 1: forced (m_parameters.f90:264)                 */
    int32_t force_type;  /* 1: Machiels band forcing (m_force.f90:158)                     */
    int32_t kfmax;       /* forced shells 1..kfmax (m_parameters.f90:309)                  */
    int32_t n_scalars;   /* passive scalars, <= HIT3D_MAX_SCALARS (m_parameters.f90:424)   */
    int32_t precision;   /* 0: FP64 transforms; 1: FP32 nonlinear-term transforms with FP64
                            state, integrator and reductions (no reference counterpart)    */
    int32_t les_model;   /* 0: none; 1: Smagorinsky (m_les.f90:94-106); 2: dynamic localization
                            model (m_les.f90:111-123); 3: the same with the lag model for
                            the dissipation (m_les.f90:124-137); 4, 5: dynamic structure
                            model with the algebraic / lag dissipation (m_les.f90:138-190);
                            6, 7: mixed models, dynamic structure + C_mixed Smagorinsky
                            (m_les.f90:208-300); 10: one-equation mixed model with the
                            lag model and no k_sgs equation (m_les.f90:303-358).  2, 4, 6
                            carry k_sgs as state field 3+n_scalars; 3, 5, 7 k_sgs,
                            (B T_B), (eps T_eps) as fields 3+n_scalars .. 5+n_scalars;
                            10 (B T_B), (eps T_eps) as 3+n_scalars, 4+n_scalars; 2-10:
                            FP64 only, no passive scalars (so model 10's Harlow scalar
                            fluxes are not built); HIT3D_LES_LEARNED (20): learned
                            closure (hit3d_gpu_les_set_mlp; no reference counterpart). */
    int32_t scalar_type[HIT3D_MAX_SCALARS]; /* 0 = uniform mean gradient source            */
    int32_t device;      /* CUDA device ordinal                                            */
    int32_t reserved;
    double nu;           /* 1/RE (m_parameters.f90:275)                                    */
    double dt;           /* time step > 0 (m_parameters.f90:277-284)                       */
    double famp;         /* FAMP (m_parameters.f90:312)                                    */
    double c_smag;       /* Smagorinsky constant; the reference hard-codes 0.18 (m_les.f90:1148) */
    double sc[HIT3D_MAX_SCALARS]; /* Schmidt numbers; PE = nu/sc (m_parameters.f90:451)    */
    double c_t;          /* lag-model constant C_T of les_model 5 (the reference reads c_t.in,
                            m_les.f90:189-207); les_models 3 and 7 use C_T = 1             */
    double c_mixed;      /* fraction C_mixed of the Smagorinsky viscosity in les_models 6, 7,
                            10 (the reference reads c_mixed.in, m_les.f90:213-335)        */
    double reac_sc[HIT3D_MAX_SCALARS]; /* reaction rates; used by scalar_type 311 with
                            phase-shift dealiasing (rhs_scalars.f90:281-303)               */
} hit3d_params;

/* Allocate the device state, transform plans and wavenumber tables.
 * Replaces m_fields_init, m_work_init, x_fftw_allocate(1), x_fftw_init and
 * m_force_init (main.f90:27-36; x_fftw.f90:81-317; m_force.f90:13-97). */
int hit3d_gpu_init(const hit3d_params *p, hit3d_ctx **out);

/* Release everything (x_fftw_allocate(-1), x_fftw.f90:134-142). */
void hit3d_gpu_finalize(hit3d_ctx *ctx);

/* Message of the last failure on this thread. */
const char *hit3d_gpu_last_error(void);

/* Copy nfields Fourier-space fields between the host array fields(ld1, ny, nz, nfields)
 * (ld1 >= nx+2 reals) and the device.  nfields = 3 + n_scalars covers the state of
 * m_fields.f90:21.  Used where the reference reads or writes `fields` on the host:
 * begin_new/begin_restart (main.f90:56-60), restart_write_parallel (main.f90:173). */
int hit3d_gpu_upload_fields(hit3d_ctx *ctx, const double *fields, int64_t ld1, int32_t nfields);
int hit3d_gpu_download_fields(hit3d_ctx *ctx, double *fields, int64_t ld1, int32_t nfields);

/* Same for the AB2 history rhs_old (m_work.f90:109), so that a run can be moved
 * between host and device without restarting the integrator. */
int hit3d_gpu_upload_rhs_old(hit3d_ctx *ctx, const double *rhs_old, int64_t ld1, int32_t nfields);
int hit3d_gpu_download_rhs_old(hit3d_ctx *ctx, double *rhs_old, int64_t ld1, int32_t nfields);

/* Advance nsteps time steps, all on the device: rhs_scalars, AB2 scalars,
 * rhs_velocity (2/3 rule or phase shift, + Smagorinsky), force_velocity, AB2
 * velocities, pressure (main.f90:124-167).  *fov / *fos are the reference's
 * first-order flags (main.f90:71-72): non-zero means "take an Euler step"; both
 * are cleared on return as the reference clears them.  *courant receives the
 * Courant number of the last step (rhs_velocity.f90:31-38).  Particles, if
 * uploaded, move with the level-n velocity of every step (main.f90:235-247). */
int hit3d_gpu_step(hit3d_ctx *ctx, int32_t nsteps, int32_t *fov, int32_t *fos, double *courant);

/* Restart image in the reference's file layout, packed on the device
 * (restart_io.f90:240-334, restart_write_parallel): the 36-byte header (nx, ny,
 * nz, nums, nles as int32; TIME and DT as float64) followed, per variable, by the
 * Fourier array's first nx of its nx+2 rows ((nx, ny, nz) float64, column-major),
 * for the velocity, the first `nums` passive scalars (0..n_scalars; the host loop
 * writes 0 until the scalars are switched on) and the LES fields.  `image`: host
 * memory of hit3d_gpu_restart_bytes(ctx, nums) bytes (-1 on bad arguments); one
 * device-to-host copy per variable, no host re-layout.  The host writes the image
 * to <run_name>.64.<itime> as is. */
int64_t hit3d_gpu_restart_bytes(hit3d_ctx *ctx, int32_t nums);
int hit3d_gpu_restart_pack(hit3d_ctx *ctx, int32_t nums, double time, double dt, void *image);
/* The inverse (restart_read_parallel, restart_io.f90:341-506): checks the header's
 * dimensions against the context (the error names both) and the image size
 * against the header, loads the velocity, min(nums, n_scalars) scalars and
 * min(nles, the context's) LES fields, and zeroes the fields the image lacks
 * (the caller initialises added scalars, as init_scalar does in the reference)
 * and every kx = N/2 mode.  Returns TIME, DT and the header's counts. */
int hit3d_gpu_restart_unpack(hit3d_ctx *ctx, const void *image, int64_t bytes, double *time, double *dt,
                             int32_t *nums_file, int32_t *nles_file);

/* Steps with host-owned fields, pipelined over PCIe (no counterpart in the
 * reference, whose host owns `fields` and calls the step between copies,
 * main.f90:124-167).  For i = 0..nio-1: upload in[i] (nf fields in the reference
 * layout (ld1, ny, nz)), advance nsteps steps (flags as hit3d_gpu_step: the
 * first step of the call takes *fov/*fos), download the state into out[i].  The
 * upload of in[i+1] runs while step i and the download of out[i] run, on copy
 * streams of their own, so the host-to-device and device-to-host copies overlap.
 * in[i+1] must not share memory with out[i]; every array stays valid until the
 * call returns, and pinned host memory gives the full PCIe rate.  The staging
 * fields (3 nf fields in the reference layout: one input set, two output sets
 * used in turn) are allocated on first use.
 * band_only = 1 (2/3 rule only): only the modes with every |k_i| <= N/3 cross
 * PCIe (29.5 % of the array at 512^3), as box copies of the host arrays: the
 * values of in[i] outside that band are taken as zero, which a dealiased state
 * has there, and out[i] is written inside the band only (it must hold zeros
 * outside, e.g. from a download with band_only = 0).  The bytes a call moves
 * per input: hit3d_gpu_step_host_bytes(ctx, nf, band_only), each way. */
int hit3d_gpu_step_host(hit3d_ctx *ctx, int32_t nio, const double *const *in, double *const *out, int64_t ld1,
                        int32_t nf, int32_t nsteps, int32_t *fov, int32_t *fos, int32_t band_only);
int64_t hit3d_gpu_step_host_bytes(hit3d_ctx *ctx, int32_t nf, int32_t band_only);

/* The CUDA stream (cudaStream_t) every kernel of this context runs on, for
 * callers that time or order work around the library (the reference's
 * system_clock stage timers, m_timing.f90:48-73, x_fftw.f90:871-889). */
void *hit3d_gpu_stream(hit3d_ctx *ctx);

/* hit3d_gpu_step with CUDA events between the stages of every step;
 * ms[0..8) accumulates device time per stage: 0 inverse z pass (with spectral
 * pre-operation), 1 inverse y pass, 2 fused x pass (c2r, products, r2c),
 * 3 forward y pass, 4 forward z pass, 5 RHS/forcing/AB2/pressure update,
 * 6 Smagorinsky stress, 7 everything else (forcing energy, particles).  The
 * replacement of the reference's benchmark counters bm(1..12)
 * (main.f90:307-356). */
int hit3d_gpu_step_profile(hit3d_ctx *ctx, int32_t nsteps, int32_t *fov, int32_t *fos, double *ms);

/* Launch-shape tuner (no reference counterpart): times every launch-shape
 * variant of the fused x pass (row pairs per CTA, threads per CTA) on this
 * context's own work buffers and keeps the fastest; the state is not touched.
 * *variant receives the choice, ms[0..HIT3D_FUSED_VARIANTS) the time of each
 * variant (unused entries are left untouched).
 * hit3d_gpu_set_variant fixes a variant by hand. */
#define HIT3D_FUSED_VARIANTS 15
int hit3d_gpu_autotune(hit3d_ctx *ctx, int32_t *variant, double *ms);
/* Column-tile shape of the strided y and z passes (0: the default, 1: half, 2:
 * twice the kx columns per CTA, grids up to 512; 3: the pipelined passes, a grid
 * of resident CTAs that bring the tile after next into shared memory while they
 * transform the current one, every grid): times the passes of one step on the
 * context's work fields (the state is read, never written) and keeps the
 * fastest.  *tile receives it, ms[0..4) the times (0 for shapes not tried).  No
 * counterpart in the reference. */
int hit3d_gpu_autotune_columns(hit3d_ctx *ctx, int32_t *tile, double *ms);
/* Fix the column-tile shape (0-3 as above) instead of tuning it. */
int hit3d_gpu_set_column_tile(hit3d_ctx *ctx, int32_t tile);
int hit3d_gpu_set_variant(hit3d_ctx *ctx, int32_t variant);

/* 2/3-rule pruning (no reference counterpart; on by default).  With the 2/3
 * rule, when every mode with some |k_i| > N/3 is zero in the state (the
 * reference dealiases at start, dealias_all.f90, and its update keeps those
 * modes zero), the transforms of a step skip the columns, rows and outputs
 * that are zero or that the update masks (rhs_velocity.f90:85-142).  The
 * result is bit-identical; the state is checked on the device before the
 * first step after every change, and a state with energy beyond N/3 runs the
 * full transforms.  hit3d_gpu_pruned returns 1 if the next step is pruned. */
int hit3d_gpu_set_pruning(hit3d_ctx *ctx, int32_t on);
int hit3d_gpu_pruned(hit3d_ctx *ctx);

/* Without LES and with the 2/3 rule, the z forward pass of the six velocity
 * products runs inside the update kernel, so that the product spectra never
 * reach HBM, and within one hit3d_gpu_step call that kernel also writes the
 * next step's z inverse of the new velocity (the fields agree with the
 * separate passes to rounding; off by default, as the separate z passes +
 * update measured faster).  No counterpart in the reference. */
int hit3d_gpu_set_update_fusion(hit3d_ctx *ctx, int32_t on);

/* Failure detection (no reference counterpart: a diverged run of the
 * reference carries NaN into its files).  Counts, on the device, the
 * non-finite components of the state and the AB2 history; the host loop
 * checks it with the statistics and ends the run with an error status. */
int hit3d_gpu_check_finite(hit3d_ctx *ctx, int64_t *nonfinite);

/* The les.gp quantities of the last step of a dynamic-localization run
 * (les_model 2-7, 10; m_les.f90:876-892, the write of les_rhs_scalars):
 * out4 = {mean k_sgs ((B T_B) + (eps T_eps) for les_model 10), mean
 * production (2 nu_t S:S, -tau_ij du_i/dx_j for
 * the dynamic structure models, their sum for the mixed ones), mean B (0
 * without the lag model), mean dissipation (k^(3/2)/Delta; with the lag
 * model (eps T_eps)^(3/2)/(Delta C_T^(3/2)))}, all from the state at the
 * start of that step.  An error for any other les_model, as the reference
 * writes les.gp only when n_les > 0. */
int hit3d_gpu_les_stats(hit3d_ctx *ctx, double *out4);

/* Number of kernels this context has launched since hit3d_gpu_init. */
int64_t hit3d_gpu_launch_count(hit3d_ctx *ctx);

/* Change dt (my_dt.f90) and start/stop advancing scalars (int_scalars, main.f90:199-204). */
int hit3d_gpu_set_dt(hit3d_ctx *ctx, double dt);
int hit3d_gpu_set_scalars_active(hit3d_ctx *ctx, int32_t active);

/* Zero every mode with some |k_i| > kmax (dealias_all.f90:97-131). */
int hit3d_gpu_dealias_all(hit3d_ctx *ctx);

/* Initial velocity (init_velocity.f90:1-246): RANDu stream seeded with rn1 and
 * Box-Muller on the host (bit-exact with the reference), transform, curl and
 * shell rescale on the device.  isp_type -1 Taylor-Green, 0 Kolmogorov,
 * 1 exponential (peak_wavenum), 3 von Karman as the reference; 2 =
 * k^ir_exp exp(-2 (k/peak_wavenum)^2), a spectrum the reference does not have. */
int hit3d_gpu_init_velocity(hit3d_ctx *ctx, double rn1, int32_t isp_type, double peak_wavenum, double ir_exp);

/* Velocity statistics (m_stats.f90:99-289): e_spec[0..kmax) and
 * out[12] = energy, eps_v, eta, etakmax, uvar, x_length, lambda, re_lambda,
 * re_lambda1, tau_e, enstrophy, and the velocity-derivative skewness
 * (mean over a of <(du_a/dx_a)^3>/<(du_a/dx_a)^2>^{3/2}; no reference counterpart). */
int hit3d_gpu_stats(hit3d_ctx *ctx, double *e_spec, int32_t kmax, double *out12);

/* Scalar statistics for scalar s (m_stats.f90:295-440): spectrum[0..kmax)
 * (already doubled like the reference) and out5 = dissipation, mean, variance,
 * min, max. */
int hit3d_gpu_scalar_stats(hit3d_ctx *ctx, int32_t s, double *spectrum, int32_t kmax, double *out5);

/* init_scalar (init_scalars.f90:41-345) for passive scalar s, by its
 * scalar_type: 0 zero; 1, 2, 3 a random field with the normalised spectrum
 * of peak wavenumber `peak` (the RANDu stream of rn2 = RN2, continuing the
 * generator state the velocity's initial condition left, as the reference's
 * module state does; 3 then clipped to +-0.9); 11, 12, 13 the reference's
 * tanh and sine profiles.  Modes with some |k_i| > N/3 are zeroed. */
int hit3d_gpu_init_scalar(hit3d_ctx *ctx, int32_t s, double rn2, double peak);

/* particles_move with particles_filter_size > 0 (m_particles.f90:759-766): the
 * particles see the velocity filtered with the Gaussian of width delta
 * (m_filter_xfftw.f90:197-220).  delta <= 0 switches the filter off;
 * delta < 3 dx is an error, as in the reference. */
int hit3d_gpu_particles_filter(hit3d_ctx *ctx, double delta);

/* Lagrangian particles (m_particles.f90:157-337, 815-1230).  xyzp(3, np) in the
 * reference's grid units (x/dx + 1); uvwp(3, np) starts at -999 (Euler first
 * step).  scheme 0 = trilinear, 1 = 4-point cubic (CINT).  The whole field is
 * resident, so the slab halos and migration of the reference become periodic
 * wrap-around on one slab. */
int hit3d_gpu_particles_upload(hit3d_ctx *ctx, const double *xyzp, const double *uvwp, int64_t np, int32_t scheme);
int hit3d_gpu_particles_download(hit3d_ctx *ctx, double *xyzp, double *uvwp);

/* One 3-D transform of a single host array in the reference layout
 * (xFFT3d(flag, n), x_fftw.f90:852-1085): flag 1 physical -> Fourier
 * (unnormalised), flag -1 Fourier -> physical (times 1/N^3).  in and out are
 * (ld1, ny, nz) host arrays and may alias. */
int hit3d_gpu_xfft3d(hit3d_ctx *ctx, int32_t flag, const double *in, double *out, int64_t ld1);

/* Forward 3-D transform (as hit3d_gpu_xfft3d with flag 1) of one DEVICE array
 * that allocates nothing, for callers that cannot call cudaMalloc (a host whose
 * device memory is all handed out by its own pool allocator, or a loop that must
 * not risk the device-wide synchronisation of cudaMalloc/cudaFree).  No
 * counterpart in the reference.  `in` is a physical (nx+2, ny, nz) device array,
 * `out` receives the Fourier (nx+2, ny, nz) array; both belong to the caller
 * and must be 16-byte aligned.  They may be the same buffer (an in-place
 * transform) or overlap: the whole input is copied into the scratch array before
 * anything is written to `out`.  Work is queued on `stream` (a cudaStream_t,
 * NULL = default stream) and the caller synchronises.  Grid sizes 32, 48, 64 and
 * 128 only: the one scratch field lives in a file-scope __device__ array (17 MB,
 * held on every GPU that loads the library until the process exits).  The first
 * call in each CUDA context of a device (again after a device reset) resolves
 * that array's address and uploads twiddle tables, so make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race and
 * must be serialised by the caller. */
int hit3d_gpu_xfft3d_static(int32_t n, const double *in, double *out, void *stream);

/* Filter Fourier-space field `field` of the state in place
 * (filter_xfftw_fields, m_filter_xfftw.f90:74-110).  kind 2 = Gaussian kernel
 * built in physical space and transformed as the reference does
 * (m_filter_xfftw.f90:197-220); kind 4 = box filter of width delta, transfer
 * function prod sin(k delta/2)/(k delta/2) (no reference counterpart). */
int hit3d_gpu_filter_field(hit3d_ctx *ctx, int32_t kind, double delta, int32_t field);

/* Training data of a learned subgrid closure from the current (DNS) state: with
 * the filter of hit3d_gpu_filter_field (kind 2 Gaussian, 4 box of width delta),
 * out receives 18 compact float32 fields (nx, ny, nz) in this order:
 *   ubar_1..3   filtered velocity,
 *   tau_11, tau_12, tau_13, tau_22, tau_23, tau_33   exact subgrid stress
 *               filter(u_i u_j) - ubar_i ubar_j (the Leonard-stress formula of
 *               m_les.f90:1847-1865 applied to the DNS field),
 *   A_ij = d ubar_i / dx_j, i-major (9 fields).
 * Needs FP64 transforms (precision 0); uses 6 extra fields of device memory. */
int hit3d_gpu_sgs_fields(hit3d_ctx *ctx, int32_t kind, double delta, float *out);
/* The same on every stride-th point per axis (stride divides nx):
 * out(18, m, m, m) with m = nx / stride. */
int hit3d_gpu_sgs_samples(hit3d_ctx *ctx, int32_t kind, double delta, int32_t stride, float *out);

/* Physical-space copies of the first nf state fields, out(ld1, ny, nz, nf), with
 * every mode of |k|^2 > k2max zeroed first when k2max > 0 (the spherical
 * truncation and inverse transforms of io_write_4, io_write_4.f90:21-90; the
 * caller converts to real*4 and writes the files). */
int hit3d_gpu_physical_fields(hit3d_ctx *ctx, int32_t nf, double k2max, double *out, int64_t ld1);

/* Rescale the velocity to the initial spectrum of type isp_type for decaying
 * runs (velocity_rescale.f90:1-159); called by the host every TRESCALE in time
 * (main.f90:111-121). */
int hit3d_gpu_velocity_rescale(hit3d_ctx *ctx, int32_t isp_type, double peak_wavenum, double ir_exp);

/* Physical-space velocity (x, y, z) of the current state, as the reference's
 * wrk1..3 after rhs_scalars (main.f90:126): out(ld1, ny, nz, 3). */
int hit3d_gpu_physical_velocity(hit3d_ctx *ctx, double *out, int64_t ld1);

/* ---------------------------------------------------------------------------
 * Batched form (no reference counterpart: the reference runs one simulation per
 * MPI job).  Many independent runs of uneven sizes, each with its own
 * parameters (Re, seeds), on one GPU.  Runs that share a grid size, precision
 * and forcing and carry the velocity only with the 2/3 rule form a size class:
 * their state and work fields sit in one slab, and every pass of a step is one
 * launch over all the class's runs (per-run viscosity, time step and forcing
 * energy in device tables).  Other runs step on their own.  hit3d_batch_step
 * takes the first-order step of new runs eagerly, then records `graph_steps`
 * Adams-Bashforth steps of all classes and runs into one CUDA graph (a branch
 * per class or lone run) and replays it, one launch per chunk.  dt and the
 * scalar switch are baked into the recording: change them (hit3d_gpu_set_dt,
 * hit3d_gpu_set_scalars_active on a run's context) only between calls; the next
 * call re-records the graph when either, or graph_steps, has changed.
 * ------------------------------------------------------------------------- */
typedef struct hit3d_batch hit3d_batch;
int hit3d_batch_create(const hit3d_params *p /* [nruns] */, int32_t nruns, hit3d_batch **out);
/* The context of run r, for initial conditions, transfers and statistics. */
int hit3d_batch_context(hit3d_batch *b, int32_t r, hit3d_ctx **ctx);
int hit3d_batch_step(hit3d_batch *b, int32_t nsteps, int32_t graph_steps);
/* Number of graph launches so far. */
int64_t hit3d_batch_graph_launches(hit3d_batch *b);
/* Number of size classes (ordered by their first run). */
int hit3d_batch_nclasses(hit3d_batch *b);
/* Per size class, time the fused x-pass launch shapes that walk several runs
 * (variants 8-14) and the column-tile shapes of the strided passes (0: the
 * default, 1: half, 2: twice the kx columns per CTA, grids up to 512; 3: the
 * pipelined passes) on the
 * class's own buffers, reading the state without changing it, and keep the
 * fastest of each.  choice[2k], choice[2k+1] receive class k's picks; ms (may
 * be NULL) receives 11 times in ms per class (7 x-pass variants, then 4 tiles,
 * NaN-free: tiles not tried report 0).  The next step re-records the graph. */
int hit3d_batch_autotune(hit3d_batch *b, int32_t *choice, double *ms);
void hit3d_batch_destroy(hit3d_batch *b);

/* ---------------------------------------------------------------------------
 * Learned subgrid closure (no reference counterpart; the reference's LES models
 * are in m_les.f90, and its Smagorinsky model, m_les.f90:1142-1215, is the
 * fallback).  A network g = MLP(x), 6 -> 64 -> 64 -> 64 -> 5 with GELU, maps
 * five invariants of the normalised filtered velocity gradient and the filter
 * width to the coefficients of a five-tensor basis, and
 *     tau_ij = Delta^2 |S|^2 sum_n g_n T^(n)_ij      (deviatoric).
 * Weights are bf16, every product is accumulated in fp32.  Parameters are a
 * flat fp32 vector of hit3d_mlp_nparam() values: W1[64][6] b1[64] W2[64][64]
 * b2[64] W3[64][64] b3[64] W4[5][64] b4[5].  Gradient fields A are [9][P]
 * with A[3i+j] = d u_i / d x_j; stresses are [6][P] in the order
 * 11 12 13 22 23 33.
 * ------------------------------------------------------------------------- */
typedef struct hit3d_mlp hit3d_mlp;
int hit3d_mlp_nparam(void);
/* Glorot-uniform initial weights from `seed`. */
int hit3d_mlp_create(int32_t device, uint64_t seed, hit3d_mlp **out);
int hit3d_mlp_destroy(hit3d_mlp *m);
/* fp32 master parameters; setting them also resets the Adam moments. */
int hit3d_mlp_set_params(hit3d_mlp *m, const float *w);
int hit3d_mlp_get_params(hit3d_mlp *m, float *w);
/* the bf16 weights the kernels use (raw bf16 bit patterns) */
int hit3d_mlp_get_bf16(hit3d_mlp *m, uint16_t *wb);
/* Training data from filtered DNS (hit3d_gpu_sgs_fields): gradients and
 * stresses at P points, filter width delta.  Stresses are made deviatoric. */
int hit3d_mlp_set_data(hit3d_mlp *m, const float *A, const float *tau, int64_t P, double delta);
/* out2 = {1 / mean |tau|_F^2, 1 / mean (tau:S)^2} over the data set */
int hit3d_mlp_norms(hit3d_mlp *m, double *out2);
/* Loss and its gradient with respect to the parameters (evaluated at the bf16
 * weights) for the data points idx[0..np):
 *   L = n1/np sum |tau_pred - tau|_F^2 + lam n2/np sum (tau_pred:S - tau:S)^2 */
int hit3d_mlp_loss_grad(hit3d_mlp *m, const int32_t *idx, int64_t np, double lam, float *loss, float *grad);
/* nsteps Adam steps (lr, betas 0.9/0.999) on minibatches of `batch` points
 * drawn from the data set by a hash of (seed, step); losses[nsteps] may be null. */
int hit3d_mlp_train(hit3d_mlp *m, int32_t nsteps, int64_t batch, double lr, double lam, uint64_t seed, float *losses);
/* Stresses predicted at np points; with clip, points whose predicted
 * dissipation -tau:S is negative get tau = 0.  kernel 0 keeps every
 * activation in fp32 on the CUDA cores (the training kernels' arithmetic);
 * kernel 1 runs the two hidden 64x64 layers on the tensor cores (tcgen05,
 * TMEM accumulators) with their inputs rounded to bf16. */
int hit3d_mlp_predict(hit3d_mlp *m, const float *A, int64_t np, double delta, int32_t clip, int32_t kernel,
                      float *tau);
/* Use a trained network as the context's subgrid model (les_model 20): nparam
 * bf16 weights, the filter width they were trained for, the clip switch and
 * the inference kernel (as in hit3d_mlp_predict). */
int hit3d_gpu_les_set_mlp(hit3d_ctx *ctx, const uint16_t *bf16_weights, int64_t nparam, double delta, int32_t clip,
                          int32_t kernel);

#ifdef __cplusplus
}
#endif

#endif /* HIT3D_GPU_H */
