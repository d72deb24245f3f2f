/*
 * fgpe.h -- C ABI of the B200 split-step spinor GPE propagator.
 *
 * The reference FORTRESS programs (SRC/cgpe1d.f90, cgpe2d.f90, cgpe3d.f90) keep
 * the state in module globals PHI/PHIF and advance it with argument-less
 * subroutines called from the main loop:
 *     FFT, KE, SOC, BFT, SE, SP, NORMC, NORMT      (cgpe1d.f90:433-474)
 *     ENERGY, RAD, CONV/CONV_EN                     (cgpe1d.f90:476-487)
 * with their interfaces declared at cgpe1d.f90:117-198 (2D: cgpe2d.f90:118-200,
 * 3D: cgpe3d.f90:122-205).  This header is the seam that replaces them: a
 * handle owns the device-resident state, one call advances whole split steps
 * (imaginary-time renormalisation included), and the observables come back as
 * plain doubles.  A Fortran host binds it with ISO_C_BINDING.
 *
 * Conventions
 *   - Every function returns 0 (FGPE_OK) on success and a negative FGPE_E*
 *     code on failure; fgpe_last_error() gives a message for the handle.
 *   - State arrays on the host are Fortran column-major PHI(NX,NY,NZ,M),
 *     M = 2*SPIN+1, complex128 stored as interleaved (re, im) doubles, exactly
 *     the reference's PHI layout.
 *   - One host thread per handle; calls on a handle are ordered on the
 *     handle's CUDA stream.  The library owns all device memory of a handle.
 *   - There is no CPU fallback: without a usable sm_100 device every call that
 *     needs the GPU fails with FGPE_E_CUDA.
 */
#ifndef FGPE_H
#define FGPE_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    FGPE_OK = 0,
    FGPE_E_ARG = -1,        /* invalid argument / unsupported size */
    FGPE_E_CUDA = -2,       /* CUDA runtime error (message in fgpe_last_error) */
    FGPE_E_STATE = -3,      /* call out of order (e.g. no state set) */
    FGPE_E_NONFINITE = -4,  /* a reduction produced NaN/Inf */
    FGPE_E_NEWTON = -5,     /* spin-2 magnetisation projection: Newton-Raphson
                               did not converge (cgpe1d.f90:1287-1290) */
    FGPE_E_TIMEOUT = -6     /* a bounded device-side wait of the persistent
                               batch kernel ran out; the batch's states are
                               not those of whole steps */
};

enum { FGPE_FP64 = 0, FGPE_FP32 = 1 };
enum { FGPE_KERNELS_AUTO = 0, FGPE_KERNELS_GENERIC = 1,
       FGPE_KERNELS_FAST_ROW_ONLY = 2, FGPE_KERNELS_FAST_COL_ONLY = 3,
       FGPE_KERNELS_SPLIT_1D = 4,  /* 1D: the N1 x N2 split as two passes per
                                      step, even for short lines */
       FGPE_KERNELS_SINGLE_1D = 5, /* 1D: the single-block kernel whenever the
                                      line fits one block (200 KB) */
       FGPE_KERNELS_CLUSTER_1D = 6,/* 1D: the N1 x N2 split on one 8-CTA
                                      thread-block cluster for a whole call,
                                      even for short lines (N1 and N2 multiples
                                      of 8; fgpe_create fails otherwise).  The
                                      default for split lines of N*M <= 10240
                                      when the cluster fits. */
       FGPE_KERNELS_WARP_ROW = 7,  /* size-specialised kernels with the row pass
                                      on one warp per x row (warp-private
                                      shared memory, no block barriers in the
                                      transforms) where the MS lines of a row
                                      fit 16 KB, in either precision; AUTO
                                      takes this row pass for FP64 */
       FGPE_KERNELS_BLOCK_ROW = 8  /* size-specialised kernels with the
                                      block-tiled row pass everywhere */ };

/* Step flags for fgpe_step_ex. */
enum {
    FGPE_STEP_DEFAULT = 0,
    FGPE_STEP_NO_SNAPSHOT = 1   /* keep the state in the spectral work buffer
                                   only; the real-space copy is rebuilt lazily */
};

/* Physical and numerical parameters of one instance.  Field meanings follow
 * the reference's input records (README.md:53-86) and derived quantities
 * (cgpe1d.f90:263-271, 321-332). */
typedef struct fgpe_params {
    int dim;            /* 1, 2 or 3 (which cgpe{1,2,3}d program) */
    int spin;           /* SPIN: 1 or 2 */
    int nx, ny, nz;     /* NX, NY, NZ (unused dimensions = 1) */
    double dx, dy, dz;  /* DX, DY, DZ */
    double dt;          /* DT */
    int imag_time;      /* SWITCH_IM: 1 imaginary time (CDT=-i DT), 0 real */
    double tau[3];      /* TAU(0:2) in the reference's units (tau includes x2) */
    double gamma[3];    /* GAMMAX, GAMMAY, GAMMAZ */
    double alpha[3];    /* ALPHAX, ALPHAY, ALPHAZ = NU{X,Y,Z}/NUX */
    int precision;      /* FGPE_FP64 or FGPE_FP32 (FP32 FFTs/exponentials,
                           FP64 reductions and renormalisation) */
    int kernels;        /* FGPE_KERNELS_AUTO: size-specialised persistent
                           kernels where compiled, else generic;
                           FGPE_KERNELS_GENERIC: generic kernels only */
    double mag;         /* MAG: magnetisation imposed in imaginary time when
                           all GAMMA are zero (cgpe1d.f90:257, 443-470) */
    int reserved[4];
} fgpe_params;

typedef struct fgpe_s fgpe_t;

/* Handle lifecycle.  Replaces ALLOCATE_MEM/INITIALIZE's grid set-up and
 * CREATE_PLANS (cgpe1d.f90:568-589, 692-710, 796-807). */
int fgpe_create(const fgpe_params *p, fgpe_t **out);
int fgpe_destroy(fgpe_t *h);                      /* DEALLOCATE_MEM, DESTROY_PLANS */
const char *fgpe_last_error(const fgpe_t *h);     /* NULL handle: last global error */
int fgpe_set_stream(fgpe_t *h, void *cuda_stream);/* cudaStream_t, NULL = library's own */

/* State transfer (host buffers, layout above).  Replaces the direct access to
 * module PHI and the initial_sol reader's assignment (cgpe1d.f90:377-391). */
int fgpe_set_state(fgpe_t *h, const double *phi_host);
int fgpe_get_state(fgpe_t *h, double *phi_host);
/* Device-pointer variants (complex128 or complex64 per precision is NOT used
 * here: these always take complex128 in the same layout). */
int fgpe_set_state_device(fgpe_t *h, const void *phi_dev);
int fgpe_get_state_device(fgpe_t *h, void *phi_dev);

/* Advance nsteps whole Lie split steps
 *   FFT -> KE -> SOC -> BFT -> SE -> SP -> NORMC [-> NORMT if imaginary time]
 * (cgpe1d.f90:433-474 for the SO-coupled branch). */
int fgpe_step(fgpe_t *h, int nsteps);
int fgpe_step_ex(fgpe_t *h, int nsteps, int flags);

/* NORMT (cgpe1d.f90:998-1031): divide the state by sqrt(total Simpson norm);
 * tnorm (may be NULL) receives TNORM. */
int fgpe_normalize(fgpe_t *h, double *tnorm);

/* NORMC of the state after the last step's SP, before renormalisation
 * (cgpe1d.f90:441; what file1/file3 report).  Before any step: NORMC of the
 * current state.  norm[M]. */
int fgpe_norms(fgpe_t *h, double *norm);

/* ENERGY + RAD of the current state (cgpe1d.f90:1077-1240, 1036-1072):
 * en, mu[M], mz, rms[M] exactly as the reference defines them (not halved). */
int fgpe_observables(fgpe_t *h, double *en, double *mu, double *mz, double *rms);

/* max |PHI - PHI_OLD| over all points and components, PHI_OLD being the state
 * one step before the current one (cgpe1d.f90:482, without the STP*2*DT
 * divisor).  Valid after an fgpe_step call of at least one step. */
int fgpe_conv(fgpe_t *h, double *max_dphi);

/* Component values at the grid centre PHI(NX/2+1, NY/2+1, NZ/2+1, :) (the
 * |phi| columns of file1, cgpe1d.f90:407).  out[2*M] interleaved. */
int fgpe_center(fgpe_t *h, double *out);

/* Unfused single operators in the reference's order, for operator-level
 * parity checks.  They act on the handle's state: FGPE_OP_FFT moves it to
 * Fourier space (unnormalised), KE/SOC act there, FGPE_OP_BFT moves it back
 * (divided by NX*NY*NZ), SE/SP act in real space.  Replaces the individual
 * subroutines FFT/KE/SOC/BFT/SE/SP (cgpe1d.f90:1324, 826, 1504, 1343, 1363,
 * 847). */
enum { FGPE_OP_FFT = 1, FGPE_OP_KE = 2, FGPE_OP_SOC = 3, FGPE_OP_BFT = 4,
       FGPE_OP_SE = 5, FGPE_OP_SP = 6 };
int fgpe_apply_op(fgpe_t *h, int op);

/* Non-blocking variant of fgpe_norms: enqueues the copy of the last step's
 * NORMC (M doubles) into dst, valid after the handle's stream has been
 * synchronised.  Pinned host memory and device memory of the handle's device
 * are written by a one-warp kernel in the step chain (no copy-engine
 * transfer between steps); other memory takes an asynchronous copy. */
int fgpe_norms_async(fgpe_t *h, double *dst);

/* Per-step NORMC without a call per step: after this call, every split step
 * of the handle appends its NORMC (M doubles) to the ring dst[count][M], in
 * step order, wrapping after count records; the step's own last block writes
 * it (no extra kernel or copy).  dst is pinned host memory or memory of the
 * handle's device, valid after the handle's stream has been synchronised; the
 * record index restarts at 0 with each call.  dst = NULL stops it.  A batch
 * graph captured before the call keeps the ring it was captured with. */
int fgpe_norms_sink(fgpe_t *h, double *dst, int count);

/* Kernel timing with CUDA events recorded on the handle's stream around
 * every kernel that fgpe_step launches.  fgpe_profile_read synchronises,
 * adds the elapsed times per kernel class -- [0] row pass (x), [1] column
 * pass y, [2] column pass z, [3] single-block 1D kernel -- into ms[4] and the
 * launch counts into n[4], and clears the record when reset != 0. */
int fgpe_profile_enable(fgpe_t *h, int on);
int fgpe_profile_read(fgpe_t *h, double *ms, long long *n, int reset);

/* ------------------------------------------------------------------ batches
 * Many independent instances (ragged grid sizes, per-instance parameters)
 * advanced together: every instance's split steps are captured as a parallel
 * branch of one CUDA graph (instance i on branch i % width) and the graph is
 * replayed with one launch per steps_per_graph steps.  The reference has no
 * counterpart (it runs one configuration per process); this is the sweep
 * launcher over parameter points.  Instances are ordinary handles: set their
 * states and read their observables through fgpe_batch_instance(). */
typedef struct fgpe_batch_s fgpe_batch_t;
int fgpe_batch_create(const fgpe_params *p, int count, fgpe_batch_t **out);
int fgpe_batch_destroy(fgpe_batch_t *b);
int fgpe_batch_size(const fgpe_batch_t *b);
int fgpe_batch_instance(fgpe_batch_t *b, int i, fgpe_t **h);
const char *fgpe_batch_last_error(const fgpe_batch_t *b);
/* width: concurrent graph branches (<= count); steps_per_graph: steps
 * captured per graph launch (>= 2).  Non-positive values keep the setting. */
int fgpe_batch_config(fgpe_batch_t *b, int width, int steps_per_graph);
int fgpe_batch_step(fgpe_batch_t *b, int nsteps);
/* As fgpe_batch_step, and device_ms receives the device time between CUDA
 * events recorded on the batch's launch stream around its graph launches.
 * nsteps >= 2 and nsteps % steps_per_graph != 1 (whole graphs only). */
int fgpe_batch_step_timed(fgpe_batch_t *b, int nsteps, double *device_ms);
/* For every instance i in order, 3+3*M_i doubles: EN, MZ, CONV (max|dphi|
 * of the last step, or -1), MU[M_i], RMS[M_i], NORM[M_i]. */
int fgpe_batch_observables(fgpe_batch_t *b, double *out, int with_conv);

/* Launch organisation of a batch.  FGPE_BATCH_BRANCHES (the default): every
 * instance's passes are launches of their own, in parallel graph branches.
 * FGPE_BATCH_GROUPED: instances that share a q2D grid shape, spin and
 * precision (both axes of a size-specialised length: 128, 192, 256, 384,
 * 512) advance together, one column-pass and one row-pass launch per step
 * for the whole group, each launch walking the tiles of all its instances;
 * the other instances keep their own branches.  The results are those of
 * the single-instance passes up to the NORMC summation order. */
/* FGPE_BATCH_PERSISTENT: the same instances (any mix of those grid sizes,
 * per spin and precision) advance by ONE persistent kernel launch per
 * captured graph of K steps.  Its blocks take work items (column tiles, then
 * row chunks, of every instance, step after step) from a device ticket
 * counter; per-instance device counters order a step's row pass after its
 * column pass and the next step after the NORMC of this one, so instances
 * of different sizes overlap.  Every device-side wait is bounded
 * (fgpe_batch_wait_bound); when one runs out the step call returns
 * FGPE_E_TIMEOUT.  No counterpart in the reference (one instance per
 * ./cgpe.x process; its loop at cgpe2d.f90:440-531). */
enum { FGPE_BATCH_BRANCHES = 0, FGPE_BATCH_GROUPED = 1, FGPE_BATCH_PERSISTENT = 2 };
int fgpe_batch_mode(fgpe_batch_t *b, int mode);

/* Persistent kernel variant (0 .. fgpe_batch_variants()-1) of the batch:
 * variant >= 0 selects one, -1 keeps the current; *current (may be NULL)
 * receives the selection.  fgpe_batch_variant_shape writes the variant's
 * shape[4] = {threads per block, values per row tile, bytes of x per column
 * tile row, radix plan of the y lines (0: radix 8 first, then 4 or 2;
 * 1: 4*4 in place of a trailing 8*2; 2: plan 0 reversed; 3: a radix-16
 * pass first where it saves a pass, 128 = 16*8, 256 = 16*16, 384 = 16*8*3)}. */
int fgpe_batch_variant(fgpe_batch_t *b, int variant, int *current);
int fgpe_batch_variant_shape(int variant, int *shape);
int fgpe_batch_variants(void);
/* Bound on one device-side wait of the persistent kernel (ms of device
 * time, default 2000).  stall_instance >= 0 is a test hook: that instance's
 * first row wait then waits for a count no block produces, so the bound
 * runs out and the step returns FGPE_E_TIMEOUT (-1: none). */
int fgpe_batch_wait_bound(fgpe_batch_t *b, double wait_ms, int stall_instance);

/* Autotuner: times kernel family per grid-size class, branch width and
 * steps per graph with one graph branch per instance, the grouped mode, and
 * the persistent mode with every kernel variant (threads per block, row and
 * column tile shapes, radix plan of the y lines), on the batch itself
 * (states saved and restored) and keeps the fastest; cache_path (may be
 * NULL) remembers the choice per batch signature.  fgpe_batch_tuning
 * reports the current width and steps, fgpe_batch_mode-/variant the rest. */
int fgpe_batch_autotune(fgpe_batch_t *b, int trial_steps, const char *cache_path);
int fgpe_batch_tuning(const fgpe_batch_t *b, int *width, int *steps_per_graph);

/* Switch one handle between the size-specialised and the generic kernels
 * (same data layout, so this can happen between any two calls). */
int fgpe_set_kernels(fgpe_t *h, int kernels);

/* Full-precision checkpoint of the handle's state (no reference
 * counterpart: FORTRESS restarts only from the F18.10 text of initial_sol).
 * The raw device buffers, pending scales, last NORMC and the projection's
 * Newton start values are written, so fgpe_checkpoint_load into a handle of
 * the same grid, spin and precision continues bit-identically.  step and
 * user[8] (may be NULL) are stored for the caller (e.g. II and EN_OLD).
 * The file is written to path.tmp and renamed; a checksum guards loading. */
int fgpe_checkpoint_save(fgpe_t *h, const char *path, long long step, const double *user);
int fgpe_checkpoint_load(fgpe_t *h, const char *path, long long *step, double *user);

/* NORMC of a spinor the caller already holds on the device, with no handle
 * and no allocation of any kind: for callers that may not allocate device
 * memory, such as a host code whose device memory is reserved up front by
 * its own pool or a solver that must not synchronise the device in the
 * middle of a run (cudaMalloc/cudaFree synchronise).  No counterpart in the
 * reference.
 *   phi_dev: complex128, the PHI layout of fgpe_set_state; norm_dev: 2*spin+1
 *   doubles of device memory; stream: cudaStream_t (NULL = legacy default).
 * Asynchronous: the result is in norm_dev once the stream reaches it.
 * Limits: every used axis an even number >= 8 of points (the reference's
 * Simpson rule), and (ny*nz lines) x (2*spin+1) <= 262144, the size of the
 * library's fixed 2 MiB scratch; larger grids return FGPE_E_ARG.  Every call
 * looks the scratch up (cudaGetSymbolAddress) in the context current at the
 * call; the first call in a context also loads the library's device code
 * there, so make it before any stream capture.  Calls on one device share
 * the scratch: never have two in flight at once. */
int fgpe_normc_noalloc(int dim, int spin, int nx, int ny, int nz, double dx, double dy, double dz,
                       const void *phi_dev, double *norm_dev, void *stream);

/* Library / device information. */
int fgpe_version(void);
int fgpe_device_ok(void);                /* 1 if an sm_100 device is usable */
int fgpe_kernel_launches(fgpe_t *h, long long *count);  /* kernels launched */
/* FP64 FMA throughput of the current device in TFLOP/s (2 flops per FMA),
 * from a CUDA-event-timed launch of independent FMA chains on every SM: the
 * compute-roofline denominator of the step kernels, whose exponentials,
 * spin-2 matrix products and FFT butterflies run on the FP64 pipe.  No
 * counterpart in the reference (a measurement aid). */
int fgpe_fp64_fma_rate(int iters, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* FGPE_H */
