/*
 * fdtd_b200.h - C ABI of the B200-native FDTD leapfrog step.
 *
 * This is the drop-in boundary for fdtd3d's GPU step path.  In the reference,
 * Scheme<...> drives the step through the InternalSchemeGPU object protocol
 * (initFromCPU / initOnGPU / copyFromCPU / copyToGPU / the *KernelLaunch
 * methods / copyBackToCPU).  Each entry point below replaces one part of that
 * protocol; the comment on each names the reference interface it replaces
 * (paths relative to the fdtd3d source tree).
 *
 * Conventions
 *  - Every entry returns an int status: 0 = FDTD_OK, negative = error
 *    (fdtd_status_str gives the text).  No entry calls exit, abort or
 *    __trap; the reference's cudaCheckError -> exit(1) and ALWAYS_ASSERT
 *    become status codes the caller maps back.
 *  - Arrays are x-major with z fastest, the order of the reference's
 *    CudaGrid linear index x*sy*sz + y*sz + z (Source/Grid/CudaGrid.cu:1096)
 *    and of its TXT dumps.  2-D TMz arrays are (x, y) with y fastest.
 *  - Host input arrays are borrowed for the duration of the call and copied.
 *    Output buffers are owned by the caller.
 *  - Calls on one context are serialised by the caller; separate contexts
 *    may live on separate host threads.
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fdtd_ctx fdtd_ctx;

/* status codes */
#define FDTD_OK 0
#define FDTD_ERR_ARG (-1)        /* invalid argument or configuration */
#define FDTD_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define FDTD_ERR_NOMEM (-3)      /* device or host allocation failed */
#define FDTD_ERR_TIMEOUT (-4)    /* bounded wait ran out */
#define FDTD_ERR_UNSUPPORTED (-5)/* mode/option combination not provided */
#define FDTD_ERR_STATE (-6)      /* call out of order (e.g. step before setup) */
#define FDTD_ERR_DEVICE (-7)     /* a kernel reported an error flag */

/* modes (fdtd3d SchemeType).  A 2-D mode keeps the fields of one plane;
 * its grid has size 1 along the third axis (size[] of that axis is ignored)
 * and its arrays are the plane's two axes in x, y, z order, the second
 * fastest. */
#define FDTD_MODE_TMZ 2          /* Dim2_TMz: Ez, Hx, Hy in the x-y plane */
#define FDTD_MODE_DIM3 3         /* Dim3: Ex, Ey, Ez, Hx, Hy, Hz */
#define FDTD_MODE_TEX 4          /* Dim2_TEx: Ey, Ez, Hx in the y-z plane */
#define FDTD_MODE_TEY 5          /* Dim2_TEy: Ex, Ez, Hy in the x-z plane */
#define FDTD_MODE_TEZ 6          /* Dim2_TEz: Ex, Ey, Hz in the x-y plane */
#define FDTD_MODE_TMX 7          /* Dim2_TMx: Ex, Hy, Hz in the y-z plane */
#define FDTD_MODE_TMY 8          /* Dim2_TMy: Ey, Hx, Hz in the x-z plane */
/* 1-D modes keep one axis (sizes of the other two are ignored) */
#define FDTD_MODE_EXHY 10        /* Dim1_ExHy: Ex, Hy along z */
#define FDTD_MODE_EXHZ 11        /* Dim1_ExHz: Ex, Hz along y */
#define FDTD_MODE_EYHX 12        /* Dim1_EyHx: Ey, Hx along z */
#define FDTD_MODE_EYHZ 13        /* Dim1_EyHz: Ey, Hz along x */
#define FDTD_MODE_EZHX 14        /* Dim1_EzHx: Ez, Hx along y */
#define FDTD_MODE_EZHY 15        /* Dim1_EzHy: Ez, Hy along x */

/* arithmetic forms */
#define FDTD_PREC_FP64_PLAIN 0   /* reference formulation, FP64, bit-faithful */
#define FDTD_PREC_FP32 1         /* fused step, FP32 storage and compute */
#define FDTD_PREC_FP16S 2        /* fused step, FP16 field storage, FP32 compute */

/* field components (fdtd3d GridType order) */
#define FDTD_EX 0
#define FDTD_EY 1
#define FDTD_EZ 2
#define FDTD_HX 3
#define FDTD_HY 4
#define FDTD_HZ 5

/* material grids (fdtd3d GridType EPS, MU, OMEGAPE, OMEGAPM, GAMMAE, GAMMAM) */
#define FDTD_MAT_EPS 0
#define FDTD_MAT_MU 1
#define FDTD_MAT_OMEGAPE 2
#define FDTD_MAT_OMEGAPM 3
#define FDTD_MAT_GAMMAE 4
#define FDTD_MAT_GAMMAM 5

/* reductions */
#define FDTD_REDUCE_ENERGY 0     /* sum over cells of eps*E^2 + mu*H^2 (FP64, compensated) */
#define FDTD_REDUCE_L2 1         /* sum over cells of E^2 + H^2, per component (6 doubles) */

/*
 * Run configuration.  Mirrors fdtd3d's Settings flags (Source/Settings/Settings.inc.h):
 * --3d/--2d-te{x,y,z}/--2d-tm{x,y,z}/--1d-*, --size, --pml-size, --tfsf-size-left/right, --dx, --wavelength,
 * --courant-factor, --angle-teta/phi/psi, --use-pml, --use-tfsf,
 * --use-metamaterials, --point-source, --point-source-e*, --layout-type.
 * Float flags hold the values exactly as the reference parses them
 * (std::stof, i.e. rounded to float).
 */
typedef struct
{
  int mode;                 /* FDTD_MODE_* */
  int size[3];              /* the axis a 2-D mode drops is ignored */
  int pml[3];
  int tfsf_left[3];         /* >= 1 */
  int tfsf_right[3];        /* >= 0 (0: no face on that side) */
  double dx;
  double wavelength;
  double courant;
  double angle_teta;        /* degrees */
  double angle_phi;
  double angle_psi;
  int use_pml;
  int use_tfsf;
  int use_metamaterials;    /* requires use_pml, as in the reference */
  int point_source[3];
  int point_source_mask;    /* bit c: hard source on component c */
  int point_source_kind;    /* 0: the reference's sin(2 pi f t); 1: Gaussian-modulated (see below) */
  double point_source_bandwidth; /* kind 1: spectral FWHM / f (e.g. 0.5) */
  int precision;            /* FDTD_PREC_* */
  int layout;               /* 0 = E_CENTERED, 1 = H_CENTERED (--layout-type) */
  int source_phase;         /* 0: sine sources; 1: cosine sources.  The reference's complex-field
                               build drives sin + i cos (InternalScheme.inc.h:2888-2890, 3312-3313);
                               with real materials its fields are the run with phase 0 plus i times
                               the run with phase 1 */
  int current_source[3];    /* --current-source: the cell of the J / M current sources */
  int current_source_mask;  /* bit c: current on component c (Jx Jy Jz = 0-2, Mx My Mz = 3-5;
                               --current-source-jx .. -mz).  After the curl update of that
                               component, before D -> E, the cell takes -= I dx Cb with
                               I = s(t) mu0 / dt / 2, t the component's time (t on E, t + 1/2
                               on H) (Scheme.inc.h:1171-1260, InternalScheme.inc.h:2423-2449) */
  int current_phase;        /* s(t): 0 = sin(w t), the real build; 1 / 2 = the real / imaginary
                               part of the complex build's cos(w (t - 1)) - i sin(w (t - 1)) */
  int double_material_precision; /* --use-double-material-precision: eps, mu and the PML sigma
                               live on a grid of twice the resolution on every kept axis (2 n, PML
                               2 p cells); a component averages the 2 x 2 x 2 fine cells around it
                               (YeeGridLayout.h:866-1030, Approximation.cpp:48-54,
                               SchemeHelper.h:596-718).  fdtd_upload_material then takes eps and mu
                               on that grid.  Not with metamaterials (the reference's eight-point
                               Drude average is unreachable, Approximation.cpp:167-197) */
  int reserved[1];
} fdtd_config;

/* Point-source kinds.  Kind 0 is the reference's hard source
 * sin(2 pi f dt (t + 1/2)) on E, (t + 1) on H (InternalScheme.inc.h:2818-2895).
 * Kind 1 (no counterpart in the reference) is a Gaussian-modulated pulse at
 * the same instants tau: exp(-((tau - t0) / w)^2) sin(2 pi f (tau - t0)),
 * w = 4 sqrt(ln 2) / (pi f B), t0 = 3 w, B = point_source_bandwidth. */
#define FDTD_SOURCE_SINE 0
#define FDTD_SOURCE_GAUSSIAN 1

/* Replaces InternalSchemeGPU::initFromCPU + initOnGPU
 * (Source/Scheme/InternalScheme.specific.h:506-563) and the set-up half of
 * InternalScheme::initScheme (Source/Scheme/InternalScheme.inc.h:3359-3394):
 * computes dt, frequency, relPhaseVelocity, sigma profiles and the TF/SF
 * geometry, and allocates device-resident SoA arrays on `device`. */
int fdtd_create (const fdtd_config *cfg, int device, fdtd_ctx **out);

/* Replaces the material half of InternalSchemeGPU::copyFromCPU/copyToGPU
 * (InternalScheme.specific.h:200-362) for Eps, Mu, OmegaPE, OmegaPM, GammaE,
 * GammaM.  `host` holds size-N doubles.  Unset grids keep the reference
 * defaults (eps = mu = 1, Drude terms 0).  The values are staged and checked
 * on the device first: a NaN or an infinity returns FDTD_ERR_ARG (the
 * message names the first such cell) and changes nothing.  (The
 * asynchronous and device-pointer uploads below do not check: a non-finite
 * value there propagates into the fields.) */
int fdtd_upload_material (fdtd_ctx *ctx, int which, const double *host);

/* Dump helpers of Scheme::saveGrids (Source/Scheme/Scheme.inc.h:4113-4530):
 * fdtd_download_field_scattered writes the component's current level minus
 * the incident wave on the TF/SF box's cells (makeGridScattered; needs
 * TF/SF); fdtd_download_incident writes the current 1-D incident grid,
 * family 0 = EInc, 1 = HInc, of fdtd_incident_length () values (0 without
 * TF/SF), as --save-tfsf-e-incident / --save-tfsf-h-incident dump it. */
int fdtd_download_field_scattered (fdtd_ctx *ctx, int component, double *host);
int fdtd_incident_length (const fdtd_ctx *ctx);
int fdtd_download_incident (fdtd_ctx *ctx, int family, double *host, int len);

/* Host copies that overlap the time steps (no reference counterpart: the
 * reference copies synchronously around each block, Source/Scheme/
 * Scheme.inc.h:45-56, 461-472).  `host` should be pinned (cudaHostAlloc or
 * cudaHostRegister; pageable memory works but does not overlap) and stays
 * untouched until fdtd_sync returns.  fdtd_upload_material_async copies on a
 * host-to-device copy stream and applies the grid on the context's stream
 * ahead of every later fdtd_step; fdtd_download_field_async snapshots the
 * component's current level on the context's stream, in order with the steps
 * before and after it, and copies it out on a device-to-host copy stream
 * while later steps run.  fdtd_sync also waits for both copy streams. */
int fdtd_upload_material_async (fdtd_ctx *ctx, int which, const double *host);
int fdtd_download_field_async (fdtd_ctx *ctx, int component, double *host);

/* Sets the current time level (level 1 in the reference's Grid) of a field
 * component from size-N host doubles; replaces copyFromCPU for Ex..Hz. */
int fdtd_upload_field (fdtd_ctx *ctx, int component, const double *host);

/* Replaces Scheme::performNStepsForBlock (Source/Scheme/Scheme.inc.h:28-473)
 * for time steps t_start .. t_start + n_steps - 1: incident-wave steps,
 * E and H updates with PML, Drude and TF/SF, point sources.  Asynchronous on
 * the context's stream. */
int fdtd_step (fdtd_ctx *ctx, uint32_t t_start, uint32_t n_steps);

/* Waits for queued work.  timeout_ns < 0 waits without limit; otherwise the
 * wait polls and returns FDTD_ERR_TIMEOUT when the limit passes (the work
 * keeps running).  Also reports device-side error flags. */
int fdtd_sync (fdtd_ctx *ctx, int64_t timeout_ns);

/* Replaces InternalSchemeGPU::copyBackToCPU (InternalScheme.specific.h:363-504)
 * for one component: writes the current time level (what Scheme::saveGrids
 * dumps) as size-N doubles into caller-owned `host`.  Synchronous. */
int fdtd_download_field (fdtd_ctx *ctx, int component, double *host);

/* Device-resident variants for callers that keep their own device buffers
 * (no host round trip): `dev` is a device pointer to size-N doubles. */
int fdtd_upload_material_device (fdtd_ctx *ctx, int which, const double *dev);
int fdtd_download_field_device (fdtd_ctx *ctx, int component, double *dev);

/* Time-integrated / global quantities in FP64 with compensated summation
 * (no reference counterpart; the reference's exact-norm kernel,
 * InternalScheme.inc.h:310-348, is test-only).  `out` receives 1 double for
 * FDTD_REDUCE_ENERGY and 6 for FDTD_REDUCE_L2. */
int fdtd_reduce (fdtd_ctx *ctx, int what, double *out);

/* Reported set-up scalars: out[0] = dt, out[1] = frequency,
 * out[2] = relPhaseVelocity (InternalScheme.inc.h:3359-3394). */
int fdtd_scalars (const fdtd_ctx *ctx, double out[3]);

/* Number of kernel launches this context issued so far. */
int64_t fdtd_launch_count (const fdtd_ctx *ctx);

/* Running DFT (no counterpart in the reference, which saves snapshots
 * only): from this call on, every time step adds
 *   F_j += v * exp(-i 2 pi f_j t_c)
 * for component `component` (FDTD_EX..FDTD_HZ) on the plane x_axis = index
 * (axis 0, 1, 2 = x, y, z; in 2-D the plane z = 0 is the whole grid), with
 * t_c = (t + 1/2) dt for E and (t + 1) dt for H, the times of the step's
 * point sources.  Sums are FP64 with compensation, whatever the field
 * precision.  Up to 64 frequencies; calling it again restarts from zero.
 * fdtd_dft_read writes nfreq x plane cells x (re, im) doubles, the plane's
 * cells ordered as the two remaining axes with the later one fastest. */
int fdtd_dft_setup (fdtd_ctx *ctx, int component, int axis, int index, int nfreq, const double *freq_hz);
int fdtd_dft_read (fdtd_ctx *ctx, double *out);

/* Near-to-far-field transform of the reference's complex-field build, 3-D;
 * replaces Scheme::Pointing_scat / Pointing_inc and the ntffN3D_* /
 * ntffL3D_* face sums behind Scheme::saveNTFF (Source/Scheme/Scheme.inc.h:
 * 4037-4095, 4535-4645; Source/Scheme/SchemeHelper.h:1036-2121).  `re` and
 * `im` are the two runs of one configuration with source_phase 0 and 1 (their
 * fields are the real and imaginary parts of the complex build's), both in
 * the same form, stepped to the same time; FP32 / FP16-storage runs need
 * fdtd_keep_previous_level before they step (the N sums average H over the
 * current and the previous level; the sums run in FP64 on the stored values
 * either way).  The box has its faces at
 * left[a] and right[a] on axis a (the reference's leftNTFF / rightNTFF:
 * right = size - left + 1, both moved in by the --ntff-diff step), with
 * 1 <= left[a] < right[a] <= size[a] - 1.  For each azimuth phi[i]
 * (radians) at polar angle teta, out[i] is the reference's "NTFF value": the
 * scattered far-field Poynting value over the incident one. */
int fdtd_ntff (fdtd_ctx *re, fdtd_ctx *im, const int left[3], const int right[3], double teta, int nphi,
               const double *phi, double *out);

/* FP32 / FP16 storage: keep the previous level of H at the end of every
 * fdtd_step call (on = 1), as the FP64 plain form's time levels do
 * (Grid::shiftInTime; the reference's NTFF reads the previous H level,
 * Source/Scheme/SchemeHelper.h:1036-2095).  The one-sweep 3-D path then ends
 * each call on a single step (its other buffer set holds the previous
 * level); the per-cell path copies H before the last H update of the call.
 * No effect on the FP64 plain form.  Without a reference counterpart. */
int fdtd_keep_previous_level (fdtd_ctx *ctx, int on);

/* Name of the kernel that performs this context's field update (no
 * reference counterpart): "plain_fp64" (FP64 plain form), "sweep2_tma"
 * (two steps per pass: the last call ended on a pair), "sweep3d_tma"
 * (TMA-pipelined one-sweep 3-D kernel), "fused3d_regblock" (register-blocked
 * one-sweep 3-D kernel), "per_cell" (one launch per half-step), or
 * "not_stepped" before the first update.  Null for a null context. */
const char *fdtd_step_kernel (const fdtd_ctx *ctx);

/* The cudaStream_t (as void *) every launch of this context goes to, so a
 * caller can order its own work or record CUDA events against it. */
void *fdtd_stream (const fdtd_ctx *ctx);

/* Field-kernel timing (no reference counterpart; the reference only prints
 * wall-clock "Total time", Source/main.cpp:1175-1213).  While enabled, every
 * field half-step launch is bracketed by CUDA events on the context stream.
 * fdtd_kernel_time waits for the stream, then returns the summed kernel
 * milliseconds and the number of timed launches since the last call (or
 * since enabling), and resets both. */
int fdtd_profile (fdtd_ctx *ctx, int enable);
int fdtd_kernel_time (fdtd_ctx *ctx, double *ms, int64_t *launches);

/* Releases every device resource of the context; replaces
 * InternalSchemeGPU::uninitFromCPU/uninitOnGPU. */
void fdtd_destroy (fdtd_ctx *ctx);

/*
 * Adjoint (reverse-mode) gradient of a 2-D TMz run (no counterpart in the
 * reference, which has no differentiation; the backward entry the
 * reference-side glue would call to get design gradients).  The context
 * supplies the geometry, PML, point source and eps as uploaded; the run
 * starts from zero fields at t = 0 on the context's stream and leaves the
 * context's own fields untouched.  The objective is
 *   J = sum over t = 0 .. steps - 1 of sum over the probe box of Ez_t^2
 * (Ez after the E half-step and point source of step t), accumulated in
 * FP64 with compensation.  precision FDTD_PREC_FP32 runs the library's FP32
 * TMz step and its exact discrete adjoint; FDTD_PREC_FP64_PLAIN runs the
 * same formulation in FP64.  The reverse sweep keeps the state every
 * checkpoint_every steps and recomputes one segment at a time, so device
 * memory is about (steps / K + K) grids.  TF/SF and metamaterials are not
 * provided (FDTD_ERR_UNSUPPORTED).
 */
typedef struct
{
  uint32_t steps;              /* time steps of the forward run */
  uint32_t checkpoint_every;   /* K */
  int probe_lo[2];             /* probe box [lo, hi) in x and y, inside 1 .. n - 2 */
  int probe_hi[2];
  int precision;               /* FDTD_PREC_FP32 or FDTD_PREC_FP64_PLAIN */
  int reserved[3];
} fdtd_adjoint_cfg;

/* Forward run only: the objective. */
int fdtd_objective (fdtd_ctx *ctx, const fdtd_adjoint_cfg *cfg, double *objective);
/* Forward run with checkpoints, then the reverse sweep: the objective and
 * dJ/d eps for every cell (host buffer of nx * ny doubles, y fastest). */
int fdtd_backward (fdtd_ctx *ctx, const fdtd_adjoint_cfg *cfg, double *objective, double *dobj_deps);

/*
 * Batched 2-D TMz (no counterpart in the reference, whose runs are one grid
 * per process): many Dim2_TMz simulations of different sizes advanced
 * together by one persistent kernel launch per fdtd_batch_step call,
 * captured in a CUDA graph.  `base` gives the shared physics (dx,
 * wavelength, Courant factor, PML width, point-source kind/bandwidth and the
 * Ez bit of point_source_mask); precision must be FDTD_PREC_FP32 and TF/SF
 * and metamaterials are not provided.  `sizes` holds count (nx, ny) pairs;
 * every instance's point source sits at (nx/2, ny/2).  Semantics per
 * instance are those of fdtd_step on the same configuration.
 */
typedef struct fdtd_batch fdtd_batch;
int fdtd_batch_create (const fdtd_config *base, int count, const int *sizes, int device, fdtd_batch **out);
/* eps of one instance: nx*ny host doubles, (x, y) with y fastest */
int fdtd_batch_upload_eps (fdtd_batch *b, int instance, const double *host);
/* Times every candidate launch shape (x chunk of a warp tile, warps per CTA,
 * CTAs per SM) over `steps` steps of the real batch, keeps the fastest,
 * then resets the fields to t = 0.  choice[3] receives the shape. */
int fdtd_batch_tune (fdtd_batch *b, int steps, int *choice);
int fdtd_batch_step (fdtd_batch *b, uint32_t t_start, uint32_t n_steps);
int fdtd_batch_sync (fdtd_batch *b, int64_t timeout_ns);
/* component: FDTD_EZ, FDTD_HX or FDTD_HY of one instance, nx*ny doubles */
int fdtd_batch_download (fdtd_batch *b, int instance, int component, double *host);
/* total cells, whether the last step ran from a CUDA graph, and the device
 * milliseconds of the last launch (valid after fdtd_batch_sync) */
int fdtd_batch_info (const fdtd_batch *b, int64_t *cells, int *graph_used, double *last_ms);
const char *fdtd_batch_last_error (const fdtd_batch *b);
/* Time limit of one wait at the batch kernel's grid barrier between steps
 * (limit_ns <= 0 restores the default, 5 s).  A barrier that runs out sets
 * the device error flag and every CTA leaves the launch; fdtd_batch_sync
 * then returns FDTD_ERR_DEVICE and the batch's fields are left part-way
 * through a step (destroy it).  No counterpart in the reference, whose
 * kernels have no waits; it exits on any CUDA error
 * (Source/Helpers/CudaInclude.h:41-47). */
int fdtd_batch_set_wait_limit (fdtd_batch *b, int64_t limit_ns);
void fdtd_batch_destroy (fdtd_batch *b);

/* Compensated FP64 sum of weight[i] * src[i]^2 * scale over n elements,
 * written to out_dev (a caller-owned device double), for callers that must
 * not allocate device memory while they run (an application whose own
 * allocator owns the device memory budget, or a real-time step loop where
 * cudaMalloc can stall and cudaFree synchronises the device).  It allocates
 * nothing: the per-block partial sums live in one fixed static device array
 * of 1024 (sum, compensation) pairs.  src (n elements) by src_kind:
 * 0 double, 1 float, 2 half.  weight (n elements, or null) by weight_kind:
 * 0 no weight (weight ignored), 1 float, 2 double; any other kind is
 * rejected with FDTD_ERR_ARG.  blocks = 0 picks the block count;
 * blocks > 1024 is rejected with FDTD_ERR_ARG.  Every call looks the
 * array's address up with cudaGetSymbolAddress on the caller's current
 * device; the first call on a device also loads the library's device code
 * there, so that first call must come before any capture of work into a
 * stream.  Looking the address up per call keeps it valid after a
 * cudaDeviceReset.  All calls share the array: calls that overlap on the
 * GPU race, and the caller must order them.  Failures set
 * fdtd_last_error(); an error left pending by earlier, unrelated CUDA work
 * is neither reported nor cleared.  No counterpart in the reference. */
int fdtd_reduce_sq_noalloc (const void *src, int src_kind, size_t n, const void *weight, int weight_kind,
                            double scale, int blocks, double *out_dev, void *stream);

/* Time limit of one wait at the grid barriers of the context's adjoint
 * kernel (fdtd_objective / fdtd_backward); limit_ns <= 0 restores the
 * default, 2 s.  A barrier that runs out sets the device error flag, every
 * CTA leaves, and the call returns FDTD_ERR_DEVICE; the next call starts
 * afresh.  (The TMA pipeline waits of the 3-D sweep keep their fixed 1 s
 * limit.)  No counterpart in the reference (see above). */
int fdtd_set_wait_limit (fdtd_ctx *ctx, int64_t limit_ns);

/* Host-side fault injection: the next `after` device and pinned host
 * allocations the library makes succeed and every later one fails as an
 * out-of-memory error would, so the call that needs it returns
 * FDTD_ERR_NOMEM and releases what it had taken; after < 0 turns the
 * injection off.  Process-wide.  No counterpart in the reference (which
 * exits on any CUDA error, Source/Helpers/CudaInclude.h:41-47). */
int fdtd_inject_alloc_failure (int64_t after);

const char *fdtd_status_str (int status);

/* Text of the last error raised on the calling host thread (diagnostics). */
const char *fdtd_last_error (void);

#ifdef __cplusplus
}
#endif

#endif /* FDTD_B200_H */
