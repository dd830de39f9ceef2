// kernels.h - launchers of the device kernels (host-callable, no CUDA types
// beyond cudaStream_t).  Each launcher returns the number of kernels it
// launched so the context can count its launches.
#pragma once

#include <cuda_runtime.h>

#include "params.h"

namespace fdtdb {

// FP32 / FP16-storage fused form: one half-step of all E or all H components.
// Fields are stored in place (one time level); the PML auxiliary fields are
// touched only in PML cells; H is stored scaled by the free-space impedance
// so E and H share one magnitude range (needed for FP16 storage).
struct FastHalf
{
  GeomDev g;
  int is_h;
  int use_pml;
  int use_tfsf;
  int fp16;                   // 1: fields stored as __half
  CompDev comp[3];
  void *f[3];                 // updated family (float* or __half*)
  float *aux[3];              // PML auxiliary (D/eps0 or c*B), full size, PML cells only
  const void *opp[3];         // opposite family (null when absent)
  const float *mat;           // eps (E) or mu (H); null = uniform 1
  float courant;              // c*dt/dx
  float inc_scale[6];         // incident value -> stored units (eta0 for H, 1 for E)
  const float *tab[3][6];     // per component: ca1, sq1 (curl axis), p5, q5 (axis c2), g4p, g4m (axis c0)
  int ilo[3][3], ihi[3][3];   // per component per axis: sigma == 0 range
  const double *inc;          // incident grid at level 1
  int inc_len;
  int cs_mask;                // bit ci: a J / M current source on component ci of this family
  int cs[3];                  // its cell
  const double *cs_val;       // this half step's current I (device)
  float cs_scale;             // I dx -> curl units (eta0 for E, 1 for H)
  const float *matc[3];       // double material precision: per-component averaged material (null: mat)
  // Drude media (metamaterials, with PML): the family's plasma frequency and
  // collision rate per cell (FP32, rad/s), and per component the last
  // increment of X, Z = D1 or eta0 B1 and the last increment of Z, updated
  // in place (the one-sweep kernels keep the previous levels instead: a 3-D
  // Drude run whose mu map is uploaded after it has stepped changes form
  // with Drude state of the other meaning; upload mu before stepping)
  int meta;
  float dt;
  const float *om, *ga;
  float *xpp[3], *zd[3], *zpp[3];
};

int launch_plain_half (const PlainHalf &p, int inc_len, int *err, int sm_count, cudaStream_t s);

// FP64 plain form, PML coefficients per component as 1-D tables along the
// axis each one varies on: [0] ca, [1] cb (curl step, axis sig_cacb),
// [2] ca2, [3] the E-from-D denominator (axis sig5), [4], [5] the E-from-D
// numerators 2 eps0 +/- sigma dt (axis sig4).  Computed on the device by
// the per-cell code's own expressions (bit-identical values); entries whose
// averaging stencil leaves the axis stay 0 (no cell reads them).
struct PlainTabs
{
  const double *t[3][6];
};
int launch_plain_tables (const PlainHalf &p, double *const out[3][6], cudaStream_t s);
// One half-step of the FP64 plain form without a current source: one
// launch, each block on one component (interleaved by block index, so that
// the blocks reading the same opposite-family cells run together), the
// component's parameters resolved once per thread and the PML coefficients
// read from the tables; the same arithmetic per cell as plain_half_kernel.
// Returns the launches.
int launch_plain_fast (const PlainHalf &p, const PlainTabs &t, int inc_len, int *err, int sm_count,
                       cudaStream_t s);
int launch_incident_e (double *e_new, const double *e_old, const double *h_old, int len, double modifier,
                       const double *src, int src_index, cudaStream_t s);
int launch_incident_h (double *h_new, const double *h_old, const double *e_new, int len, double modifier,
                       cudaStream_t s);
int launch_point_source (double *f, size_t index, const double *src, int src_index, cudaStream_t s);

// Double material precision: per coarse cell, the average of the fine cells
// (mul * p + off[j]) of a grid nf (mul = 2 on a kept axis, 0 on a dropped one).
struct FineAvg
{
  int n[3], nf[3], mul[3];
  int off[8][3];
};
int launch_fine_average (const double *fine, double *out64, float *out32, const FineAvg &a, int sm_count,
                         cudaStream_t s);
// f -= incident value of component k on the TF/SF box's cells (a dump of the
// scattered field)
int launch_scattered (double *f, const GeomDev &g, int k, const double *inc, int inc_len, const double left[3],
                      const double right[3], int *err, int sm_count, cudaStream_t s);

int launch_fast_half (const FastHalf &p, int *err, int sm_count, cudaStream_t s);
int launch_fast_point_source (void *f, int fp16, size_t index, const double *src, int src_index, float scale,
                              cudaStream_t s);

// conversions between host-order FP64 arrays and the stored forms
int launch_convert_in (void *dst, int dst_kind, const double *src, size_t n, double scale, cudaStream_t s);
int launch_convert_out (double *dst, const void *src, int src_kind, size_t n, double scale, cudaStream_t s);
// kinds: 0 = double, 1 = float, 2 = __half
// *first = min(*first, index of every NaN / Inf among src[0 .. n))
int launch_find_nonfinite (const double *src, size_t n, unsigned long long *first, cudaStream_t s);

// compensated FP64 reductions: out[0..parts) partial pairs (sum, compensation)
// weight kinds: 0 = none, 1 = float, 2 = double
int launch_reduce_sq (const void *src, int kind, size_t n, const void *weight, int wkind, double scale,
                      double *partials, int nblocks, cudaStream_t s);
int launch_fill (double *dst, size_t n, double value, cudaStream_t s);
// one step of the running DFT of a stored field (kind 0 double, 1 float,
// 2 half) on the plane x_axis = index; phase: (cos, sin) per frequency;
// acc: (re, re comp., im, im comp.) per frequency and plane cell
int launch_dft (const void *src, int kind, int axis, int index, const int n[3], double scale, const double *phase,
                int nf, double *acc, int sm_count, cudaStream_t s);
int launch_reduce_final (const double *partials, int nblocks, double *out, cudaStream_t s);
// the two reduction launches with their own launch status (cudaLaunchKernel)
cudaError_t launch_reduce_sq_checked (const void *src, int kind, size_t n, const void *weight, int wkind,
                                      double scale, double *partials, int nblocks, cudaStream_t s);
cudaError_t launch_reduce_final_checked (const double *partials, int nblocks, double *out, cudaStream_t s);

// Sets the text fdtd_last_error() returns on the calling host thread.
void set_last_error (const char *msg);

// Every device and pinned host allocation of the library goes through these
// two, so that fdtd_inject_alloc_failure can make them fail on the host as
// an out-of-memory error would (cudaErrorMemoryAllocation, *p = null).
cudaError_t device_malloc (void **p, size_t bytes);
cudaError_t pinned_malloc (void **p, size_t bytes);

}  // namespace fdtdb
