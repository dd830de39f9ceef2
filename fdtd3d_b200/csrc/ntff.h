// ntff.h - near-to-far-field transform on the device (3-D).
//
// The reference computes it in its complex-field build only, on the host,
// one face sum at a time (Source/Scheme/Scheme.inc.h:4037-4095 Pointing_scat,
// Source/Scheme/SchemeHelper.h:1036-2121 ntffN3D_* / ntffL3D_*).  Here the
// complex fields are two FP64 plain runs (sine sources: real part; cosine
// sources: imaginary part) and one kernel evaluates every face point for
// every azimuth at once.
#pragma once

#include <cuda_runtime.h>

namespace fdtdb {

struct NtffParams
{
  int n[3];                    // grid size
  int left[3], right[3];       // the box: faces at left and right on every axis
  double diff0[3];             // phase origin: n / 2 (integer division)
  double dx;                   // grid step
  double k;                    // 2 pi / wavelength
  double teta;                 // polar angle (radians)
  int h_centered;              // layout
  double min_fp[6][3];         // component positions
  // [0] real part (sine run), [1] imaginary part (cosine run): every
  // component's current level, and the previous level of H (the N sums
  // average H over the two time levels); stored as double (kind 0), float
  // (1) or half (2), value = stored * scale[component]
  const void *cur[2][6];
  const void *prev[2][6];
  int kind;
  double scale[6];
  int64_t points;              // face points over the six faces
};

// out[i * 8 + 0..7]: N_teta, N_phi, L_teta, L_phi (re, im each) at phi[i].
// partial: scratch of nphi * blocks * 8 doubles.  Returns launches issued.
int launch_ntff (const NtffParams &p, const double *phi_dev, int nphi, double *partial, int blocks, double *out,
                 cudaStream_t s);

}  // namespace fdtdb
