// params.h - kernel parameter blocks shared by the host launcher and kernels.
// Plain structs passed by value as kernel arguments (no device globals), so
// contexts on different devices or with different geometry never interfere.
#pragma once

#include <cstdint>

#ifndef FDTDB_HD
#if defined(__CUDACC__)
#define FDTDB_HD __host__ __device__
#else
#define FDTDB_HD
#endif
#endif

namespace fdtdb {

constexpr int kMaxTerms = 4;   // TF/SF terms per component (slots 11/12/21/22 pairs)

// One TF/SF term as the kernels see it (see TfsfTerm in setup.h).
struct TermDev
{
  int lo[3];
  int hi[3];
  int aux[3];
  int slot;        // neighbour value modified: 0 p11, 1 p12, 2 p21, 3 p22
  int inc_comp;    // component whose incident projection is used
  double negate;
};

// Layout of one updated component as the kernels see it.
struct CompDev
{
  int exists;
  int opp1, opp2;  // index 0..2 into the opposite family (E: Hx Hy Hz, H: Ex Ey Ez)
  int d11[3], d12[3], d21[3], d22[3];
  int sig_cacb, sig4, sig5;
  int nmat;
  int m[4][3];
  int nterms;
  TermDev term[kMaxTerms];
};

// Geometry scalars common to every half-step.
struct GeomDev
{
  int n[3];
  int drop;                   // bit a: axis a has size 1 (2-D / 1-D modes)
  int inc_ax[2];              // 2-D / 1-D: incident distance u k0 + v k1 along these axes
  double inc_k[2];
  double dt, dx;
  double s1, c1, s2, c2;
  double zero_inc[3];
  double proj[6];
  double min_fp[6][3];
};

// FP64 plain form: one half-step (the three E or the three H components).
struct PlainHalf
{
  GeomDev g;
  int is_h;
  int use_pml, use_tfsf, use_meta;
  double mat_modifier;         // eps0 for E, mu0 for H
  CompDev comp[3];
  double *f[3][3];             // [component][level] field E or H
  double *dd[3][3];            // D or B (PML)
  double *d1[3][3];            // D1 or B1 (metamaterials)
  const double *opp[3];        // opposite family at level 1 (null when absent)
  const double *mat;           // eps (E) or mu (H)
  const double *omega;         // omegape / omegapm
  const double *gamma;         // gammae / gammam
  const double *sigma[3];      // 1-D sigma profiles
  const double *inc;           // incident grid at level 1 (HInc for E, EInc for H)
  int cs_mask;                 // bit ci: a J / M current source on component ci of this family
  int cs[3];                   // its cell
  const double *cs_val;        // this half step's current I (device)
  // per component: its material grid and its three sigma profiles - mat and
  // sigma, or with double material precision the material averaged over its
  // eight fine cells and the profiles averaged at its position (the
  // component's stencil is then one point)
  const double *matc[3];
  const double *sigc[3][3];
  int dmp;                     // 1: the kernel reads matc / sigc (double material precision)
};

}  // namespace fdtdb
