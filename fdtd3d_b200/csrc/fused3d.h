// fused3d.h - parameters and launcher of the one-sweep 3-D E+H kernel.
#pragma once

#include <cuda_runtime.h>

#include "params.h"

namespace fdtdb {

struct FusedParams
{
  GeomDev g;
  int use_pml;
  int use_tfsf;
  int tfsf_post;               // TF/SF corrections applied by the post-pass kernel (sweep3d only)
  int fp16;
  int x_chunk;                 // x planes per CTA
  int shape;                   // tile / occupancy variant (see launch_fused3d)
  CompDev comp[6];             // Ex..Hz
  const void *e_old[3];
  const void *h_old[3];
  void *e_new[3];
  void *h_new[3];
  const float *aux_old[6];
  float *aux_new[6];
  const float *eps;            // null = uniform 1 (mu must be uniform 1)
  float courant;
  float inc_scale[6];
  const float *tab[6][6];
  int ilo[6][3], ihi[6][3];
  int face[3][4];              // TF/SF face planes per axis (-1 = unused)
  const double *inc_h;         // HInc before this step's H-incident update (E corrections)
  const double *inc_e;         // EInc after this step's E-incident update (H corrections)
  int inc_len;
  int ps[3];
  int ps_mask;
  const double *src;           // per-step table; src[src_index] E value, src[src_index + 1] H value
  int src_index;
  float ps_scale_h;

  // Drude (metamaterials): per-cell bit k set when component k sees a
  // non-zero averaged plasma frequency or collision rate; state of those
  // cells: X (in aux), X two steps back, Z = D1/eps0... scaled, Z one step back
  int use_meta;
  float dt;
  const unsigned char *dflag;
  const float *omega[2];       // omegape (E side), omegapm (H side)
  const float *gamma[2];       // gammae, gammam
  const float *xpp_old[6];
  float *xpp_new[6];
  const float *z_old[6];
  float *z_new[6];
  const float *zpp_old[6];
  float *zpp_new[6];
};

int launch_fused3d (const FusedParams &p, int *err, cudaStream_t s);
// owned y rows of one CTA for a shape variant
int fused_rows_per_cta (int shape);

// Cells x = lo[0] .. hi[0] - 1 (and the same for y, z).
struct DrudeBox
{
  int lo[3], hi[3];
};

// Bounding box of the cells with a Drude flag into box[6] (device ints:
// lowest x, y, z, then highest; INT_MAX / -1 when no cell has one).
int launch_drude_box (const unsigned char *flags, int nx, int ny, int nz, int *box, cudaStream_t s);

// Drude fix-up of a TMA sweep step over the Drude cells of `box` (two
// launches; returns how many).
int launch_drude_fixup (const FusedParams &p, const DrudeBox &box, cudaStream_t s);

// J / M current source of a one-sweep step (Scheme.inc.h:1171-1260,
// InternalScheme.inc.h:2423-2449): the sweep updates every cell without it;
// the source enters the curl of its components at one cell (curl -= I dx,
// in the scaled units), so the step's fields take the linear response: the
// E components at the cell, then the H components whose curl reads them
// (at the cell and one cell below along the third axis), then the H
// components at the cell.  Used when the cell and those neighbours are
// outside the PML for every component involved (interior update F += S
// im curl).  `src` is this step's row of the source table (E current at
// [0], H current at [1]).
struct CurrentFix
{
  int pos[3];
  int mask_e, mask_h;          // bit c: a current on component c of the family
  float scale_e, scale_h;      // I dx -> curl units (eta0 for E, 1 for H)
};
int launch_current_fix (const FusedParams &p, const CurrentFix &cf, const double *src, cudaStream_t s);

// Recomputes the per-cell Drude bitmask from the four material arrays.
int launch_drude_flags (unsigned char *flags, const float *ome, const float *gae, const float *omm, const float *gam,
                        int nx, int ny, int nz, cudaStream_t s);

}  // namespace fdtdb
