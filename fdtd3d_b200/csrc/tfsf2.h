// tfsf2.h - TF/SF corrections of a pair of time steps taken by the
// two-step sweep (tfsf2.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fused3d.h"

namespace fdtdb {

struct Tf2Box
{
  int lo[3], hi[3];            // cells lo .. hi - 1 per axis
  unsigned mask;               // bit 4k + t: term t of component k (Ex .. Hz) covers the box
};

struct Tf2Pass
{
  // regions as disjoint boxes (device): 0 T_E (the E term cells), 1 R_H1
  // (support of the first step's H corrections), 2 R_E (of the E
  // corrections), 3 R_H2 (of the second step's H corrections)
  Tf2Box *boxes[4] = {};
  int2 *blk[4] = {};           // per CTA: the box and the first of its cells
  int nblk[4] = {};
  // first-step E (3) and H (3) and second-step E (3) corrections:
  // full-size, zero outside T_E, R_H1 and R_E
  float *scratch[9] = {};
};

// The passes' regions as disjoint boxes (from the TF/SF term boxes), or the
// reason the scheme cannot serve the geometry (a region cell too close to
// the grid's faces or to a PML cell).
std::string tfsf2_regions (const FusedParams &p, std::vector<Tf2Box> r[4]);

// CTA table of a region (256 cells per CTA).
std::string tfsf2_blocks (const std::vector<Tf2Box> &boxes, std::vector<int2> &blk);

// Adds the TF/SF corrections of the pair of steps to p.e_new / p.h_new:
// inc_h1 / inc_e1 are the incident H before the first step's H update and
// the incident E after its E update, inc_h2 / inc_e2 the same for the second
// step (four launches; returns how many).
int launch_tfsf2 (const Tf2Pass &pass, const FusedParams &p, const double *inc_h1, const double *inc_e1,
                  const double *inc_h2, const double *inc_e2, int *err, cudaStream_t s);

}  // namespace fdtdb
