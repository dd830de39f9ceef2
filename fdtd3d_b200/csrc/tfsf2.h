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
  unsigned mask;               // bit 4k + t: term t of component k (Ex .. Hz) reaches the box
};

// A tile of the correction kernel: own box lo .. hi - 1, the terms that
// reach it, and per phase (dE1, dH1, dE2) the box of cells that can be
// nonzero, in coordinates relative to lo - 1 (lo .. hi - 1; empty when
// lo >= hi on an axis).
struct Tf2Tile
{
  int lo[3], hi[3];
  unsigned mask;               // bit 4k + t: term t of component k reaches the tile
  short ph[3][6];
};

struct Tf2Pass
{
  Tf2Tile *tiles = nullptr;    // device: the tiles
  int ntiles = 0;
  unsigned smem = 0;           // dynamic shared memory per CTA
};

// The corrections' supports as disjoint boxes (from the TF/SF term boxes):
// r[0] the E term cells, r[1] the support of the first step's H
// corrections, r[2] that of the E corrections, r[3] that of the second
// step's H corrections (which holds the others); or the reason the scheme
// cannot serve the geometry (a support cell too close to the grid's faces
// or to a PML cell).
std::string tfsf2_regions (const FusedParams &p, std::vector<Tf2Box> r[4]);

// Splits the last support into the kernel's tiles, with each tile's term
// mask and phase boxes, and the shared memory a tile needs at most.
std::string tfsf2_tiles (const FusedParams &p, const std::vector<Tf2Box> r[4], std::vector<Tf2Tile> &tiles,
                         unsigned &smem);

// Raises the kernel's dynamic shared-memory limit to smem bytes.
std::string tfsf2_configure (unsigned smem);

// Adds the TF/SF corrections of the pair of steps to p.e_new / p.h_new:
// inc_h1 / inc_e1 are the incident H before the first step's H update and
// the incident E after its E update, inc_h2 / inc_e2 the same for the second
// step (one launch; returns how many).
int launch_tfsf2 (const Tf2Pass &pass, const FusedParams &p, const double *inc_h1, const double *inc_e1,
                  const double *inc_h2, const double *inc_e2, int *err, cudaStream_t s);

}  // namespace fdtdb
